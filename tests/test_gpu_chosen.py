"""The FP32 chosen form (ZFV_PREC_FP32) against the FP64 oracle.

The chosen form is the same scheme evaluated in FP32 with a compensated
update, so it is compared to the FP64 oracle by error norms, not bitwise:
L1 / Linf of the depth after a number of steps, plus the properties the form
is built for — an exactly well-balanced lake at rest, FP64-accurate mass.
"""
import numpy as np
import pytest

from cases import config2_strip_setup, setup
from zoomy_amrex_b200._abi import ZFV_PREC_FP32
from zoomy_amrex_b200.models import SWE
from zoomy_amrex_b200.settings import config_from_settings

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(parity_oracle):
    """The FP64 authority: the reference's own make_rhs.H under the oracle's
    driver (oracle/_ref) where it was built, else the restatement."""
    return parity_oracle


def bumps(seed, n_b=8, hump=0.3, eta0=1.0, wet_everywhere=False, moving=False):
    def ic(x):
        rng = np.random.default_rng(seed)
        b = np.zeros(x.shape[1])
        for _ in range(n_b):
            cx, cy = rng.uniform(0, 100, 2)
            a, w = rng.uniform(0.2, 1.5), rng.uniform(2.0, 10.0)
            b += a * np.exp(-((x[0] - cx) ** 2 + (x[1] - cy) ** 2) / (2 * w * w))
        e0 = b.max() + 0.5 if wet_everywhere else eta0
        hx, hy = rng.uniform(20, 80, 2)
        eta = e0 + hump * np.exp(-((x[0] - hx) ** 2 + (x[1] - hy) ** 2) / (2 * 5.0 ** 2))
        h = np.maximum(eta - b, 0.0)
        hu = 0.05 * h * np.sin(x[1] / 7.0) if moving else np.zeros_like(h)
        hv = -0.05 * h * np.cos(x[0] / 9.0) if moving else np.zeros_like(h)
        return np.array([b, h, hu, hv])
    return ic


def _settings(n, steps, **kw):
    s = dict(dimension=2, domain=[0, 100, 0, 100], n_cells=[n, n], spatial_order=2, cfl=0.45,
             time_end=1e30, max_step=steps, well_balanced=True, implicit_source=True)
    s.update(kw)
    return s


def run_fp32(model, settings):
    from zoomy_amrex_b200.level import Level
    cfg64, Q0, A0 = setup(model, settings)
    cfg = config_from_settings(model, settings, precision=ZFV_PREC_FP32)
    lev = Level(cfg, Q0, A0)
    try:
        st = lev.run(chunk=32)
        return lev.state64().cpu().numpy(), lev.aux.cpu().numpy(), st, lev.log(), (cfg64, Q0, A0)
    finally:
        lev.close()


def test_lake_at_rest_is_exact_in_fp32(cuda):
    """Config 2's lake-at-rest variant (still water over the bumps, no hump),
    fully wet, order 2, Manning implicit: u stays exactly zero (the FP32 bound
    required is 1e-6) and eta does not move."""
    model = SWE(2, "wall", bumps(3, hump=0.0, wet_everywhere=True), parameters={"n_m": 0.03})
    Q, _, st, _, (cfg, Q0, A0) = run_fp32(model, _settings(96, 200))
    assert st["step"] == 200
    u = np.abs(Q[2:]) / np.maximum(Q[1], 1e-300)
    assert u.max() < 1e-6
    assert np.abs(Q[2:]).max() == 0.0
    assert np.abs((Q[0] + Q[1]) - (Q0[0] + Q0[1])).max() < 1e-12


def test_lake_at_rest_with_dry_islands_order1(cuda):
    """With emerging bumps (dry islands) the reference scheme is exactly
    well-balanced at order 1 (Audusse); so is the FP32 form at order 1 (the
    generic tile kernels' forward-Euler stage): the momenta stay exactly
    zero and eta does not move."""
    model = SWE(2, "wall", bumps(5, hump=0.0), parameters={"n_m": 0.03})
    s = _settings(64, 100, spatial_order=1)
    from zoomy_amrex_b200.level import Level
    cfg64, Q0, A0 = setup(model, s)
    assert (Q0[1] == 0).any()
    lev = Level(cfg64, Q0, A0)
    lev.run(chunk=50)
    Q = lev.Q.cpu().numpy()
    lev.close()
    assert np.abs(Q[2:]).max() < 1e-12
    Q32, _, st, _, _ = run_fp32(model, s)
    assert st["step"] == 100
    assert np.abs(Q32[2:]).max() == 0.0
    wet = Q0[1] > 0
    assert np.abs((Q32[0] + Q32[1]) - (Q0[0] + Q0[1]))[wet].max() < 1e-12
    # dry cells did not move: their exported depth is the import/export round
    # trip's, the FP32 remainder of eta = b (b is stored in FP32)
    b32 = Q0[0].astype(np.float32).astype(np.float64)
    lo = (Q0[0] - b32).astype(np.float32).astype(np.float64)
    assert np.array_equal(Q32[1][~wet], lo[~wet])


@pytest.mark.parametrize("moving", [False, True])
def test_fp32_order1_error_vs_fp64_oracle(cuda, oracle, moving):
    """Order 1 (one forward-Euler stage per step) of the chosen form: L1 /
    Linf depth error after 150 steps of the wet/dry hump over bumps against
    the FP64 reference (Manning implicit, WB, walls), every tile variant
    giving the same bits."""
    from zoomy_amrex_b200.batch import generic_tile_variants
    from zoomy_amrex_b200.level import Level
    model = SWE(2, "wall", bumps(7, moving=moving), parameters={"n_m": 0.03})
    s = _settings(80, 150, spatial_order=1)
    cfg64, Q0, A0 = setup(model, s)
    cfg = config_from_settings(model, s, precision=ZFV_PREC_FP32)
    outs = []
    for v in range(len(generic_tile_variants())):
        lev = Level(cfg, Q0, A0, variant=v)
        try:
            st = lev.run(chunk=50)
            outs.append((lev.state64().cpu().numpy(), st))
        finally:
            lev.close()
    for Q, _ in outs[1:]:
        assert np.array_equal(Q, outs[0][0])
    Q32, st = outs[0]
    Qo, Ao, n, t, logo, _ = oracle.run(cfg64, Q0, A0)
    assert st["step"] == n == 150
    assert abs(st["time"] - t) <= 1e-6 * t
    dh = np.abs(Q32[1] - Qo[1])
    l1, linf = dh.mean(), dh.max()
    print(f"[fp32 order 1 vs fp64 oracle] moving={moving}: L1 {l1:.3e} Linf {linf:.3e} "
          f"mom {np.abs(Q32[2:] - Qo[2:]).max():.3e}")
    assert l1 <= 1e-6, l1
    assert linf <= 1e-4, linf
    assert np.abs(Q32[2:] - Qo[2:]).max() <= 1e-4
    assert ((Q32[1] <= 1e-6) == (Qo[1] <= 1e-6)).mean() > 0.999


@pytest.mark.parametrize("moving", [False, True])
def test_fp32_depth_error_vs_fp64_oracle(cuda, oracle, moving):
    """L1 / Linf depth error of the chosen form after 150 steps of a wet/dry
    hump over bumps (Manning implicit, WB, walls, order 2)."""
    model = SWE(2, "wall", bumps(7, moving=moving), parameters={"n_m": 0.03})
    s = _settings(80, 150)
    Q32, A32, st, log32, (cfg, Q0, A0) = run_fp32(model, s)
    Qo, Ao, n, t, logo, _ = oracle.run(cfg, Q0, A0)
    assert st["step"] == n == 150
    assert abs(st["time"] - t) <= 1e-6 * t
    dh = np.abs(Q32[1] - Qo[1])
    l1, linf = dh.mean(), dh.max()
    print(f"[fp32 vs fp64 oracle] moving={moving}: L1 {l1:.3e} Linf {linf:.3e} "
          f"mom {np.abs(Q32[2:] - Qo[2:]).max():.3e} dt-time {abs(st['time'] - t):.3e}")
    assert l1 <= 1e-6, l1
    assert linf <= 1e-4, linf
    assert np.abs(Q32[2:] - Qo[2:]).max() <= 1e-4
    # dry cells agree on being dry
    assert ((Q32[1] <= 1e-6) == (Qo[1] <= 1e-6)).mean() > 0.999


def test_fp32_config2_strip_error_vs_fp64_oracle(cuda, oracle):
    """The benchmark's own fields (a 4096 x 64 strip of the 4096^2 level: 16
    seeded bumps, hump, Manning n = 0.03, walls, WB, order 2), 200 steps:
    L1 / Linf depth error of the chosen form against the FP64 oracle."""
    from zoomy_amrex_b200.level import Level
    from zoomy_amrex_b200.workloads import fp64_twin
    cfg64, Q0, A0 = config2_strip_setup(steps=200)
    cfg = fp64_twin(cfg64)
    cfg.precision = ZFV_PREC_FP32
    lev = Level(cfg, Q0, A0)
    try:
        st = lev.run(chunk=50)
        Q32 = lev.state64().cpu().numpy()
    finally:
        lev.close()
    Qo, Ao, n, t, logo, _ = oracle.run(cfg64, Q0, A0)
    assert st["step"] == n == 200
    dh = np.abs(Q32[1] - Qo[1])
    l1, linf = dh.mean(), dh.max()
    print(f"[fp32 vs fp64 oracle, config-2 strip] L1 {l1:.3e} Linf {linf:.3e} "
          f"mom {np.abs(Q32[2:] - Qo[2:]).max():.3e}")
    assert l1 <= 1e-6, l1
    assert linf <= 1e-4, linf
    assert ((Q32[1] <= 1e-6) == (Qo[1] <= 1e-6)).mean() > 0.999


def test_fp32_mass_is_conserved_with_walls(cuda):
    model = SWE(2, "wall", bumps(9, moving=True), parameters={"n_m": 0.03})
    Q, _, st, log, (cfg, Q0, A0) = run_fp32(model, _settings(72, 120))
    dx = dy = 100.0 / 72
    # the FP32 form's initial mass: depth measured from its FP32 bed
    b32 = Q0[0].astype(np.float32).astype(np.float64)
    m0 = ((Q0[1] + Q0[0]) - b32).sum() * dx * dy
    m = log[:, 2]
    assert np.abs(m - m0).max() / m0 < 1e-10
    assert abs(Q[1].sum() * dx * dy - m0) / m0 < 1e-10
    assert abs(m0 - Q0[1].sum() * dx * dy) / m0 < 1e-7


def test_fp32_import_export_round_trip(cuda):
    import torch
    from zoomy_amrex_b200.level import Level
    model = SWE(2, "wall", bumps(11, moving=True))
    s = _settings(40, 1)
    cfg64, Q0, A0 = setup(model, s)
    cfg = config_from_settings(model, s, precision=ZFV_PREC_FP32)
    lev = Level(cfg, Q0, A0)
    back = lev.state64().cpu().numpy()
    lev.close()
    b32 = Q0[0].astype(np.float32).astype(np.float64)
    assert np.array_equal(back[0], b32)
    # eta = h + b is carried as float + float remainder (~48 bits)
    eta0, eta = Q0[0] + Q0[1], back[0] + back[1]
    assert np.abs(eta - eta0).max() <= 1e-13 * max(1.0, np.abs(eta0).max())
    # the depth is measured from the FP32 bed: within half an FP32 ulp of b
    assert np.abs(back[1] - Q0[1]).max() <= 6e-8 * max(1.0, np.abs(Q0[0]).max())
    assert np.abs(back[2:] - Q0[2:]).max() <= 1e-14


def test_fp32_runs_are_deterministic(cuda):
    model = SWE(2, "wall", bumps(13, moving=True), parameters={"n_m": 0.03})
    a = run_fp32(model, _settings(48, 40))
    b = run_fp32(model, _settings(48, 40))
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[3], b[3])


@pytest.mark.parametrize("shape", [(7, 5), (2, 9), (65, 2), (3, 3), (61, 33)])
def test_fp32_tiny_and_ragged_grids_every_strip_shape(cuda, oracle, shape):
    """Grids smaller than one strip, one or two cells wide, or one column
    past a strip boundary: every compiled strip shape (scalar and packed
    columns, odd widths that force the per-element path) follows the FP64
    oracle to FP32 accuracy and conserves mass with walls."""
    from zoomy_amrex_b200.batch import Batch, tile_variants
    nx, ny = shape
    model = SWE(2, "wall", bumps(17, moving=True, wet_everywhere=True), parameters={"n_m": 0.03})
    s = dict(dimension=2, domain=[0, 100, 0, 100 * ny / nx], n_cells=[nx, ny], spatial_order=2,
             cfl=0.45, time_end=1e30, max_step=20, well_balanced=True, implicit_source=True)
    cfg64, Q0, A0 = setup(model, s)
    Qo, _, n, t, _, _ = oracle.run(cfg64, Q0, A0)
    cfg = config_from_settings(model, s, precision=ZFV_PREC_FP32)
    for v in range(len(tile_variants())):
        b = Batch([cfg], [Q0], [A0], variant=v)
        b.begin()
        b.evolve(20)
        st = b.status()[0]
        Q = b.state64()[0].cpu().numpy()
        b.close()
        assert st["step"] == 20
        err = np.abs(Q[1:] - Qo[1:]).max()
        assert err <= 1e-4, (v, err)
        b32 = Q0[0].astype(np.float32).astype(np.float64)   # depth measured from the FP32 bed
        m0, m1 = ((Q0[1] + Q0[0]) - b32).sum(), Q[1].sum()
        assert abs(m1 - m0) <= 1e-10 * m0, (v, abs(m1 - m0) / m0)


def test_fp32_level_with_device_made_aux(cuda):
    """An FP32 level created without a host aux (init_solution on the device)
    runs and exports bit for bit like one given the host aux: the FP32 stages
    never read aux, and the export refreshes its hinv row."""
    from zoomy_amrex_b200.level import Level
    model = SWE(2, "wall", bumps(19, moving=True), parameters={"n_m": 0.03})
    s = _settings(56, 30)
    cfg64, Q0, A0 = setup(model, s)
    cfg = config_from_settings(model, s, precision=ZFV_PREC_FP32)
    out = []
    for aux0 in (A0, None):
        lev = Level(cfg, Q0, aux0)
        try:
            assert np.array_equal(lev.aux.cpu().numpy(), A0)
            st = lev.run(chunk=8)
            out.append((lev.state64().cpu().numpy(), lev.aux.cpu().numpy(), st["step"], st["time"]))
        finally:
            lev.close()
    (Qa, Aa, na, ta), (Qb, Ab, nb, tb) = out
    assert na == nb == 30 and ta == tb
    assert np.array_equal(Qa, Qb) and np.array_equal(Aa, Ab)


def _dry_dam(x):
    r = np.sqrt((x[0] - 3.0) ** 2 + (x[1] - 5.0) ** 2)
    h = np.where(r < 2.0, 1.0, 0.0)
    z = np.zeros_like(h)
    b = 0.1 * np.sin(x[0]) * np.cos(x[1])
    return np.array([b, h, z, z])


def test_fp32_mood_whole_step_redo(cuda, oracle):
    """positivity = "mood" in the FP32 form (generic tile kernels): order-2
    candidates with a negative or non-finite depth are discarded and the
    step is redone at order 1 from Q^n (ZoomyAmr.cpp:685-720). A circular
    dam break onto a dry bed (cfl 1, WB, walls) troubles about half of the
    FP64 reference's steps; the FP32 form redoes steps too (which ones can
    differ: a candidate depth of -1e-17 in FP64 can be exactly 0 in the
    FP32 form's eta storage), stays finite and close to the reference, and
    gives the same bits on a plain and a TMA-staged tile."""
    from zoomy_amrex_b200.level import Level
    model = SWE(2, "wall", _dry_dam)
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[40, 32], spatial_order=2, cfl=1.0,
             time_end=1e30, max_step=60, positivity="mood", well_balanced=True)
    cfg64, Q0, A0 = setup(model, s)
    Qo, Ao, n, t, logo, redos = oracle.run(cfg64, Q0, A0)
    assert redos > 0
    cfg = config_from_settings(model, s, precision=ZFV_PREC_FP32)
    from zoomy_amrex_b200.batch import generic_tile_variants
    shapes = generic_tile_variants()
    tma0 = next(k for k, sh in enumerate(shapes) if sh[2])   # the first TMA-staged variant
    outs = []
    for v in (0, tma0):
        lev = Level(cfg, Q0, A0, variant=v)
        try:
            st = lev.run(chunk=20)
            outs.append((lev.state64().cpu().numpy(), st))
        finally:
            lev.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    Q32, st = outs[0]
    dh = np.abs(Q32[1] - Qo[1])
    print(f"[fp32 mood] redos {st['mood_redos']} (fp64 {redos}), time {st['time']:.4f} (fp64 {t:.4f}), "
          f"depth L1 {dh.mean():.3e} Linf {dh.max():.3e}, min h {Q32[1].min():.3e} (fp64 {Qo[1].min():.3e})")
    assert st["step"] == n and st["mood_redos"] > 0 and st["flags"] & 2
    assert np.isfinite(Q32).all()


def test_fp32_mood_untroubled_steps_equal_plain_steps(cuda):
    """The MOOD candidate + commit path of the FP32 tile kernels gives the
    plain SSP-RK2 step's bits when no step is troubled (a shallow-moment
    case made fully wet, 0.5 m more depth everywhere, cfl 0.45)."""
    from cases import CASES_SME
    from zoomy_amrex_b200.level import Level
    from zoomy_amrex_b200.workloads import fp64_twin
    cfg64, Q0, A0 = setup(*CASES_SME["sme2d_wetdry_wb_impl_o2"])
    Q0 = Q0.copy()
    Q0[1] += 0.5
    res = []
    for mood in (0, 1):
        cfg = fp64_twin(cfg64)
        cfg.precision = ZFV_PREC_FP32
        cfg.positivity_mood = mood
        lev = Level(cfg, Q0, A0, variant=1)
        try:
            st = lev.run(chunk=25)
            res.append((lev.state64().cpu().numpy(), st))
        finally:
            lev.close()
    assert res[1][1]["mood_redos"] == 0 and res[0][1]["step"] == res[1][1]["step"]
    assert np.array_equal(res[0][0], res[1][0])
