"""The shallow-moment model (level 2, csrc/models/sme.H) on the sm_100a
kernels: the FP64 plain form against the CPU oracle, through the C ABI.

The FP64 stage kernels are generic in Model::n_dof_q, so the 8-row moment
model runs the same fused kernels as the shallow-water model; state, aux,
step count, time and every dt must equal the reference's make_rhs.H under
the oracle's driver bit for bit (the mass, a reduction in another order, to
1e-13). Cases: wet/dry bumps with well-balancing and the point-implicit
Navier-slip solve (8 x 8 elimination, make_rhs.H:429-509), mixed walls and
extrapolation with a moving start, order 1, a 7 x 5 grid, 1-D, and a strip
of the benchmark level itself.
"""
import numpy as np
import pytest

from cases import CASES_SME, setup, sme_strip_setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(parity_oracle):
    """The reference's own make_rhs.H under the oracle's driver (oracle/_ref)
    where it was built, else the restatement (equal to it bitwise on every
    case here, tests/test_oracle_golden.py)."""
    return parity_oracle


def run_gpu(cfg, Q0, A0, use_graph=False, chunk=16):
    from zoomy_amrex_b200.level import Level
    lev = Level(cfg, Q0, A0)
    try:
        st = lev.run(chunk=chunk, use_graph=use_graph)
        return lev.Q.cpu().numpy(), lev.aux.cpu().numpy(), st, lev.log()
    finally:
        lev.close()


def assert_same_run(cfg, Q0, A0, oracle, use_graph=False):
    Qo, Ao, n, t, logo, _ = oracle.run(cfg, Q0, A0)
    Qg, Ag, st, logg = run_gpu(cfg, Q0, A0, use_graph=use_graph)
    assert np.isfinite(Qo).all()
    assert st["step"] == n, (st["step"], n)
    assert st["time"] == t
    bad = np.argwhere(Qg != Qo)
    assert bad.size == 0, f"{len(bad)} state values differ, first {bad[:3].tolist()}, max {np.abs(Qg - Qo).max():.3e}"
    assert np.array_equal(Ag, Ao), f"aux max diff {np.abs(Ag - Ao).max():.3e}"
    k = min(len(logo), len(logg))
    assert np.array_equal(logg[-k:, :2], logo[-k:, :2]), "dt/time sequence differs"
    np.testing.assert_allclose(logg[-k:, 2], logo[-k:, 2], rtol=1e-13, atol=0)
    return Qg, Ag, st


@pytest.mark.parametrize("name", sorted(CASES_SME))
def test_sme_cases_bitwise_vs_oracle(cuda, oracle, name):
    assert_same_run(*setup(*CASES_SME[name]), oracle)


def test_sme_benchmark_strip_bitwise_vs_oracle(cuda, oracle):
    """Rows 0..31 of the 2048^2 shallow-moment benchmark level, 20 steps."""
    assert_same_run(*sme_strip_setup(steps=20), oracle)


def test_sme_graph_replay_is_bitwise_eager(cuda):
    cfg, Q0, A0 = setup(*CASES_SME["sme2d_wetdry_wb_impl_o2"])
    a = run_gpu(cfg, Q0, A0, use_graph=False)
    b = run_gpu(cfg, Q0, A0, use_graph=True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("name", ["sme2d_wetdry_wb_impl_o2", "sme2d_moving_mixed_bc_o2"])
def test_sme_rhs_and_ghosts_bitwise(cuda, oracle, name):
    """One stage's RHS (make_rhs.H:346-399) and the ghost fill with the wall
    mirror of the whole velocity profile, from a moving state."""
    import torch
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = setup(*CASES_SME[name])
    Q1, A1, _, _, _, _ = oracle.run(cfg, Q0, A0, max_steps=3)
    for impl in (0, 1):
        cfg.implicit_source = impl
        R_o = oracle.rhs(cfg, Q1, A1, 0.5)
        lev = Level(cfg, Q1, A1)
        R = lev.rhs(0.5)
        Qg, Ag = lev.fill_ghosts(0.25)
        torch.cuda.synchronize()
        R, Qg, Ag = R.cpu().numpy(), Qg.cpu().numpy(), Ag.cpu().numpy()
        lev.close()
        assert np.array_equal(R, R_o), f"max diff {np.abs(R - R_o).max():.3e}"
        Qg_o, Ag_o = oracle.fill_ghosts(cfg, Q1, A1, 0.25)
        assert np.array_equal(Qg, Qg_o) and np.array_equal(Ag, Ag_o)


def test_sme_lake_at_rest_is_exact(cuda):
    """Still water over bumps with every moment zero, fully wet, order 2,
    well-balanced, implicit friction: nothing moves (|u| < 1e-12)."""
    from zoomy_amrex_b200.models import SME
    from cases import _bumps

    def ic(x):
        b = _bumps(x, 17)
        h = b.max() + 0.5 - b
        z = np.zeros_like(h)
        return np.array([b, h, z, z, z, z, z, z])
    model = SME(level=2, dimension=3, bc="wall", initial_conditions=ic)
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[64, 48], spatial_order=2, cfl=0.45, time_end=1e30,
             max_step=200, well_balanced=True, implicit_source=True)
    cfg, Q0, A0 = setup(model, s)
    Q, _, st, _ = run_gpu(cfg, Q0, A0)
    assert st["step"] == 200
    assert np.abs(Q[2:]).max() < 1e-12
    assert np.abs((Q[0] + Q[1]) - (Q0[0] + Q0[1])).max() < 1e-12


# --- the FP32 chosen form of the shallow-moment model (generic tile kernels) ---

def run_fp32(cfg64, Q0, A0, variant=None, chunk=25):
    from zoomy_amrex_b200._abi import ZFV_PREC_FP32
    from zoomy_amrex_b200.level import Level
    from zoomy_amrex_b200.workloads import fp64_twin
    cfg = fp64_twin(cfg64)
    cfg.precision = ZFV_PREC_FP32
    lev = Level(cfg, Q0, A0, variant=variant)
    try:
        st = lev.run(chunk=chunk)
        return lev.state64().cpu().numpy(), lev.aux.cpu().numpy(), st, lev.log()
    finally:
        lev.close()


@pytest.mark.parametrize("name", ["sme2d_wetdry_wb_impl_o2", "sme2d_moving_mixed_bc_o2", "sme2d_o1_impl_wb"])
def test_sme_fp32_error_vs_fp64_oracle(cuda, oracle, name):
    """L1 / Linf error of the FP32 chosen form against the FP64 oracle, depth
    and moments (the FP32 form has no bitwise target)."""
    cfg, Q0, A0 = setup(*CASES_SME[name])
    Q32, A32, st, _ = run_fp32(cfg, Q0, A0)
    Qo, Ao, n, t, _, _ = oracle.run(cfg, Q0, A0)
    assert st["step"] == n
    assert abs(st["time"] - t) <= 1e-6 * t
    dh = np.abs(Q32[1] - Qo[1])
    dm = np.abs(Q32[2:] - Qo[2:])
    print(f"[sme fp32 vs fp64 oracle] {name}: depth L1 {dh.mean():.3e} Linf {dh.max():.3e}, "
          f"momenta/moments Linf {dm.max():.3e}")
    assert dh.mean() <= 1e-6 and dh.max() <= 1e-4
    assert dm.max() <= 1e-4
    # export refreshes aux with the model's FP64 hinv of the exported depth
    h4 = Q32[1] ** 4
    np.testing.assert_allclose(A32[0], np.sqrt(2.0) * Q32[1] / np.sqrt(h4 + np.maximum(h4, 1e-24)), rtol=1e-14)


def test_sme_fp32_benchmark_strip_error(cuda, oracle):
    """Rows 0..31 of the 2048^2 shallow-moment benchmark level, 100 steps."""
    cfg, Q0, A0 = sme_strip_setup(steps=100)
    Q32, _, st, _ = run_fp32(cfg, Q0, A0)
    Qo, _, n, _, _, _ = oracle.run(cfg, Q0, A0)
    assert st["step"] == n == 100
    dh = np.abs(Q32[1] - Qo[1])
    print(f"[sme fp32 vs fp64 oracle, benchmark strip] depth L1 {dh.mean():.3e} Linf {dh.max():.3e} "
          f"moments Linf {np.abs(Q32[4:] - Qo[4:]).max():.3e}")
    assert dh.mean() <= 1e-6 and dh.max() <= 1e-4


def test_sme_fp32_lake_at_rest_is_exact(cuda):
    """Fully wet still water over bumps, no moments, order 2, WB, implicit:
    the FP32 form keeps every momentum and moment exactly zero."""
    from zoomy_amrex_b200.models import SME
    from cases import _bumps

    def ic(x):
        b = _bumps(x, 19)
        h = b.max() + 0.5 - b
        z = np.zeros_like(h)
        return np.array([b, h, z, z, z, z, z, z])
    model = SME(level=2, dimension=3, bc="wall", initial_conditions=ic)
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[64, 48], spatial_order=2, cfl=0.45, time_end=1e30,
             max_step=200, well_balanced=True, implicit_source=True)
    cfg, Q0, A0 = setup(model, s)
    Q, _, st, _ = run_fp32(cfg, Q0, A0)
    assert st["step"] == 200
    assert np.abs(Q[2:]).max() == 0.0
    assert np.abs((Q[0] + Q[1]) - (Q0[0] + Q0[1])).max() < 1e-12


def test_sme_fp32_tile_shapes_agree_and_mass_is_conserved(cuda):
    """Every tile shape, staged by plain loads or by TMA boxes, computes the
    same faces in the same order: identical results. With walls the FP64
    mass of the compensated state is conserved."""
    from zoomy_amrex_b200.batch import generic_tile_variants
    cfg, Q0, A0 = setup(*CASES_SME["sme2d_wetdry_wb_impl_o2"])
    variants = generic_tile_variants()
    assert len(variants) == 6 and [v[2] for v in variants] == [0, 0, 0, 1, 1, 1]
    assert cfg.nx % 4 == 0
    outs = [run_fp32(cfg, Q0, A0, variant=v) for v in range(len(variants))]
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
    log = outs[0][3]
    b32 = Q0[0].astype(np.float32).astype(np.float64)
    m0 = ((Q0[1] + Q0[0]) - b32).sum() * (10.0 / 48) * (10.0 / 40)
    assert np.abs(log[:, 2] - m0).max() / m0 < 1e-10
