"""sm_100a kernels against the CPU oracle, through the C ABI.

FP64 with --fmad=false on the GPU and -ffp-contract=off on the CPU evaluate
the same IEEE operations in the same order, so state, aux, step count, time
and dt are required to match BITWISE; the mass (a reduction whose summation
order differs) to 1e-13 relative.
"""
import numpy as np
import pytest

from cases import CASES_1D, CASES_2D, GOLDEN_CASES, config2_strip_setup, golden_setup, setup, wetdry_ic
from zoomy_amrex_b200.models import SWE

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(parity_oracle):
    """Every comparison in this module is against the reference's own
    make_rhs.H under the oracle's driver (oracle/_ref) where it was built,
    else against the restatement (which equals it bitwise on every case here,
    tests/test_oracle_golden.py)."""
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
    assert st["step"] == n, (st["step"], n)
    assert st["time"] == t
    bad = np.argwhere(Qg != Qo)
    assert bad.size == 0, f"{len(bad)} state values differ, first {bad[:3].tolist()}, max {np.abs(Qg - Qo).max():.3e}"
    assert np.array_equal(Ag, Ao), f"aux max diff {np.abs(Ag - Ao).max():.3e}"
    k = min(len(logo), len(logg))
    assert np.array_equal(logg[-k:, :2], logo[-k:, :2]), "dt/time sequence differs"
    np.testing.assert_allclose(logg[-k:, 2], logo[-k:, 2], rtol=1e-13, atol=0)
    return Qg, Ag, st


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_golden_cases_bitwise_vs_oracle(cuda, oracle, name):
    assert_same_run(*golden_setup(name), oracle)


@pytest.mark.parametrize("name", sorted(CASES_2D))
def test_2d_cases_bitwise_vs_oracle(cuda, oracle, name):
    assert_same_run(*setup(*CASES_2D[name]), oracle)


@pytest.mark.parametrize("name", sorted(CASES_1D))
def test_1d_cases_bitwise_vs_oracle(cuda, oracle, name):
    assert_same_run(*setup(*CASES_1D[name]), oracle)


def test_config2_strip_bitwise_vs_oracle(cuda, oracle):
    """The benchmark's own fields (16 seeded bumps over [0,100]^2 m at 4096
    cells across, hump, Manning n = 0.03, walls, WB, order 2): a 4096 x 64
    strip of rows for 20 steps, bitwise."""
    assert_same_run(*config2_strip_setup(steps=20), oracle)


def test_explicit_friction_blow_up_is_reproduced(cuda, oracle):
    """Explicit Manning friction on thin films is unstable (make_rhs.H:411-416
    explains why the reference moved to the point-implicit source); the GPU
    must follow the oracle through the blow-up value for value, NaNs included."""
    model, s = CASES_2D["wetdry_moving_o2_mixed_bc"]
    cfg, Q0, A0 = setup(model, dict(s, implicit_source=False, max_step=12))
    Qo, Ao, n, t, _, _ = oracle.run(cfg, Q0, A0)
    Qg, Ag, st, _ = run_gpu(cfg, Q0, A0)
    assert np.isnan(Qo).any() and st["step"] == n
    assert np.array_equal(np.isnan(Qg), np.isnan(Qo))
    assert np.array_equal(Qg, Qo, equal_nan=True)


def test_graph_replay_is_bitwise_eager(cuda, oracle):
    cfg, Q0, A0 = setup(*CASES_2D["wetdry_wb_manning_o2"])
    a = run_gpu(cfg, Q0, A0, use_graph=False)
    b = run_gpu(cfg, Q0, A0, use_graph=True)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("dim", [1, 2])
def test_ghost_fill_bitwise(cuda, oracle, order, dim):
    """FillPatch + FillPhysicalBC_mf (ZoomyAmr.cpp:342-443): mirror indices,
    x-first corners, wall reflection, identity aux BC."""
    import torch
    from zoomy_amrex_b200.level import Level
    if dim == 2:
        model, s = CASES_2D["wetdry_moving_o2_mixed_bc"]
    else:
        model, s = CASES_1D["bump_o1_explicit_manning"]
    s = dict(s, spatial_order=order)
    cfg, Q0, A0 = setup(model, s)
    rng = np.random.default_rng(0)
    A0 = A0 + rng.uniform(0, 1, A0.shape)       # carried aux rows must pass through unchanged
    Qg_o, Ag_o = oracle.fill_ghosts(cfg, Q0, A0, 0.25)
    lev = Level(cfg, Q0, A0)
    Qg, Ag = lev.fill_ghosts(0.25)
    torch.cuda.synchronize()
    Qg, Ag = Qg.cpu().numpy(), Ag.cpu().numpy()
    lev.close()
    if dim == 1:   # only the j = 0 row (and its x ghosts) holds data in a 1-D run
        ng = Qg.shape[1] // 2
        Qg, Ag, Qg_o, Ag_o = (a[:, ng:ng + 1, :] for a in (Qg, Ag, Qg_o, Ag_o))
    assert np.array_equal(Qg, Qg_o)
    assert np.array_equal(Ag, Ag_o)


@pytest.mark.parametrize("name", ["dambreak_o2", "wetdry_wb_manning_o2", "wetdry_o1_impl"])
def test_rhs_bitwise(cuda, oracle, name):
    """One stage's RHS (make_rhs.H:346-399) from a moving, partly dry state."""
    import torch
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = setup(*CASES_2D[name])
    Q1, A1, _, _, _, _ = oracle.run(cfg, Q0, A0, max_steps=3)   # a non-trivial state
    for impl in (0, 1):
        cfg.implicit_source = impl
        R_o = oracle.rhs(cfg, Q1, A1, 0.5)
        lev = Level(cfg, Q1, A1)
        R = lev.rhs(0.5)
        torch.cuda.synchronize()
        R = R.cpu().numpy()
        lev.close()
        assert np.array_equal(R, R_o), f"max diff {np.abs(R - R_o).max():.3e}"


def test_compute_dt_and_mass(cuda, oracle):
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = setup(*CASES_2D["wetdry_moving_o2_mixed_bc"])
    Q1, A1, _, _, _, _ = oracle.run(cfg, Q0, A0, max_steps=4)
    dt_o, mi_o = oracle.compute_dt(cfg, Q1, A1)
    lev = Level(cfg, Q1, A1)
    lev.begin()
    dt, mi = lev.compute_dt()
    m = lev.total_mass()
    lev.close()
    assert dt == dt_o and mi == mi_o
    dx = (cfg.prob_hi[0] - cfg.prob_lo[0]) / cfg.nx
    dy = (cfg.prob_hi[1] - cfg.prob_lo[1]) / cfg.ny
    np.testing.assert_allclose(m, Q1[1].sum() * (dx * dy), rtol=1e-13)


def test_first_dt_uses_stored_aux(cuda, oracle):
    """ZoomyAmr::Evolve's first ComputeDt reads the aux init_solution wrote
    (hinv = 0), not an updated one: a moving start must reproduce that."""
    cfg, Q0, A0 = setup(*CASES_2D["wetdry_o1_impl"])
    Qo, Ao, n, t, logo, _ = oracle.run(cfg, Q0, A0, max_steps=1)
    from zoomy_amrex_b200.level import Level
    lev = Level(cfg, Q0, A0)
    lev.begin()
    lev.evolve(1)
    log = lev.log()
    lev.close()
    assert log[0, 0] == logo[0, 0]


def test_update_state_bitwise(cuda, oracle):
    import torch
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = setup(*CASES_2D["wetdry_moving_o2_mixed_bc"])
    cfg.clamp_positivity = 1
    Q0 = Q0.copy(); Q0[1, 3, 3] = -1e-3          # a negative depth for the clamp
    Qo, Ao = oracle.update_state(cfg, Q0, A0, 0.0)
    lev = Level(cfg, Q0, A0)
    lev.update_state(0.0)
    torch.cuda.synchronize()
    assert np.array_equal(lev.Q.cpu().numpy(), Qo) and np.array_equal(lev.aux.cpu().numpy(), Ao)
    lev.close()


def test_run_is_deterministic(cuda):
    cfg, Q0, A0 = setup(*CASES_2D["dambreak_o2"])
    a = run_gpu(cfg, Q0, A0)
    b = run_gpu(cfg, Q0, A0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[3], b[3])


def test_mood_whole_step_redo_bitwise(cuda, oracle):
    """positivity = "mood" (ZoomyAmr.cpp:685-720): order-2 candidates with a
    negative or non-finite depth are discarded and the whole step is redone at
    order 1 from Q^n; the GPU redoes exactly the same steps."""
    model = SWE(2, "wall", wetdry_ic(5, moving=True))
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[40, 32], spatial_order=2, cfl=1.0,
             time_end=1e30, max_step=60, positivity="mood")
    cfg, Q0, A0 = setup(model, s)
    Qo, Ao, n, t, logo, redos = oracle.run(cfg, Q0, A0)
    assert redos > 0
    for graph in (False, True):
        Qg, Ag, st, logg = run_gpu(cfg, Q0, A0, use_graph=graph)
        assert st["step"] == n and st["time"] == t
        assert st["mood_redos"] == redos and st["flags"] & 2
        assert np.array_equal(Qg, Qo) and np.array_equal(Ag, Ao)
        assert np.array_equal(logg[:, :2], logo[:, :2])


@pytest.mark.parametrize("name", ["dambreak_o2", "wetdry_o1_impl", "wetdry_moving_o2_mixed_bc"])
def test_init_solution_on_device_bitwise(cuda, oracle, name):
    """zfv_init_solution writes init_solution's fields (init_solution.cpp:78-116)
    bit for bit as the oracle does, for the state's and the aux's component
    counts; a level created with aux0 = None (aux made on the device) runs
    bitwise like one given the host aux."""
    import torch
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = setup(*CASES_2D[name])
    Qi, Ai = oracle.init_solution(cfg)
    lev = Level(cfg, Q0, None)
    try:
        for ref in (Qi, Ai):
            f = torch.full(ref.shape, float("nan"), dtype=torch.float64, device=lev.device)
            _lib.check(_lib.lib().zfv_init_solution(lev.handle, f.data_ptr(), ref.shape[0], lev._s()),
                       "zfv_init_solution")
            lev.sync()
            assert np.array_equal(f.cpu().numpy(), ref)
        assert np.array_equal(lev.aux.cpu().numpy(), A0)
        st = lev.run(chunk=16)
        Qg, Ag = lev.Q.cpu().numpy(), lev.aux.cpu().numpy()
    finally:
        lev.close()
    Qo, Ao, n, t, _, _ = oracle.run(cfg, Q0, A0)
    assert st["step"] == n and st["time"] == t
    assert np.array_equal(Qg, Qo) and np.array_equal(Ag, Ao)


@pytest.mark.parametrize("shape", [(1, 37, 1), (2, 33, 17)])
def test_init_solution_odd_grids_and_offsets(cuda, oracle, shape):
    """Grids with an odd cell count and a shifted x range (the split point is
    then a cell boundary or a cell centre), 1-D and 2-D."""
    import torch
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.level import Level
    from zoomy_amrex_b200._abi import ZFV_MODEL_SWE1D, ZFV_MODEL_SWE2D, make_config
    dim, nx, ny = shape
    model = ZFV_MODEL_SWE1D if dim == 1 else ZFV_MODEL_SWE2D
    cfg = make_config(model, nx, ny, (-3.25, 0.0), (7.0, 1.0), spatial_order=2, bc=("extrapolation",) * 4)
    Qi, Ai = oracle.init_solution(cfg)
    lev = Level(cfg, Qi, None)
    try:
        assert np.array_equal(lev.aux.cpu().numpy(), Ai)
        for ref in (Qi, Ai):
            f = torch.empty(ref.shape, dtype=torch.float64, device=lev.device)
            _lib.check(_lib.lib().zfv_init_solution(lev.handle, f.data_ptr(), ref.shape[0], lev._s()),
                       "zfv_init_solution")
            lev.sync()
            assert np.array_equal(f.cpu().numpy(), ref)
    finally:
        lev.close()
