"""The AMR hierarchy (zoomy_amrex_b200/amr.py) on the FP32 batch engine."""
import numpy as np
import pytest

from zoomy_amrex_b200._abi import ZFV_MODEL_SWE2D, ZFV_PREC_FP32, make_config

pytestmark = pytest.mark.gpu


def _fields(nx, ny, L, dam=True, seed=3):
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * (L / nx)
    y = (np.arange(ny) + 0.5) * (L * ny / nx / ny)
    y = (np.arange(ny) + 0.5) * (L / nx)
    X, Y = np.meshgrid(x, y)
    b = np.zeros_like(X)
    for _ in range(6):
        cx, cy = rng.uniform(0, L), rng.uniform(0, L * ny / nx)
        b += rng.uniform(0.2, 0.8) * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * (0.08 * L) ** 2))
    eta = np.where(X < 0.4 * L, 2.0, 1.2) if dam else np.full_like(X, b.max() + 0.3)
    h = np.maximum(eta - b, 0.0)
    return np.array([b, h, 0 * h, 0 * h])


def _cfg(nx, ny, L):
    return make_config(ZFV_MODEL_SWE2D, nx, ny, (0.0, 0.0), (L, L * ny / nx), spatial_order=2,
                       well_balanced=True, implicit_source=True, cfl=0.45, time_end=1e30, max_step=-1,
                       bc=("wall",) * 4, params={"n_m": 0.03})


def test_amr_base_level_only_matches_single_level(cuda, oracle):
    """No refinement: the boxes of the base level, coupled through their ghost
    frames, advance like one FP32 level (and like the FP64 oracle)."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    from zoomy_amrex_b200.level import Level
    nx, ny, L, steps = 256, 192, 50.0, 40
    Q0 = _fields(nx, ny, L)
    cfg = _cfg(nx, ny, L)
    A0 = np.zeros((7, ny, nx))
    hier = AmrHierarchy(cfg, Q0, max_level=0, B=64)
    hier.run(steps)
    Qa = hier.level_state(0)
    hier.close()
    c32 = _cfg(nx, ny, L); c32.precision = ZFV_PREC_FP32; c32.max_step = steps
    lev = Level(c32, Q0, A0)
    st = lev.run(chunk=20)
    Qs = lev.state64().cpu().numpy()
    lev.close()
    assert st["step"] == steps
    c64 = _cfg(nx, ny, L); c64.max_step = steps
    Qo, _, n, _, _, _ = oracle.run(c64, Q0, A0)
    d_single = np.abs(Qa[1] - Qs[1])
    d_oracle = np.abs(Qa[1] - Qo[1])
    print(f"[amr base only] vs single FP32 level: L1 {d_single.mean():.2e} Linf {d_single.max():.2e}; "
          f"vs FP64 oracle: L1 {d_oracle.mean():.2e} Linf {d_oracle.max():.2e}")
    assert d_single.mean() < 1e-6 and d_oracle.mean() < 1e-5
    assert d_oracle.max() < 1e-3


def test_amr_lake_at_rest_on_three_levels(cuda):
    """Still water over bumps refined everywhere to three levels stays at
    rest: the ghost interpolation keeps eta flat, so the well-balanced faces
    at coarse-fine boundaries see a lake at rest too."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    nx, ny, L = 128, 128, 40.0
    Q0 = _fields(nx, ny, L, dam=False)
    hier = AmrHierarchy(_cfg(nx, ny, L), Q0, max_level=2, B=32, threshold=-1.0)
    assert len(hier.levels) == 3
    hier.run(20)
    eta0 = Q0[0, 0, 0] + Q0[1, 0, 0]
    for lev in range(3):
        q = hier.level_state(lev)
        m = ~np.isnan(q[1])
        assert np.abs(q[2][m]).max() == 0.0 and np.abs(q[3][m]).max() == 0.0, lev
        assert np.abs((q[0] + q[1])[m] - eta0).max() < 1e-5, lev
    hier.close()


def test_amr_dam_break_refines_the_front(cuda):
    """A dam break over bumps on three levels: the front is refined, regrids
    follow it, the solution stays finite and the base-level mass drifts only
    by the coarse-fine flux mismatch (no flux register, as in the reference)."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    nx, ny, L = 256, 256, 50.0
    Q0 = _fields(nx, ny, L)
    hier = AmrHierarchy(_cfg(nx, ny, L), Q0, max_level=2, B=32, threshold=0.01, regrid_int=2)
    n_levels0 = len(hier.levels)
    m0 = hier.mass()
    start = [list(lv.blocks) for lv in hier.levels]
    counts, moved = [], False
    for _ in range(8):
        hier.run(50)
        counts.append([lv.n for lv in hier.levels])
        moved |= [list(lv.blocks) for lv in hier.levels] != start
    m1 = hier.mass()
    q = hier.level_state(0)
    print(f"[amr dam break] levels at start {n_levels0}, boxes per level every 50 coarse steps {counts}, "
          f"mass drift {(m1 - m0) / m0:.2e}, time {hier.time:.4f}")
    assert n_levels0 == 3
    assert moved, "the refined boxes never followed the front"
    assert np.isfinite(q).all()
    assert abs(m1 - m0) / m0 < 1e-3
    assert (q[1] >= -1e-6).all()
    hier.close()


def test_amr_graph_replay_equals_eager_launches(cuda):
    """A coarse step replayed from its CUDA graph (device-side dt_0) gives the
    same bits as the same launches issued one by one, regrids included."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    nx, ny, L = 128, 128, 50.0
    Q0 = _fields(nx, ny, L)
    out = []
    for use_graph in (True, False):
        hier = AmrHierarchy(_cfg(nx, ny, L), Q0, max_level=2, B=32, threshold=0.01, regrid_int=2)
        hier.use_graph = use_graph
        hier.run(9)
        out.append(([hier.level_state(l) for l in range(len(hier.levels))], hier.time,
                    [list(lv.blocks) for lv in hier.levels]))
        hier.close()
    (qa, ta, ba), (qb, tb, bb) = out
    assert ta == tb and ba == bb
    for a, b in zip(qa, qb):
        assert np.array_equal(np.nan_to_num(a, nan=-7.0), np.nan_to_num(b, nan=-7.0))


def test_amr_reference_tagging_and_time_end(cuda):
    """The reference's ErrorEst criterion (undivided |grad h| or h > 1e-2, gated
    by b < b_max) refines every wet block of the dam break, a b_max below every
    bed value refines nothing; evolve() lands on time_end like
    ZoomyAmr::TimeStep."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    nx, ny, L = 128, 128, 50.0
    Q0 = _fields(nx, ny, L)
    cfg = _cfg(nx, ny, L)
    cfg.time_end = 0.05
    full = AmrHierarchy(cfg, Q0, max_level=1, B=32, threshold=0.01, tag="reference")
    gated = AmrHierarchy(cfg, Q0, max_level=1, B=32, threshold=0.01, tag="reference",
                         tag_b_max=float(Q0[0].min()))
    n_full, n_gated = full.levels[1].n, len(gated.levels) - 1
    steps = full.evolve()
    t = full.time
    q = full.level_state(1)
    full.close()
    gated.close()
    print(f"[amr reference tags] level-1 blocks {n_full}, {steps} steps to t = {t!r}")
    assert n_full == (2 * nx // 32) * (2 * ny // 32)     # every wet block, refined with full nesting
    assert n_gated == 0
    assert abs(t - 0.05) < 1e-12
    assert np.isfinite(q[~np.isnan(q)]).all()


def test_amr_plotfile_holds_every_level(cuda, tmp_path):
    """write_plotfile puts every level's patches into one AMReX plotfile (the
    multi-level format the reference's reader accepts, pinned by
    tests/test_plotfile.py); read back, each level equals level_state and the
    aux hinv row is 1/h of the written depth on wet cells."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    from zoomy_amrex_b200.plotfile import read_plotfile
    nx, ny, L = 128, 128, 50.0
    Q0 = _fields(nx, ny, L)
    hier = AmrHierarchy(_cfg(nx, ny, L), Q0, max_level=2, B=32, threshold=0.01, regrid_int=2)
    hier.run(6)
    path = hier.write_plotfile(tmp_path, "amr")
    head, levels = read_plotfile(path)
    assert head["finest_level"] == len(hier.levels) - 1 and head["ref_ratios"] == [2] * head["finest_level"]
    assert abs(head["time"] - hier.time) < 1e-15
    for lev, Lr in enumerate(levels):
        dense = hier.level_state(lev)
        assert Lr.step == 6 << lev
        assert sum(P.data.shape[1] * P.data.shape[2] for P in Lr.patches) == hier.levels[lev].n * 32 * 32
        for P in Lr.patches:
            i0, j0 = P.lo
            ny_, nx_ = P.data.shape[1:]
            assert np.array_equal(P.data[:4], dense[:, j0:j0 + ny_, i0:i0 + nx_])
            h = P.data[1]
            wet = h > 1e-3
            assert np.allclose(P.data[-1][wet], 1.0 / h[wet], rtol=1e-6)
    hier.close()


def test_amr_levels_come_and_go(cuda):
    """Raising the threshold mid-run removes the refined levels at the next
    regrid and lowering it brings them back; the coarse step's CUDA graph is
    recaptured each time and the run stays finite with the base-level mass
    drifting only by coarse-fine flux mismatch."""
    from zoomy_amrex_b200.amr import AmrHierarchy
    nx, ny, L = 128, 128, 50.0
    Q0 = _fields(nx, ny, L)
    hier = AmrHierarchy(_cfg(nx, ny, L), Q0, max_level=2, B=32, threshold=0.01, regrid_int=2)
    m0 = hier.mass()
    n_start = len(hier.levels)
    hier.run(4)
    hier.threshold = 1e9
    hier.run(4)
    n_mid = len(hier.levels)
    hier.threshold = 0.01
    hier.run(6)
    n_end = len(hier.levels)
    q = hier.level_state(0)
    m1 = hier.mass()
    hier.close()
    print(f"[amr levels] {n_start} -> {n_mid} -> {n_end}, mass drift {(m1 - m0) / m0:.2e}")
    assert n_start == 3 and n_mid == 1 and n_end == 3
    assert np.isfinite(q).all()
    assert abs(m1 - m0) / m0 < 1e-3


@pytest.mark.parametrize("dt_mode", ["fixed", "level"])
def test_two_levels_with_refinement_match_the_multilevel_oracle(cuda, dt_mode):
    """A base level of 128^2 with a fine level around a moving hump (eta
    gradient tags, 16^2 blocks, never regridded), 30 coarse steps: the FP32
    hierarchy against the FP64 two-level oracle (oracle/fv_oracle_amr.H: the
    same subcycling, coarse-fine ghost interpolation and average-down) by
    L1 / Linf on both levels, and the fine level's initial interpolation.
    dt_mode "fixed": a dt below both levels' CFL steps (the time-aligned law
    then takes it); "level": the reference's per-level CFL law
    (ZoomyAmr.cpp:739-749), each level's dt from its own current state."""
    from oracle.oracle import amr2_run
    from zoomy_amrex_b200.amr import AmrHierarchy
    n, L, steps, B = 128, 10.0, 30, 16
    x = (np.arange(n) + 0.5) * (L / n)
    X, Y = np.meshgrid(x, x)
    b = 0.4 * np.exp(-((X - 4.0) ** 2 + (Y - 6.5) ** 2) / 1.5) + 0.2 * np.exp(-((X - 7.0) ** 2 + (Y - 3.0) ** 2))
    eta = 1.0 + 0.25 * np.exp(-((X - 6.0) ** 2 + (Y - 5.0) ** 2) / 0.8)
    h = np.maximum(eta - b, 0.0)
    Q0 = np.array([b, h, 0 * h, 0 * h])
    # below both levels' CFL steps (base: 0.45 / 6 * dx / (|u| + sqrt(g h)) >= 1.3e-3
    # for |u| + sqrt(g h) < 4.5 m/s; the fine level allows twice its half step)
    dt = 1.0e-3 if dt_mode == "fixed" else 1.0
    cfg = make_config(ZFV_MODEL_SWE2D, n, n, (0.0, 0.0), (L, L), spatial_order=2, well_balanced=True,
                      implicit_source=True, cfl=0.45, dtmax=dt, time_end=1e30, max_step=-1,
                      bc=("wall",) * 4, params={"n_m": 0.03})
    hier = AmrHierarchy(cfg, Q0, max_level=1, B=B, threshold=0.02, regrid_int=0,
                        dt_mode="aligned" if dt_mode == "fixed" else "level")
    try:
        assert len(hier.levels) == 2
        patches = hier.levels[1].patches
        nblk = sum(nbx * nby for _, _, nbx, nby in patches)
        assert 0 < nblk < (2 * n // B) ** 2, nblk       # refined somewhere, not everywhere
        rects = [(bx * B, by * B, nbx * B, nby * B) for bx, by, nbx, nby in patches]
        F0 = hier.level_state(1)
        _, fine0 = amr2_run(cfg, Q0, rects, 0, dt)
        for (i0, j0, w, hh), f in zip(rects, fine0):
            d = np.abs(F0[:, j0:j0 + hh, i0:i0 + w] - f)
            assert d[1].max() < 1e-6 and d[0].max() < 1e-6
        hier.run(steps)
        t_gpu = hier.time
        G0, G1 = hier.level_state(0), hier.level_state(1)
    finally:
        hier.close()
    Qo, fine, t_or = amr2_run(cfg, Q0, rects, steps, dt if dt_mode == "fixed" else None, return_time=True)
    print(f"[amr 2 levels vs oracle, {dt_mode}] time gpu {t_gpu:.9f} oracle {t_or:.9f}")
    assert abs(t_gpu - t_or) <= 1e-6 * t_or
    d0 = np.abs(G0[1] - Qo[1])
    m0 = np.abs(G0[2:] - Qo[2:])
    print(f"[amr 2 levels vs oracle, {dt_mode}] base: depth L1 {d0.mean():.2e} Linf {d0.max():.2e}, "
          f"momenta Linf {m0.max():.2e}")
    assert d0.mean() < 1e-6 and d0.max() < 1e-4 and m0.max() < 1e-4
    worst = 0.0
    for (i0, j0, w, hh), f in zip(rects, fine):
        g = G1[:, j0:j0 + hh, i0:i0 + w]
        assert np.isfinite(g).all()
        d1 = np.abs(g[1] - f[1])
        worst = max(worst, d1.max())
        assert d1.mean() < 1e-6 and np.abs(g[2:] - f[2:]).max() < 1e-4
    print(f"[amr 2 levels vs oracle, {dt_mode}] fine patches {len(rects)}: depth Linf {worst:.2e}")
    assert worst < 1e-4
