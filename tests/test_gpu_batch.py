"""The FP32 batch engine: many independent levels, one launch per stage.

A batch advances every instance exactly as a single FP32 level with the same
configuration would (the same kernels on the same strips), so per-instance
results are compared bitwise with single-level runs; the single levels are
checked against the FP64 oracle in test_gpu_chosen.py.
"""
import numpy as np
import pytest

from zoomy_amrex_b200.workloads import dam_break_ensemble, fp64_twin

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle(parity_oracle):
    """The FP64 authority: the reference's own make_rhs.H under the oracle's
    driver (oracle/_ref) where it was built, else the restatement."""
    return parity_oracle


def _single(cfg, Q0, A0, steps_chunk=16, variant=None):
    from zoomy_amrex_b200.level import Level
    lev = Level(cfg, Q0, A0, variant=variant)
    try:
        st = lev.run(chunk=steps_chunk)
        return lev.state64().cpu().numpy(), lev.aux.cpu().numpy(), st, lev.log()
    finally:
        lev.close()


def _ens(n, seed, side_range=(24, 160), **kw):
    return dam_break_ensemble(n, seed=seed, side_range=side_range, **kw)


def test_batch_equals_single_levels(cuda):
    """Uneven boxes, own bathymetry / dam ratio / friction / stop step."""
    from zoomy_amrex_b200.batch import Batch
    ens = _ens(6, seed=1)
    for k, (cfg, _, _) in enumerate(ens):
        cfg.max_step = 20 + 7 * k           # instances stop at different steps
        cfg.params[3] = 0.01 * (k + 1)      # own Manning n
    cfgs, Q0s, A0s = zip(*ens)
    b = Batch(cfgs, Q0s, A0s, variant=0)
    st = b.run(chunk=16)
    Qb = [q.cpu().numpy() for q in b.state64()]
    Ab = [a.cpu().numpy() for a in b.aux]
    b.close()
    for k, (cfg, Q0, A0) in enumerate(ens):
        Qs, As, ss, _ = _single(cfg, Q0, A0, variant=0)   # the same strip shape
        assert st[k]["step"] == ss["step"] == cfg.max_step
        assert st[k]["time"] == ss["time"]
        assert np.array_equal(Qb[k], Qs), k
        assert np.array_equal(Ab[k], As), k


def test_batch_graph_replay_equals_eager(cuda):
    from zoomy_amrex_b200.batch import Batch
    ens = _ens(5, seed=2)
    cfgs, Q0s, A0s = zip(*ens)
    a = Batch(cfgs, Q0s, A0s, variant=0)
    a.begin(); a.evolve(24)
    Qa = [q.cpu().numpy() for q in a.state64()]
    sa = a.status()
    a.close()
    g = Batch(cfgs, Q0s, A0s, variant=0)
    g.begin()
    g.capture(8)
    for _ in range(3):
        g.replay()
    Qg = [q.cpu().numpy() for q in g.state64()]
    sg = g.status()
    g.close()
    for k in range(len(ens)):
        assert sa[k]["step"] == sg[k]["step"] == 24
        assert sa[k]["time"] == sg[k]["time"]
        assert np.array_equal(Qa[k], Qg[k])


def test_batch_strip_variants_agree(cuda):
    """Every compiled strip shape advances the same instances to FP32
    accuracy. Shapes move the boundary between interior and edge strips,
    whose code paths the compiler contracts into FMAs differently, and the
    packed sweep uses FP32 pair instructions, so values agree to rounding,
    not bitwise."""
    from zoomy_amrex_b200.batch import Batch, tile_variants
    ens = _ens(4, seed=3, side_range=(40, 300))
    cfgs, Q0s, A0s = zip(*ens)
    shapes = tile_variants()
    ref = None
    for v, shape in enumerate(shapes):
        b = Batch(cfgs, Q0s, A0s, variant=v)
        b.begin(); b.evolve(30)
        Q = [q.cpu().numpy() for q in b.state64()]
        st = b.status()
        b.close()
        if ref is None:
            ref = (Q, st)
            continue
        for k in range(len(ens)):
            dh = np.abs(Q[k][1] - ref[0][k][1])
            print(f"[strip shape {shape} vs {shapes[0]}] instance {k}: "
                  f"L1 {dh.mean():.2e} Linf {dh.max():.2e} bitwise {np.array_equal(Q[k], ref[0][k])}")
            assert dh.mean() <= 1e-6 and dh.max() <= 1e-4
            assert abs(st[k]["time"] - ref[1][k]["time"]) <= 1e-6 * ref[1][k]["time"]
            assert abs(st[k]["mass"] - ref[1][k]["mass"]) <= 1e-9 * abs(ref[1][k]["mass"])


@pytest.mark.parametrize("variant", [0, 3, 7, 9])
def test_batch_depth_error_vs_fp64(cuda, oracle, variant):
    """Batch members against the FP64 oracle (L1 depth, 60 steps), scalar and
    packed sweeps."""
    from zoomy_amrex_b200.batch import Batch
    ens = _ens(3, seed=5, side_range=(32, 130), max_step=60)
    cfgs, Q0s, A0s = zip(*ens)
    b = Batch(cfgs, Q0s, A0s, variant=variant)
    st = b.run(chunk=32)
    Qb = [q.cpu().numpy() for q in b.state64()]
    b.close()
    for k, (cfg, Q0, A0) in enumerate(ens):
        Qo, _, n, t, _, _ = oracle.run(fp64_twin(cfg), Q0, A0)
        assert st[k]["step"] == n == 60
        assert abs(st[k]["time"] - t) <= 1e-6 * t
        dh = np.abs(Qb[k][1] - Qo[1])
        print(f"[batch vs fp64 oracle] {cfg.nx}x{cfg.ny}: L1 {dh.mean():.3e} Linf {dh.max():.3e}")
        assert dh.mean() <= 1e-5     # the FP32 form's L1 depth bound
        assert dh.max() <= 1e-3


def test_packed_sweep_keeps_lake_at_rest(cuda):
    """Still water over bumps, fully wet, order 2, WB, implicit Manning: the
    packed sweep keeps the momenta exactly zero (even and odd row lengths)."""
    from zoomy_amrex_b200.batch import Batch
    from zoomy_amrex_b200.workloads import dam_break_ensemble
    ens = dam_break_ensemble(2, seed=8, side_range=(70, 140))
    cfgs, Q0s, A0s = [], [], []
    for k, (c, Q0, A0) in enumerate(ens):
        Q = Q0.copy()
        Q[1] = (Q0[0].max() + 0.5) - Q0[0]
        Q[2:] = 0.0
        cfgs.append(c); Q0s.append(Q); A0s.append(A0)
    cfgs[1].nx -= 1 if cfgs[1].nx % 2 == 0 else 0          # one odd row length
    Q0s[1] = Q0s[1][:, :, :cfgs[1].nx].copy()
    A0s[1] = A0s[1][:, :, :cfgs[1].nx].copy()
    cfgs[1].prob_hi[0] = cfgs[1].nx * 0.1
    b = Batch(cfgs, Q0s, A0s, variant=3)
    b.begin(); b.evolve(100)
    Q = [q.cpu().numpy() for q in b.state64()]
    b.close()
    for k in range(2):
        assert np.abs(Q[k][2:]).max() == 0.0, k
        assert np.abs((Q[k][0] + Q[k][1]) - (Q0s[k][0] + Q0s[k][1])).max() < 1e-12


def test_batch_rejects_mixed_schemes(cuda):
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.batch import Batch
    ens = _ens(2, seed=6)
    ens[1][0].implicit_source = 0
    cfgs, Q0s, A0s = zip(*ens)
    with pytest.raises(_lib.ZfvError, match="share well_balanced"):
        Batch(cfgs, Q0s, A0s)


def test_single_level_strip_shape_selection(cuda):
    """An FP32 level starts on the library's default strip shape, switches
    shape on request (a batch of one on the same shape gives the same bits),
    and the FP64 form refuses a shape."""
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.batch import DEFAULT_VARIANT, Batch, tile_variants
    from zoomy_amrex_b200.level import Level
    cfg, Q0, A0 = _ens(1, seed=9, side_range=(150, 151))[0]
    cfg.max_step = 12
    lev = Level(cfg, Q0, A0, variant=None)
    try:
        from zoomy_amrex_b200.autotune import cached_variant
        want = cached_variant(4, "fp32", cfg.nx * cfg.ny)
        assert lev.variant == (DEFAULT_VARIANT if want is None else want)
        for v in (0, 3, len(tile_variants()) - 1):
            lev.set_variant(v)
            assert lev.variant == v
        with pytest.raises(_lib.ZfvError):
            lev.set_variant(len(tile_variants()))
    finally:
        lev.close()
    for v in (1, 11):
        Qs, _, ss, _ = _single(cfg, Q0, A0, variant=v)
        b = Batch([cfg], [Q0], [A0], variant=v)
        st = b.run(chunk=16)
        Qb = b.state64()[0].cpu().numpy()
        b.close()
        assert st[0]["step"] == ss["step"] == 12
        assert np.array_equal(Qb, Qs), v
    from zoomy_amrex_b200.workloads import fp64_twin
    lev64 = Level(fp64_twin(cfg), Q0, A0)
    try:
        assert lev64.variant == -1
        with pytest.raises(_lib.ZfvError):
            lev64.set_variant(0)
    finally:
        lev64.close()
