"""The hand-written CUDA adjoint of the FP64 SWE2D step (zoomy_amrex_b200/adjoint.py).

Checked three ways: the recording forward is bitwise the solver's forward;
the gradients equal FP64 torch autograd of the plain tensor restatement
(oracle/torch_swe.py) of the same scheme; and directional derivatives equal
central finite differences of the GPU forward.
"""
import ctypes as C

import numpy as np
import pytest

from zoomy_amrex_b200._abi import ZFV_MODEL_SWE2D, make_config

pytestmark = pytest.mark.gpu

PAR = dict(g=9.81, ex=0.0, ey=0.0, h_floor=1e-6, eps=1e-24)
BC = ("wall", "extrapolation", "wall", "wall")
BC_I = (1, 0, 1, 1)


def case(nx, ny, seed, dry=False, n_m=0.03, wb=True, moving=True):
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx * 10.0
    y = (np.arange(ny) + 0.5) / ny * 10.0
    X, Y = np.meshgrid(x, y)
    b = 0.3 * np.exp(-((X - 4) ** 2 + (Y - 6) ** 2) / 4.0) + 0.02 * rng.random((ny, nx))
    if dry:
        b = b + 1.3 * np.exp(-((X - 5) ** 2 + (Y - 5) ** 2) / 1.0)
    eta = 1.0 + 0.2 * np.exp(-((X - 7) ** 2 + (Y - 3) ** 2) / 2.0)
    h = np.maximum(eta - b, 0.0)
    hu = h * (0.2 + 0.05 * np.sin(Y)) if moving else 0 * h
    hv = h * (-0.1 + 0.05 * np.cos(X)) if moving else 0 * h
    Q0 = np.array([b, h, hu, hv])
    A0 = np.zeros((7, ny, nx))
    cfg = make_config(ZFV_MODEL_SWE2D, nx, ny, (0, 0), (10, 10), spatial_order=2, well_balanced=wb,
                      implicit_source=True, cfl=0.45, time_end=1e30, max_step=-1, bc=BC,
                      params={"n_m": n_m})
    return cfg, Q0, A0


def test_record_is_the_forward(cuda):
    """zfv_adj_record advances the state exactly like zfv_evolve."""
    import torch
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.adjoint import _Solver, forward_only
    cfg, Q0, A0 = case(37, 29, 1, dry=True)
    ref = forward_only(torch.from_numpy(Q0).cuda(), torch.from_numpy(A0).cuda(), cfg, 9)
    sol = _Solver(cfg, torch.device("cuda:0"))
    L = _lib.lib()
    Q = torch.from_numpy(Q0).cuda().contiguous()
    A = torch.from_numpy(A0).cuda().contiguous()
    tape = torch.empty(int(L.zfv_adj_tape_bytes(sol.h, 9)), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    _lib.check(L.zfv_begin(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), sol.s()), "begin")
    _lib.check(L.zfv_adj_record(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), tape.data_ptr(),
                                9, sol.s()), "record")
    sol.stream.synchronize()
    sol.close()
    assert torch.equal(Q, ref)


def _loss(QT, eta_obs):
    eta = QT[0] + QT[1]
    return 0.5 * ((eta - eta_obs) ** 2).sum()


@pytest.mark.parametrize("dry", [False, True])
def test_adjoint_equals_torch_autograd(cuda, dry):
    import torch
    from oracle import torch_swe as T
    from zoomy_amrex_b200.adjoint import evolve_differentiable
    nx, ny, steps = 40, 32, 12
    cfg, Q0, A0 = case(nx, ny, 2, dry=dry)
    rng = np.random.default_rng(3)
    eta_obs = torch.from_numpy(Q0[0] + Q0[1] + 0.01 * rng.standard_normal((ny, nx)))
    # ours (CUDA reverse)
    q = torch.from_numpy(Q0).cuda().requires_grad_(True)
    nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
    QT = evolve_differentiable(q, nm, torch.from_numpy(A0).cuda(), cfg, steps, checkpoint_every=5)
    loss = _loss(QT, eta_obs.cuda())
    loss.backward()
    gq, gnm = q.grad.cpu().numpy(), float(nm.grad)
    # torch autograd of the tensor restatement, FP64 on the CPU
    qt = torch.from_numpy(Q0).clone().requires_grad_(True)
    nmt = torch.tensor(0.03, dtype=torch.float64, requires_grad=True)
    QTt, _ = T.run(qt, torch.from_numpy(A0[6]), nmt, steps, PAR, 10.0 / nx, 10.0 / ny, BC_I)
    assert torch.allclose(QTt, QT.detach().cpu(), rtol=0, atol=1e-12)
    _loss(QTt, eta_obs).backward()
    gt, gnmt = qt.grad.numpy(), float(nmt.grad)
    for r in range(4):
        err = np.abs(gq[r] - gt[r]).max() / max(np.abs(gt[r]).max(), 1e-30)
        print(f"[adjoint vs autograd] dry={dry} row {r}: max rel {err:.2e}")
        assert err < 1e-8, (r, err)
    print(f"[adjoint vs autograd] dry={dry} n_m: {gnm:.12e} vs {gnmt:.12e}")
    assert abs(gnm - gnmt) <= 1e-8 * abs(gnmt)


def test_adjoint_directional_derivatives_vs_fd(cuda):
    """Central differences of the GPU forward on random directions.

    The scheme is piecewise smooth (minmod branch switches, max wave speed,
    wet/dry): over a 1e-8 perturbation of every cell a few limiter switches
    are crossed, so the central difference at eps = 1e-6 differs from the
    derivative by ~2e-5 relative; the same gap appears between the tensor
    restatement's own finite differences and its torch autograd gradient, and
    it shrinks with eps (checked at 1e-8)."""
    import torch
    from zoomy_amrex_b200.adjoint import evolve_differentiable, forward_only
    nx, ny, steps = 96, 80, 30
    cfg, Q0, A0 = case(nx, ny, 4)
    rng = np.random.default_rng(5)
    eta_obs = torch.from_numpy(Q0[0] + Q0[1] + 0.01 * rng.standard_normal((ny, nx))).cuda()
    A = torch.from_numpy(A0).cuda()
    q = torch.from_numpy(Q0).cuda().requires_grad_(True)
    nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
    loss = _loss(evolve_differentiable(q, nm, A, cfg, steps, checkpoint_every=7), eta_obs)
    loss.backward()
    base = torch.from_numpy(Q0).cuda()
    for eps, tol in ((1e-6, 1e-4), (1e-8, 1e-5)):
        worst = 0.0
        for k in range(4):
            V = torch.from_numpy(rng.standard_normal(Q0.shape) * 0.01).cuda()
            lp = _loss(forward_only(base + eps * V, A, cfg, steps), eta_obs)
            lm = _loss(forward_only(base - eps * V, A, cfg, steps), eta_obs)
            fd = float(lp - lm) / (2 * eps)
            an = float((q.grad * V).sum())
            err = abs(fd - an) / (abs(fd) + abs(an))
            worst = max(worst, err)
            print(f"[adjoint vs FD] eps {eps:.0e} dir {k}: fd {fd:.10e} adjoint {an:.10e} rel {err:.2e}")
        assert worst < tol, (eps, worst)
    lp = _loss(forward_only(base, A, cfg, steps, n_m=0.03 + 1e-7), eta_obs)
    lm = _loss(forward_only(base, A, cfg, steps, n_m=0.03 - 1e-7), eta_obs)
    fd = float(lp - lm) / 2e-7
    print(f"[adjoint vs FD] n_m: fd {fd:.10e} adjoint {float(nm.grad):.10e}")
    assert abs(fd - float(nm.grad)) <= 1e-5 * (abs(fd) + abs(float(nm.grad)))


def test_adjoint_tile_shapes_agree(cuda):
    """Every compiled face-reverse tile shape gives the same gradients (the
    per-cell gather order is fixed, so only FMA contraction differs)."""
    import torch
    from zoomy_amrex_b200 import _lib
    from zoomy_amrex_b200.adjoint import evolve_differentiable
    L = _lib.lib()
    nx, ny, steps = 83, 45, 7
    cfg, Q0, A0 = case(nx, ny, 5, dry=True)
    eta_obs = torch.from_numpy(Q0[0] + Q0[1]).cuda() + 0.01
    grads = []
    try:
        for v in range(int(L.zfv_adj_variants())):
            _lib.check(L.zfv_adj_set_variant(v), "zfv_adj_set_variant")
            q = torch.from_numpy(Q0).cuda().requires_grad_(True)
            nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
            QT = evolve_differentiable(q, nm, torch.from_numpy(A0).cuda(), cfg, steps, checkpoint_every=3)
            _loss(QT, eta_obs).backward()
            grads.append((q.grad.detach().clone(), float(nm.grad)))
    finally:
        _lib.check(L.zfv_adj_set_variant(6), "zfv_adj_set_variant")   # the library default
    g0, n0 = grads[0]
    scale = float(g0.abs().max())
    for v, (g, n) in enumerate(grads):
        assert float((g - g0).abs().max()) <= 1e-12 * scale, v
        assert abs(n - n0) <= 1e-12 * abs(n0), v


def _bench_case(m):
    from zoomy_amrex_b200.workloads import bump_workload_config, bump_workload_fields
    Q0, A0 = bump_workload_fields(m)
    cfg = bump_workload_config(m)
    cfg.time_end = 1e30
    return cfg, Q0, A0


def test_adjoint_equals_torch_autograd_at_benchmark_scale(cuda):
    """The benchmark's wet/dry bump level at 256^2 (Manning implicit, WB,
    walls), 200 steps, checkpoints every 20: the tensor restatement's forward
    is the CUDA forward bit for bit (same IEEE operations in the same order),
    so torch autograd of it takes the same minmod / max / wet-dry branches as
    the hand-written reverse, and the two gradients agree to 1e-10."""
    import torch
    from oracle import torch_swe as T
    from zoomy_amrex_b200.adjoint import evolve_differentiable
    m, steps = 256, 200
    cfg, Q0, A0 = _bench_case(m)
    rng = np.random.default_rng(11)
    eta_obs = torch.from_numpy(Q0[0] + Q0[1] + 0.01 * rng.standard_normal((m, m))).cuda()
    A = torch.from_numpy(A0).cuda()
    q = torch.from_numpy(Q0).cuda().requires_grad_(True)
    nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
    QT = evolve_differentiable(q, nm, A, cfg, steps, checkpoint_every=20)
    _loss(QT, eta_obs).backward()
    qt = torch.from_numpy(Q0).cuda().requires_grad_(True)
    nmt = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
    QTt, _ = T.run(qt, A[6], nmt, steps, PAR, 100.0 / m, 100.0 / m, (1, 1, 1, 1), checkpoint=True)
    assert torch.equal(QTt.detach(), QT.detach()), float((QTt - QT).abs().max())
    _loss(QTt, eta_obs).backward()
    for r in range(4):
        err = float((q.grad[r] - qt.grad[r]).abs().max() / qt.grad[r].abs().max())
        print(f"[adjoint vs autograd, 256^2 x 200] row {r}: max rel {err:.2e}")
        assert err <= 1e-10, (r, err)
    e_nm = abs(float(nm.grad) - float(nmt.grad)) / abs(float(nmt.grad))
    print(f"[adjoint vs autograd, 256^2 x 200] n_m: rel {e_nm:.2e}")
    assert e_nm <= 1e-10


def test_adjoint_taylor_remainder_is_second_order(cuda):
    """Taylor test of x -> L(Q_T(x)) at a generic point of a fully wet level
    (the benchmark's bumps and hump with 0.6 m more depth everywhere,
    N(0, 1e-3^2) seeded noise on b, h, hu and hv; Manning implicit, WB,
    walls): the remainder |L(x + eps d) - L(x) - eps g.d| falls as eps^2 on
    seeded directions over (b, h, hu, hv). The map is continuous and
    piecewise smooth (minmod, the hydrostatic max(b_L, b_R), the Rusanov and
    CFL maxima); a kink crossed inside +-eps adds at most eps times its slope
    jump and is crossed with probability ~eps, so the slope stays 2 -- as
    long as the base point is not itself on kinks. A lake at rest is: zero
    momentum and near-flat stretches of the smooth bed put the minmod
    arguments at (or within rounding of) zero, where no derivative exists
    and the remainder falls only as eps; hence the noise. (With dry cells
    the discrete map also has jumps, e.g. the friction Jacobian's Heaviside
    at h = h_floor.)"""
    import torch
    from zoomy_amrex_b200.adjoint import evolve_differentiable, forward_only
    m, steps = 128, 100
    cfg, Q0, A0 = _bench_case(m)
    Q0 = Q0.copy()
    Q0[1] = Q0[1] + 0.6                                  # every cell wet, the hump kept
    nrng = np.random.default_rng(13)
    for r in range(4):                                   # off the kinks of the lake at rest
        Q0[r] += 1e-3 * nrng.standard_normal((m, m))
    assert Q0[1].min() >= 0.59
    rng = np.random.default_rng(12)
    eta_obs = torch.from_numpy(Q0[0] + Q0[1] + 0.01 * rng.standard_normal((m, m))).cuda()
    A = torch.from_numpy(A0).cuda()
    q = torch.from_numpy(Q0).cuda().requires_grad_(True)
    nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
    L0 = _loss(evolve_differentiable(q, nm, A, cfg, steps, checkpoint_every=20), eta_obs)
    L0.backward()
    base = torch.from_numpy(Q0).cuda()
    wet = torch.from_numpy((Q0[1] > 0).astype(np.float64)).cuda()
    epss = [1e-2, 1e-3, 1e-4, 1e-5]
    rem = np.zeros((8, len(epss)))
    for k in range(8):
        V = torch.from_numpy(rng.standard_normal(Q0.shape) * 1e-2).cuda()
        V[1:] *= wet
        gd = float((q.grad * V).sum())
        for e, eps in enumerate(epss):
            Le = float(_loss(forward_only(base + eps * V, A, cfg, steps), eta_obs))
            rem[k, e] = abs(Le - float(L0) - eps * gd)
    med = np.median(rem, axis=0)
    slope = np.polyfit(np.log10(epss), np.log10(med), 1)[0]
    print(f"[adjoint Taylor test 128^2 x 100] median remainders {med}, slope {slope:.2f}")
    assert slope >= 1.8
