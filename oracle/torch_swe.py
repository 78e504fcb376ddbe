"""Plain tensor restatement of the 2-D shallow-water SSP-RK2 step (FP64), for
autograd. TEST INFRASTRUCTURE: the adjoint tests differentiate this with
torch.autograd and compare with the hand-written CUDA reverse; nothing in the
package imports it.

Same scheme as the oracle (oracle/fv_oracle.H) for ZFV_MODEL_SWE2D, order 2,
no clamp, no MOOD:
  * ghost cells by mirroring (ZoomyAmr.cpp:399-406), walls flip the normal
    momentum (the SWE boundary_conditions);
  * per face: minmod MUSCL on b, h, hu, hv (make_rhs.H:9-13, 31-83), Audusse
    hydrostatic reconstruction when well-balanced (make_rhs.H:84-98), hinv of
    the face states (make_rhs.H:114-115), central flux + Rusanov D+- with the
    bed product g (hL+hR)/2 (bR-bL) (make_rhs.H:129-130);
  * cell RHS -(f_r - f_l) - D-_r - D+_l per direction over dx, plus the WB bed
    source 0.5 g (h*_L,r^2 - h*_R,l^2)/dx (make_rhs.H:142-163, 346-399);
  * point-implicit Manning source with hinv of the stage input held fixed
    (make_rhs.H:429-509; the 4x4 system reduces to the 2x2 momentum block);
  * Heun average, dt from the CFL max over cells (ZoomyAmr.cpp:448-515, 665-675).
"""
from __future__ import annotations

import math

import torch

SQRT2 = math.sqrt(2.0)


def sdiv(a, s):
    """a / s for a Python scalar s, correctly rounded per element (PyTorch
    turns a division by a CPU scalar into a multiplication by its
    reciprocal, which rounds twice)."""
    return a / torch.full_like(a, s)


def rdiv(s, a):
    """s / a for a Python scalar s, correctly rounded (scalar / tensor is
    a reciprocal followed by a multiplication in PyTorch)."""
    return torch.full_like(a, s) / a


class _Sqrt(torch.autograd.Function):
    """Correctly rounded square root (IEEE, as the oracle's std::sqrt and the
    kernels' FP64 sqrt): PyTorch's CPU sqrt goes through a vector math
    library that can be one ulp off; on the GPU torch.sqrt is IEEE."""

    @staticmethod
    def forward(ctx, x):
        if x.is_cuda:
            y = torch.sqrt(x)
        else:
            import numpy as np
            y = torch.from_numpy(np.sqrt(x.detach().numpy()))
        ctx.save_for_backward(y)
        return y

    @staticmethod
    def backward(ctx, g):
        (y,) = ctx.saved_tensors
        return g * 0.5 / y


def csqrt(x):
    return _Sqrt.apply(x)


def hinv(h, eps):
    x0 = (h * h) * (h * h)
    return SQRT2 * h / csqrt(x0 + torch.where(x0 < eps, torch.full_like(x0, eps), x0))


def minmod(a, b):
    z = torch.zeros_like(a)
    pick_a = torch.abs(a) < torch.abs(b)
    v = torch.where(pick_a, a, b)
    return torch.where(a * b <= 0, z, v)


def _mirror_index(n, lo_pad, hi_pad, device):
    i = torch.arange(-lo_pad, n + hi_pad, device=device)
    out = (i < 0) | (i >= n)
    m = torch.where(i < 0, -1 - i, torch.where(i >= n, 2 * n - 1 - i, i))
    return m.clamp(0, n - 1), out


def pad2(Q, bc, ng=2):
    """(4, ny, nx) -> (4, ny, nx + 2 ng) x-padded and (4, ny + 2 ng, nx) y-padded."""
    _, ny, nx = Q.shape
    ix, ox = _mirror_index(nx, ng, ng, Q.device)
    iy, oy = _mirror_index(ny, ng, ng, Q.device)
    Qx = Q[:, :, ix]
    Qy = Q[:, iy, :]
    sx = torch.ones(nx + 2 * ng, dtype=Q.dtype, device=Q.device)
    sx[:ng] = -1.0 if bc[0] == 1 else 1.0
    sx[nx + ng:] = -1.0 if bc[1] == 1 else 1.0
    sy = torch.ones(ny + 2 * ng, dtype=Q.dtype, device=Q.device)
    sy[:ng] = -1.0 if bc[2] == 1 else 1.0
    sy[ny + ng:] = -1.0 if bc[3] == 1 else 1.0
    Qx = torch.stack([Qx[0], Qx[1], Qx[2] * sx[None, :], Qx[3]])
    Qy = torch.stack([Qy[0], Qy[1], Qy[2], Qy[3] * sy[:, None]])
    return Qx, Qy


def faces(c0, c1, c2, c3, D, p, wb):
    """Face outputs for stencils c0..c3 (each (4, ...)): flux (3), D+ (3), D- (3), h*_L, h*_R."""
    g, eps = p["g"], p["eps"]
    qL = c1 + 0.5 * minmod(c1 - c0, c2 - c1)
    qR = c2 - 0.5 * minmod(c2 - c1, c3 - c2)
    bL, hL, mLx, mLy = qL
    bR, hR, mRx, mRy = qR
    if wb:
        bf = torch.where(bL < bR, bR, bL)
        tL = hL + bL - bf
        tR = hR + bR - bf
        hsL = torch.where(0.0 < tL, tL, torch.zeros_like(tL))
        hsR = torch.where(0.0 < tR, tR, torch.zeros_like(tR))
        sL = torch.where(hL > 0, hsL / torch.where(hL > 0, hL, torch.ones_like(hL)), torch.zeros_like(hL))
        sR = torch.where(hR > 0, hsR / torch.where(hR > 0, hR, torch.ones_like(hR)), torch.zeros_like(hR))
        mLx, mLy, mRx, mRy = mLx * sL, mLy * sL, mRx * sR, mRy * sR
        hL, hR = hsL, hsR
        bL = bR = bf
    hiL, hiR = hinv(hL, eps), hinv(hR, eps)
    mL = (mLx, mLy)
    mR = (mRx, mRy)
    FL = [mL[D]]
    FR = [mR[D]]
    for k in range(2):
        FL.append(mL[k] * mL[D] * hiL + (0.5 * g * hL * hL if k == D else 0.0))
        FR.append(mR[k] * mR[D] * hiR + (0.5 * g * hR * hR if k == D else 0.0))

    evL = torch.abs(mL[D] * hiL) + _sqrt_g(hL, g)
    evR = torch.abs(mR[D] * hiR) + _sqrt_g(hR, g)
    s = torch.where(evL < evR, evR, evL)
    db = bR - bL
    Bn = g * (0.5 * (hL + hR))
    dq = [hR - hL, mRx - mLx, mRy - mLy]
    flux, dp, dm = [], [], []
    for n in range(3):
        flux.append(0.5 * (FL[n] + FR[n]))
        bdq = Bn * db if n == 1 + D else 0.0
        dp.append(0.5 * bdq + 0.5 * s * dq[n])
        dm.append(0.5 * bdq - 0.5 * s * dq[n])
    return flux, dp, dm, hL, hR


def explicit_stage(X, dt, p, dx, dy, bc, wb):
    """q* = X + dt RHS(X)."""
    _, ny, nx = X.shape
    Qx, Qy = pad2(X, bc)
    # x-faces a = 0..nx between cells a-1 and a: stencil padded columns a .. a+3
    cx = [Qx[:, :, k:k + nx + 1] for k in range(4)]
    fx, dpx, dmx, hLx, hRx = faces(*cx, 0, p, wb)
    cy = [Qy[:, k:k + ny + 1, :] for k in range(4)]
    fy, dpy, dmy, hLy, hRy = faces(*cy, 1, p, wb)
    rows = [X[0]]
    for n in range(3):
        Fx = -(fx[n][:, 1:] - fx[n][:, :-1]) - dmx[n][:, 1:] - dpx[n][:, :-1]
        Fy = -(fy[n][1:, :] - fy[n][:-1, :]) - dmy[n][1:, :] - dpy[n][:-1, :]
        rhs = sdiv(Fx, dx) + sdiv(Fy, dy)
        if wb and n == 1:
            rhs = rhs + sdiv(0.5 * p["g"] * (hLx[:, 1:] * hLx[:, 1:] - hRx[:, :-1] * hRx[:, :-1]), dx)
        if wb and n == 2:
            rhs = rhs + sdiv(0.5 * p["g"] * (hLy[1:, :] * hLy[1:, :] - hRy[:-1, :] * hRy[:-1, :]), dy)
        rows.append(X[n + 1] + dt * rhs)
    return torch.stack(rows)


class _InvCbrt(torch.autograd.Function):
    """m^(-1/3) for m > 0 (normal numbers), bit for bit the model's
    zb::inv_cbrt_pos (exponent reduction m = f 2^e, e = 3q + r, a cubic first
    guess of f^(-1/3) scaled by 2^(-r/3), three multiply-only Newton steps,
    times 2^(-q)); the derivative is the analytic -(1/3) y / m."""

    @staticmethod
    def forward(ctx, m):
        mant, ex = torch.frexp(m)            # m = mant 2^ex, mant in [0.5, 1)
        f = mant * 2.0                       # f in [1, 2), exact
        e = ex.to(torch.int64) - 1
        q = torch.div(e, 3, rounding_mode="floor")
        r = e - 3 * q
        one = torch.ones_like(m)
        w = f * torch.where(r == 0, one, torch.where(r == 1, 2.0 * one, 4.0 * one))
        c = torch.where(r == 0, one, torch.where(r == 1, 0.7937005259840998 * one, 0.6299605249474366 * one))
        y = (1.53701885 + f * (-0.801366717 + f * (0.312967226 + f * -0.0490997445))) * c
        for _ in range(3):
            y3 = y * y * y
            y = y + y * (1.0 - w * y3) * (1.0 / 3.0)
        y = torch.ldexp(y, -q)
        ctx.save_for_backward(m, y)
        return y

    @staticmethod
    def backward(ctx, g):
        m, y = ctx.saved_tensors
        return g * (-(1.0 / 3.0)) * y / m


def inv_cbrt(m):
    return _InvCbrt.apply(m)


def implicit(qs, hv, dt, p, n_m):
    g, hf = p["g"], p["h_floor"]
    h, mx, my = qs[1], qs[2], qs[3]
    m = torch.where(h < hf, torch.full_like(h, hf), h)
    k = g * n_m * n_m * inv_cbrt(m)
    ux, uy = mx * hv, my * hv
    sp2 = ux * ux + uy * uy
    pos = sp2 > 0
    sp = torch.where(pos, csqrt(torch.where(pos, sp2, torch.ones_like(sp2))), torch.zeros_like(sp2))
    S0 = g * p["ex"] * h - k * ux * sp
    S1 = g * p["ey"] * h - k * uy * sp
    rsp = torch.where(pos, 1.0 / torch.where(pos, sp, torch.ones_like(sp)), torch.zeros_like(sp))
    dsx, dsy = ux * hv * rsp, uy * hv * rsp
    # dk/dh through max(h, h_floor)^(-1/3): Heaviside(h - h_floor, 1/2)
    ic = inv_cbrt(m)
    heav = torch.where(h - hf > 0, torch.ones_like(h), torch.where(h - hf < 0, torch.zeros_like(h),
                                                                   torch.full_like(h, 0.5)))
    dk_dh = -k * (ic * ic * ic) * (1.0 / 3.0) * heav
    z = torch.zeros_like(h)
    J = [[z, z, z, z], [z, z, z, z],
         [z, g * p["ex"] - dk_dh * ux * sp, -k * (hv * sp + ux * dsx), -k * (ux * dsy)],
         [z, g * p["ey"] - dk_dh * uy * sp, -k * (uy * dsx), -k * (hv * sp + uy * dsy)]]
    S = [z, z, S0, S1]
    q0 = [qs[0], qs[1], mx, my]
    return torch.stack(point_implicit(q0, S, J, dt))


def point_implicit(q0, S, J, dt):
    """make_rhs.H:429-509 elementwise over a field: A = I - dt J, rhs dt S,
    Gaussian elimination with partial pivoting in the same operation order as
    the oracle and the kernels (so the branch choices and the rounding are
    theirs), q = q0 + dq; the explicit update q0 + dt S (or q0 where that is
    not finite) if a pivot vanishes or a component is not finite."""
    n = len(q0)
    one = torch.ones_like(q0[0])
    A = [[(one if r == c else torch.zeros_like(one)) - dt * J[r][c] for c in range(n)] for r in range(n)]
    b = [dt * S[r] for r in range(n)]
    ok = torch.ones_like(one, dtype=torch.bool)
    for k in range(n):
        best = torch.abs(A[k][k])
        piv = torch.full_like(one, float(k))
        for r in range(k + 1, n):
            take = torch.abs(A[r][k]) > best
            best = torch.where(take, torch.abs(A[r][k]), best)
            piv = torch.where(take, torch.full_like(one, float(r)), piv)
        ok = ok & (best > 0) & torch.isfinite(best)
        for r in range(k + 1, n):
            sw = piv == float(r)
            for c in range(k, n):
                A[k][c], A[r][c] = torch.where(sw, A[r][c], A[k][c]), torch.where(sw, A[k][c], A[r][c])
            b[k], b[r] = torch.where(sw, b[r], b[k]), torch.where(sw, b[k], b[r])
        piv_nz = torch.where(ok, A[k][k], one)     # keep the unused branch finite
        for r in range(k + 1, n):
            f = A[r][k] / piv_nz
            for c in range(k, n):
                A[r][c] = A[r][c] - f * A[k][c]
            b[r] = b[r] - f * b[k]
    dq = [None] * n
    for r in range(n - 1, -1, -1):
        s = torch.zeros_like(one)
        for c in range(r + 1, n):
            s = s + A[r][c] * dq[c]
        dq[r] = (b[r] - s) / torch.where(ok, A[r][r], one)
        ok = ok & torch.isfinite(dq[r])
    out = []
    for r in range(n):
        v = q0[r] + dt * S[r]
        fb = torch.where(torch.isfinite(v), v, q0[r])
        out.append(torch.where(ok, q0[r] + dq[r], fb))
    return out


def _sqrt_g(h, g):
    # sqrt(g max(h, 0)) with the derivative 0 at h <= 0 (no 0/0 in autograd)
    pos = h > 0
    return torch.where(pos, csqrt(g * torch.where(pos, h, torch.ones_like(h))), torch.zeros_like(h))


def max_inv(Q, hv, p, dx, dy):
    c = _sqrt_g(Q[1], p["g"])
    ix = sdiv(torch.abs(Q[2] * hv) + c, dx)
    iy = sdiv(torch.abs(Q[3] * hv) + c, dy)
    return torch.maximum(ix.max(), iy.max())


def step(Q, hv_dt, n_m, p, dx, dy, bc, wb=True, impl=True, cfl=0.45, cfl_div=6.0, dtmin=1e-7, dtmax=1.0):
    """One SSP-RK2 step from Q with the CFL dt from the aux hinv ``hv_dt``
    (ZoomyAmr.cpp:448-515, 538-731); returns (Q_next, hinv of Q_next, dt)."""
    M = max_inv(Q, hv_dt, p, dx, dy)
    dt = rdiv(cfl, cfl_div * M)
    dt = torch.clamp(dt, max=dtmax, min=dtmin)
    X = Q
    for _ in range(2):
        hv = hinv(X[1], p["eps"])
        qs = explicit_stage(X, dt, p, dx, dy, bc, wb)
        X = implicit(qs, hv, dt, p, n_m) if impl else qs
    Q = 0.5 * Q + 0.5 * X
    return Q, hinv(Q[1], p["eps"]), dt


def run(Q0, aux_hinv0, n_m, steps, p, dx, dy, bc, wb=True, impl=True, cfl=0.45, cfl_div=6.0,
        dtmin=1e-7, dtmax=1.0, checkpoint=False):
    """`steps` SSP-RK2 steps from Q0 (4, ny, nx); returns Q_T and the dts.
    With ``checkpoint`` each step's autograd graph is recomputed during the
    backward pass instead of being kept (torch.utils.checkpoint), so long
    runs fit in memory."""
    Q = Q0
    hv_dt = aux_hinv0
    dts = []
    kw = dict(wb=wb, impl=impl, cfl=cfl, cfl_div=cfl_div, dtmin=dtmin, dtmax=dtmax)

    def one(Q, hv_dt, n_m):
        return step(Q, hv_dt, n_m, p, dx, dy, bc, **kw)

    for n in range(steps):
        if checkpoint:
            from torch.utils.checkpoint import checkpoint as ck
            Q, hv_dt, dt = ck(one, Q, hv_dt, n_m, use_reentrant=False)
        else:
            Q, hv_dt, dt = one(Q, hv_dt, n_m)
        dts.append(dt)
    return Q, dts
