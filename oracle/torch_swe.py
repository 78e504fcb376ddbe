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


def hinv(h, eps):
    x0 = (h * h) * (h * h)
    return SQRT2 * h / torch.sqrt(x0 + torch.where(x0 < eps, torch.full_like(x0, eps), x0))


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
        rhs = Fx / dx + Fy / dy
        if wb and n == 1:
            rhs = rhs + 0.5 * p["g"] * (hLx[:, 1:] * hLx[:, 1:] - hRx[:, :-1] * hRx[:, :-1]) / dx
        if wb and n == 2:
            rhs = rhs + 0.5 * p["g"] * (hLy[1:, :] * hLy[1:, :] - hRy[:-1, :] * hRy[:-1, :]) / dy
        rows.append(X[n + 1] + dt * rhs)
    return torch.stack(rows)


def inv_cbrt(m):
    return m ** (-1.0 / 3.0)


def implicit(qs, hv, dt, p, n_m):
    g, hf = p["g"], p["h_floor"]
    h, mx, my = qs[1], qs[2], qs[3]
    m = torch.where(h < hf, torch.full_like(h, hf), h)
    k = g * n_m * n_m * inv_cbrt(m)
    ux, uy = mx * hv, my * hv
    sp2 = ux * ux + uy * uy
    pos = sp2 > 0
    sp = torch.where(pos, torch.sqrt(torch.where(pos, sp2, torch.ones_like(sp2))), torch.zeros_like(sp2))
    S0 = g * p["ex"] * h - k * ux * sp
    S1 = g * p["ey"] * h - k * uy * sp
    rsp = torch.where(pos, 1.0 / torch.where(pos, sp, torch.ones_like(sp)), torch.zeros_like(sp))
    dsx, dsy = ux * hv * rsp, uy * hv * rsp
    J00 = -k * (hv * sp + ux * dsx)
    J01 = -k * (ux * dsy)
    J10 = -k * (uy * dsx)
    J11 = -k * (hv * sp + uy * dsy)
    a, b = 1 - dt * J00, -dt * J01
    c, d = -dt * J10, 1 - dt * J11
    det = a * d - b * c
    r0, r1 = dt * S0, dt * S1
    dq0 = (r0 * d - b * r1) / det
    dq1 = (a * r1 - c * r0) / det
    return torch.stack([qs[0], qs[1], mx + dq0, my + dq1])


def _sqrt_g(h, g):
    # sqrt(g max(h, 0)) with the derivative 0 at h <= 0 (no 0/0 in autograd)
    pos = h > 0
    return torch.where(pos, torch.sqrt(g * torch.where(pos, h, torch.ones_like(h))), torch.zeros_like(h))


def max_inv(Q, hv, p, dx, dy):
    c = _sqrt_g(Q[1], p["g"])
    ix = (torch.abs(Q[2] * hv) + c) / dx
    iy = (torch.abs(Q[3] * hv) + c) / dy
    return torch.maximum(ix.max(), iy.max())


def run(Q0, aux_hinv0, n_m, steps, p, dx, dy, bc, wb=True, impl=True, cfl=0.45, cfl_div=6.0,
        dtmin=1e-7, dtmax=1.0):
    """`steps` SSP-RK2 steps from Q0 (4, ny, nx); returns Q_T and the dts."""
    Q = Q0
    hv_dt = aux_hinv0
    dts = []
    for n in range(steps):
        M = max_inv(Q, hv_dt, p, dx, dy)
        dt = cfl / (cfl_div * M)
        dt = torch.clamp(dt, max=dtmax, min=dtmin)
        dts.append(dt)
        X = Q
        for _ in range(2):
            hv = hinv(X[1], p["eps"])
            qs = explicit_stage(X, dt, p, dx, dy, bc, wb)
            X = implicit(qs, hv, dt, p, n_m) if impl else qs
        Q = 0.5 * Q + 0.5 * X
        hv_dt = hinv(Q[1], p["eps"])
    return Q, dts
