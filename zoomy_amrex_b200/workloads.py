"""Seeded synthetic inputs for the benchmark workloads.

The reference quotes no public dataset for this path; these generators give
the shapes and value distributions of its scenarios:

* ``bump_workload_fields`` / ``bump_workload_config``: the 2-D wet/dry hump
  over 16 Gaussian bumps (the benchmark's headline level);

* ``bump_field``: Gaussian-bump bathymetry (centres uniform in the box,
  amplitudes U(0.2, 1.5) m, widths U(2, 10) m) under still water at eta0 plus
  an optional Gaussian hump;
* ``sme_workload_fields`` / ``sme_workload_config``: the shallow-moment
  level-2 scenario on [0,50]^2 m: the same bump generator, the same surface
  (1 m plus a 0.3 m hump), fluid at rest in the mean with seeded moments
  h alpha_j, h beta_j = h U(-0.05, 0.05) m/s;
* ``dam_break_ensemble``: independent shallow-water boxes of uneven size
  (sides log-uniform per axis), each with its own bumps and a dam-break ratio
  drawn U(1.2, 3.0), as a list of (config, Q0, aux0) for the FP32 batch engine.
"""
from __future__ import annotations

import numpy as np

from ._abi import ZFV_MODEL_SME2D_L2, ZFV_MODEL_SWE2D, ZFV_PREC_FP32, ZFV_PREC_FP64, make_config

BUMP_SEED = 2026
BUMP_DOMAIN = 100.0


def _bumps(rng, n_bumps, x_extent, y_extent, width=(2.0, 10.0)):
    cx, cy = rng.uniform(0, x_extent, n_bumps), rng.uniform(0, y_extent, n_bumps)
    amp, wid = rng.uniform(0.2, 1.5, n_bumps), rng.uniform(width[0], width[1], n_bumps)
    return cx, cy, amp, wid


def _bed(xs, ys, bumps):
    cx, cy, amp, wid = bumps
    b = np.zeros((len(ys), len(xs)))
    for k in range(len(cx)):
        gx = np.exp(-((xs - cx[k]) ** 2) / (2 * wid[k] ** 2))
        gy = np.exp(-((ys - cy[k]) ** 2) / (2 * wid[k] ** 2))
        b += amp[k] * np.outer(gy, gx)
    return b


def dam_break_ensemble(n_inst: int = 256, seed: int = 4, side_range=(32, 512), dx: float = 0.1,
                       n_bumps: int = 6, precision: int = ZFV_PREC_FP32, max_step: int = -1,
                       time_end: float = 1.0e30, n_m: float = 0.03):
    """``n_inst`` dam breaks over bumps on boxes of nx x ny cells of size dx.

    Per instance: nx, ny = round(exp(U(log lo, log hi))); bumps with centres in
    the box, amplitudes U(0.2, 1.5) m and widths U(0.05, 0.2) x the shorter
    box side; eta = r on the left half and 1 m on the right half with
    r ~ U(1.2, 3.0); h = max(eta - b, 0); walls; Manning n; order 2,
    well-balanced, point-implicit source.
    """
    rng = np.random.default_rng(seed)
    lo, hi = np.log(side_range[0]), np.log(side_range[1])
    out = []
    for _ in range(n_inst):
        nx, ny = (int(round(np.exp(v))) for v in rng.uniform(lo, hi, 2))
        ratio = rng.uniform(1.2, 3.0)
        Lx, Ly = nx * dx, ny * dx
        s = min(Lx, Ly)
        bumps = _bumps(rng, n_bumps, Lx, Ly, width=(0.05 * s, 0.2 * s))
        xs = (np.arange(nx) + 0.5) * dx
        ys = (np.arange(ny) + 0.5) * dx
        b = _bed(xs, ys, bumps)
        eta = np.where(xs < 0.5 * Lx, ratio, 1.0)[None, :]
        Q0 = np.zeros((4, ny, nx))
        Q0[0] = b
        Q0[1] = np.maximum(eta - b, 0.0)
        aux0 = np.zeros((7, ny, nx))
        cfg = make_config(ZFV_MODEL_SWE2D, nx, ny, (0.0, 0.0), (Lx, Ly), spatial_order=2,
                          well_balanced=True, implicit_source=True, cfl=0.45, dtmin=1e-7,
                          dtmax=1.0, time_end=time_end, max_step=max_step, bc=("wall",) * 4,
                          params={"n_m": n_m}, precision=precision)
        out.append((cfg, Q0, aux0))
    return out


def bump_workload_fields(n: int, seed: int = BUMP_SEED, rows: slice | None = None):
    """Wet/dry hump over 16 seeded Gaussian bumps on n x n cells over
    [0,100]^2 m: bumps with centres U(domain), amplitudes U(0.2,1.5) m,
    widths U(2,10) m; eta = 1 m plus a 0.3 m Gaussian hump; h = max(eta - b, 0).
    ``rows`` selects a strip of rows of the same grid. Returns Q0 (4, ny, n),
    aux0 (7, ny, n) (aux row 1 carries the init_solution dam pattern)."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0, BUMP_DOMAIN, 16), rng.uniform(0, BUMP_DOMAIN, 16)
    amp, wid = rng.uniform(0.2, 1.5, 16), rng.uniform(2.0, 10.0, 16)
    hx, hy, hw = rng.uniform(0, BUMP_DOMAIN), rng.uniform(0, BUMP_DOMAIN), rng.uniform(2.0, 10.0)
    dx = BUMP_DOMAIN / n
    x = (np.arange(n) + 0.5) * dx
    ys = x if rows is None else x[rows]
    ny = len(ys)
    b = np.zeros((ny, n))
    for k in range(16):
        gx = np.exp(-((x - cx[k]) ** 2) / (2 * wid[k] ** 2))
        gy = np.exp(-((ys - cy[k]) ** 2) / (2 * wid[k] ** 2))
        b += amp[k] * np.outer(gy, gx)
    eta = 1.0 + 0.3 * np.outer(np.exp(-((ys - hy) ** 2) / (2 * hw ** 2)),
                               np.exp(-((x - hx) ** 2) / (2 * hw ** 2)))
    h = np.maximum(eta - b, 0.0)
    Q0 = np.zeros((4, ny, n))
    Q0[0], Q0[1] = b, h
    aux0 = np.zeros((7, ny, n))
    aux0[1] = np.where(x < 0.5 * BUMP_DOMAIN, 2.0, 1.0)[None, :]   # init_solution on aux
    return Q0, aux0


def bump_workload_config(n: int, ny: int | None = None, y_extent: float | None = None):
    """The matching configuration: SWE2D, order 2, WB, point-implicit Manning n = 0.03, walls,
    cfl 0.45, no stop time (callers set max_step / time_end)."""
    ny = n if ny is None else ny
    ye = BUMP_DOMAIN if y_extent is None else y_extent
    return make_config(ZFV_MODEL_SWE2D, n, ny, (0.0, 0.0), (BUMP_DOMAIN, ye), spatial_order=2,
                       well_balanced=True, implicit_source=True, clamp_positivity=False,
                       cfl=0.45, dtmin=1e-7, dtmax=1.0, time_end=1e30, max_step=-1,
                       bc=("wall",) * 4, params={"n_m": 0.03, "h_floor": 1e-6, "eps": 1e-24})


def dam_break_level(n: int, seed: int = 2029, L: float = 100.0, n_bumps: int = 16):
    """One n x n dam break over Gaussian bumps on [0, L]^2 (the AMR
    benchmark's base level): eta = r ~ U(1.2, 3.0) left of x = 0.4 L and 1 m
    to the right, bumps with amplitudes U(0.2, 1.5) m and widths U(2, 10) m
    scaled to L = 100, walls, Manning n = 0.03. Returns (cfg, Q0)."""
    rng = np.random.default_rng(seed)
    ratio = rng.uniform(1.2, 3.0)
    bumps = _bumps(rng, n_bumps, L, L, width=(0.02 * L, 0.1 * L))
    xs = (np.arange(n) + 0.5) * (L / n)
    b = _bed(xs, xs, bumps)
    eta = np.where(xs < 0.4 * L, ratio, 1.0)[None, :]
    Q0 = np.zeros((4, n, n))
    Q0[0] = b
    Q0[1] = np.maximum(eta - b, 0.0)
    cfg = make_config(ZFV_MODEL_SWE2D, n, n, (0.0, 0.0), (L, L), spatial_order=2, well_balanced=True,
                      implicit_source=True, cfl=0.45, dtmin=1e-7, dtmax=1.0, time_end=1.0e30, max_step=-1,
                      bc=("wall",) * 4, params={"n_m": 0.03})
    return cfg, Q0


def fp64_twin(cfg):
    """The same configuration in the FP64 plain form."""
    import ctypes as C
    c = type(cfg)()
    C.memmove(C.byref(c), C.byref(cfg), C.sizeof(cfg))
    c.precision = ZFV_PREC_FP64
    return c


SME_SEED = 2030
SME_DOMAIN = 50.0


def sme_workload_fields(n: int, seed: int = SME_SEED, rows: slice | None = None):
    """Shallow-moment level-2 state on n x n cells over [0,50]^2 m: 16 seeded
    Gaussian bumps (centres U(domain), amplitudes U(0.2,1.5) m, widths
    U(2,10) m), eta = 1 m plus a 0.3 m Gaussian hump, h = max(eta - b, 0),
    zero mean velocity, moments h alpha_1, h alpha_2, h beta_1, h beta_2 =
    h U(-0.05, 0.05) m/s (seeded per cell). ``rows`` selects a strip of rows
    of the same grid (the moments of those rows are the full grid's). Returns
    Q0 (8, ny, n), aux0 (1, ny, n)."""
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0, SME_DOMAIN, 16), rng.uniform(0, SME_DOMAIN, 16)
    amp, wid = rng.uniform(0.2, 1.5, 16), rng.uniform(2.0, 10.0, 16)
    hx, hy, hw = rng.uniform(0, SME_DOMAIN), rng.uniform(0, SME_DOMAIN), rng.uniform(2.0, 10.0)
    dx = SME_DOMAIN / n
    x = (np.arange(n) + 0.5) * dx
    sel = slice(0, n) if rows is None else rows
    ys = x[sel]
    ny = len(ys)
    b = np.zeros((ny, n))
    for k in range(16):
        gx = np.exp(-((x - cx[k]) ** 2) / (2 * wid[k] ** 2))
        gy = np.exp(-((ys - cy[k]) ** 2) / (2 * wid[k] ** 2))
        b += amp[k] * np.outer(gy, gx)
    eta = 1.0 + 0.3 * np.outer(np.exp(-((ys - hy) ** 2) / (2 * hw ** 2)),
                               np.exp(-((x - hx) ** 2) / (2 * hw ** 2)))
    h = np.maximum(eta - b, 0.0)
    Q0 = np.zeros((8, ny, n))
    Q0[0], Q0[1] = b, h
    # per-cell moment draws of the whole grid, row-major, so that a strip of
    # rows sees the same values as the full grid
    mrng = np.random.default_rng(seed + 1)
    start = 0 if rows is None else (rows.start or 0)
    mrng.uniform(-0.05, 0.05, (start, 4, n)) if start else None
    m = mrng.uniform(-0.05, 0.05, (ny, 4, n))
    for k in range(4):
        Q0[4 + k] = h * m[:, k, :]
    return Q0, np.zeros((1, ny, n))


def sme_workload_config(n: int, ny: int | None = None, y_extent: float | None = None,
                        well_balanced: bool = True):
    """The matching configuration: SME level 2 (2-D), order 2, point-implicit
    Navier-slip friction (viscosity 1e-3, slip length 0.1), walls, cfl 0.45,
    no stop time (callers set max_step / time_end)."""
    ny = n if ny is None else ny
    ye = SME_DOMAIN if y_extent is None else y_extent
    return make_config(ZFV_MODEL_SME2D_L2, n, ny, (0.0, 0.0), (SME_DOMAIN, ye), spatial_order=2,
                       well_balanced=well_balanced, implicit_source=True, cfl=0.45, dtmin=1e-7, dtmax=1.0,
                       time_end=1e30, max_step=-1, bc=("wall",) * 4,
                       params={"nu": 1.0e-3, "lambda": 0.1, "eps": 1e-24})
