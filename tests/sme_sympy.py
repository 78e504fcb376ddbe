"""Symbolic derivation of the shallow-moment equations (test infrastructure).

An independent route to the system that zoomy_amrex_b200/csrc/models/sme.H
hand-codes from coefficient tables: here every term is obtained by
integrating the assumed velocity profiles over the scaled vertical
coordinate zeta in [0, 1] with sympy, following the Galerkin projection of
Kowalski & Torrilhon (Commun. Comput. Phys. 25, 2019):

  u(zeta) = u_m + sum_j alpha_j phi_j(zeta),  v(zeta) = v_m + sum_j beta_j phi_j(zeta),
  phi_j(zeta) = (1/j!) d^j/dzeta^j (zeta - zeta^2)^j,

  mass:               d_t h + d_x(h u_m) + d_y(h v_m) = 0
  momentum / moments: (2i+1) int_0^1 phi_i [ d_t(h u) + d_x(h u^2 + g h^2/2) + d_y(h u v)
                         + d_zeta(h u omega) + g h d_x b - d_zeta(sigma_xz) ] dzeta = 0
  with h omega(zeta) = -sum_j (d_x(h alpha_j) + d_y(h beta_j)) int_0^zeta phi_j,
  sigma_xz = (nu/h) d_zeta u, sigma_xz(0) = (nu/lambda) u(0), sigma_xz(1) = 0.

The conserved variables are Q = [b, h, hu, hv, h alpha_1.., h beta_1..]
(2-D) or [b, h, hu, h alpha_1..] (1-D); the quasi-linear form is
d_t Q + d_x F(Q) + d_y G(Q) + B_x(Q) d_x Q + B_y(Q) d_y Q = S(Q).
"""
from __future__ import annotations

from functools import lru_cache

import sympy as sp

ZETA = sp.Symbol("zeta")


def phi(j: int):
    return sp.expand(sp.diff((ZETA - ZETA ** 2) ** j, ZETA, j) / sp.factorial(j))


def big_phi(j: int):
    """int_0^zeta phi_j."""
    return sp.integrate(phi(j), (ZETA, 0, ZETA))


def _int(e):
    return sp.integrate(sp.expand(e), (ZETA, 0, 1))


@lru_cache(maxsize=None)
def derive(level: int, dim: int = 2):
    """Symbols and the system's terms. Returns a dict with
    q (list of conserved symbols, bed first), hinv (symbol standing for 1/h in
    the source), F[d] (flux along d), B[d] (n x n non-conservative matrix
    along d), S (source in terms of q and hinv), params (g, ex, ey, nu, lam)."""
    b, h, qu, qv = sp.symbols("b h qu qv")
    g, ex, ey, nu, lam, hinv = sp.symbols("g ex ey nu lam hinv")
    a = list(sp.symbols(f"a1:{level + 1}")) if level else []
    be = list(sp.symbols(f"be1:{level + 1}")) if (level and dim == 2) else []
    if dim == 2:
        q = [b, h, qu, qv] + a + be
    else:
        q = [b, h, qu] + a
    n = len(q)
    u = qu / h + sum(a[j - 1] / h * phi(j) for j in range(1, level + 1))
    v = (qv / h + sum(be[j - 1] / h * phi(j) for j in range(1, level + 1))) if dim == 2 else 0
    # row index of each equation: 0 bed, 1 mass, then the projections of the
    # x- and y-momentum equations onto phi_0 (mean) .. phi_L
    rows_x = [2] + [2 + dim + j - 1 for j in range(1, level + 1)]
    rows_y = ([3] + [4 + level + j - 1 for j in range(1, level + 1)]) if dim == 2 else []
    cols_ax = [2 + dim + j - 1 for j in range(1, level + 1)]               # h alpha_j columns
    cols_by = [4 + level + j - 1 for j in range(1, level + 1)] if dim == 2 else []

    F = [sp.zeros(n, 1) for _ in range(dim)]
    Bm = [sp.zeros(n, n) for _ in range(dim)]
    S = sp.zeros(n, 1)
    F[0][1] = qu
    if dim == 2:
        F[1][1] = qv
    for comp, rows in ((u, rows_x), (v, rows_y)):
        if not rows:
            continue
        is_x = comp is u
        for i, r in enumerate(rows):
            c = 2 * i + 1
            wgt = phi(i)
            F[0][r] = sp.simplify(c * h * _int(wgt * comp * u) + (g * h ** 2 / 2 if (i == 0 and is_x) else 0))
            if dim == 2:
                F[1][r] = sp.simplify(c * h * _int(wgt * comp * v) + (g * h ** 2 / 2 if (i == 0 and not is_x) else 0))
            # vertical coupling: (2i+1) int phi_i d_zeta(h comp omega)
            #   = (2i+1) sum_j d(h gamma_j) int phi_i' comp Phi_j
            for j in range(1, level + 1):
                coef = sp.simplify(c * _int(sp.diff(wgt, ZETA) * comp * big_phi(j)))
                Bm[0][r, cols_ax[j - 1]] += coef
                if dim == 2:
                    Bm[1][r, cols_by[j - 1]] += coef
            # friction: (2i+1) [ -phi_i(0) sigma(0) - int phi_i' sigma ], sigma = (nu/h) d_zeta comp
            comp_h = comp.subs(h, 1 / hinv)
            sig0 = nu / lam * comp_h.subs(ZETA, 0)
            S[r] = sp.simplify(c * (-wgt.subs(ZETA, 0) * sig0
                                    - nu * hinv * _int(sp.diff(wgt, ZETA) * sp.diff(comp_h, ZETA))))
        # bed and gravity along the slope (mean momentum rows only)
        Bm[0 if is_x else 1][rows[0], 0] += g * h
        S[rows[0]] += g * (ex if is_x else ey) * h
    return dict(q=q, hinv=hinv, F=F, B=Bm, S=S, params=(g, ex, ey, nu, lam), n=n)


@lru_cache(maxsize=None)
def numeric(level: int, dim: int = 2):
    """Lambdified terms: f(q, params) -> flux_d / B_d / S / dS/dq (hinv fixed)
    / quasi-linear matrix dF_d/dq + B_d, all with hinv = 1/h."""
    d = derive(level, dim)
    q, hv, par = d["q"], d["hinv"], d["params"]
    h = q[1]
    out = {}
    args = (q, par)
    for k in range(dim):
        out[f"F{k}"] = sp.lambdify(args, d["F"][k], "numpy")
        out[f"B{k}"] = sp.lambdify(args, d["B"][k], "numpy")
        A = d["F"][k].jacobian(sp.Matrix(q)) + d["B"][k]
        out[f"A{k}"] = sp.lambdify(args, A, "numpy")
    S1 = d["S"].subs(hv, 1 / h)
    out["S"] = sp.lambdify(args, S1, "numpy")
    JS = d["S"].jacobian(sp.Matrix(q)).subs(hv, 1 / h)
    out["dSdq"] = sp.lambdify(args, JS, "numpy")
    JA = sp.diff(d["S"], hv).subs(hv, 1 / h)
    out["dSdhinv"] = sp.lambdify(args, JA, "numpy")
    out["n"] = d["n"]
    return out
