"""The shallow-moment model header (zoomy_amrex_b200/csrc/models/sme.H), host build.

sme.H codes the projected system from tabulated Legendre coefficients; here
it is compared, at random states, with an independent symbolic derivation
from the velocity profiles (tests/sme_sympy.py): fluxes, the non-conservative
products, the friction source and its Jacobians, and the Gershgorin bound of
the quasi-linear matrix (which must also bound its eigenvalues). With every
moment zero the flux and the non-conservative products reduce bit for bit to
the shallow-water model's.
"""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
CSRC = ROOT / "zoomy_amrex_b200" / "csrc"
BUILD = ROOT / "tests" / "_build"
PAR = np.array([9.81, 0.0, 0.0, 1.0e-3, 0.1, 1.0e-24])      # g, ex, ey, nu, lambda, eps


@pytest.fixture(scope="module")
def host():
    BUILD.mkdir(exist_ok=True)
    so = BUILD / "libmodelhost.so"
    src = ROOT / "tests" / "model_host.cpp"
    deps = [src, CSRC / "models" / "sme.H", CSRC / "models" / "swe.H"]
    if not so.exists() or any(d.stat().st_mtime > so.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                        "-I", str(CSRC), "-I", str(CSRC / "amrex_compat"), "-I", str(CSRC / "models"),
                        str(src), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    p = C.c_void_p
    L.model_eval.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, p, p, p, p]
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def ev(L, model, dim, level, what, D, q, dq=None, par=PAR, size=None):
    n = len(q)
    out = np.zeros(size or (2 * n * n + 2 * n))
    dq = np.zeros(n) if dq is None else np.ascontiguousarray(dq, dtype=np.float64)
    rc = L.model_eval(model, dim, level, what, D, _p(np.ascontiguousarray(q, dtype=np.float64)), _p(dq),
                      _p(np.ascontiguousarray(par, dtype=np.float64)), _p(out))
    assert rc == 0
    return out


def rand_state(rng, dim, level, scale=0.3):
    n = 2 + dim * (1 + level)
    q = np.zeros(n)
    q[0] = rng.uniform(0.0, 1.0)                 # bed
    q[1] = rng.uniform(0.3, 2.0)                 # depth
    q[2:] = q[1] * rng.uniform(-scale, scale, n - 2)
    return q


CASES = [(2, 1), (2, 2), (2, 3), (1, 2), (1, 3)]


@pytest.mark.parametrize("dim,level", CASES)
def test_flux_and_products_match_symbolic_derivation(host, dim, level):
    from sme_sympy import numeric
    f = numeric(level, dim)
    par = tuple(PAR[:5])
    rng = np.random.default_rng(10 * dim + level)
    for _ in range(20):
        q = rand_state(rng, dim, level)
        dq = rng.standard_normal(len(q))
        for D in range(dim):
            F = ev(host, 1, dim, level, 0, D, q)[:len(q)]
            Fs = np.asarray(f[f"F{D}"](q, par), dtype=float).ravel()
            np.testing.assert_allclose(F, Fs, rtol=1e-12, atol=1e-14)
            # moment rows of B_D(q) dq (the bed product sits in the numerics)
            Bq = ev(host, 1, dim, level, 1, D, q, dq)[:len(q)]
            Bs = np.asarray(f[f"B{D}"](q, par), dtype=float) @ dq
            mom = np.arange(2 + dim, len(q))
            np.testing.assert_allclose(Bq[mom], Bs[mom], rtol=1e-12, atol=1e-14)
            # the bed column of B_D is g h on the mean momentum along D
            assert np.allclose(np.asarray(f[f"B{D}"](q, par), dtype=float)[2 + D, 0], PAR[0] * q[1])


@pytest.mark.parametrize("dim,level", CASES)
def test_source_and_jacobians_match_symbolic_derivation(host, dim, level):
    from sme_sympy import numeric
    f = numeric(level, dim)
    rng = np.random.default_rng(100 + 10 * dim + level)
    for _ in range(20):
        q = rand_state(rng, dim, level)
        par = np.array([9.81, rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1), rng.uniform(1e-4, 1e-2),
                        rng.uniform(0.01, 1.0), 1e-24])
        ps = tuple(par[:5])
        n = len(q)
        S = ev(host, 1, dim, level, 2, 0, q, par=par)[:n]
        np.testing.assert_allclose(S, np.asarray(f["S"](q, ps), float).ravel(), rtol=1e-12, atol=1e-15)
        J = ev(host, 1, dim, level, 3, 0, q, par=par)[:n * n].reshape(n, n)
        np.testing.assert_allclose(J, np.asarray(f["dSdq"](q, ps), float), rtol=1e-12, atol=1e-15)
        Ja = ev(host, 1, dim, level, 4, 0, q, par=par)[:n]
        np.testing.assert_allclose(Ja, np.asarray(f["dSdhinv"](q, ps), float).ravel(), rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("dim,level", CASES)
def test_gershgorin_bound(host, dim, level):
    """local_max_abs_eigenvalue is the largest absolute row sum of the
    quasi-linear matrix dF/dQ + B over the evolved rows and columns, so it
    bounds every eigenvalue of that matrix."""
    from sme_sympy import numeric
    f = numeric(level, dim)
    par = tuple(PAR[:5])
    rng = np.random.default_rng(200 + 10 * dim + level)
    for _ in range(30):
        q = rand_state(rng, dim, level, scale=0.6)
        for D in range(dim):
            A = np.asarray(f[f"A{D}"](q, par), dtype=float)[1:, 1:]
            want = np.abs(A).sum(axis=1).max()
            got = ev(host, 1, dim, level, 5, D, q)[0]
            np.testing.assert_allclose(got, want, rtol=1e-12)
            assert got >= np.abs(np.linalg.eigvals(A)).max() * (1 - 1e-12)


@pytest.mark.parametrize("dim", [1, 2])
def test_zero_moments_reduce_to_shallow_water_bitwise(host, dim):
    """Every moment zero: the SME flux and the path products are the
    shallow-water model's bit for bit, and the moment rows stay zero."""
    rng = np.random.default_rng(7 + dim)
    swe_par = np.array([9.81, 0.0, 0.0, 0.0, 1e-6, 1e-24])
    for level in (1, 2, 3):
        n = 2 + dim * (1 + level)
        for _ in range(20):
            qs = rand_state(rng, dim, 0)
            qr = rand_state(rng, dim, 0)
            q = np.zeros(n); q[:len(qs)] = qs
            r = np.zeros(n); r[:len(qr)] = qr
            for D in range(dim):
                F = ev(host, 1, dim, level, 0, D, q)[:n]
                Fw = ev(host, 0, dim, 0, 0, D, qs, par=swe_par)[:len(qs)]
                assert np.array_equal(F[:len(qs)], Fw) and not F[len(qs):].any()
                B = ev(host, 1, dim, level, 8, D, q, r)[:n]
                Dw = ev(host, 0, dim, 0, 7, D, qs, qr, par=swe_par)[:2 * len(qs)]
                # SWE's D+ + D- = B~ dq (the Rusanov parts cancel exactly only
                # up to rounding, so compare the bed product directly)
                bed = 9.81 * (0.5 * (qs[1] + qr[1])) * (qr[0] - qs[0])
                assert B[2 + D] == bed and not B[len(qs):].any()
                assert np.isfinite(Dw).all()


def test_wall_reflects_the_whole_velocity_profile(host):
    """A wall ghost mirrors the velocity profile u(z): the normal mean
    momentum and every normal moment flip sign, the transverse ones are kept."""
    rng = np.random.default_rng(3)
    for dim, level in CASES:
        q = rand_state(rng, dim, level)
        for D in range(dim):
            g = ev(host, 1, dim, level, 9, D, q)[:len(q)]
            want = q.copy()
            want[2 + D] *= -1
            first = 2 + dim + D * level
            want[first:first + level] *= -1
            assert np.array_equal(g, want)


@pytest.mark.parametrize("dim,level", CASES)
def test_block_point_implicit_step_solves_the_linear_system(host, dim, level):
    """zb_implicit_increment (the FP32 kernels' structured solve) returns
    the solution of (I - dt J) dq = dt S with J = dS/dQ at fixed hinv
    (make_rhs.H:429-509's system), J and S from the symbolic derivation."""
    from sme_sympy import numeric
    f = numeric(level, dim)
    rng = np.random.default_rng(300 + 10 * dim + level)
    for _ in range(20):
        q = rand_state(rng, dim, level)
        par = np.array([9.81, rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1), rng.uniform(1e-4, 1e-2),
                        rng.uniform(0.01, 1.0), 1e-24])
        dt = float(rng.uniform(1e-4, 5e-2))
        n = len(q)
        d = np.zeros(n); d[0] = dt
        got = ev(host, 1, dim, level, 10, 0, q, d, par=par)[:n]
        ps = tuple(par[:5])
        J = np.asarray(f["dSdq"](q, ps), float)
        S = np.asarray(f["S"](q, ps), float).ravel()
        want = np.linalg.solve(np.eye(n) - dt * J, dt * S)
        # the bed and depth rows have no source: their increment is exactly zero
        assert got[0] == 0.0 and got[1] == 0.0
        np.testing.assert_allclose(got[2:], want[2:], rtol=1e-11, atol=1e-15)


@pytest.mark.parametrize("dim,level", CASES)
def test_implicit_system_block_structure(host, dim, level):
    """The structure the FP64 kernels' block elimination relies on
    (zb_implicit_blocks): the source and its Jacobian vanish in rows b and h,
    column b is zero, and no entry couples the blocks {mean momentum and
    moments of direction d}. Checked exactly on the header's Jacobian and
    against the symbolic derivation's sparsity."""
    from sme_sympy import numeric
    f = numeric(level, dim)
    n = 2 + dim * (1 + level)
    block = np.full(n, -1)
    for d in range(dim):
        block[2 + d] = d
        block[2 + dim + d * level: 2 + dim + (d + 1) * level] = d
    rng = np.random.default_rng(400 + 10 * dim + level)
    for _ in range(20):
        q = rand_state(rng, dim, level)
        par = np.array([9.81, rng.uniform(-0.1, 0.1), rng.uniform(-0.1, 0.1), rng.uniform(1e-4, 1e-2),
                        rng.uniform(0.01, 1.0), 1e-24])
        S = ev(host, 1, dim, level, 2, 0, q, par=par)[:n]
        J = ev(host, 1, dim, level, 3, 0, q, par=par)[:n * n].reshape(n, n)
        Js = np.asarray(f["dSdq"](q, tuple(par[:5])), float)
        assert S[0] == 0.0 and S[1] == 0.0
        assert not J[0].any() and not J[1].any() and not J[:, 0].any()
        for r in range(2, n):
            for c in range(2, n):
                if block[r] != block[c]:
                    assert J[r, c] == 0.0 and Js[r, c] == 0.0, (r, c)
