"""The hand-written stage adjoint (zoomy_amrex_b200/csrc/swe_adjoint.H), host build.

The same header is compiled into the sm_100a adjoint kernels; here it runs on
the CPU (tests/adjoint_host.cpp) so that its arithmetic is checked without a
GPU: the flat forward stage against the oracle's SSP-RK2 step, and the
reverse maps against central finite differences of the forward maps.
"""
import ctypes as C
import pathlib
import subprocess

import numpy as np
import pytest

from zoomy_amrex_b200._abi import ZFV_MODEL_SWE2D, make_config

ROOT = pathlib.Path(__file__).resolve().parent.parent
CSRC = ROOT / "zoomy_amrex_b200" / "csrc"
BUILD = ROOT / "tests" / "_build"
PAR = np.array([9.81, 0.0, 0.0, 0.03, 1e-6, 1e-24])


def _host_lib(name, defines=()):
    BUILD.mkdir(exist_ok=True)
    so = BUILD / name
    src = ROOT / "tests" / "adjoint_host.cpp"
    deps = [src, CSRC / "swe_adjoint.H", CSRC / "models" / "zb_portable_math.H"]
    if not so.exists() or any(d.stat().st_mtime > so.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC",
                        *[f"-D{d}" for d in defines],
                        "-I", str(CSRC), "-I", str(CSRC / "amrex_compat"), "-I", str(CSRC / "models"),
                        str(src), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    d, i, p = C.c_double, C.c_int, C.c_void_p
    L.adj_stage_fwd.argtypes = [i, i, d, d, p, p, i, i, p, d, p]
    L.adj_stage_rev.argtypes = [i, i, d, d, p, p, i, i, p, d, p, p, p, p]
    L.adj_face_fwd.argtypes = [i, i, p, p, p]
    L.adj_face_rev.argtypes = [i, i, p, p, p, p]
    return L


@pytest.fixture(scope="module")
def adj():
    return _host_lib("libadjhost.so")


@pytest.fixture(scope="module")
def adj_fwd_branches():
    """The same reverse with every wave-speed max decided from speeds
    recomputed with the forward's operations."""
    return _host_lib("libadjhost_fwdbranch.so", ("ZADJ_FORWARD_BRANCHES",))


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def wet_state(nx, ny, seed, dry=False):
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    b = 0.4 * np.exp(-((X - 0.4) ** 2 + (Y - 0.6) ** 2) / 0.05) + 0.05 * rng.random((ny, nx))
    eta = 1.0 + 0.1 * np.exp(-((X - 0.7) ** 2 + (Y - 0.3) ** 2) / 0.02)
    if dry:
        b = b + 1.2 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    h = np.maximum(eta - b, 0.0)
    hu = h * (0.3 + 0.2 * rng.standard_normal((ny, nx)))
    hv = h * (-0.2 + 0.2 * rng.standard_normal((ny, nx)))
    return np.ascontiguousarray(np.array([b, h, hu, hv]))


class Stage:
    def __init__(self, L, nx, ny, bc, wb, impl, par=PAR):
        self.L, self.nx, self.ny = L, nx, ny
        self.dx, self.dy = 1.0 / nx, 1.0 / ny
        self.bc = np.array(bc, dtype=np.int32)
        self.wb, self.impl = int(wb), int(impl)
        self.par = np.array(par, dtype=np.float64)

    def fwd(self, X, dt, par=None):
        Y = np.zeros_like(X)
        pr = self.par if par is None else np.asarray(par, np.float64)
        self.L.adj_stage_fwd(self.nx, self.ny, self.dx, self.dy, _p(self.bc), _p(pr), self.wb,
                             self.impl, _p(np.ascontiguousarray(X)), dt, _p(Y))
        return Y

    def rev(self, X, dt, lamY):
        lamX = np.zeros_like(X)
        lnm, ldt = C.c_double(0.0), C.c_double(0.0)
        self.L.adj_stage_rev(self.nx, self.ny, self.dx, self.dy, _p(self.bc), _p(self.par), self.wb,
                             self.impl, _p(np.ascontiguousarray(X)), dt,
                             _p(np.ascontiguousarray(lamY)), _p(lamX), C.byref(lnm), C.byref(ldt))
        return lamX, lnm.value, ldt.value


def test_flat_stage_matches_oracle_step(adj, oracle):
    """Two flat stages + Heun reproduce the oracle's SSP-RK2 step."""
    nx, ny = 14, 11
    Q = wet_state(nx, ny, 1)
    for wb in (False, True):
        st = Stage(adj, nx, ny, (1, 0, 1, 1), wb, True)
        cfg = make_config(ZFV_MODEL_SWE2D, nx, ny, (0, 0), (1, 1), spatial_order=2, well_balanced=wb,
                          implicit_source=True, bc=("wall", "extrapolation", "wall", "wall"),
                          params={"n_m": 0.03})
        dt = 2e-3
        Y1 = st.fwd(Q, dt)
        Y2 = st.fwd(Y1, dt)
        ours = 0.5 * Q + 0.5 * Y2
        A = np.zeros((7, ny, nx))
        Qo, _ = oracle.advance(cfg, Q, A, 0.0, dt)
        assert np.abs(ours - Qo).max() <= 1e-13 * max(1.0, np.abs(Qo).max()), wb


@pytest.mark.parametrize("D", [0, 1])
@pytest.mark.parametrize("wb", [0, 1])
def test_face_reverse_vs_fd(adj, D, wb):
    rng = np.random.default_rng(10 + D + 2 * wb)
    worst = 0.0
    for trial in range(200):
        c = np.zeros((4, 4))
        c[:, 0] = rng.uniform(0.0, 0.5, 4)
        c[:, 1] = rng.uniform(0.05, 2.0, 4)
        c[:, 2:] = rng.normal(0, 0.5, (4, 2))
        c = np.ascontiguousarray(c)
        lo = rng.normal(size=11)
        v = rng.normal(size=(4, 4))
        lc = np.zeros((4, 4))
        adj.adj_face_rev(D, wb, _p(PAR), _p(c), _p(lo), _p(lc))
        eps = 1e-6
        op, om = np.zeros(11), np.zeros(11)
        cp = np.ascontiguousarray(c + eps * v)
        cm = np.ascontiguousarray(c - eps * v)
        adj.adj_face_fwd(D, wb, _p(PAR), _p(cp), _p(op))
        adj.adj_face_fwd(D, wb, _p(PAR), _p(cm), _p(om))
        fd = lo @ (op - om) / (2 * eps)
        an = (lc * v).sum()
        err = abs(fd - an) / max(1e-8, abs(fd) + abs(an))
        worst = max(worst, err)
    # random stencils sit at kinks only with probability ~0 at eps = 1e-6
    assert worst < 1e-6, worst


@pytest.mark.parametrize("wb,impl,bc", [(True, True, (1, 1, 1, 1)), (False, True, (0, 1, 1, 0)),
                                        (True, False, (0, 0, 1, 1))])
def test_stage_reverse_vs_fd(adj, wb, impl, bc):
    nx, ny = 13, 9
    st = Stage(adj, nx, ny, bc, wb, impl)
    X = wet_state(nx, ny, 3)
    dt = 1.5e-3
    rng = np.random.default_rng(4)
    lamY = rng.normal(size=X.shape)
    lamX, lnm, ldt = st.rev(X, dt, lamY)
    eps = 1e-6
    for k in range(6):
        V = rng.normal(size=X.shape)
        fd = (lamY * (st.fwd(X + eps * V, dt) - st.fwd(X - eps * V, dt))).sum() / (2 * eps)
        an = (lamX * V).sum()
        assert abs(fd - an) <= 1e-6 * (abs(fd) + abs(an)), (k, fd, an)
    # dt and Manning n
    fd = (lamY * (st.fwd(X, dt + eps * dt) - st.fwd(X, dt - eps * dt))).sum() / (2 * eps * dt)
    assert abs(fd - ldt) <= 1e-6 * (abs(fd) + abs(ldt)), (fd, ldt)
    if impl:
        pp, pm = PAR.copy(), PAR.copy()
        pp[3] += 1e-7; pm[3] -= 1e-7
        fd = (lamY * (st.fwd(X, dt, pp) - st.fwd(X, dt, pm))).sum() / 2e-7
        assert abs(fd - lnm) <= 1e-6 * (abs(fd) + abs(lnm)), (fd, lnm)


def test_stage_reverse_with_dry_cells(adj):
    """Dry islands: the adjoint is the derivative of the branch taken."""
    nx, ny = 16, 12
    st = Stage(adj, nx, ny, (1, 1, 1, 1), True, True)
    X = wet_state(nx, ny, 5, dry=True)
    assert (X[1] == 0).any()
    dt = 1e-3
    rng = np.random.default_rng(6)
    lamY = rng.normal(size=X.shape)
    lamX, _, _ = st.rev(X, dt, lamY)
    assert np.isfinite(lamX).all()
    # directions that keep dry cells dry (perturb wet cells only)
    wet = (X[1] > 0)[None]
    eps = 1e-7
    for k in range(4):
        V = rng.normal(size=X.shape) * wet
        fd = (lamY * (st.fwd(X + eps * V, dt) - st.fwd(X - eps * V, dt))).sum() / (2 * eps)
        an = (lamX * V).sum()
        assert abs(fd - an) <= 1e-5 * (abs(fd) + abs(an)), (k, fd, an)


@pytest.mark.parametrize("wb", [0, 1])
@pytest.mark.parametrize("dry", [False, True])
def test_near_tie_branches_are_the_forwards(adj, adj_fwd_branches, wb, dry):
    """The face reverse forms hinv and the Audusse ratio a few ulps off the
    forward's, and decides the Rusanov max near ties by bracketing the
    forward's speeds. A state whose velocities are constant along x (x-face
    speeds tie to an ulp) and water at rest with ulp-level momenta (every
    speed ties to an ulp) must give the reverse of the build that recomputes
    every speed with the forward's operations, to rounding."""
    nx, ny = 40, 32
    rng = np.random.default_rng(2)
    x = (np.arange(nx) + 0.5) / nx * 10.0
    y = (np.arange(ny) + 0.5) / ny * 10.0
    X, Y = np.meshgrid(x, y)
    b = 0.3 * np.exp(-((X - 4) ** 2 + (Y - 6) ** 2) / 4.0) + 0.02 * rng.random((ny, nx))
    if dry:
        b = b + 1.3 * np.exp(-((X - 5) ** 2 + (Y - 5) ** 2) / 1.0)
    eta = 1.0 + 0.2 * np.exp(-((X - 7) ** 2 + (Y - 3) ** 2) / 2.0)
    h = np.maximum(eta - b, 0.0)
    moving = np.array([b, h, h * (0.2 + 0.05 * np.sin(Y)), h * (-0.1 + 0.05 * np.cos(X))])
    h1 = np.maximum(1.0 - b, 0.0)
    at_rest = np.array([b, h1, 1e-15 * rng.standard_normal((ny, nx)) * h1,
                        1e-15 * rng.standard_normal((ny, nx)) * h1])
    lam = np.random.default_rng(5).standard_normal(moving.shape)
    for Q in (moving, at_rest):
        Q = np.ascontiguousarray(Q)
        st, sf = (Stage(L, nx, ny, (1, 0, 1, 1), wb, True) for L in (adj, adj_fwd_branches))
        for k in range(8):
            ga, _, _ = st.rev(Q, 0.01, lam)
            gb, _, _ = sf.rev(Q, 0.01, lam)
            for r in range(4):
                err = np.abs(ga[r] - gb[r]).max() / np.abs(gb[r]).max()
                assert err <= 1e-14, (k, r, err)
            Q = np.ascontiguousarray(st.fwd(Q, 0.01))
