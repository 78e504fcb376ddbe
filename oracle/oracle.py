"""ctypes front end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Two builds share one API:
  * ``liboracle.so``       — the C++ restatement of Source/make_rhs.H and the
                             single-level ZoomyAmr driver (oracle/fv_oracle.H);
  * ``_ref/libzoomyref.so`` — the same driver with the per-cell work done by the
                             reference's own Source/make_rhs.H (built by
                             ``make -C oracle ref REF_SRC=<reference tree>/Source``).

Only tests, the smoke check and the benchmark's CPU baseline use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

from zoomy_amrex_b200._abi import MODELS, zfv_config

HERE = pathlib.Path(__file__).resolve().parent
LIB_ORACLE = HERE / "liboracle.so"
LIB_REF = HERE / "_ref" / "libzoomyref.so"

_D = C.POINTER(C.c_double)
_libs: dict = {}


def build(ref: bool | None = None) -> None:
    """Compile the oracle, and the reference build when the environment variable
    REF_SRC names the reference's Source directory (holding make_rhs.H)."""
    import subprocess
    targets = ["all"]
    if ref is None:
        ref = bool(os.environ.get("REF_SRC")) and pathlib.Path(os.environ["REF_SRC"], "make_rhs.H").exists()
    if ref:
        if not os.environ.get("REF_SRC"):
            raise RuntimeError("building the reference kernels needs REF_SRC=<reference tree>/Source")
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE)] + targets, check=True)


def _load(kind: str):
    if kind in _libs:
        return _libs[kind]
    path, prefix = (LIB_ORACLE, "oracle_") if kind == "oracle" else (LIB_REF, "ref_")
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built (make -C {HERE} {'all' if kind == 'oracle' else 'ref'})")
    lib = C.CDLL(str(path))
    cfgp = C.POINTER(zfv_config)
    f = getattr(lib, prefix + "run")
    f.argtypes = [cfgp, _D, _D, C.c_int, C.c_int, _D, C.c_int, C.POINTER(C.c_int64), _D,
                  C.POINTER(C.c_int)]
    f = getattr(lib, prefix + "fill_ghosts")
    f.argtypes = [cfgp, _D, _D, C.c_double, _D, _D]
    f = getattr(lib, prefix + "rhs")
    f.argtypes = [cfgp, _D, _D, C.c_double, C.c_int, _D]
    f = getattr(lib, prefix + "compute_dt")
    f.argtypes = [cfgp, _D, _D, _D, _D]
    f = getattr(lib, prefix + "update_state")
    f.argtypes = [cfgp, _D, _D, C.c_double]
    f = getattr(lib, prefix + "advance")
    f.argtypes = [cfgp, _D, _D, C.c_double, C.c_double, C.c_int]
    getattr(lib, prefix + "set_threads").argtypes = [C.c_int]
    if kind == "oracle":
        lib.oracle_init_solution.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _D]
        lib.oracle_amr2_run.argtypes = [cfgp, _D, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_double, C.c_int, _D,
                                        _D]
    _libs[kind] = (lib, prefix)
    return _libs[kind]


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _shapes(cfg: zfv_config):
    m = MODELS[cfg.model]
    return (m["n_q"], cfg.ny, cfg.nx), (m["n_aux"], cfg.ny, cfg.nx)


class Oracle:
    """One CPU implementation (``kind`` = "oracle" or "ref")."""

    def __init__(self, kind: str = "oracle", threads: int | None = None):
        self.kind = kind
        self.lib, self.prefix = _load(kind)
        if threads:
            self._fn("set_threads")(int(threads))

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def max_threads(self) -> int:
        return int(self._fn("max_threads")())

    def init_solution(self, cfg: zfv_config):
        """Default state and aux as init_solution writes them (dam break in x)."""
        lib, _ = _load("oracle")
        qs, as_ = _shapes(cfg)
        Q = np.zeros(qs); A = np.zeros(as_)
        lo = (C.c_double * 2)(*cfg.prob_lo); hi = (C.c_double * 2)(*cfg.prob_hi)
        lib.oracle_init_solution(qs[0], cfg.nx, cfg.ny, lo, hi, _p(Q))
        lib.oracle_init_solution(as_[0], cfg.nx, cfg.ny, lo, hi, _p(A))
        return Q, A

    def run(self, cfg: zfv_config, Q, A, max_steps: int = -1, face_based: bool = True,
            log_cap: int = 100000):
        """Evolve from (Q, A); returns (Q, A, steps, time, log[steps, 3], mood_redos)."""
        Q = np.ascontiguousarray(Q, dtype=np.float64).copy()
        A = np.ascontiguousarray(A, dtype=np.float64).copy()
        log = np.zeros((log_cap, 3))
        ns = C.c_int64(0); t = C.c_double(0.0); mr = C.c_int(0)
        rc = self._fn("run")(C.byref(cfg), _p(Q), _p(A), int(max_steps), int(face_based), _p(log),
                            log_cap, C.byref(ns), C.byref(t), C.byref(mr))
        if rc != 0:
            raise RuntimeError(f"{self.kind}_run failed ({rc})")
        n = int(ns.value)
        return Q, A, n, float(t.value), log[:min(n, log_cap)], int(mr.value)

    def fill_ghosts(self, cfg: zfv_config, Q, A, time: float = 0.0):
        ng = 2 if cfg.spatial_order == 2 else 1
        m = MODELS[cfg.model]
        Qg = np.zeros((m["n_q"], cfg.ny + 2 * ng, cfg.nx + 2 * ng))
        Ag = np.zeros((m["n_aux"], cfg.ny + 2 * ng, cfg.nx + 2 * ng))
        rc = self._fn("fill_ghosts")(C.byref(cfg), _p(np.ascontiguousarray(Q, np.float64)),
                                     _p(np.ascontiguousarray(A, np.float64)), time, _p(Qg), _p(Ag))
        if rc != 0:
            raise RuntimeError("fill_ghosts failed")
        return Qg, Ag

    def rhs(self, cfg: zfv_config, Q, A, time: float = 0.0, face_based: bool = True):
        qs, _ = _shapes(cfg)
        R = np.zeros(qs)
        rc = self._fn("rhs")(C.byref(cfg), _p(np.ascontiguousarray(Q, np.float64)),
                             _p(np.ascontiguousarray(A, np.float64)), time, int(face_based), _p(R))
        if rc != 0:
            raise RuntimeError("rhs failed")
        return R

    def compute_dt(self, cfg: zfv_config, Q, A):
        dt = C.c_double(0); mi = C.c_double(0)
        rc = self._fn("compute_dt")(C.byref(cfg), _p(np.ascontiguousarray(Q, np.float64)),
                                    _p(np.ascontiguousarray(A, np.float64)), C.byref(dt), C.byref(mi))
        if rc != 0:
            raise RuntimeError("compute_dt failed")
        return float(dt.value), float(mi.value)

    def update_state(self, cfg: zfv_config, Q, A, time: float = 0.0):
        Q = np.ascontiguousarray(Q, dtype=np.float64).copy()
        A = np.ascontiguousarray(A, dtype=np.float64).copy()
        if self._fn("update_state")(C.byref(cfg), _p(Q), _p(A), time) != 0:
            raise RuntimeError("update_state failed")
        return Q, A

    def advance(self, cfg: zfv_config, Q, A, time: float, dt: float, face_based: bool = True):
        Q = np.ascontiguousarray(Q, dtype=np.float64).copy()
        A = np.ascontiguousarray(A, dtype=np.float64).copy()
        if self._fn("advance")(C.byref(cfg), _p(Q), _p(A), time, dt, int(face_based)) != 0:
            raise RuntimeError("advance failed")
        return Q, A


def amr2_run(cfg: zfv_config, Q0, rects, n_steps: int, dt: float | None, return_time: bool = False):
    """Two-level AMR run of the restatement (oracle/fv_oracle_amr.H): base
    state Q0 (4, ny, nx), fine patches ``rects`` = [(i0, j0, nx, ny)] in fine
    cells (started as the interpolation of the base state), ``n_steps``
    coarse steps of ``dt`` (None: the reference's per-level CFL law).
    Returns (base state, [fine patch states]) (and the final time)."""
    lib, _ = _load("oracle")
    Q = np.ascontiguousarray(Q0, dtype=np.float64).copy()
    r = np.ascontiguousarray(np.asarray(rects, dtype=np.int32).reshape(-1, 4))
    out = np.zeros(int(sum(4 * int(w) * int(h) for _, _, w, h in r)))
    t = C.c_double(0.0)
    rc = lib.oracle_amr2_run(C.byref(cfg), _p(Q), r.ctypes.data_as(C.POINTER(C.c_int)), len(r), int(n_steps),
                             0.0 if dt is None else float(dt), 1 if dt is None else 0, _p(out), C.byref(t))
    if rc != 0:
        raise RuntimeError(f"oracle_amr2_run failed ({rc})")
    fine, off = [], 0
    for _, _, w, h in r:
        n = 4 * int(w) * int(h)
        fine.append(out[off:off + n].reshape(4, int(h), int(w)))
        off += n
    return (Q, fine, float(t.value)) if return_time else (Q, fine)
