"""One refinement level on one B200: PyTorch tensors + a libzoomyfv handle.

This is the in-process replacement for the part of the reference's AMReX
executable that a zoomy_amrex run spends its time in: the level data
(Q, Qaux: ZoomyAmr.H:81-84) live in HBM as component-major torch tensors, and
each call enqueues SSP-RK2 steps whose dt, time and stop test stay on the
device (ZoomyAmr::Evolve's loop, ZoomyAmr.cpp:782-810). The host reads the run
status only when asked.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._abi import MODELS, ZFV_MODEL_SWE2D, ZFV_PREC_FP32, zfv_config, zfv_status


def fp32_kernel_family(cfg: zfv_config) -> str:
    """Which FP32 kernels run a level, and so which shapes its variant
    indexes: "fp32" = the shallow-water column sweep (2-D SWE, order 2, no
    MOOD; batch.tile_variants()), "fp32-tile" = the generic tile kernels (every
    other FP32 case; batch.generic_tile_variants()). The autotuner caches
    the two under these names."""
    sweep = cfg.model == ZFV_MODEL_SWE2D and cfg.spatial_order == 2 and not cfg.positivity_mood
    return "fp32" if sweep else "fp32-tile"

_DTYPE = torch.float64


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class Level:
    """A single-level solver state on ``device``.

    FP64 plain form (cfg.precision == ZFV_PREC_FP64):
      Q:   (n_q, ny, nx) float64, rows [b, h, hu, (hv)]
    FP32 chosen form (ZFV_PREC_FP32, 2-D shallow water):
      Q:   (4, ny, nx) float32, rows [b, eta = h + b, hu, hv] at import; steps
           ping-pong the state between Q and a scratch buffer and keep the
           low-order remainders of eta, hu, hv in scratch, so the state is
           read through state64() (the reference layout, FP64), which also
           refreshes aux's hinv row.
    aux: (n_aux, ny, nx) float64, last row hinv (both forms); aux0 = None
         creates it on the device as init_solution does (zfv_init_solution)
    """

    def __init__(self, cfg: zfv_config, Q0, aux0=None, device: str | torch.device = "cuda:0",
                 stream: torch.cuda.Stream | None = None, variant: int | None = None):
        if not torch.cuda.is_available():
            raise _lib.ZfvError("zoomy_amrex_b200 needs a CUDA device (no CPU fallback)")
        self.cfg = cfg
        self.info = MODELS[cfg.model]
        self.device = torch.device(device)
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.zfv_create(C.byref(cfg), C.byref(h)), "zfv_create")
        self._h = h
        nq, na = self.info["n_q"], self.info["n_aux"]
        shape_q, shape_a = (nq, cfg.ny, cfg.nx), (na, cfg.ny, cfg.nx)
        self.fp32 = cfg.precision == ZFV_PREC_FP32
        nbytes = int(L.zfv_scratch_bytes(h))
        self.scratch = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
        # A dedicated stream: CUDA graphs cannot be captured on the default stream.
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        if aux0 is None:
            # init_solution on the device, as InitData fills Qaux (ZoomyAmr.cpp:174-175)
            self.aux = torch.empty(shape_a, dtype=_DTYPE, device=self.device)
            self.stream.wait_stream(torch.cuda.current_stream(self.device))
            _lib.check(L.zfv_init_solution(h, _ptr(self.aux), na, self._s()), "zfv_init_solution")
        else:
            self.aux = self._as_tensor(aux0, shape_a)
        if self.fp32:
            q64 = self._as_tensor(Q0, shape_q)
            self.Q = torch.empty(shape_q, dtype=torch.float32, device=self.device)
            self.stream.wait_stream(torch.cuda.current_stream(self.device))
            _lib.check(L.zfv_state_import(h, _ptr(q64), _ptr(self.Q), _ptr(self.scratch), self._s()),
                       "zfv_state_import")
            self.stream.synchronize()
            del q64
        else:
            self.Q = self._as_tensor(Q0, shape_q)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        self._graph = None
        self._graph_steps = 0
        if self.fp32:
            if variant is None:   # the autotuner's pick for this size, if one was measured
                from .autotune import cached_variant
                variant = cached_variant(nq, fp32_kernel_family(cfg), cfg.nx * cfg.ny)
            if variant is not None:
                self.set_variant(variant)
        elif variant is not None:
            raise ValueError("strip shapes (variant) are a property of the FP32 form")

    def _as_tensor(self, a, shape):
        t = torch.as_tensor(np.asarray(a) if not torch.is_tensor(a) else a)
        t = t.to(device=self.device, dtype=_DTYPE).reshape(shape).contiguous().clone()
        return t

    @property
    def handle(self):
        return self._h

    @property
    def variant(self) -> int:
        """Shape of the FP32 stage kernels (index into batch.tile_variants() for the
        shallow-water sweep, batch.generic_tile_variants() otherwise, see
        fp32_kernel_family); -1 for FP64."""
        return int(_lib.lib().zfv_get_variant(self._h))

    def set_variant(self, variant: int):
        """Select the FP32 strip shape (drops a captured graph)."""
        self._graph = None
        _lib.check(_lib.lib().zfv_set_variant(self._h, int(variant), self._s()), "zfv_set_variant")

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._graph = None
            _lib.lib().zfv_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's driver entry points -------------------------------------
    def begin(self):
        """Reset time/step and compute the first dt from (Q, aux) as stored."""
        _lib.check(_lib.lib().zfv_begin(self._h, _ptr(self.Q), _ptr(self.aux), _ptr(self.scratch),
                                        self._s()), "zfv_begin")

    def evolve(self, n_steps: int):
        """Enqueue up to n_steps time steps (no host synchronization)."""
        _lib.check(_lib.lib().zfv_evolve(self._h, _ptr(self.Q), _ptr(self.aux), _ptr(self.scratch),
                                         int(n_steps), self._s()), "zfv_evolve")

    def capture(self, n_steps: int):
        """Capture `evolve(n_steps)` into a CUDA graph for replay()."""
        g = torch.cuda.CUDAGraph()
        self.stream.synchronize()
        with torch.cuda.stream(self.stream):
            with torch.cuda.graph(g, stream=self.stream):
                _lib.check(_lib.lib().zfv_evolve(self._h, _ptr(self.Q), _ptr(self.aux),
                                                 _ptr(self.scratch), int(n_steps),
                                                 C.c_void_p(torch.cuda.current_stream().cuda_stream)),
                           "zfv_evolve (capture)")
        self._graph, self._graph_steps = g, int(n_steps)
        return g

    def replay(self):
        if self._graph is None:
            raise RuntimeError("capture() first")
        with torch.cuda.stream(self.stream):
            self._graph.replay()

    def status(self) -> dict:
        st = zfv_status()
        _lib.check(_lib.lib().zfv_get_status(self._h, _ptr(self.scratch), C.byref(st), self._s()),
                   "zfv_get_status")
        return dict(time=st.time, dt=st.dt, mass=st.mass, max_inv=st.max_inv, step=int(st.step),
                    flags=int(st.flags), done=bool(st.flags & 4), mood_redos=int(st.mood_redos))

    def run(self, max_steps: int | None = None, chunk: int = 64, use_graph: bool = False) -> dict:
        """Evolve until time_end / max_step (or max_steps), syncing once per chunk.
        With implicit_global the steps always run uncaptured (the Newton-Krylov
        iteration reads norms on the host)."""
        if self.cfg.implicit_source and self.cfg.implicit_global:
            use_graph = False
        self.begin()
        done_steps = 0
        last_step = -1
        while True:
            n = chunk if max_steps is None else min(chunk, max_steps - done_steps)
            if n <= 0:
                break
            if use_graph:
                if self._graph is None or self._graph_steps != n:
                    self.capture(n)
                self.replay()
            else:
                self.evolve(n)
            done_steps += n
            st = self.status()
            if st["done"]:
                break
            if st["step"] <= last_step:   # the device did not advance: stop, do not spin
                raise _lib.ZfvError(f"no progress after {done_steps} requested steps: status {st}")
            last_step = st["step"]
        return self.status()

    def implicit_global_stats(self) -> dict:
        """Field solves, Newton iterations and GMRES iterations of the global
        implicit source since the last begin (zeros for the point-implicit form)."""
        v = [C.c_longlong(0) for _ in range(3)]
        _lib.check(_lib.lib().zfv_implicit_global_stats(self._h, *[C.byref(x) for x in v]),
                   "zfv_implicit_global_stats")
        return dict(solves=v[0].value, newton=v[1].value, gmres=v[2].value)

    def state64(self) -> torch.Tensor:
        """The state in the reference layout [b, h, hu, (hv)], float64 (synchronizes)."""
        if not self.fp32:
            self.stream.synchronize()
            return self.Q.clone()
        out = torch.empty(self.Q.shape, dtype=_DTYPE, device=self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        _lib.check(_lib.lib().zfv_state_export(self._h, _ptr(self.Q), _ptr(self.scratch), _ptr(out),
                                               self._s()), "zfv_state_export")
        self.stream.synchronize()
        return out

    def log(self) -> np.ndarray:
        """(steps, 3) array of (dt, time, mass) per completed step (last 4096 kept)."""
        L = _lib.lib()
        cap = int(L.zfv_log_capacity(self._h))
        out = (C.c_double * (3 * cap))()
        first = C.c_int64(0); n = C.c_int(0)
        _lib.check(L.zfv_read_log(self._h, _ptr(self.scratch), out, cap, C.byref(first), C.byref(n),
                                  self._s()), "zfv_read_log")
        return np.frombuffer(out, dtype=np.float64, count=3 * n.value).reshape(n.value, 3).copy()

    # -- validation entries -------------------------------------------------------
    def sync(self):
        """Wait for this level's stream (host reads of Q/aux need it)."""
        self.stream.synchronize()

    def rhs(self, time: float = 0.0) -> torch.Tensor:
        out = torch.empty_like(self.Q)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        _lib.check(_lib.lib().zfv_rhs(self._h, _ptr(self.Q), _ptr(self.aux), _ptr(out), float(time),
                                      self._s()), "zfv_rhs")
        return out

    def fill_ghosts(self, time: float = 0.0):
        ng = 2 if self.cfg.spatial_order == 2 else 1
        nq, na = self.info["n_q"], self.info["n_aux"]
        Qg = torch.empty((nq, self.cfg.ny + 2 * ng, self.cfg.nx + 2 * ng), dtype=_DTYPE, device=self.device)
        Ag = torch.empty((na, self.cfg.ny + 2 * ng, self.cfg.nx + 2 * ng), dtype=_DTYPE, device=self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        _lib.check(_lib.lib().zfv_fill_ghosts(self._h, _ptr(self.Q), _ptr(self.aux), _ptr(Qg), _ptr(Ag),
                                              float(time), self._s()), "zfv_fill_ghosts")
        return Qg, Ag

    def update_state(self, time: float = 0.0):
        _lib.check(_lib.lib().zfv_update_state(self._h, _ptr(self.Q), _ptr(self.aux), float(time),
                                               self._s()), "zfv_update_state")

    def compute_dt(self) -> tuple[float, float]:
        _lib.check(_lib.lib().zfv_compute_dt(self._h, _ptr(self.Q), _ptr(self.aux), _ptr(self.scratch),
                                             self._s()), "zfv_compute_dt")
        st = self.status()
        return st["dt"], st["max_inv"]

    def total_mass(self) -> float:
        _lib.check(_lib.lib().zfv_total_mass(self._h, _ptr(self.Q), _ptr(self.scratch), self._s()),
                   "zfv_total_mass")
        return self.status()["mass"]
