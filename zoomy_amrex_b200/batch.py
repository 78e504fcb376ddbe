"""Many independent FP32 shallow-water levels advanced by one launch per stage.

The instances are the boxes of one AMR level or the members of an ensemble:
each has its own grid size, bathymetry, initial state, parameters, boundary
tags, dt, time and stop test, exactly as if each were a separate
`ZoomyAmr` run (ZoomyAmr.cpp:782-810 per instance), but a step of all of them
is two kernel launches over one work list of strips (libzoomyfv's
zfv_batch_* entry points). All instances share the scheme switches
(spatial order 2, well_balanced, implicit_source).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
import torch

from . import _lib
from ._abi import MODELS, ZFV_MODEL_SWE2D, ZFV_PREC_FP32, zfv_config, zfv_status


# The strip shape batches and FP32 levels use until one is selected (the
# library's default: 4 warps x 8 rows, column pairs, flags 3).
DEFAULT_VARIANT = 9


def tile_variants() -> list[tuple[int, int, int, int]]:
    """The compiled strip shapes as (warps per block, rows per warp, columns
    per lane, flags: bit 0 stage-2 staging, bit 1 stage-2 kernel capped at
    128 registers)."""
    L = _lib.lib()
    nw = (C.c_int * 32)()
    cpt = (C.c_int * 32)()
    cols = (C.c_int * 32)()
    pf = (C.c_int * 32)()
    n = int(L.zfv_tile_variants(nw, cpt, cols, pf, 32))
    return [(nw[k], cpt[k], cols[k], pf[k]) for k in range(n)]


def generic_tile_variants() -> list[tuple[int, int, int]]:
    """Tile variants of the generic FP32 kernels (the shallow-moment model's
    FP32 form) as (tile width, tile height, staging: 0 plain loads, 1 TMA)."""
    L = _lib.lib()
    tx = (C.c_int * 32)()
    ty = (C.c_int * 32)()
    tma = (C.c_int * 32)()
    n = int(L.zfv_generic_tile_variants(tx, ty, tma, 32))
    return [(tx[k], ty[k], tma[k]) for k in range(n)]


class Batch:
    """A batch of FP32 SWE2D instances on one device.

    Per instance k: ``Q[k]`` (4, ny, nx) float32 rows [b, eta, hu, hv] and
    ``aux[k]`` (7, ny, nx) float64; the remainders and ping-pong planes live in
    one shared scratch tensor.
    """

    def __init__(self, cfgs: Sequence[zfv_config], Q0s, A0s, device="cuda:0",
                 stream: torch.cuda.Stream | None = None, variant: int | None = None,
                 groups: Sequence[int] | None = None):
        if not torch.cuda.is_available():
            raise _lib.ZfvError("zoomy_amrex_b200 needs a CUDA device (no CPU fallback)")
        if (Q0s is not None and len(Q0s) != len(cfgs)) or (A0s is not None and len(A0s) != len(cfgs)):
            raise ValueError("cfgs, Q0s and A0s must have the same length")
        for c in cfgs:
            if c.model != ZFV_MODEL_SWE2D or c.precision != ZFV_PREC_FP32:
                raise ValueError("Batch instances must be SWE2D configs with precision ZFV_PREC_FP32")
        L = _lib.lib()
        self.device = torch.device(device)
        self.n = len(cfgs)
        arr = (zfv_config * self.n)(*cfgs)
        self.cfgs = list(arr)
        h = C.c_void_p()
        if groups is None:
            _lib.check(L.zfv_batch_create(arr, self.n, C.byref(h)), "zfv_batch_create")
        else:
            g = (C.c_int * self.n)(*[int(x) for x in groups])
            _lib.check(L.zfv_batch_create_grouped(arr, self.n, g, C.byref(h)), "zfv_batch_create_grouped")
        self._h = h
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        info = MODELS[ZFV_MODEL_SWE2D]
        self.Q, self.aux = [], []
        for c, a0 in zip(self.cfgs, A0s if A0s is not None else [None] * self.n):
            self.Q.append(torch.empty((info["n_q"], c.ny, c.nx), dtype=torch.float32, device=self.device))
            shape = (info["n_aux"], c.ny, c.nx)
            self.aux.append(self._f64(a0, shape) if a0 is not None
                            else torch.zeros(shape, dtype=torch.float64, device=self.device))
        self.scratch = torch.zeros(int(L.zfv_batch_scratch_bytes(h)), dtype=torch.uint8, device=self.device)
        self._qp = (C.c_void_p * self.n)(*[q.data_ptr() for q in self.Q])
        self._ap = (C.c_void_p * self.n)(*[a.data_ptr() for a in self.aux])
        torch.cuda.synchronize(self.device)
        _lib.check(L.zfv_batch_bind(h, self._qp, self._ap, C.c_void_p(self.scratch.data_ptr()), self._s()),
                   "zfv_batch_bind")
        if variant is None:   # the autotuner's pick for this state width and box size
            from .autotune import cached_variant
            variant = cached_variant(info["n_q"], "fp32", np.mean([c.nx * c.ny for c in self.cfgs]))
        if variant is not None:
            self.set_variant(variant)
        self.variant = DEFAULT_VARIANT if variant is None else int(variant)
        if Q0s is not None:
            self.load(Q0s)
        self._graph = None
        self._graph_steps = 0

    def _f64(self, a, shape):
        t = a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a))
        return t.to(device=self.device, dtype=torch.float64).reshape(shape).contiguous().clone()

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._graph = None
            _lib.lib().zfv_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def units(self) -> int:
        return int(_lib.lib().zfv_batch_units(self._h))

    def set_variant(self, variant: int):
        """Switch the strip shape (re-uploads the work list; drops a captured graph)."""
        self._graph = None
        _lib.check(_lib.lib().zfv_batch_set_variant(self._h, int(variant), self._s()), "zfv_batch_set_variant")
        self.variant = int(variant)

    def load(self, Q0s):
        """Import FP64 reference-layout states [b, h, hu, hv] (one per instance)."""
        q64 = [self._f64(q, (4, c.ny, c.nx)) for q, c in zip(Q0s, self.cfgs)]
        ptrs = (C.c_void_p * self.n)(*[q.data_ptr() for q in q64])
        torch.cuda.synchronize(self.device)
        _lib.check(_lib.lib().zfv_batch_import(self._h, ptrs, self._s()), "zfv_batch_import")
        del q64

    @property
    def descriptors(self) -> int:
        """Device address of the instance descriptors (for the AMR kernels)."""
        return int(_lib.lib().zfv_batch_descriptors(self._h) or 0)

    def set_frames(self, frames):
        """Ghost frames (one float32 tensor (4, ny+4, nx+4) per instance, or None)."""
        ptrs = (C.c_void_p * self.n)(*[(f.data_ptr() if f is not None else None) for f in frames])
        _lib.check(_lib.lib().zfv_batch_set_frames(self._h, ptrs, self._s()), "zfv_batch_set_frames")

    def set_dt(self, dts: torch.Tensor):
        """Next dt of every instance from a device float64 tensor (enqueued)."""
        _lib.check(_lib.lib().zfv_batch_set_dt(self._h, dts.data_ptr(), self._s()), "zfv_batch_set_dt")

    def compute_dt(self):
        """Next dt of every run record from the CFL law on its current state
        (ZoomyAmr::ComputeDt; enqueued)."""
        _lib.check(_lib.lib().zfv_batch_compute_dt(self._h, self._s()), "zfv_batch_compute_dt")

    def stage(self, k: int):
        """Stage k (1 or 2) of one step of every instance (enqueued)."""
        _lib.check(_lib.lib().zfv_batch_stage(self._h, int(k), self._s()), "zfv_batch_stage")

    def begin(self):
        _lib.check(_lib.lib().zfv_batch_begin(self._h, self._s()), "zfv_batch_begin")

    def evolve(self, n_steps: int):
        _lib.check(_lib.lib().zfv_batch_evolve(self._h, int(n_steps), self._s()), "zfv_batch_evolve")

    def capture(self, n_steps: int):
        g = torch.cuda.CUDAGraph()
        self.stream.synchronize()
        with torch.cuda.stream(self.stream):
            with torch.cuda.graph(g, stream=self.stream):
                _lib.check(_lib.lib().zfv_batch_evolve(
                    self._h, int(n_steps), C.c_void_p(torch.cuda.current_stream().cuda_stream)),
                    "zfv_batch_evolve (capture)")
        self._graph, self._graph_steps = g, int(n_steps)
        return g

    def replay(self):
        if self._graph is None:
            raise RuntimeError("capture() first")
        with torch.cuda.stream(self.stream):
            self._graph.replay()

    def status(self) -> list[dict]:
        out = (zfv_status * self.n)()
        _lib.check(_lib.lib().zfv_batch_status(self._h, out, self._s()), "zfv_batch_status")
        return [dict(time=s.time, dt=s.dt, mass=s.mass, max_inv=s.max_inv, step=int(s.step),
                     flags=int(s.flags), done=bool(s.flags & 4)) for s in out]

    def run(self, max_steps: int | None = None, chunk: int = 64, use_graph: bool = False) -> list[dict]:
        """Evolve every instance to its own stop (time_end / max_step)."""
        self.begin()
        done_steps = 0
        last_steps = -1
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
            if all(s["done"] for s in st):
                break
            steps = sum(s["step"] for s in st)
            if steps <= last_steps:   # the device did not advance: stop, do not spin
                raise _lib.ZfvError(f"no progress after {done_steps} requested steps")
            last_steps = steps
        return self.status()

    def state64(self) -> list[torch.Tensor]:
        """Every instance's state in the reference layout [b, h, hu, hv], float64."""
        outs = [torch.empty((4, c.ny, c.nx), dtype=torch.float64, device=self.device) for c in self.cfgs]
        ptrs = (C.c_void_p * self.n)(*[o.data_ptr() for o in outs])
        torch.cuda.synchronize(self.device)
        _lib.check(_lib.lib().zfv_batch_export(self._h, ptrs, self._s()), "zfv_batch_export")
        self.stream.synchronize()
        return outs

    def sync(self):
        self.stream.synchronize()
