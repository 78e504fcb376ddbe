"""Gradients of a final-time misfit through the FP64 shallow-water solver.

``evolve_differentiable(Q0, n_m, aux0, cfg, n_steps)`` runs ``n_steps`` SSP-RK2
steps of the FP64 SWE2D form on the GPU and returns Q_T as a torch tensor
whose backward runs the hand-written CUDA reverse (libzoomyfv's
zfv_adj_record / zfv_adj_step): gradients with respect to the initial state
(bathymetry row b included) and the Manning coefficient n_m.

Memory: the forward keeps one checkpoint (Q and the 128-byte device run
record) every ``checkpoint_every`` steps; the backward re-runs each segment
from its checkpoint, recording the tape of that segment only (about 14 state
planes per step), then walks it backwards. The last segment is recorded by
the forward itself (its tape is kept until the backward), so the backward
re-runs all segments but that one. The map differentiated is the one
the solver applies, including dt_n = cfl / (d (2k+1) max_inv(Q^n)); the
forward recomputation is bitwise identical to the original run.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._abi import MODELS, ZFV_MODEL_SWE2D, ZFV_PREC_FP64, zfv_config

N_M_SLOT = 3   # Manning coefficient in the SWE parameter vector


def _copy_cfg(cfg: zfv_config) -> zfv_config:
    c = zfv_config()
    C.memmove(C.byref(c), C.byref(cfg), C.sizeof(cfg))
    return c


# One side stream per device for every solver of this module: the caching
# allocator keeps freed blocks per stream, so checkpoints and tapes of one
# gradient computation are reused by the next one instead of being allocated
# again (a 2 GB tape allocated inside a backward can cost more than the
# backward's kernels).
_STREAMS: dict = {}


def _side_stream(device) -> "torch.cuda.Stream":
    d = torch.device(device)
    key = d.index if d.index is not None else torch.cuda.current_device()
    if key not in _STREAMS:
        _STREAMS[key] = torch.cuda.Stream(d)
    return _STREAMS[key]


class _Solver:
    """A handle plus the buffers the forward/backward share."""

    def __init__(self, cfg: zfv_config, device):
        if cfg.model != ZFV_MODEL_SWE2D or cfg.precision != ZFV_PREC_FP64 or cfg.spatial_order != 2:
            raise ValueError("the adjoint runs the FP64 SWE2D form at spatial_order 2")
        L = _lib.lib()
        self.cfg = cfg
        h = C.c_void_p()
        _lib.check(L.zfv_create(C.byref(cfg), C.byref(h)), "zfv_create")
        self.h = h
        self.device = device
        self.stream = _side_stream(device)
        self.scratch = torch.zeros(int(L.zfv_scratch_bytes(h)), dtype=torch.uint8, device=device)
        self.rs_bytes = int(L.zfv_run_state_bytes())
        info = MODELS[cfg.model]
        self.nq, self.na = info["n_q"], info["n_aux"]

    def s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def close(self):
        if self.h is not None and self.h.value:
            _lib.lib().zfv_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _check_steps(sol: _Solver, expect_step: int):
    from ._abi import zfv_status
    st = zfv_status()
    _lib.check(_lib.lib().zfv_get_status(sol.h, sol.scratch.data_ptr(), C.byref(st), sol.s()), "zfv_get_status")
    if st.step != expect_step:
        raise RuntimeError(f"the run stopped at step {st.step} (expected {expect_step}); "
                           "raise time_end / max_step so the recorded steps all run")
    return st


class SWEEvolve(torch.autograd.Function):
    """Q_T = evolve(Q0; n_m) for n_steps steps (see the module docstring)."""

    @staticmethod
    def forward(ctx, Q0, n_m, aux0, cfg, n_steps, checkpoint_every):
        device = Q0.device
        c = _copy_cfg(cfg)
        c.params[N_M_SLOT] = float(n_m)
        c.max_step = -1
        sol = _Solver(c, device)
        L = _lib.lib()
        Q = Q0.detach().to(torch.float64).contiguous().clone()
        A = aux0.detach().to(torch.float64).contiguous().clone()
        sol.stream.wait_stream(torch.cuda.current_stream(device))
        _lib.check(L.zfv_begin(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), sol.s()), "zfv_begin")
        ckpts = []
        last = None       # (start, n, tape) of the segment the forward recorded
        done = 0
        with torch.cuda.stream(sol.stream):
            while done < n_steps:
                n = min(checkpoint_every, n_steps - done)
                if done + n == n_steps:
                    # the last segment: record its tape now (the same launches
                    # as zfv_evolve plus the tape writes) instead of re-running
                    # it in the backward
                    tape = torch.empty(int(L.zfv_adj_tape_bytes(sol.h, n)), dtype=torch.uint8, device=device)
                    _lib.check(L.zfv_adj_record(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(),
                                                tape.data_ptr(), n, sol.s()), "zfv_adj_record")
                    last = (done, n, tape)
                else:
                    rs = torch.empty(sol.rs_bytes, dtype=torch.uint8, device=device)
                    _lib.check(L.zfv_save_run_state(sol.h, sol.scratch.data_ptr(), rs.data_ptr(), sol.s()),
                               "zfv_save_run_state")
                    ckpts.append((done, Q.clone(), rs))
                    _lib.check(L.zfv_evolve(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), n,
                                            sol.s()), "zfv_evolve")
                done += n
        _check_steps(sol, n_steps)
        torch.cuda.current_stream(device).wait_stream(sol.stream)
        ctx.sol = sol
        ctx.ckpts = ckpts
        ctx.last = last
        ctx.aux0 = aux0.detach().to(torch.float64).contiguous()
        ctx.n_steps = n_steps
        ctx.every = checkpoint_every
        return Q

    @staticmethod
    def backward(ctx, gQ):
        sol = ctx.sol
        L = _lib.lib()
        device = gQ.device
        lam = gQ.detach().to(torch.float64).contiguous().clone()
        grad = torch.zeros(2, dtype=torch.float64, device=device)
        work = torch.zeros(int(L.zfv_adj_work_bytes(sol.h)), dtype=torch.uint8, device=device)
        sol.stream.wait_stream(torch.cuda.current_stream(device))

        def reverse(start, n, tape):
            # the segment's steps n-1 .. 0 in one call (no host round trip per step)
            aux0 = ctx.aux0.data_ptr() if start == 0 else None
            _lib.check(L.zfv_adj_steps(sol.h, tape.data_ptr(), n, lam.data_ptr(), grad.data_ptr(), aux0,
                                       work.data_ptr(), sol.s()), "zfv_adj_steps")

        with torch.cuda.stream(sol.stream):
            if ctx.last is not None:
                start, n, tape_last = ctx.last
                reverse(start, n, tape_last)
            if ctx.ckpts:
                tape = torch.empty(int(L.zfv_adj_tape_bytes(sol.h, ctx.every)), dtype=torch.uint8, device=device)
                Q = torch.empty_like(ctx.ckpts[0][1])
                A = ctx.aux0.clone()
            for start, Qc, rs in reversed(ctx.ckpts):
                n = min(ctx.every, ctx.n_steps - start)
                Q.copy_(Qc)
                _lib.check(L.zfv_load_run_state(sol.h, sol.scratch.data_ptr(), rs.data_ptr(), sol.s()),
                           "zfv_load_run_state")
                _lib.check(L.zfv_adj_record(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(),
                                            tape.data_ptr(), n, sol.s()), "zfv_adj_record")
                reverse(start, n, tape)
        torch.cuda.current_stream(device).wait_stream(sol.stream)
        sol.stream.synchronize()
        ctx.sol = None
        ctx.last = None
        sol.close()
        g_nm = grad[0].reshape(()).to(gQ.dtype)
        return lam, g_nm, None, None, None, None


def evolve_differentiable(Q0: torch.Tensor, n_m: torch.Tensor, aux0: torch.Tensor, cfg: zfv_config,
                          n_steps: int, checkpoint_every: int = 20) -> torch.Tensor:
    """Q_T after n_steps steps, differentiable in Q0 (all rows) and n_m."""
    return SWEEvolve.apply(Q0, n_m, aux0, cfg, int(n_steps), int(checkpoint_every))


def forward_only(Q0: torch.Tensor, aux0: torch.Tensor, cfg: zfv_config, n_steps: int,
                 n_m: float | None = None) -> torch.Tensor:
    """The same forward map without a graph (for finite differences)."""
    c = _copy_cfg(cfg)
    if n_m is not None:
        c.params[N_M_SLOT] = float(n_m)
    c.max_step = -1
    sol = _Solver(c, Q0.device)
    L = _lib.lib()
    Q = Q0.detach().to(torch.float64).contiguous().clone()
    A = aux0.detach().to(torch.float64).contiguous().clone()
    sol.stream.wait_stream(torch.cuda.current_stream(Q0.device))
    _lib.check(L.zfv_begin(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), sol.s()), "zfv_begin")
    _lib.check(L.zfv_evolve(sol.h, Q.data_ptr(), A.data_ptr(), sol.scratch.data_ptr(), int(n_steps), sol.s()),
               "zfv_evolve")
    _check_steps(sol, n_steps)
    sol.stream.synchronize()
    sol.close()
    return Q
