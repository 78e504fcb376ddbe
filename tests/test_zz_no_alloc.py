"""zfv_evolve_static — the entry point for callers that cannot allocate device
memory (code inside another framework's memory pool, under a caching allocator
that owns the device, or in a plugin that must not allocate at call time).

It must give the same run as zfv_begin + zfv_evolve with caller-provided
scratch, call after call, while using only the library's built-in 64 MiB
scratch array. Collected last (file name) so that a failure here never hides
the other tests; it passes alone in a fresh process and after the others
(each comparison starts with restart=1, which clears the shared run record).
"""
import ctypes as C

import numpy as np
import pytest

from cases import setup
from zoomy_amrex_b200 import _lib
from zoomy_amrex_b200._abi import make_config, ZFV_MODEL_SWE2D, zfv_status
from zoomy_amrex_b200.models import SWE

pytestmark = pytest.mark.gpu


def _bumpy(x):
    b = 0.9 * np.exp(-((x[0] - 3.0) ** 2 + (x[1] - 6.0) ** 2) / 3.0)
    eta = 1.0 + 0.25 * np.exp(-((x[0] - 7.0) ** 2 + (x[1] - 3.0) ** 2))
    h = np.maximum(eta - b, 0.0)
    return np.array([b, h, 0.05 * h, -0.03 * h])


CASE = (SWE(2, {"West": "wall", "East": "extrapolation", "South": "wall", "North": "wall"}, _bumpy,
            parameters={"n_m": 0.03}),
        dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[96, 80], spatial_order=2, cfl=0.9,
             time_end=1e30, max_step=-1, well_balanced=True, implicit_source=True))

STEPS = 7   # per call


def _vp(t):
    return C.c_void_p(t.data_ptr())


def _create(lib, cfg):
    h = C.c_void_p()
    rc = lib.zfv_create(C.byref(cfg), C.byref(h))
    assert rc == 0, lib.zfv_last_error()
    return h


def _reference_path(lib, cfg, Q0, A0, torch):
    """Two zfv_evolve calls with caller-allocated scratch (the existing entry point)."""
    h = _create(lib, cfg)
    stream = torch.cuda.Stream()
    s = C.c_void_p(stream.cuda_stream)
    Q = torch.as_tensor(Q0, device="cuda").contiguous().clone()
    A = torch.as_tensor(A0, device="cuda").contiguous().clone()
    scratch = torch.zeros(lib.zfv_scratch_bytes(h), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    out = []
    assert lib.zfv_begin(h, _vp(Q), _vp(A), _vp(scratch), s) == 0
    for _ in range(2):
        assert lib.zfv_evolve(h, _vp(Q), _vp(A), _vp(scratch), STEPS, s) == 0, lib.zfv_last_error()
        st = zfv_status()
        assert lib.zfv_get_status(h, _vp(scratch), C.byref(st), s) == 0
        out.append((Q.cpu().numpy(), A.cpu().numpy(), st.step, st.time, st.dt))
    lib.zfv_destroy(h)
    return out


def _static_path(lib, cfg, Q0, A0, torch):
    """The same two calls through zfv_evolve_static (no scratch argument)."""
    h = _create(lib, cfg)
    stream = torch.cuda.Stream()
    s = C.c_void_p(stream.cuda_stream)
    Q = torch.as_tensor(Q0, device="cuda").contiguous().clone()
    A = torch.as_tensor(A0, device="cuda").contiguous().clone()
    torch.cuda.synchronize()
    out = []
    for call in range(2):
        st = zfv_status()
        rc = lib.zfv_evolve_static(h, _vp(Q), _vp(A), STEPS, 1 if call == 0 else 0, C.byref(st), s)
        assert rc == 0, lib.zfv_last_error()
        out.append((Q.cpu().numpy(), A.cpu().numpy(), st.step, st.time, st.dt))
    lib.zfv_destroy(h)
    return out


def test_static_scratch_matches_caller_scratch(cuda):
    import torch
    lib = _lib.lib()
    cfg, Q0, A0 = setup(*CASE)
    ref = _reference_path(lib, cfg, Q0, A0, torch)
    got = _static_path(lib, cfg, Q0, A0, torch)
    for k, (a, b) in enumerate(zip(ref, got)):
        assert b[2] == a[2] == STEPS * (k + 1)
        assert b[3] == a[3] and b[4] == a[4], f"call {k}: time/dt differ"
        # FP64 parity in this suite is bitwise
        assert np.array_equal(a[0], b[0]), f"call {k}: state differs, max {np.abs(a[0] - b[0]).max():.3e}"
        assert np.array_equal(a[1], b[1]), f"call {k}: aux differs"
        assert np.isfinite(b[0]).all()
    # a second run on the same device restarts cleanly from the shared array
    again = _static_path(lib, cfg, Q0, A0, torch)
    assert np.array_equal(again[1][0], got[1][0])


def test_static_scratch_rejects_levels_that_do_not_fit(cuda):
    import torch
    lib = _lib.lib()
    cfg = make_config(ZFV_MODEL_SWE2D, 2048, 2048, (0.0, 0.0), (1.0, 1.0), spatial_order=2)
    h = _create(lib, cfg)
    assert lib.zfv_scratch_bytes(h) > (64 << 20)
    # the size check fails before any device access, so no real buffers are needed
    Q = torch.empty(16, dtype=torch.float64, device="cuda")
    st = zfv_status()
    rc = lib.zfv_evolve_static(h, _vp(Q), _vp(Q), 1, 1, C.byref(st), None)
    msg = lib.zfv_last_error().decode()
    lib.zfv_destroy(h)
    assert rc != 0 and "static" in msg and "too large" in msg


def test_static_scratch_refuses_fp32_and_foreign_continuations(cuda):
    import torch
    from zoomy_amrex_b200._abi import ZFV_PREC_FP32
    lib = _lib.lib()
    Q = torch.empty(16, dtype=torch.float64, device="cuda")
    st = zfv_status()
    # the FP32 form keeps its state remainder in scratch that only the
    # import/export entry points reach, so it is refused before any device work
    cfg32 = make_config(ZFV_MODEL_SWE2D, 64, 64, (0.0, 0.0), (1.0, 1.0), spatial_order=2,
                        precision=ZFV_PREC_FP32)
    h32 = _create(lib, cfg32)
    rc = lib.zfv_evolve_static(h32, _vp(Q), _vp(Q), 1, 1, C.byref(st), None)
    msg = lib.zfv_last_error().decode()
    lib.zfv_destroy(h32)
    assert rc != 0 and "FP64" in msg
    # continuing (restart == 0) with a handle that did not make the last restart
    # on this device is refused before any kernel runs
    cfg = make_config(ZFV_MODEL_SWE2D, 64, 64, (0.0, 0.0), (1.0, 1.0), spatial_order=2)
    h = _create(lib, cfg)
    rc = lib.zfv_evolve_static(h, _vp(Q), _vp(Q), 1, 0, C.byref(st), None)
    msg = lib.zfv_last_error().decode()
    lib.zfv_destroy(h)
    assert rc != 0 and "restart" in msg
