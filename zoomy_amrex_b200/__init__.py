"""zoomy_amrex_b200 — a B200 (sm_100a) implementation of zoomy-amrex's
per-level finite-volume right-hand side and SSP-RK2 time step.

The hot path lives in ``csrc/`` (CUDA, built into ``lib/libzoomyfv.so`` behind
the C ABI in ``include/zoomy_fv.h``); this package is the host side that
mirrors the reference's Python entry points (``solvers.HyperbolicSolver``,
``run_case.run_case``) and passes PyTorch CUDA tensors through ctypes.
"""
from ._abi import (ZFV_MODEL_SWE1D, ZFV_MODEL_SWE2D, ZFV_PREC_FP32, ZFV_PREC_FP64, MODELS,
                   make_config, zfv_config, zfv_status)

__all__ = ["ZFV_MODEL_SWE1D", "ZFV_MODEL_SWE2D", "ZFV_PREC_FP32", "ZFV_PREC_FP64", "MODELS", "make_config",
           "zfv_config", "zfv_status"]
