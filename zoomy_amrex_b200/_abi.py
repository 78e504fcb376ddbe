"""ctypes mirror of include/zoomy_fv.h (structs and constants only).

The struct layouts here must match the C header field for field; the
library checks ``sizeof(zfv_config)`` against what Python passes.
"""
from __future__ import annotations

import ctypes as C

ZFV_MAX_PARAMS = 16

ZFV_MODEL_SWE1D = 1
ZFV_MODEL_SWE2D = 2
ZFV_MODEL_SME2D_L2 = 3
ZFV_MODEL_SME1D_L2 = 4

ZFV_PREC_FP64 = 0
ZFV_PREC_FP32 = 1

ZFV_FLAG_NONFINITE_DT = 1
ZFV_FLAG_MOOD_REDO = 2
ZFV_FLAG_DONE = 4
ZFV_FLAG_DEVICE_WAIT = 8

# Model registry: id -> (n_q, n_aux, n_params, dimension, parameter names,
# default parameters, boundary tags). Mirrors the compiled Model::
# constants (zoomy_amrex_b200/csrc/models/swe.H, sme.H).
SWE_PARAM_NAMES = ("g", "ex", "ey", "n_m", "h_floor", "eps")
SWE_DEFAULTS = (9.81, 0.0, 0.0, 0.0, 1.0e-6, 1.0e-24)
SWE_TAGS = ("extrapolation", "wall")
SME_PARAM_NAMES = ("g", "ex", "ey", "nu", "lambda", "eps")
SME_DEFAULTS = (9.81, 0.0, 0.0, 1.0e-3, 0.1, 1.0e-24)

MODELS = {
    ZFV_MODEL_SWE1D: dict(name="swe1d", n_q=3, n_aux=4, n_params=6, dimension=1,
                          param_names=SWE_PARAM_NAMES, defaults=SWE_DEFAULTS, tags=SWE_TAGS),
    ZFV_MODEL_SWE2D: dict(name="swe2d", n_q=4, n_aux=7, n_params=6, dimension=2,
                          param_names=SWE_PARAM_NAMES, defaults=SWE_DEFAULTS, tags=SWE_TAGS),
    ZFV_MODEL_SME2D_L2: dict(name="sme2d_l2", n_q=8, n_aux=1, n_params=6, dimension=2, level=2,
                             param_names=SME_PARAM_NAMES, defaults=SME_DEFAULTS, tags=SWE_TAGS),
    ZFV_MODEL_SME1D_L2: dict(name="sme1d_l2", n_q=5, n_aux=1, n_params=6, dimension=1, level=2,
                             param_names=SME_PARAM_NAMES, defaults=SME_DEFAULTS, tags=SWE_TAGS),
}


class zfv_config(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("precision", C.c_int),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("prob_lo", C.c_double * 2),
        ("prob_hi", C.c_double * 2),
        ("spatial_order", C.c_int),
        ("well_balanced", C.c_int),
        ("implicit_source", C.c_int),
        ("clamp_positivity", C.c_int),
        ("positivity_mood", C.c_int),
        ("implicit_global", C.c_int),
        ("cfl", C.c_double),
        ("dtmin", C.c_double),
        ("dtmax", C.c_double),
        ("time_end", C.c_double),
        ("max_step", C.c_int),
        ("cfl_dimension", C.c_int),
        ("cfl_degree_factor", C.c_int),
        ("bc_tag", C.c_int * 4),
        ("n_params", C.c_int),
        ("params", C.c_double * ZFV_MAX_PARAMS),
    ]


class zfv_status(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("mass", C.c_double),
        ("max_inv", C.c_double),
        ("step", C.c_int64),
        ("flags", C.c_uint32),
        ("mood_redos", C.c_uint32),
        ("pad", C.c_uint32 * 4),
    ]


class zfv_amr_level(C.Structure):
    _fields_ = [("insts", C.c_void_p), ("map", C.c_void_p), ("nbx", C.c_int), ("nby", C.c_int),
                ("B", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("wall", C.c_int), ("pad", C.c_int)]


def make_config(model: int, nx: int, ny: int, prob_lo, prob_hi, *, spatial_order: int = 1,
                well_balanced: bool = False, implicit_source: bool = False,
                clamp_positivity: bool = False, positivity: str = "none", cfl: float = 0.9,
                dtmin: float = 1.0e-7, dtmax: float = 1.0, time_end: float = 1.0,
                max_step: int = -1, cfl_dimension: int | None = None,
                cfl_degree_factor: int | None = None, bc=("extrapolation",) * 4,
                params: dict | None = None, precision: int = ZFV_PREC_FP64,
                implicit_global: bool = False) -> zfv_config:
    """Build a zfv_config the way the reference's deck + MarchConstants.H define it.

    ``bc`` names the boundary tag per side (x_lo, x_hi, y_lo, y_hi); each name
    is resolved against the model's sorted tag list, and an unknown non-empty
    name is an error (ZoomyAmr.cpp:361-372). ``cfl_dimension`` defaults to the
    model dimension d and ``cfl_degree_factor`` to 2k+1 with k = order - 1
    (zoomy_amrex/_constants.py:8-13, run_case.py:391-395). ``implicit_global``
    (solver.implicit_global, ZoomyAmr.cpp:48) solves the implicit source for
    the whole field by Jacobian-free Newton-Krylov.
    """
    info = MODELS[model]
    if positivity not in ("none", "mood"):
        raise ValueError(f"positivity must be 'none' or 'mood', got {positivity!r}")
    if spatial_order not in (1, 2):
        raise ValueError(f"spatial_order must be 1 or 2, got {spatial_order}")
    c = zfv_config()
    c.model = model
    c.precision = precision
    c.nx, c.ny = int(nx), int(ny)
    c.prob_lo[0], c.prob_lo[1] = float(prob_lo[0]), float(prob_lo[1])
    c.prob_hi[0], c.prob_hi[1] = float(prob_hi[0]), float(prob_hi[1])
    c.spatial_order = int(spatial_order)
    c.well_balanced = int(bool(well_balanced))
    c.implicit_source = int(bool(implicit_source))
    c.clamp_positivity = int(bool(clamp_positivity))
    c.positivity_mood = int(positivity == "mood")
    c.implicit_global = int(bool(implicit_global))
    c.cfl, c.dtmin, c.dtmax, c.time_end = float(cfl), float(dtmin), float(dtmax), float(time_end)
    c.max_step = int(max_step)
    c.cfl_dimension = int(info["dimension"] if cfl_dimension is None else cfl_dimension)
    c.cfl_degree_factor = int(2 * (spatial_order - 1) + 1 if cfl_degree_factor is None
                              else cfl_degree_factor)
    tags = info["tags"]
    for s in range(4):
        name = bc[s] if s < len(bc) else ""
        if not name:
            c.bc_tag[s] = 0
        elif name in tags:
            c.bc_tag[s] = tags.index(name)
        else:
            raise ValueError(f"boundary tag {name!r} is not declared by this model; "
                             f"known tags: {list(tags)}")
    pv = list(info["defaults"])
    for k, v in (params or {}).items():
        if k not in info["param_names"]:
            raise KeyError(f"unknown parameter {k!r}; known: {list(info['param_names'])}")
        pv[info["param_names"].index(k)] = float(v)
    c.n_params = len(pv)
    for k, v in enumerate(pv):
        c.params[k] = v
    return c
