"""Settings -> solver configuration, with the reference's key semantics.

Mirrors what zoomy_amrex/run_case.py does with a settings dict before it
writes the AMReX inputs deck: the grid (run_case.py:75-84), the deck values
write_inputs emits (build.py:55-120; run_case.py:235-288) and the march
constants (run_case.py:390-395, _constants.py:8-13). The reference then
compiles and launches a binary; here the result is a zfv_config for
libzoomyfv.so.
"""
from __future__ import annotations

from ._abi import ZFV_PREC_FP64, make_config
from .models import SWE


def grid(settings: dict):
    """(dimension, nx, ny, prob_lo, prob_hi) as run_case._grid builds them.

    1-D: ny = 1 and the y extent is one cell, [0, (x1 - x0)/nx]."""
    dim = int(settings.get("dimension", 2))
    dom = settings["domain"]
    nc = settings["n_cells"]
    if dim == 1:
        nx = int(nc[0] if isinstance(nc, (list, tuple)) else nc)
        ny = 1
        x0, x1 = float(dom[0]), float(dom[1])
        y0, y1 = 0.0, (x1 - x0) / nx
    else:
        nx, ny = (int(nc[0]), int(nc[1])) if isinstance(nc, (list, tuple)) else (int(nc), int(nc))
        x0, x1, y0, y1 = [float(v) for v in dom[:4]]
    return dim, nx, ny, (x0, y0), (x1, y1)


def config_from_settings(model: SWE, settings: dict, *, precision: int = ZFV_PREC_FP64):
    """Build the zfv_config for ``model`` on the grid ``settings`` describes.

    Keys (defaults as the reference's run_case/write_inputs apply them):
      time_end (0.1), cfl (0.45), spatial_order (1), well_balanced (False),
      positivity ("none"), dtmax (time_end), dtmin (1e-7), max_step (-1),
      implicit_source (False), implicit_global (False: the deck's
      solver.implicit_global, ZoomyAmr.cpp:48), clamp_positivity (False),
      params ({}).
    """
    dim, nx, ny, lo, hi = grid(settings)
    if dim != model.dimension:
        raise ValueError(f"settings dimension {dim} does not match the model's {model.dimension}")
    tend = float(settings.get("time_end", 0.1))
    order = int(settings.get("spatial_order", 1))
    dtmax = settings.get("dtmax")
    dtmin = settings.get("dtmin")
    max_step = settings.get("max_step")
    params = dict(model.parameters)
    params.update(settings.get("params", {}) or {})
    return make_config(
        model.model_id, nx, ny, lo, hi,
        spatial_order=order,
        well_balanced=bool(settings.get("well_balanced", False)),
        implicit_source=bool(settings.get("implicit_source", False)),
        clamp_positivity=bool(settings.get("clamp_positivity", False)),
        positivity=str(settings.get("positivity", "none")),
        cfl=float(settings.get("cfl", 0.45)),
        dtmin=1.0e-7 if dtmin is None else float(dtmin),
        dtmax=tend if dtmax is None else float(dtmax),
        time_end=tend,
        max_step=-1 if max_step is None else int(max_step),
        cfl_dimension=dim,
        cfl_degree_factor=2 * max(0, order - 1) + 1,
        bc=model.side_kinds(),
        params=params,
        precision=precision,
        implicit_global=bool(settings.get("implicit_global", False)),
    )
