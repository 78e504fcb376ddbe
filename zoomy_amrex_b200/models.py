"""Model descriptors for the compiled Model::/Numerics:: families.

The reference builds a zoomy_core SystemModel, prints it to Model.H /
Numerics.H and compiles the driver against it (zoomy_amrex/run_case.py:43-71,
210-230). Here the model families are compiled ahead of time into
libzoomyfv.so (csrc/models/), and a descriptor selects one and carries what
the reference keeps on the model object: boundary conditions per side, the
initial condition, and parameter values.

Dimension convention: ``SWE(dimension=d)`` counts horizontal directions
(1 or 2). ``SME(level=0, dimension=n)`` follows zoomy_core's convention, which
counts the vertical too (tests/test_swe_2d.py:129-131: dimension=3 is 2-D).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, Mapping

import numpy as np

from ._abi import MODELS, ZFV_MODEL_SME1D_L2, ZFV_MODEL_SME2D_L2, ZFV_MODEL_SWE1D, ZFV_MODEL_SWE2D

SIDES_2D = ("West", "East", "South", "North")   # run_case.py:281-283
SIDES_1D = ("West", "East")

# BC kinds accepted per side; "swashes" is the reference suite's alias for
# extrapolation (tests/cases.py:182-186).
_BC_ALIASES = {"extrapolation": "extrapolation", "swashes": "extrapolation", "wall": "wall"}


@dataclass
class SWE:
    """Shallow-water equations with state [b, h, hu(, hv)].

    bc: one kind for every side ("extrapolation" | "wall" | "swashes"), or a
        mapping side name -> kind with sides West/East(/South/North).
    initial_conditions: callable X -> Q with X of shape (2, ncell) (cell
        centres, x then y, cells ordered i + nx*j) returning (n_q, ncell);
        the same contract as the reference's sampled IC rasters
        (run_case.py:98-115). None keeps the driver's default dam break.
    parameters: overrides of the model parameters (params.<name> in the deck).
    """

    dimension: int = 2
    bc: str | Mapping[str, str] = "extrapolation"
    initial_conditions: Callable | None = None
    parameters: dict = field(default_factory=dict)

    @property
    def model_id(self) -> int:
        if self.dimension not in (1, 2):
            raise ValueError(f"SWE dimension must be 1 or 2 horizontal directions, got {self.dimension}")
        return ZFV_MODEL_SWE1D if self.dimension == 1 else ZFV_MODEL_SWE2D

    @property
    def info(self) -> dict:
        return MODELS[self.model_id]

    def state_names(self) -> list[str]:
        """Names of the state rows, in the order Q stores them."""
        return ["b", "h", "hu", "hv"][:2 + self.dimension]

    def side_kinds(self) -> tuple:
        """BC kind per side in (x_lo, x_hi, y_lo, y_hi) order ('' = unused side)."""
        sides = SIDES_1D if self.dimension == 1 else SIDES_2D
        if isinstance(self.bc, str):
            kinds = {s: self.bc for s in sides}
        else:
            unknown = set(self.bc) - set(sides)
            if unknown:
                raise ValueError(f"unknown boundary sides {sorted(unknown)}; this model has {sides}")
            kinds = dict(self.bc)
        out = []
        for s in SIDES_2D:
            if s not in sides:
                out.append("")
                continue
            k = kinds.get(s, "")
            if k and k not in _BC_ALIASES:
                raise ValueError(f"unknown BC kind {k!r} on side {s}; use one of {sorted(_BC_ALIASES)}")
            out.append(_BC_ALIASES.get(k, ""))
        return tuple(out)


@dataclass
class ShallowMoments(SWE):
    """Shallow-moment equations of level ``level`` (csrc/models/sme.H): state
    [b, h, hu, (hv), h alpha_1..h alpha_L, (h beta_1..h beta_L)], Navier-slip
    bed friction with viscosity ``nu`` and slip length ``lambda`` (parameters
    g, ex, ey, nu, lambda, eps). Same bc / initial_conditions / parameters
    contract as SWE; initial_conditions return all n_q rows."""

    level: int = 2

    @property
    def model_id(self) -> int:
        if self.level != 2:
            raise NotImplementedError(f"shallow-moment level {self.level} is not compiled (levels 0 and 2 are)")
        if self.dimension not in (1, 2):
            raise ValueError(f"SME dimension must be 1 or 2 horizontal directions, got {self.dimension}")
        return ZFV_MODEL_SME1D_L2 if self.dimension == 1 else ZFV_MODEL_SME2D_L2

    def state_names(self) -> list[str]:
        names = ["b", "h", "hu", "hv"][:2 + self.dimension]
        names += [f"halpha_{j}" for j in range(1, self.level + 1)]
        if self.dimension == 2:
            names += [f"hbeta_{j}" for j in range(1, self.level + 1)]
        return names


def SME(level: int = 0, dimension: int = 3, **kw) -> SWE:
    """zoomy_core-style constructor (dimension counts the vertical too): level
    0 is the shallow-water model, level 2 the two-moment shallow-moment model."""
    if level == 0:
        return SWE(dimension=dimension - 1, **kw)
    if level == 2:
        return ShallowMoments(dimension=dimension - 1, level=level, **kw)
    raise NotImplementedError(f"shallow-moment level {level} is not compiled (levels 0 and 2 are)")


def cell_centres(nx: int, ny: int, prob_lo, prob_hi, dimension: int) -> np.ndarray:
    """(2, nx*ny) cell centres, ordered i + nx*j (run_case.py:87-95)."""
    dx = (prob_hi[0] - prob_lo[0]) / nx
    xc = prob_lo[0] + (np.arange(nx) + 0.5) * dx
    if dimension == 1:
        return np.vstack([xc, np.zeros_like(xc)])
    dy = (prob_hi[1] - prob_lo[1]) / ny
    yc = prob_lo[1] + (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(xc, yc, indexing="xy")
    return np.vstack([X.ravel(order="C"), Y.ravel(order="C")])


def default_fields(n_comp: int, nx: int, ny: int, prob_lo, prob_hi) -> np.ndarray:
    """init_solution (Source/init_solution.cpp:78-116): zeros, and for fields
    with >= 2 components a flat-bed dam break b = 0, h = 2 | 1 split at the
    x mid-point. The reference applies it to the aux field too
    (ZoomyAmr.cpp:174-175), which is why aux row 1 carries the pattern."""
    v = np.zeros((n_comp, ny, nx))
    if n_comp >= 2:
        dx = (prob_hi[0] - prob_lo[0]) / nx
        x = prob_lo[0] + (np.arange(nx) + 0.5) * dx
        x_mid = 0.5 * (prob_lo[0] + prob_hi[0])
        v[1] = np.where(x < x_mid, 2.0, 1.0)[None, :]
    return v


def initial_state(model: SWE, nx: int, ny: int, prob_lo, prob_hi):
    """(Q0, aux0) as the reference's InitData leaves them (ZoomyAmr.cpp:112-156):
    init_solution on both fields, then the IC rasters overwrite every state row."""
    info = model.info
    Q = default_fields(info["n_q"], nx, ny, prob_lo, prob_hi)
    A = default_fields(info["n_aux"], nx, ny, prob_lo, prob_hi)
    if model.initial_conditions is not None:
        X = cell_centres(nx, ny, prob_lo, prob_hi, model.dimension)
        vals = np.asarray(model.initial_conditions(X), dtype=np.float64)
        if vals.shape != (info["n_q"], nx * ny):
            raise ValueError(f"initial_conditions returned {vals.shape}, expected ({info['n_q']}, {nx * ny})")
        Q = vals.reshape(info["n_q"], ny, nx).copy()
    return Q, A
