"""``HyperbolicSolver`` — the reference's solver front end, on the GPU.

Mirrors zoomy_amrex.solvers.HyperbolicSolver (zoomy_amrex/solvers.py:104-124):
the same parameters (CFL, order, well_balanced, positivity) and the same
``solve(model, mesh, settings)`` call, where ``mesh`` is a descriptor
``{"domain": [...], "n_cells": [...]}`` and ``settings`` is structured
(``time_end``, ``output.directory`` (required, as in the reference's
``_output_dir``, solvers.py:96-100), ``max_level``). ``solve`` returns the
run's ``.pvd`` path like the reference; ``run`` takes the same arguments and
returns the in-memory ``CaseResult`` (``output.directory`` optional there).
The reference's ``param.Parameterized`` base is replaced by a dataclass
(``param`` is not a dependency here); bounds are checked the same way.
"""
from __future__ import annotations

from dataclasses import dataclass

from .run_case import CaseResult, run_case


def _get(obj, dotted, default=None):
    """Dotted lookup through dicts / attribute objects (solvers.py:137-146)."""
    cur = obj
    for key in dotted.split("."):
        if cur is None:
            return default
        cur = cur.get(key) if isinstance(cur, dict) else getattr(cur, key, None)
    return default if cur is None else cur


def _mesh_domain_ncells(mesh, settings):
    if isinstance(mesh, dict):
        return mesh["domain"], mesh["n_cells"]
    raise NotImplementedError("mesh files (.msh) are not supported; pass {'domain', 'n_cells'}")


@dataclass
class HyperbolicSolver:
    """Explicit finite-volume march for hyperbolic models (SWE / SME)."""

    CFL: float = 0.45
    order: int = 1
    well_balanced: bool = True
    positivity: str = "none"

    def __post_init__(self):
        if not (0.0 <= self.CFL <= 1.0):
            raise ValueError(f"CFL must be in [0, 1], got {self.CFL}")
        if self.order not in (1, 2):
            raise ValueError(f"order must be 1 or 2, got {self.order}")
        if self.positivity not in ("none", "mood"):
            raise ValueError(f"positivity must be 'none' or 'mood', got {self.positivity!r}")

    def _legacy_settings(self, mesh, settings) -> dict:
        domain, n_cells = _mesh_domain_ncells(mesh, settings)
        nc = list(n_cells) if isinstance(n_cells, (list, tuple)) else [n_cells]
        dim = 1 if len(domain) == 2 else 2
        s = {"dimension": dim, "domain": list(domain), "n_cells": nc,
             "time_end": _get(settings, "time_end", 1.0),
             "output_snapshots": _get(settings, "output.snapshots", 10),
             "max_level": _get(settings, "max_level", 0)}
        for k in ("dtmax", "dtmin", "max_step", "params", "implicit_source", "implicit_global", "precision",
                  "max_grid_size"):
            v = _get(settings, k)
            if v is not None:
                s[k] = v
        return s

    def _settings(self, mesh, settings) -> dict:
        s = self._legacy_settings(mesh, settings)
        s.update(cfl=self.CFL, spatial_order=self.order, well_balanced=self.well_balanced,
                 positivity=self.positivity)
        return s

    def solve(self, model, mesh, settings, on_progress=None) -> str:
        """Run and return the path of the run's ``.pvd`` (solvers.py:120-124)."""
        d = _get(settings, "output.directory")
        if d is None:
            raise ValueError("solve: settings['output']['directory'] is required")
        return run_case(model, self._settings(mesh, settings), d, on_progress=on_progress)

    def run(self, model, mesh, settings, on_progress=None) -> CaseResult:
        """``solve`` returning the final state, time, step count and log in memory."""
        return run_case(model, self._settings(mesh, settings), _get(settings, "output.directory"),
                        on_progress=on_progress, return_result=True)
