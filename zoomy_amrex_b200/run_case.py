"""``run_case`` — run a model on a structured single-level grid on the GPU.

Same entry shape as zoomy_amrex.run_case.run_case (zoomy_amrex/run_case.py:346-426):
``run_case(model, settings, output_dir)``. The reference generates C++,
compiles it, runs it as a subprocess and converts AMReX plotfiles to VTK; here
the model family is precompiled into libzoomyfv.so and the march runs
in-process on PyTorch CUDA tensors. The final state is returned (and, when
``output_dir`` is given, saved to ``<output_dir>/final.npz`` with the per-step
dt/time/mass log).
"""
from __future__ import annotations

import pathlib
from dataclasses import dataclass

import numpy as np

from .models import SWE, initial_state
from .settings import config_from_settings, grid


@dataclass
class CaseResult:
    Q: np.ndarray          # (n_q, ny, nx) final state
    Qaux: np.ndarray       # (n_aux, ny, nx) final aux
    time: float
    steps: int
    log: np.ndarray        # (steps, 3): dt, time, mass per step
    path: str | None = None


def run_case(model: SWE, settings: dict, output_dir: str | None = None, on_progress=None,
             device: str = "cuda:0", use_graph: bool = True, chunk: int = 64) -> CaseResult:
    """March ``model`` to settings['time_end'] (or settings['max_step'] steps)."""
    from .level import Level   # needs torch + the CUDA library

    if settings.get("max_level", 0):
        raise NotImplementedError("adaptive refinement (max_level > 0) is not part of this build")
    if settings.get("mpi_ranks", 1) not in (None, 1):
        raise NotImplementedError("one level runs on one GPU; mpi_ranks must be 1")
    cfg = config_from_settings(model, settings)
    _, nx, ny, lo, hi = grid(settings)
    Q0, A0 = initial_state(model, nx, ny, lo, hi)
    lev = Level(cfg, Q0, A0, device=device)
    try:
        lev.begin()
        while True:
            if use_graph:
                if lev._graph is None:
                    lev.capture(chunk)
                lev.replay()
            else:
                lev.evolve(chunk)
            st = lev.status()
            if on_progress is not None:
                on_progress(st["step"], st["time"], st["dt"])
            if st["done"]:
                break
        Q = lev.Q.cpu().numpy()
        A = lev.aux.cpu().numpy()
        log = lev.log()
    finally:
        lev.close()
    res = CaseResult(Q=Q, Qaux=A, time=st["time"], steps=st["step"], log=log)
    if output_dir is not None:
        out = pathlib.Path(output_dir)
        out.mkdir(parents=True, exist_ok=True)
        p = out / "final.npz"
        np.savez(p, Q=Q, Qaux=A, time=res.time, steps=res.steps, log=log)
        res.path = str(p)
    return res
