"""``run_case`` — run a model on a structured single-level grid on the GPU.

Same entry shape as zoomy_amrex.run_case.run_case (zoomy_amrex/run_case.py:346-426):
``run_case(model, settings, output_dir)``. The reference generates C++,
compiles it, runs it as a subprocess and converts AMReX plotfiles to VTK; here
the model family is precompiled into libzoomyfv.so and the march runs
in-process on PyTorch CUDA tensors. The final state is returned. When
``output_dir`` is given, AMReX plotfiles of (Q, aux) are written there as the
reference's Evolve writes them (ZoomyAmr.cpp:782-812, 821-882): at the start
of the first step with time >= next plot time, next plot time advancing by
time_end / output_snapshots, and once more after the last step, named
plt_<identifier><plot index:05d>; plus ``final.npz`` with the per-step
dt/time/mass log.
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
    plotfiles: list | None = None


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
    out = pathlib.Path(output_dir) if output_dir is not None else None
    plot_dt = float(settings.get("time_end", 1.0)) / max(1, int(settings.get("output_snapshots", 10)))
    identifier = str(settings.get("identifier", "0"))
    plots = []

    def write_plot(index, st):
        from .plotfile import write_level_state
        Qp = lev.state64().cpu().numpy()
        plots.append(write_level_state(out, identifier, index, st["time"], Qp, lev.aux.cpu().numpy(),
                                       lo, hi))

    if cfg.implicit_source and cfg.implicit_global:
        use_graph = False            # the Newton-Krylov iteration reads norms on the host
    try:
        lev.begin()
        if out is not None:
            out.mkdir(parents=True, exist_ok=True)
        next_plot, plot_index, last_step = 0.0, 0, -1
        st = lev.status()
        while not st["done"]:
            n = chunk
            if out is not None:
                if st["time"] >= next_plot:
                    write_plot(plot_index, st)
                    next_plot += plot_dt
                    plot_index += 1
                # stop on the step boundary the reference writes at: single
                # steps near the next plot time, shorter chunks before it
                gap = next_plot - st["time"]
                if st["dt"] > 0 and gap < chunk * st["dt"]:
                    n = 1 if gap <= 4 * st["dt"] else max(1, int(gap / st["dt"] / 2))
            if use_graph and n == chunk:
                if lev._graph is None:
                    lev.capture(chunk)
                lev.replay()
            else:
                lev.evolve(n)
            st = lev.status()
            if on_progress is not None:
                on_progress(st["step"], st["time"], st["dt"])
            if not st["done"] and st["step"] <= last_step:   # the device did not advance
                raise RuntimeError(f"run_case: no progress at step {st['step']} (status {st})")
            last_step = st["step"]
        if out is not None:
            write_plot(plot_index, st)
        Q = lev.state64().cpu().numpy()
        A = lev.aux.cpu().numpy()
        log = lev.log()
    finally:
        lev.close()
    res = CaseResult(Q=Q, Qaux=A, time=st["time"], steps=st["step"], log=log)
    res.plotfiles = plots
    if out is not None:
        p = out / "final.npz"
        np.savez(p, Q=Q, Qaux=A, time=res.time, steps=res.steps, log=log)
        res.path = str(p)
    return res
