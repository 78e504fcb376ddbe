"""``run_case`` — run a model on a structured grid on the GPU (one level, or an
AMR hierarchy when ``max_level > 0``).

Same entry shape as zoomy_amrex.run_case.run_case (zoomy_amrex/run_case.py:346-426):
``run_case(model, settings, output_dir)`` returning the path of the run's
ParaView collection ``<output_dir>/simulation.pvd``. The reference generates
C++, compiles it, runs it as a subprocess and converts AMReX plotfiles to VTK;
here the model family is precompiled into libzoomyfv.so and the march runs
in-process on PyTorch CUDA tensors. AMReX plotfiles of (Q, aux) are written
into ``output_dir`` as the reference's Evolve writes them
(ZoomyAmr.cpp:782-812, 821-882): at the start of the first step with
time >= next plot time, next plot time advancing by time_end /
output_snapshots, and once more after the last step, named
plt_<identifier><plot index:05d>; they are converted to ``simulation.pvd`` +
``vtk/*.vtu`` like the reference's ``_plotfiles_to_vtk``
(run_case.py:128-178), and ``final.npz`` holds the final state and the
per-step dt/time/mass log. ``return_result=True`` returns the in-memory
``CaseResult`` instead (then ``output_dir`` may be None: nothing is written).
"""
from __future__ import annotations

import pathlib
from dataclasses import dataclass

import numpy as np

from .models import SWE, initial_state
from .settings import config_from_settings, grid


def _precision(settings: dict) -> int:
    """settings['precision']: "fp64" (default; the reference's arithmetic) or
    "fp32" (the FP32 chosen form: 2-D SWE at order 1 or 2, 2-D SME level 2)."""
    from ._abi import ZFV_PREC_FP32, ZFV_PREC_FP64
    p = str(settings.get("precision", "fp64")).lower()
    if p not in ("fp64", "fp32"):
        raise ValueError(f"precision must be 'fp64' or 'fp32', got {p!r}")
    return ZFV_PREC_FP32 if p == "fp32" else ZFV_PREC_FP64


@dataclass
class CaseResult:
    Q: np.ndarray          # (n_q, ny, nx) final state
    Qaux: np.ndarray       # (n_aux, ny, nx) final aux
    time: float
    steps: int
    log: np.ndarray        # (steps, 3): dt, time, mass per step
    path: str | None = None      # the .pvd written into output_dir (None without one)
    plotfiles: list | None = None


def run_case(model: SWE, settings: dict, output_dir: str | None = None, on_progress=None, *,
             return_result: bool = False, device: str = "cuda:0", use_graph: bool = True,
             chunk: int = 64):
    """March ``model`` to settings['time_end'] (or settings['max_step'] steps).

    Returns the ``.pvd`` path (a str), as the reference does, or the
    ``CaseResult`` when ``return_result`` is set."""
    if output_dir is None and not return_result:
        raise ValueError("run_case: output_dir is required (the run's .pvd and plotfiles are written there); "
                         "pass return_result=True for the in-memory result only")
    res = _run(model, settings, output_dir, on_progress, device, use_graph, chunk)
    if output_dir is not None:
        res.path = _to_vtk(model, res, output_dir)
    return res if return_result else res.path


def _to_vtk(model, res: CaseResult, output_dir) -> str:
    from .vtk import plotfiles_to_vtk
    return plotfiles_to_vtk(res.plotfiles, model.state_names(), output_dir, model.dimension)


def _run(model, settings, output_dir, on_progress, device, use_graph, chunk) -> CaseResult:
    from .level import Level   # needs torch + the CUDA library

    if settings.get("mpi_ranks", 1) not in (None, 1):
        raise NotImplementedError("one level runs on one GPU; mpi_ranks must be 1")
    riemann = settings.get("riemann")
    if riemann is not None and getattr(riemann, "__name__", riemann) != "NonconservativeRusanov":
        raise NotImplementedError(f"riemann={riemann!r}: the flux built here is the printer's default "
                                  "NonconservativeRusanov (zoomy_core's other solvers are not part of the reference)")
    if int(settings.get("max_level", 0) or 0) > 0:
        return _run_case_amr(model, settings, output_dir, on_progress, device)
    precision = _precision(settings)
    cfg = config_from_settings(model, settings, precision=precision)
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
        np.savez(out / "final.npz", Q=Q, Qaux=A, time=res.time, steps=res.steps, log=log)
    return res


def _run_case_amr(model: SWE, settings: dict, output_dir, on_progress, device) -> CaseResult:
    """max_level > 0: the AMR hierarchy (amr.AmrHierarchy, FP32 form) with the
    deck the reference's run_case writes for it (build.py:96-119: ref ratio 2,
    regrid every 2 coarse steps, tagging.threshold 0.02 with its ErrorEst
    criterion, optional tagging.b_max, boxes up to max_grid_size 64). Blocks
    are the largest power of two <= max_grid_size (>= 8) dividing both grid
    sides. Plotfiles of all levels are written at the reference's output
    times; the result holds the base level."""
    from ._abi import ZFV_PREC_FP32
    from .amr import AmrHierarchy
    if model.dimension != 2 or int(settings.get("spatial_order", 1)) != 2:
        raise NotImplementedError("AMR runs the FP32 form: 2-D SWE at spatial_order 2")
    if str(settings.get("positivity", "none")) == "mood" or settings.get("clamp_positivity"):
        raise NotImplementedError("AMR runs the FP32 form, which has no MOOD / clamp_positivity")
    cfg = config_from_settings(model, settings, precision=ZFV_PREC_FP32)
    _, nx, ny, lo, hi = grid(settings)
    Q0, _ = initial_state(model, nx, ny, lo, hi)
    mgs = int(settings.get("max_grid_size", 64))
    B = next((b for b in (64, 32, 16, 8) if b <= mgs and nx % b == 0 and ny % b == 0), None)
    if B is None:
        raise ValueError(f"AMR needs both grid sides ({nx} x {ny}) divisible by a block side of 8 .. "
                         f"{min(64, mgs)}")
    hier = AmrHierarchy(cfg, Q0, max_level=int(settings["max_level"]), B=B,
                        threshold=float(settings.get("tag_threshold", 0.02)), regrid_int=2, device=device,
                        tag="reference", tag_b_max=float(settings.get("tag_b_max", 1.0e30)))
    out = pathlib.Path(output_dir) if output_dir is not None else None
    tend = float(settings.get("time_end", 1.0))
    plot_dt = tend / max(1, int(settings.get("output_snapshots", 10)))
    identifier = str(settings.get("identifier", "0"))
    max_step = cfg.max_step
    plots = []
    try:
        if out is not None:
            out.mkdir(parents=True, exist_ok=True)
        next_plot, index = 0.0, 0
        t = hier.time
        while t < tend and (max_step < 0 or hier.steps < max_step):
            if out is not None and t >= next_plot:
                plots.append(hier.write_plotfile(out, identifier, index))
                next_plot += plot_dt
                index += 1
            hier.step()
            t_new = hier.time
            if on_progress is not None:
                on_progress(hier.steps, t_new, t_new - t)
            if not t_new > t:
                raise RuntimeError(f"run_case (AMR): no progress at coarse step {hier.steps}, time {t_new}")
            t = t_new
        if out is not None:
            plots.append(hier.write_plotfile(out, identifier, index))
        Q = hier.level_state(0)
        L0 = hier.levels[0]
        A = np.zeros((L0.batch.aux[0].shape[0], L0.ny, L0.nx))
        for (bx, by, nbx, nby), a in zip(L0.patches, L0.batch.aux):
            A[:, by * B:(by + nby) * B, bx * B:(bx + nbx) * B] = a.cpu().numpy()
        steps = hier.steps
    finally:
        hier.close()
    res = CaseResult(Q=Q, Qaux=A, time=t, steps=steps, log=np.zeros((0, 3)))
    res.plotfiles = plots
    if out is not None:
        np.savez(out / "final.npz", Q=Q, Qaux=A, time=t, steps=steps)
    return res
