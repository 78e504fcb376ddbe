"""The reference's test suite (tests/test_swe_*.py, test_wb_lake_at_rest.py,
test_parity_numpy.py, test_parallel_two_ranks.py), run through this package's
public entry points (HyperbolicSolver.solve / run_case) on the GPU and checked
the way the reference checks itself: np.allclose against the golden (Q, Qaux)
(tests/refs.py:301-312) plus each test's physical assertions."""
import pathlib

import numpy as np
import pytest

from cases import CFL_1D, CFL_2D, GOLDEN_CASES, gaussian_pulse_2d, lake_at_rest_ic, ritter_ic, stoker_ic
from zoomy_amrex_b200.models import SME, SWE
from zoomy_amrex_b200.run_case import run_case
from zoomy_amrex_b200.solvers import HyperbolicSolver

pytestmark = pytest.mark.gpu
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def check(name, Q, Qaux):   # tests/refs.py:check
    ref = np.load(GOLDEN / f"{name}.npz")
    assert np.allclose(Q, ref["Q"]), f"{name}.Q: max|diff| {np.abs(Q - ref['Q']).max():.3e}"
    assert np.allclose(Qaux, ref["Qaux"]), f"{name}.Qaux: max|diff| {np.abs(Qaux - ref['Qaux']).max():.3e}"


def march(model, settings, t_end, cfl):
    r = run_case(model, dict(settings, time_end=t_end, cfl=cfl), return_result=True)
    return r.Q, r.Qaux


ONE_D = {"dimension": 1, "domain": [0.0, 10.0], "n_cells": 100, "spatial_order": 1,
         "output_snapshots": 1, "max_level": 0}


def test_stoker_wet(cuda):
    Q, Qaux = march(SME(level=0, dimension=2, bc="swashes", initial_conditions=stoker_ic), ONE_D, 1.0, CFL_1D)
    assert np.isfinite(Q).all()
    assert Q[1].min() > 0.0
    assert np.abs(Q[2]).max() > 0.0
    check("stoker_wet", Q, Qaux)


def test_ritter_dry(cuda):
    Q, Qaux = march(SME(level=0, dimension=2, bc="swashes", initial_conditions=ritter_ic), ONE_D, 1.0, CFL_1D)
    assert np.isfinite(Q).all()
    assert Q[1].min() >= 0.0
    assert Q[1].max() > 0.0
    check("ritter_dry", Q, Qaux)


def test_lake_at_rest_over_bump(cuda):
    Q, Qaux = march(SME(level=0, dimension=2, bc="wall", initial_conditions=lake_at_rest_ic),
                    dict(ONE_D, well_balanced=True), 1.0, CFL_1D)
    eta = Q[0] + Q[1]
    u = Q[2] / np.maximum(Q[1], 1e-300)
    assert np.isfinite(Q).all()
    assert np.abs(eta - eta.mean()).max() < 1e-12
    assert np.abs(u).max() < 1e-12
    check("wb_lake", Q, Qaux)


def test_swe_2d_pulse(cuda, tmp_path):
    """HyperbolicSolver.solve returns the run's .pvd path, as the reference's
    does (solvers.py:120-124 -> run_case.py:426); the last data set's cell
    data holds the golden state and aux."""
    from zoomy_amrex_b200.vtk import read_pvd, read_vtu
    solver = HyperbolicSolver(CFL=CFL_2D, order=1, well_balanced=False)
    path = solver.solve(SME(level=0, dimension=3, bc="extrapolation", initial_conditions=gaussian_pulse_2d),
                        {"domain": [-1.0, 1.0, -1.0, 1.0], "n_cells": [32, 32]},
                        {"time_end": 0.1, "output": {"snapshots": 1, "directory": str(tmp_path)}})
    assert isinstance(path, str) and path.endswith(".pvd") and pathlib.Path(path).is_file()
    sets = read_pvd(path)
    assert sets and abs(sets[-1][0] - 0.1) < 1e-12
    d = read_vtu(sets[-1][2])
    assert d["Points"].shape == (33 * 33, 3)
    Q = np.stack([d[n].reshape(32, 32) for n in ("b", "h", "hu", "hv")])
    Qaux = np.stack([d[f"var{c}"].reshape(32, 32) for c in range(4, 11)])
    assert np.isfinite(Q).all() and Q[1].min() > 0.0
    assert np.abs(Q[2]).max() > 0.0 and np.abs(Q[3]).max() > 0.0
    check("swe_2d", Q, Qaux)
    with pytest.raises(ValueError, match="directory"):
        solver.solve(SME(level=0, dimension=3), {"domain": [-1.0, 1.0, -1.0, 1.0], "n_cells": [8, 8]},
                     {"time_end": 0.1})


@pytest.mark.parametrize("n_cells", [100, 200])
def test_numpy_parity_goldens(cuda, n_cells):
    Q, Qaux = march(SME(level=0, dimension=2, bc="swashes", initial_conditions=stoker_ic),
                    dict(ONE_D, n_cells=n_cells), 0.5, CFL_1D)
    check(f"parity_numpy_n{n_cells}", Q, Qaux)


def test_two_rank_golden_and_box_invariance(cuda):
    """The reference asserts 1 rank == 2 ranks bitwise; one GPU level is one
    box, and the result equals the 2-rank golden bitwise."""
    Q, Qaux = march(SME(level=0, dimension=2, bc="swashes", initial_conditions=stoker_ic),
                    dict(ONE_D, n_cells=128), 0.5, CFL_1D)
    ref = np.load(GOLDEN / "parallel_2rank.npz")
    assert np.abs(Q - ref["Q"]).max() == 0.0
    assert np.abs(Qaux - ref["Qaux"]).max() == 0.0


def test_plotfiles_like_evolve(cuda, oracle, tmp_path):
    """run_case with an output directory writes AMReX plotfiles where the
    reference's Evolve does (ZoomyAmr.cpp:782-812): at the start of the first
    step with time >= k * time_end / snapshots, and after the last step; the
    last plotfile holds the golden (Q, Qaux), read the way the reference's
    tests read it (tests/conftest.py:101-108)."""
    from cases import golden_setup
    from zoomy_amrex_b200.plotfile import read_plotfile
    model = SME(level=0, dimension=2, bc="swashes", initial_conditions=stoker_ic)
    settings = dict(ONE_D, time_end=1.0, cfl=CFL_1D, output_snapshots=7)
    r = run_case(model, settings, str(tmp_path), return_result=True)
    plts = sorted(tmp_path.glob("plt_*"))
    assert [p.name for p in plts] == [f"plt_0{k:05d}" for k in range(len(plts))]
    H, levels = read_plotfile(plts[-1])
    arr = levels[0].patches[0].data
    check("stoker_wet", arr[:3], arr[3:])
    # expected write times from the oracle's per-step log
    cfg, Q0, A0 = golden_setup("stoker_wet")
    _, _, n, t_end, log, _ = oracle.run(cfg, Q0, A0)
    plot_dt = 1.0 / 7
    expect, nxt, t = [], 0.0, 0.0
    for s in range(n):
        if t >= nxt:
            expect.append(t)
            nxt += plot_dt
        t = log[s, 1]
    expect.append(t)
    got = [read_plotfile(p)[0]["time"] for p in plts]
    assert got == expect
    assert r.plotfiles and pathlib.Path(r.plotfiles[-1]) == plts[-1]


def test_run_case_fp32_precision_follows_fp64(cuda):
    """settings['precision'] = 'fp32' runs the FP32 chosen form through the
    same entry point; it follows the FP64 run to FP32 accuracy."""
    def ic(x):
        b = 0.3 * np.exp(-((x[0] - 4.0) ** 2 + (x[1] - 6.0) ** 2) / 2.0)
        h = np.maximum(np.where(x[0] < 5.0, 1.5, 1.0) - b, 0.0)
        return np.array([b, h, 0 * h, 0 * h])
    model = SWE(2, "wall", ic, parameters={"n_m": 0.03})
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[64, 48], spatial_order=2, cfl=0.45, time_end=0.3,
             well_balanced=True, implicit_source=True, output_snapshots=1)
    r64 = run_case(model, dict(s), return_result=True)
    r32 = run_case(model, dict(s, precision="fp32"), return_result=True)
    assert abs(r32.time - r64.time) < 1e-9 and abs(r32.steps - r64.steps) <= 1
    assert np.abs(r32.Q[1] - r64.Q[1]).max() < 1e-4


def test_run_case_max_level_runs_the_amr_hierarchy(cuda, tmp_path):
    """max_level > 0 (the reference's AMR deck: ratio 2, regrid every 2 coarse
    steps, tagging.threshold 0.02 with its ErrorEst) runs the AMR hierarchy and
    writes multi-level plotfiles at the output times; the base level conserves
    mass up to the coarse-fine flux mismatch."""
    from zoomy_amrex_b200.plotfile import read_plotfile
    def ic(x):
        b = 0.3 * np.exp(-((x[0] - 4.0) ** 2 + (x[1] - 6.0) ** 2) / 2.0)
        h = np.maximum(np.where(x[0] < 5.0, 1.5, 1.0) - b, 0.0)
        return np.array([b, h, 0 * h, 0 * h])
    model = SWE(2, "wall", ic, parameters={"n_m": 0.03})
    s = dict(dimension=2, domain=[0, 10, 0, 10], n_cells=[128, 128], spatial_order=2, cfl=0.45, time_end=0.2,
             well_balanced=True, implicit_source=True, output_snapshots=4, max_level=2, tag_b_max=0.2)
    r = run_case(model, s, str(tmp_path), return_result=True)
    plts = sorted(tmp_path.glob("plt_*"))
    assert len(plts) >= 5 and r.plotfiles[-1] == str(plts[-1])
    from zoomy_amrex_b200.vtk import read_pvd
    parts = read_pvd(r.path)
    assert {p for _, p, _ in parts} >= {0, 1} and all(pathlib.Path(f).is_file() for _, _, f in parts)
    head, levels = read_plotfile(plts[-1])
    print(f"[run_case amr] {r.steps} coarse steps to t = {r.time}, levels {len(levels)}, "
          f"patches {[len(L.patches) for L in levels]}")
    assert abs(r.time - 0.2) < 1e-12 and head["finest_level"] >= 1
    assert np.isfinite(r.Q).all()
    dx = 10.0 / 128
    m0 = ic(np.meshgrid((np.arange(128) + 0.5) * dx, (np.arange(128) + 0.5) * dx))[1].sum()
    assert abs(r.Q[1].sum() - m0) / m0 < 1e-3
