"""AMReX plotfile writer/reader against what the reference's reader returns."""
import hashlib
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))

from make_plotfile_golden import file_hashes, sample_levels, write_sample  # noqa: E402
from zoomy_amrex_b200.plotfile import read_plotfile, write_level_state  # noqa: E402


def test_writer_bytes_are_the_ones_the_reference_reader_accepted(tmp_path):
    g = np.load(HERE / "golden" / "plotfile_ref_read.npz")
    plt = write_sample(tmp_path)
    h = file_hashes(plt)
    assert sorted(h) == list(g["files"])
    assert [h[k] for k in sorted(h)] == list(g["sha256"])


def test_reader_matches_reference_reader(tmp_path):
    g = np.load(HERE / "golden" / "plotfile_ref_read.npz")
    H, levels = read_plotfile(write_sample(tmp_path))
    assert H["names"] == list(g["names"])
    assert H["ref_ratios"] == list(g["refs"])
    for lev, L in enumerate(levels):
        ilo, jlo, nx, ny = g[f"L{lev}_ext"]
        dense = np.full((len(H["names"]), ny, nx), np.nan)
        for P in L.patches:
            c, py, px = P.data.shape
            dense[:, P.lo[1] - jlo:P.lo[1] - jlo + py, P.lo[0] - ilo:P.lo[0] - ilo + px] = P.data
        np.testing.assert_array_equal(dense, g[f"L{lev}_arr"])
    src, _ = sample_levels()
    for L, S in zip(levels, src):
        for P, Q in zip(L.patches, S.patches):
            assert np.array_equal(P.data, Q.data) and tuple(P.lo) == tuple(Q.lo)


def test_level_state_plotfile_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    Q = rng.standard_normal((4, 9, 13))
    A = rng.standard_normal((7, 9, 13))
    p = write_level_state(tmp_path, "dam", 12, 0.5, Q, A, (0.0, 0.0), (1.0, 2.0))
    assert pathlib.Path(p).name == "plt_dam00012"
    H, levels = read_plotfile(p)
    assert H["names"][:4] == ["var0", "var1", "var2", "var3"] and H["names"][4] == "aux0"
    assert H["time"] == 0.5 and H["finest_level"] == 0
    d = levels[0].patches[0].data
    assert np.array_equal(d[:4], Q) and np.array_equal(d[4:], A)


def test_plotfiles_convert_to_pvd_and_vtu(tmp_path):
    """The run's ParaView output (run_case.py:128-178 of the reference): one
    .vtu per plotfile and level, cell data by state name then var<c>, listed
    in simulation.pvd with the plotfile times."""
    from zoomy_amrex_b200.plotfile import write_level_state
    from zoomy_amrex_b200.vtk import plotfiles_to_vtk, read_pvd, read_vtu
    rng = np.random.default_rng(3)
    Q, A = rng.random((4, 5, 7)), rng.random((7, 5, 7))
    p1 = write_level_state(tmp_path, "0", 0, 0.0, Q, A, (0.0, 0.0), (7.0, 5.0))
    p2 = write_level_state(tmp_path, "0", 1, 0.5, 2 * Q, A, (0.0, 0.0), (7.0, 5.0))
    pvd = plotfiles_to_vtk([p1, p2], ["b", "h", "hu", "hv"], tmp_path, 2)
    assert pvd == str(tmp_path / "simulation.pvd")
    sets = read_pvd(pvd)
    assert [(t, part) for t, part, _ in sets] == [(0.0, 0), (0.5, 0)]
    v = read_vtu(sets[1][2])
    assert v["Points"].shape == (6 * 8, 3) and v["Points"][9, 0] == 1.0 and v["Points"][9, 1] == 1.0
    assert np.array_equal(v["h"].reshape(5, 7), 2 * Q[1])
    assert np.array_equal(v["var6"].reshape(5, 7), A[2])
    assert np.array_equal(v["connectivity"][:4], [0, 1, 9, 8])
