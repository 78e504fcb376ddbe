"""Golden fixture for the plotfile writer (zoomy_amrex_b200/plotfile.py).

Writes a two-level, multi-box plotfile with the writer, then reads it back
with the reference's own plotfile reader (deliverable.py:33-129 of the
zoomy-amrex tree: read_levels, which its tests and its VTK conversion use)
and stores what that reader returned plus the SHA-256 of every file the writer
produced. tests/test_plotfile.py regenerates the same plotfile and requires
the same bytes and, through our reader, the same arrays.

deliverable.py imports matplotlib at module level for its figures; the
reader functions do not use it, so the module is loaded with stand-in
matplotlib modules.

    python tests/golden/make_plotfile_golden.py [/path/to/zoomy-amrex]
"""
import hashlib
import importlib.util
import pathlib
import sys
import tempfile
import types

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))


def sample_levels():
    """The deterministic two-level case the fixture pins."""
    from zoomy_amrex_b200.plotfile import LevelData, PatchData
    rng = np.random.default_rng(7)
    ncomp = 11
    L0 = LevelData((0, 0), (23, 15), (0.5, 0.75),
                   [PatchData(rng.standard_normal((ncomp, 16, 12)), (0, 0)),
                    PatchData(rng.standard_normal((ncomp, 16, 12)), (12, 0))], step=3)
    L1 = LevelData((0, 0), (47, 31), (0.25, 0.375),
                   [PatchData(rng.standard_normal((ncomp, 8, 10)), (6, 4)),
                    PatchData(rng.standard_normal((ncomp, 6, 16)), (20, 14))], step=3)
    return [L0, L1], ncomp


def write_sample(out_dir):
    from zoomy_amrex_b200.plotfile import component_names, write_plotfile
    levels, ncomp = sample_levels()
    return write_plotfile(pathlib.Path(out_dir) / "plt_golden00003", levels, component_names(4, 7),
                          0.125, (0.0, 0.0), (12.0, 12.0), [2])


def file_hashes(plt):
    plt = pathlib.Path(plt)
    return {str(f.relative_to(plt)): hashlib.sha256(f.read_bytes()).hexdigest()
            for f in sorted(plt.rglob("*")) if f.is_file()}


def load_reference_reader(root):
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.patches"):
        m = types.ModuleType(name)
        m.use = lambda *a, **k: None
        m.Rectangle = object
        sys.modules.setdefault(name, m)
    spec = importlib.util.spec_from_file_location("ref_deliverable", pathlib.Path(root) / "deliverable.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main(root):
    ref = load_reference_reader(root)
    with tempfile.TemporaryDirectory() as tmp:
        plt = write_sample(tmp)
        levels, H = ref.read_levels(plt)
        arrays = {}
        for lev, ld in enumerate(levels):
            arrays[f"L{lev}_arr"] = ld["arr"]
            arrays[f"L{lev}_ext"] = np.array(ld["ext"])
            arrays[f"L{lev}_boxes"] = np.array(ld["boxes"])
            arrays[f"L{lev}_ref"] = np.array(ld["ref"])
        arrays["names"] = np.array(H["names"])
        arrays["prob_lo"] = np.array(H["prob_lo"])
        arrays["prob_hi"] = np.array(H["prob_hi"])
        arrays["refs"] = np.array(H["refs"])
        hashes = file_hashes(plt)
        arrays["files"] = np.array(sorted(hashes))
        arrays["sha256"] = np.array([hashes[k] for k in sorted(hashes)])
    np.savez(HERE / "plotfile_ref_read.npz", **arrays)
    print({k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference tree>")
    main(sys.argv[1])
