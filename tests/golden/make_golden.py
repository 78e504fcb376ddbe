"""Regenerate the golden fixtures in this directory from the reference's own
golden data (tests/refs/*.npz in the zoomy-amrex tree).

The reference stores each golden as the final (Q, Qaux) of a run written to a
plotfile; 1-D runs keep a singleton y axis, and the numpy-parity goldens keep
Q without it. Here every array is normalised to (n_comp, ny, nx) and saved
uncompressed, with the measured numpy-parity numbers kept alongside.

    python tests/golden/make_golden.py [/path/to/zoomy-amrex]
"""
import pathlib
import sys

import numpy as np

NAMES = ["stoker_wet", "ritter_dry", "wb_lake", "swe_2d", "parallel_2rank",
         "parity_numpy_n100", "parity_numpy_n200"]


def main(root):
    src = pathlib.Path(root) / "tests" / "refs"
    out = pathlib.Path(__file__).resolve().parent
    for name in NAMES:
        d = np.load(src / f"{name}.npz")
        arrays = {}
        for k in d.files:
            a = np.asarray(d[k], dtype=np.float64)
            if k in ("Q", "Qaux"):
                if a.ndim == 2:            # (n, nx): 1-D run without the y axis
                    a = a[:, None, :]
                assert a.ndim == 3, (name, k, a.shape)
            arrays[k] = a
        np.savez(out / f"{name}.npz", **arrays)
        print(name, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference tree>")
    main(sys.argv[1])
