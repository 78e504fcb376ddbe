"""Build libzoomyfv.so for sm_100a with nvcc (in-tree, no JIT cache).

    python -m zoomy_amrex_b200.build [--verbose]

The library is written to zoomy_amrex_b200/lib/libzoomyfv.so. FMA contraction
is disabled (--fmad=false) for the FP64 plain form, as in the reference's CUDA
build (build.py:33-41 of zoomy-amrex), so those kernels evaluate the same IEEE
operations as the CPU build of the same expressions; the FP32 chosen form
(zoomy_fv32.cu) is compiled with FMA.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libzoomyfv.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# (source, extra flags): the FP64 plain form keeps FMA contraction off so its
# arithmetic is bitwise the CPU build's; the FP32 chosen form uses FMA and the
# hardware's approximate FP32 division / square root (its FP64 parts are
# unaffected by these flags); the adjoint (FP64, checked to tolerances) uses FMA.
FP32_FLAGS = ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"]
N_FP32_SHAPES = 13   # kNumVariants in csrc/fv32_shapes.H
# (source, extra flags, object stem). The FP32 strip shapes are one source
# compiled once per shape (-DZFV32_SHAPE=k) so that they build in parallel.
SOURCES = ([("zoomy_fv.cu", ["--fmad=false"], "zoomy_fv"),
            ("zoomy_fv64_swe.cu", ["--fmad=false"], "zoomy_fv64_swe"),
            ("zoomy_fv64_sme.cu", ["--fmad=false"], "zoomy_fv64_sme"),
            ("zoomy_fv32.cu", FP32_FLAGS, "zoomy_fv32"),
            ("zoomy_fv32_tile.cu", FP32_FLAGS, "zoomy_fv32_tile"),
            ("zoomy_adj.cu", ["--fmad=true"], "zoomy_adj")]
           + [("zoomy_fv32_shape.cu", FP32_FLAGS + [f"-DZFV32_SHAPE={k}"], f"zoomy_fv32_shape{k}")
              for k in range(N_FP32_SHAPES)])


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def _deps():
    files = [p for p in CSRC.rglob("*") if p.suffix in (".cu", ".cuh", ".H", ".h")]
    files.append(INCLUDE / "zoomy_fv.h")
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in _deps())


def _reap(running) -> None:
    """Wait for the first of the running compilers to finish; raise if it failed."""
    import time
    while True:
        for k, (p, cmd) in enumerate(running):
            rc = p.poll()
            if rc is not None:
                running.pop(k)
                if rc != 0:
                    for q, _ in running:
                        q.wait()
                    raise subprocess.CalledProcessError(rc, cmd)
                return
        time.sleep(0.2)


def build(verbose: bool = False, force: bool = False) -> pathlib.Path:
    if not force and up_to_date():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs, jobs = [], []
    for src, flags, stem in SOURCES:
        obj = LIB_DIR / (stem + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", *flags, "-std=c++17",
               "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(CSRC / "amrex_compat"),
               "-I", str(CSRC / "models"), "-I", str(INCLUDE), "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        jobs.append((cmd, obj))
    # at most one compiler per core; the longest units first
    width = max(1, os.cpu_count() or 1)
    running = []
    for cmd, obj in jobs:
        while len(running) >= width:
            _reap(running)
        running.append((subprocess.Popen(cmd), cmd))
        objs.append(str(obj))
    while running:
        _reap(running)
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
