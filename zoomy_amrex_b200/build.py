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
SOURCES = [("zoomy_fv.cu", ["--fmad=false"]),
           ("zoomy_fv32.cu", ["--fmad=true", "-ftz=true", "-prec-div=false", "-prec-sqrt=false"]),
           ("zoomy_adj.cu", ["--fmad=true"])]


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


def build(verbose: bool = False, force: bool = False) -> pathlib.Path:
    if not force and up_to_date():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs, jobs = [], []
    for src, flags in SOURCES:
        obj = LIB_DIR / (pathlib.Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", *flags, "-std=c++17",
               "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(CSRC / "amrex_compat"),
               "-I", str(CSRC / "models"), "-I", str(INCLUDE), "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        jobs.append((cmd, obj))
    procs = [subprocess.Popen(cmd) for cmd, _ in jobs]
    for p, (cmd, obj) in zip(procs, jobs):
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, cmd)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
