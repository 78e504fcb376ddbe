"""AMReX plotfiles (the reference's output format), written and read natively.

The reference's executable writes one plotfile per output time through
amrex::WriteMultiLevelPlotfile (ZoomyAmr.cpp:821-882): components
``var0 .. var{n_q-1}`` (the state Q) then ``aux0 .. aux{n_aux-1}``, no ghost
cells, one directory ``plt_<identifier><step:05d>`` holding a text ``Header``,
and per level ``Level_<l>/Cell_H`` (the MultiFab header) plus
``Level_<l>/Cell_D_00000`` (the boxes' data, each a ``FAB`` line followed by
little-endian float64 values, component-major, x fastest). The reference's
readers (deliverable.py:33-129, used by its tests and its VTK conversion) parse
exactly these files; the layout below follows the published AMReX plotfile
format ("HyperCLaw-V1.1" header, VisMF version 1 MultiFab header).
"""
from __future__ import annotations

import os
import pathlib
import re
from dataclasses import dataclass, field

import numpy as np

_REAL_DESC = "((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))"   # IEEE float64, little-endian


def _box(lo, hi, dim):
    z = ",".join("0" for _ in range(dim))
    return "((" + ",".join(str(v) for v in lo) + ") (" + ",".join(str(v) for v in hi) + ") (" + z + "))"


@dataclass
class PatchData:
    """One box of one level: data (ncomp, ny, nx) with its lower cell index."""
    data: np.ndarray
    lo: tuple


@dataclass
class LevelData:
    domain_lo: tuple
    domain_hi: tuple
    dx: tuple
    patches: list = field(default_factory=list)
    step: int = 0


def plotfile_name(identifier: str, step: int) -> str:
    """ZoomyAmr.cpp:824: Concatenate(Concatenate("plt_", identifier), step, 5)."""
    return f"plt_{identifier}{step:05d}"


def component_names(n_q: int, n_aux: int) -> list[str]:
    return [f"var{n}" for n in range(n_q)] + [f"aux{n}" for n in range(n_aux)]


def write_plotfile(path, levels: list[LevelData], names: list[str], time: float, prob_lo, prob_hi,
                   ref_ratios: list[int] = ()) -> str:
    """Write a (multi-level) 2-D plotfile; returns its path."""
    p = pathlib.Path(path)
    p.mkdir(parents=True, exist_ok=True)
    dim = 2
    ncomp = len(names)
    finest = len(levels) - 1
    lines = ["HyperCLaw-V1.1", str(ncomp), *names, str(dim), repr(float(time)), str(finest),
             " ".join(repr(float(v)) for v in prob_lo[:dim]),
             " ".join(repr(float(v)) for v in prob_hi[:dim]),
             " ".join(str(int(r)) for r in ref_ratios[:finest]),
             " ".join(_box(L.domain_lo, L.domain_hi, dim) for L in levels),
             " ".join(str(int(L.step)) for L in levels)]
    for L in levels:
        lines.append(" ".join(repr(float(d)) for d in L.dx[:dim]))
    lines += ["0", "0"]
    for lev, L in enumerate(levels):
        lines.append(f"{lev} {len(L.patches)} {float(time)!r}")
        lines.append(str(int(L.step)))
        for P in L.patches:
            ny, nx = P.data.shape[1], P.data.shape[2]
            for d, (lo_i, n_i) in enumerate(((P.lo[0], nx), (P.lo[1], ny))):
                x0 = prob_lo[d] + lo_i * L.dx[d]
                lines.append(f"{x0!r} {x0 + n_i * L.dx[d]!r}")
        lines.append(f"Level_{lev}/Cell")
        _write_level(p / f"Level_{lev}", L, ncomp, dim)
    (p / "Header").write_text("\n".join(lines) + "\n")
    return str(p)


def _write_level(d: pathlib.Path, L: LevelData, ncomp: int, dim: int):
    d.mkdir(parents=True, exist_ok=True)
    offsets, boxes, mins, maxs = [], [], [], []
    with open(d / "Cell_D_00000", "wb") as f:
        for P in L.patches:
            data = np.ascontiguousarray(P.data, dtype="<f8")
            if data.shape[0] != ncomp:
                raise ValueError(f"patch has {data.shape[0]} components, expected {ncomp}")
            ny, nx = data.shape[1], data.shape[2]
            lo = tuple(int(v) for v in P.lo[:dim])
            hi = (lo[0] + nx - 1, lo[1] + ny - 1)
            boxes.append(_box(lo, hi, dim))
            offsets.append(f.tell())
            f.write(f"FAB {_REAL_DESC}{_box(lo, hi, dim)} {ncomp}\n".encode())
            f.write(data.tobytes())
            mins.append(data.reshape(ncomp, -1).min(axis=1))
            maxs.append(data.reshape(ncomp, -1).max(axis=1))
    n = len(L.patches)
    out = ["1", "1", str(ncomp), "0", f"({n} 0"]
    out += boxes
    out.append(")")
    out.append(str(n))
    out += [f"FabOnDisk: Cell_D_00000 {o}" for o in offsets]
    out.append("")
    out.append(f"{n},{ncomp}")
    out += ["".join(f"{v!r}," for v in m) for m in mins]
    out.append("")
    out.append(f"{n},{ncomp}")
    out += ["".join(f"{v!r}," for v in m) for m in maxs]
    (d / "Cell_H").write_text("\n".join(out) + "\n")


_BOX_RE = re.compile(r"\(\(([-\d,]+)\) \(([-\d,]+)\)")


def read_plotfile(path):
    """Read a 2-D plotfile: (header dict, [LevelData]) with each box's data."""
    p = pathlib.Path(path)
    lines = (p / "Header").read_text().splitlines()
    ncomp = int(lines[1])
    names = lines[2:2 + ncomp]
    i = 2 + ncomp
    dim = int(lines[i]); i += 1
    time = float(lines[i]); i += 1
    finest = int(lines[i]); i += 1
    prob_lo = [float(v) for v in lines[i].split()]; i += 1
    prob_hi = [float(v) for v in lines[i].split()]; i += 1
    refs = [int(v) for v in lines[i].split()]; i += 1
    doms = _BOX_RE.findall(lines[i]); i += 1
    steps = [int(v) for v in lines[i].split()]; i += 1
    dxs = []
    for _ in range(finest + 1):
        dxs.append(tuple(float(v) for v in lines[i].split())); i += 1
    levels = []
    for lev in range(finest + 1):
        lo = tuple(int(v) for v in doms[lev][0].split(","))
        hi = tuple(int(v) for v in doms[lev][1].split(","))
        L = LevelData(lo, hi, dxs[lev], step=steps[lev])
        ld = p / f"Level_{lev}"
        txt = (ld / "Cell_H").read_text()
        boxes = _BOX_RE.findall(txt)
        fods = re.findall(r"FabOnDisk:\s+(\S+)\s+(\d+)", txt)
        for (a, b), (fname, off) in zip(boxes, fods):
            blo = [int(v) for v in a.split(",")]
            bhi = [int(v) for v in b.split(",")]
            nx, ny = bhi[0] - blo[0] + 1, bhi[1] - blo[1] + 1
            with open(ld / fname, "rb") as f:
                f.seek(int(off))
                f.readline()
                data = np.frombuffer(f.read(8 * ncomp * nx * ny), dtype="<f8").reshape(ncomp, ny, nx)
            L.patches.append(PatchData(data.copy(), tuple(blo)))
        levels.append(L)
    return dict(names=names, dim=dim, time=time, finest_level=finest, prob_lo=prob_lo,
                prob_hi=prob_hi, ref_ratios=refs), levels


def write_level_state(out_dir, identifier: str, step: int, time: float, Q: np.ndarray, aux: np.ndarray,
                      prob_lo, prob_hi) -> str:
    """One single-box, single-level plotfile of (Q, aux), as WritePlotFile does for level 0."""
    n_q, ny, nx = Q.shape
    data = np.concatenate([np.asarray(Q, np.float64), np.asarray(aux, np.float64)], axis=0)
    dx = ((prob_hi[0] - prob_lo[0]) / nx, (prob_hi[1] - prob_lo[1]) / ny)
    L = LevelData((0, 0), (nx - 1, ny - 1), dx, [PatchData(data, (0, 0))], step=step)
    path = os.path.join(out_dir, plotfile_name(identifier, step))
    return write_plotfile(path, [L], component_names(n_q, aux.shape[0]), time, prob_lo, prob_hi)
