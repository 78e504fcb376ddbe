"""ParaView output of a run: a ``.pvd`` collection over ``.vtu`` files.

The reference's ``run_case`` ends by converting its AMReX plotfiles into
``<output_dir>/simulation.pvd`` plus ``<output_dir>/vtk/<plotfile>_L<level>.vtu``
and returns the ``.pvd`` path (zoomy_amrex/run_case.py:128-178, 426). This
module does the same conversion from the plotfiles written here: one ``.vtu``
per plotfile and refinement level, over the level's bounding box (cells no box
covers hold NaN, as the reference's reader fills them), structured quads in
2-D and line cells in 1-D, cell data named by the model's state names and
``var<c>`` for the remaining plotfile components. The reference writes them
through meshio; here the VTK XML is written directly (inline base64 binary,
no compression), which ParaView and meshio both read.
"""
from __future__ import annotations

import base64
import pathlib
import re
import xml.etree.ElementTree as ET

import numpy as np

from .plotfile import read_plotfile

_VTK_LINE, _VTK_QUAD = 3, 9
_TYPES = {np.dtype("<f8"): "Float64", np.dtype("<i8"): "Int64", np.dtype("u1"): "UInt8"}


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(np.uint64(len(raw)).tobytes() + raw).decode("ascii")


def _data_array(name: str, a: np.ndarray, ncomp: int = 1) -> str:
    a = np.ascontiguousarray(a)
    if a.dtype.kind == "f":
        a = a.astype("<f8")
    elif a.dtype.kind in "iu" and a.dtype != np.uint8:
        a = a.astype("<i8")
    t = _TYPES[a.dtype]
    nc = f' NumberOfComponents="{ncomp}"' if ncomp > 1 else ""
    return f'<DataArray type="{t}" Name="{name}"{nc} format="binary">{_b64(a)}</DataArray>'


def write_vtu(path, points: np.ndarray, conn: np.ndarray, cell_type: int, cell_data: dict) -> str:
    """An unstructured grid of one cell type with per-cell FP64 data."""
    n_pts, n_cells, k = points.shape[0], conn.shape[0], conn.shape[1]
    offsets = np.arange(1, n_cells + 1, dtype=np.int64) * k
    types = np.full(n_cells, cell_type, dtype=np.uint8)
    parts = ['<?xml version="1.0"?>',
             '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
             'header_type="UInt64">',
             '<UnstructuredGrid>',
             f'<Piece NumberOfPoints="{n_pts}" NumberOfCells="{n_cells}">',
             '<Points>', _data_array("Points", points, 3), '</Points>',
             '<Cells>', _data_array("connectivity", conn.reshape(-1)),
             _data_array("offsets", offsets), _data_array("types", types), '</Cells>',
             '<CellData>']
    parts += [_data_array(name, np.asarray(v, dtype=np.float64).reshape(-1)) for name, v in cell_data.items()]
    parts += ['</CellData>', '</Piece>', '</UnstructuredGrid>', '</VTKFile>']
    p = pathlib.Path(path)
    p.write_text("\n".join(parts))
    return str(p)


def read_vtu(path) -> dict:
    """Cell data of a ``.vtu`` written by write_vtu: {name: FP64 array}, plus
    the points under the key ``"Points"``."""
    root = ET.parse(path).getroot()
    out = {}
    for da in root.iter("DataArray"):
        raw = base64.b64decode(da.text.strip())
        n = int(np.frombuffer(raw[:8], dtype="<u8")[0])
        dt = {"Float64": "<f8", "Int64": "<i8", "UInt8": "u1"}[da.get("type")]
        a = np.frombuffer(raw[8:8 + n], dtype=dt)
        if da.get("Name") == "Points":
            a = a.reshape(-1, 3)
        out[da.get("Name")] = a.copy()
    return out


def _level_box_array(level, ncomp: int):
    """(ncomp, ny, nx) over the level's bounding box and (ilo, jlo)."""
    los = [p.lo for p in level.patches]
    his = [(p.lo[0] + p.data.shape[2] - 1, p.lo[1] + p.data.shape[1] - 1) for p in level.patches]
    ilo, jlo = min(l[0] for l in los), min(l[1] for l in los)
    ihi, jhi = max(h[0] for h in his), max(h[1] for h in his)
    arr = np.full((ncomp, jhi - jlo + 1, ihi - ilo + 1), np.nan)
    for p in level.patches:
        _, by, bx = p.data.shape
        arr[:, p.lo[1] - jlo:p.lo[1] - jlo + by, p.lo[0] - ilo:p.lo[0] - ilo + bx] = p.data
    return arr, ilo, jlo


def _grid(ox: float, oy: float, dx: float, dy: float, nx: int, ny: int, dim: int):
    if dim == 1:
        pts = np.zeros((nx + 1, 3))
        pts[:, 0] = ox + np.arange(nx + 1) * dx
        i = np.arange(nx, dtype=np.int64)
        return pts, np.stack([i, i + 1], axis=1), _VTK_LINE
    jj, ii = np.meshgrid(np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    pts = np.stack([ox + ii.reshape(-1) * dx, oy + jj.reshape(-1) * dy, np.zeros(ii.size)], axis=1)
    cj, ci = np.meshgrid(np.arange(ny, dtype=np.int64), np.arange(nx, dtype=np.int64), indexing="ij")
    v = ci.reshape(-1) + (nx + 1) * cj.reshape(-1)          # cells j-major, like the arrays
    conn = np.stack([v, v + 1, v + 1 + (nx + 1), v + (nx + 1)], axis=1)
    return pts, conn, _VTK_QUAD


def plotfiles_to_vtk(plotfiles, names: list[str], out_dir, dim: int) -> str:
    """Convert plotfiles (in step order) to ``out_dir/simulation.pvd`` and
    ``out_dir/vtk/*.vtu``; returns the ``.pvd`` path."""
    if not plotfiles:
        raise RuntimeError("run_case: no plotfiles were written")
    out = pathlib.Path(out_dir)
    vdir = out / "vtk"
    vdir.mkdir(parents=True, exist_ok=True)
    pvd = ['<?xml version="1.0"?>',
           '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">',
           '  <Collection>']
    for pf in plotfiles:
        pf = pathlib.Path(pf)
        head, levels = read_plotfile(pf)
        plo = head["prob_lo"]
        ncomp = len(head["names"])
        for lev, L in enumerate(levels):
            arr, ilo, jlo = _level_box_array(L, ncomp)
            dx = L.dx[0]
            dy = L.dx[1] if len(L.dx) > 1 else dx
            ny, nx = arr.shape[1], arr.shape[2]
            pts, conn, ctype = _grid(plo[0] + ilo * dx, (plo[1] if len(plo) > 1 else 0.0) + jlo * dy,
                                     dx, dy, nx, ny, dim)
            cell_data = {(names[c] if c < len(names) else f"var{c}"): arr[c].reshape(-1) for c in range(ncomp)}
            vtu = vdir / f"{pf.name}_L{lev}.vtu"
            write_vtu(vtu, pts, conn, ctype, cell_data)
            pvd.append(f'    <DataSet timestep="{head["time"]!r}" part="{lev}" file="vtk/{vtu.name}"/>')
    pvd += ['  </Collection>', '</VTKFile>']
    path = out / "simulation.pvd"
    path.write_text("\n".join(pvd))
    return str(path)


def read_pvd(path) -> list[tuple[float, int, str]]:
    """(time, part, absolute .vtu path) of every data set of a ``.pvd``."""
    p = pathlib.Path(path)
    txt = p.read_text()
    return [(float(t), int(part), str(p.parent / f))
            for t, part, f in re.findall(r'timestep="([^"]+)" part="(\d+)" file="([^"]+)"', txt)]
