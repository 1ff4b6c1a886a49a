"""VTK export of level fields and interval fields (drop-in for ``subsetix_cupy.export_vtk``).

Public names, arguments and the files' layout follow the reference's
``subsetix_cupy/export_vtk.py``: rectilinear grids (``.vtr``, ASCII) for
whole levels, ParaView collections (``.pvd``), and one unstructured grid of
quads (``.vtu``, raw appended data) whose cells carry ``level``,
``ghost_mask`` and ``u``.  The array names and types are the format a
reader of the reference's files expects.

For an interval field the quads are assembled on the device
(``sx_cell_quads``: four float32 corners and the value per cell, in one
launch) and brought back with one copy per array; the connectivity is the
identity and is made on the host.  Dense masks take the host path, as in the
reference.  Files are written on the host.
"""

from __future__ import annotations

import os
import struct
from typing import Any, Dict, List, NamedTuple, Sequence, Tuple

import numpy as np
import torch

from .._runtime import ptr, stream_handle
from .expressions import _t

_VTK_QUAD = 9


class QuadChunk(NamedTuple):
    """Quads of one group of cells: 4 float32 corners per cell, then per-cell level, ghost flag and value."""

    points: np.ndarray  # (4 n, 3) float32
    levels: np.ndarray  # (n,) int32
    ghosts: np.ndarray  # (n,) int32
    values: np.ndarray  # (n,) float32

    @property
    def cells(self) -> int:
        return int(self.values.size)


def _host(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    if hasattr(a, "get") and not isinstance(a, np.ndarray):
        return np.asarray(a.get())
    if not isinstance(a, np.ndarray) and (hasattr(a, "__cuda_array_interface__") or hasattr(a, "__dlpack__")):
        return torch.as_tensor(a).cpu().numpy()
    return np.asarray(a)


def interval_field_quads(field, level: int, dx: float, dy: float, x0: float = 0.0, y0: float = 0.0,
                         ghost: int = 0) -> QuadChunk:
    """Quads of every cell of an interval field, assembled on the device (``export_vtk.py:271-316``)."""
    from .. import _lib

    s = field.interval_set
    vals = _t(field.values)
    n = int(_t(s.begin).numel())
    cells = int(vals.numel())
    if n == 0 or cells == 0:
        return QuadChunk(np.zeros((0, 3), np.float32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                         np.zeros(0, np.float32))
    if vals.dtype not in (torch.float32, torch.float64):
        vals = vals.to(torch.float32)
    dev = vals.device
    pts = torch.empty(cells * 12, dtype=torch.float32, device=dev)
    out = torch.empty(cells, dtype=torch.float32, device=dev)
    code = _lib.SX_F64 if vals.dtype == torch.float64 else _lib.SX_F32
    _lib.check(_lib.load().sx_cell_quads(code, ptr(_t(s.row_offsets)), ptr(_t(s.rows)), int(_t(s.rows).numel()),
                                         ptr(_t(s.begin)), ptr(_t(s.end)), ptr(_t(field.interval_cell_offsets)), n,
                                         ptr(vals.contiguous()), float(dx), float(dy), float(x0), float(y0), ptr(pts),
                                         ptr(out), stream_handle(dev)), "sx_cell_quads")
    return QuadChunk(pts.cpu().numpy().reshape(-1, 3), np.full(cells, int(level), np.int32),
                     np.full(cells, int(ghost), np.int32), out.cpu().numpy())


def mask_quads(mask, u, level: int, dx: float, dy: float, x0: float = 0.0, y0: float = 0.0, ghost=None) -> QuadChunk:
    """Quads of the cells of a dense boolean mask, values sampled from ``u`` (``export_vtk.py:319-355``)."""
    m = _host(mask).astype(bool)
    ys, xs = np.nonzero(m)
    n = ys.size
    f32 = np.float32
    xl = f32(x0) + xs.astype(f32) * f32(dx)
    yb = f32(y0) + ys.astype(f32) * f32(dy)
    xr, yt = xl + f32(dx), yb + f32(dy)
    pts = np.zeros((n, 4, 3), f32)
    pts[:, 0, 0], pts[:, 0, 1] = xl, yb
    pts[:, 1, 0], pts[:, 1, 1] = xr, yb
    pts[:, 2, 0], pts[:, 2, 1] = xr, yt
    pts[:, 3, 0], pts[:, 3, 1] = xl, yt
    vals = _host(u).astype(f32)[ys, xs]
    g = np.zeros(n, np.int32) if ghost is None else _host(ghost).astype(np.int32)[ys, xs]
    return QuadChunk(pts.reshape(-1, 3), np.full(n, int(level), np.int32), g, vals)


def _chunk_of(entry) -> QuadChunk:
    if hasattr(entry[0], "interval_set"):
        if len(entry) < 7:
            raise ValueError("IntervalField entries must be (field, level, dx, dy, x0, y0, ghost_flag)")
        field, lvl, dx, dy, x0, y0, ghost = entry[:7]
        return interval_field_quads(field, int(lvl), float(dx), float(dy), float(x0), float(y0), int(ghost))
    mask, u, lvl, dx, dy, x0, y0 = entry[:7]
    return mask_quads(mask, u, int(lvl), float(dx), float(dy), float(x0), float(y0),
                      entry[7] if len(entry) > 7 else None)


def write_unstructured_quads_vtu(path: str, cells: List[Tuple[Any, ...]], origin=(0.0, 0.0)) -> None:
    """One ``.vtu`` in which every listed cell of every entry is a quad (``export_vtk.py:358-486``).

    Entries are ``(field, level, dx, dy, x0, y0, ghost_flag)`` for interval
    fields or ``(mask, u, level, dx, dy, x0, y0[, ghost])`` for dense masks.
    """
    chunks = [c for c in (_chunk_of(e) for e in cells if e) if c.cells]
    cat = (lambda xs, empty: np.concatenate(xs) if xs else empty)
    P = cat([c.points for c in chunks], np.zeros((0, 3), np.float32)).astype(np.float32)
    L = cat([c.levels for c in chunks], np.zeros(0, np.int32)).astype(np.int32)
    G = cat([c.ghosts for c in chunks], np.zeros(0, np.int32)).astype(np.int32)
    U = cat([c.values for c in chunks], np.zeros(0, np.float32)).astype(np.float32)
    n = int(L.size)
    C = np.arange(4 * n, dtype=np.int32)
    O = 4 * np.arange(1, n + 1, dtype=np.int32)
    T = np.full(n, _VTK_QUAD, np.uint8)
    blocks = [("CellData", "Int32", "level", L), ("CellData", "Int32", "ghost_mask", G),
              ("CellData", "Float32", "u", U), ("Points", "Float32", None, P),
              ("Cells", "Int32", "connectivity", C), ("Cells", "Int32", "offsets", O), ("Cells", "UInt8", "types", T)]
    offsets, pos = [], 0
    for _, _, _, arr in blocks:
        offsets.append(pos)
        pos += 8 + arr.nbytes
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    head = ['<?xml version="1.0"?>',
            '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" header_type="UInt64">',
            "  <UnstructuredGrid>", f'    <Piece NumberOfPoints="{int(P.shape[0])}" NumberOfCells="{n}">']
    section = None
    for (sec, typ, name, arr), off in zip(blocks, offsets):
        if sec != section:
            if section is not None:
                head.append(f"      </{section}>")
            head.append('      <CellData Scalars="u">' if sec == "CellData" else f"      <{sec}>")
            section = sec
        comps = ' NumberOfComponents="3"' if sec == "Points" else ""
        label = f' Name="{name}"' if name else ""
        head.append(f'        <DataArray type="{typ}"{label}{comps} format="appended" offset="{off}"/>')
    head += [f"      </{section}>", "    </Piece>", "  </UnstructuredGrid>", '  <AppendedData encoding="raw">']
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        f.write(b"_")
        for _, _, _, arr in blocks:
            data = np.ascontiguousarray(arr).tobytes()
            f.write(struct.pack("<Q", len(data)))
            f.write(data)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


def _ascii_array(name: str, arr: np.ndarray, typ: str) -> str:
    flat = arr.ravel()
    lines = [f'        <DataArray type="{typ}" Name="{name}" format="ascii">']
    for i in range(0, flat.size, 4096):
        lines.append("          " + " ".join(str(x) for x in flat[i:i + 4096].tolist()))
    lines.append("        </DataArray>")
    return "\n".join(lines)


def write_rectilinear_grid_vtr(path: str, u_cell, dx: float, dy: float, *, origin=(0.0, 0.0, 0.0),
                               cell_arrays: Dict[str, np.ndarray] | None = None) -> None:
    """A whole level as a rectilinear grid with cell data ``u`` and extra cell arrays (``export_vtk.py:35-94``)."""
    u = _host(u_cell)
    H, W = u.shape
    ox, oy, oz = (float(c) for c in origin)
    xs = np.float32(ox) + np.float32(dx) * np.arange(W + 1, dtype=np.float32)
    ys = np.float32(oy) + np.float32(dy) * np.arange(H + 1, dtype=np.float32)
    parts = ['<?xml version="1.0"?>', '<VTKFile type="RectilinearGrid" version="0.1" byte_order="LittleEndian">',
             f'  <RectilinearGrid WholeExtent="0 {W} 0 {H} 0 0">', f'    <Piece Extent="0 {W} 0 {H} 0 0">',
             '      <CellData Scalars="u">', _ascii_array("u", u.astype(np.float32), "Float32")]
    for name, arr in (cell_arrays or {}).items():
        a = _host(arr)
        if a.dtype == np.bool_ or np.issubdtype(a.dtype, np.integer):
            parts.append(_ascii_array(name, a.astype(np.int32), "Int32"))
        else:
            parts.append(_ascii_array(name, a.astype(np.float32), "Float32"))
    parts.append("      </CellData>")
    parts.append("      <Coordinates>")
    for axis, vals in (("X", xs), ("Y", ys), ("Z", np.array([oz], np.float32))):
        parts.append(f'        <DataArray type="Float32" Name="{axis}_COORDINATES" NumberOfComponents="1" '
                     'format="ascii">')
        parts.append("          " + " ".join(str(v) for v in vals.tolist()))
        parts.append("        </DataArray>")
    parts += ["      </Coordinates>", "    </Piece>", "  </RectilinearGrid>", "</VTKFile>"]
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w", encoding="utf-8") as f:
        f.write("\n".join(parts) + "\n")


def write_pvd(path: str, datasets: List[Tuple[float, List[str]]]) -> None:
    """A ParaView collection: one entry per (time, files) with a part index per file (``export_vtk.py:97-111``)."""
    lines = ['<?xml version="1.0"?>', '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">',
             "  <Collection>"]
    for t, files in datasets:
        lines += [f'    <DataSet timestep="{t}" group="" part="{k}" file="{name}"/>' for k, name in enumerate(files)]
    lines += ["  </Collection>", "</VTKFile>"]
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w", encoding="utf-8") as f:
        f.write("\n".join(lines) + "\n")


def save_amr3_step_vtr(out_dir: str, base: str, step: int, time_value: float, *, u0, u1, u2, refine0, L1_mask,
                       refine1_mid, L2_mask, dx0: float, dy0: float, dx1: float, dy1: float, dx2: float,
                       dy2: float) -> Tuple[List[str], Tuple[float, List[str]]]:
    """Three ``.vtr`` files (one per level) of a step and their collection entry (``export_vtk.py:114-175``)."""
    os.makedirs(out_dir, exist_ok=True)
    names = [f"{base}_step{step:04d}_L{k}.vtr" for k in range(3)]
    l1 = _host(L1_mask).astype(bool)
    levels = [(u0, dx0, dy0, {"coarse_only": ~_host(refine0).astype(bool)}),
              (u1, dx1, dy1, {"mid_active": l1, "mid_only": l1 & ~_host(refine1_mid).astype(bool)}),
              (u2, dx2, dy2, {"fine_active": _host(L2_mask).astype(bool)})]
    for name, (u, dx, dy, extra) in zip(names, levels):
        write_rectilinear_grid_vtr(os.path.join(out_dir, name), u, dx, dy, cell_arrays=extra)
    return names, (time_value, names)


def save_amr3_mesh_vtu(out_dir: str, base: str, step: int, *, u0, u1, u2, coarse_only, mid_only, fine_active,
                       dx0: float, dy0: float, dx1: float, dy1: float, dx2: float, dy2: float,
                       origin=(0.0, 0.0)) -> str:
    """The three levels' active cells as one quad mesh (``export_vtk.py:489-521``)."""
    os.makedirs(out_dir, exist_ok=True)
    name = f"{base}_step{step:04d}_mesh.vtu"
    x0, y0 = origin
    write_unstructured_quads_vtu(os.path.join(out_dir, name),
                                 cells=[(coarse_only, u0, 0, dx0, dy0, x0, y0), (mid_only, u1, 1, dx1, dy1, x0, y0),
                                        (fine_active, u2, 2, dx2, dy2, x0, y0)], origin=(x0, y0))
    return name


__all__ = ["QuadChunk", "interval_field_quads", "mask_quads", "write_unstructured_quads_vtu",
           "write_rectilinear_grid_vtr", "write_pvd", "save_amr3_step_vtr", "save_amr3_mesh_vtu"]
