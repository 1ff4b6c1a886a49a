"""VTK export of a two-level AMR snapshot (drop-in for ``subsetix_amr2.export``).

``save_two_level_vtk`` follows ``subsetix_amr2/export.py`` of the
reference: the coarse-only cells minus a ghost band around the refine
region, that ghost band, the fine cells and the fine ghost band are
gathered on the device, then written as one unstructured grid of quads
(``.vtu``, ASCII) with cell data ``value``, ``level`` and ``ghost``.
File output is host work and is outside the GPU path.
"""

from __future__ import annotations

import os
from typing import Dict, List, Tuple

import numpy as np
import torch

from ..subsetix_cupy import evaluate, ghost_zones, make_difference, make_input, make_intersection
from ..subsetix_cupy.expressions import IntervalSet, _t
from ..subsetix_cupy.interval_field import IntervalField
from .fields import gather_interval_subset


def _as_interval_field(field, *, name: str) -> IntervalField:
    if isinstance(field, IntervalField):
        return field
    raise TypeError(f"{name} must be an IntervalField")


def _interval_dimensions(field: IntervalField) -> Tuple[int, int]:
    height = int(field.interval_set.row_count)
    width = 0 if int(field.interval_set.begin.shape[0]) == 0 else int(_t(field.interval_set.end).max().item())
    return height, width


def _quads(field: IntervalField, dx: float, dy: float):
    """Corner points and cell values of every cell of ``field`` (host arrays)."""
    s = field.interval_set
    b = _t(s.begin).cpu().numpy().astype(np.int64)
    e = _t(s.end).cpu().numpy().astype(np.int64)
    off = _t(s.row_offsets).cpu().numpy()
    rows = _t(s.rows).cpu().numpy().astype(np.int64)
    vals = _t(field.values).cpu().numpy().astype(np.float64)
    lengths = np.maximum(e - b, 0)
    per_row = np.repeat(rows, np.diff(off))
    ys = np.repeat(per_row, lengths)
    starts = np.repeat(b, lengths)
    local = np.arange(int(lengths.sum())) - np.repeat(np.cumsum(lengths) - lengths, lengths)
    xs = starts + local
    x0, y0 = xs * dx, ys * dy
    pts = np.stack([np.stack([x0, y0], 1), np.stack([x0 + dx, y0], 1), np.stack([x0 + dx, y0 + dy], 1),
                    np.stack([x0, y0 + dy], 1)], 1)
    return pts.reshape(-1, 2), vals[: xs.size]


def write_unstructured_quads_vtu(path: str, cells: List[tuple]) -> None:
    """Write ``(field, level, dx, dy, ox, oy, ghost)`` chunks as one ``.vtu`` file of quads."""
    points, values, levels, ghosts = [], [], [], []
    for field, level, dx, dy, ox, oy, ghost in cells:
        p, v = _quads(field, dx, dy)
        p = p + np.array([ox, oy])
        points.append(p)
        values.append(v)
        levels.append(np.full(v.size, level, np.int32))
        ghosts.append(np.full(v.size, ghost, np.int32))
    pts = np.concatenate(points) if points else np.zeros((0, 2))
    val = np.concatenate(values) if values else np.zeros(0)
    lev = np.concatenate(levels) if levels else np.zeros(0, np.int32)
    gh = np.concatenate(ghosts) if ghosts else np.zeros(0, np.int32)
    n = val.size
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n')
        f.write(f'<UnstructuredGrid>\n<Piece NumberOfPoints="{4 * n}" NumberOfCells="{n}">\n')
        f.write('<Points>\n<DataArray type="Float64" NumberOfComponents="3" format="ascii">\n')
        xyz = np.concatenate([pts, np.zeros((pts.shape[0], 1))], 1)
        np.savetxt(f, xyz, fmt="%.9g")
        f.write("</DataArray>\n</Points>\n<Cells>\n")
        f.write('<DataArray type="Int64" Name="connectivity" format="ascii">\n')
        np.savetxt(f, np.arange(4 * n).reshape(-1, 4), fmt="%d")
        f.write('</DataArray>\n<DataArray type="Int64" Name="offsets" format="ascii">\n')
        np.savetxt(f, 4 * np.arange(1, n + 1), fmt="%d")
        f.write('</DataArray>\n<DataArray type="UInt8" Name="types" format="ascii">\n')
        np.savetxt(f, np.full(n, 9), fmt="%d")
        f.write("</DataArray>\n</Cells>\n<CellData>\n")
        for name, arr, typ, fmt in (("value", val, "Float64", "%.9g"), ("level", lev, "Int32", "%d"),
                                    ("ghost", gh, "Int32", "%d")):
            f.write(f'<DataArray type="{typ}" Name="{name}" format="ascii">\n')
            np.savetxt(f, arr, fmt=fmt)
            f.write("</DataArray>\n")
        f.write("</CellData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")


def save_two_level_vtk(out_dir: str, base: str, step: int, *, coarse_field, fine_field, refine_set: IntervalSet,
                       coarse_only_set: IntervalSet, fine_set: IntervalSet, dx_coarse: float, dy_coarse: float,
                       ratio: int = 2, time_value: float = 0.0, ghost_halo: int = 1, width: int | None = None,
                       height: int | None = None) -> Dict[str, str]:
    """Write ``<base>_mesh_step<step>.vtu`` in ``out_dir``; returns the file name (``export.py:34-109``)."""
    coarse = _as_interval_field(coarse_field, name="coarse_field")
    fine = _as_interval_field(fine_field, name="fine_field")
    dh, dw = _interval_dimensions(coarse)
    width = int(width if width is not None else dw)
    height = int(height if height is not None else dh)
    fw, fh = width * ratio, height * ratio
    dxf, dyf = dx_coarse / ratio, dy_coarse / ratio
    ghost_raw = ghost_zones(refine_set, halo_x=ghost_halo, halo_y=ghost_halo, width=width, height=height)
    coarse_ghost = evaluate(make_intersection(make_input(ghost_raw), make_input(coarse_only_set)))
    coarse_active = evaluate(make_difference(make_input(coarse_only_set), make_input(coarse_ghost)))
    fine_ghost = ghost_zones(fine_set, halo_x=max(0, ghost_halo * ratio), halo_y=max(0, ghost_halo * ratio),
                             width=fw, height=fh)
    chunks = [
        (gather_interval_subset(coarse, coarse_active), 0, dx_coarse, dy_coarse, 0.0, 0.0, 0),
        (gather_interval_subset(coarse, coarse_ghost), 0, dx_coarse, dy_coarse, 0.0, 0.0, 1),
        (gather_interval_subset(fine, fine_set), 1, dxf, dyf, 0.0, 0.0, 0),
        (gather_interval_subset(fine, fine_ghost), 1, dxf, dyf, 0.0, 0.0, 1),
    ]
    cells = [c for c in chunks if int(c[0].interval_set.begin.shape[0]) != 0]
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, f"{base}_mesh_step{step:04d}.vtu")
    write_unstructured_quads_vtu(path, cells)
    return {"mesh_vtu": os.path.basename(path)}


__all__ = ["save_two_level_vtk", "write_unstructured_quads_vtu"]
