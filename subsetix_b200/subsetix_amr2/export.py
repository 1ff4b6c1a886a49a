"""VTK export of a two-level AMR snapshot (drop-in for ``subsetix_amr2.export``).

``save_two_level_vtk`` follows ``subsetix_amr2/export.py`` of the
reference: the coarse-only cells minus a ghost band around the refine
region, that ghost band, the fine cells and the fine ghost band are
gathered on the device, their quads assembled on the device, and written as
one unstructured grid (``.vtu``, raw appended data) with cell data ``level``,
``ghost_mask`` and ``u`` (``subsetix_cupy.export_vtk``).
"""

from __future__ import annotations

import os
from typing import Dict, Tuple


from ..subsetix_cupy import evaluate, ghost_zones, make_difference, make_input, make_intersection
from ..subsetix_cupy.expressions import IntervalSet, _t
from ..subsetix_cupy.export_vtk import write_unstructured_quads_vtu
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
