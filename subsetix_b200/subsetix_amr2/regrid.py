"""Refinement tagging and grading (drop-in for ``subsetix_amr2.regrid``).

Follows ``subsetix_amr2/regrid.py`` of the reference.  The gradient and the
threshold run-length encoding are fused into one kernel
(``sx_threshold_rle`` with ``gradient = 1``): one warp per row, where each
lane computes the gradient magnitude of its cell, and a ballot plus popc
turn the predicate into run starts and ends.  The gradient field itself is
only materialised when asked for (:func:`gradient_magnitude_interval_field`).
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _core, _lib
from .._runtime import like, ptr, stream_handle
from ..subsetix_cupy import (
    IntervalSet,
    clip_interval_set,
    dilate_interval_set,
    evaluate,
    make_input,
    make_union,
)
from ..subsetix_cupy.expressions import _t
from ..subsetix_cupy.interval_field import IntervalField

I32 = torch.int32


def _empty_interval_set(rows: int) -> IntervalSet:
    from .._runtime import current_device

    device = current_device()
    z = torch.zeros(0, dtype=I32, device=device)
    rows_arr = torch.arange(rows, dtype=I32, device=device) if rows > 0 else z.clone()
    return IntervalSet._trusted(z, z.clone(), torch.zeros(rows + 1, dtype=I32, device=device), rows_arr,
                                rows if rows > 0 else None)


def _grid_values(field: IntervalField, width: int, height: int, check_rows: bool) -> torch.Tensor:
    width, height = int(width), int(height)
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    if int(field.values.shape[0]) != width * height:
        raise ValueError("field cell count mismatch with width/height")
    if check_rows and field.interval_set.row_count != height:
        raise ValueError("interval_set row count mismatch with height")
    v = _t(field.values)
    return (v if v.dtype == torch.float32 else v.to(torch.float32)).contiguous()


def gradient_magnitude_interval_field(field: IntervalField, *, width: int, height: int) -> IntervalField:
    """Per-cell gradient magnitude of a full-grid field, no division by dx (``regrid.py:233-274``)."""
    data = _grid_values(field, width, height, check_rows=True)
    out = torch.empty_like(data)
    lib = _lib.load()
    _lib.check(lib.sx_gradient_magnitude(ptr(data), int(width), int(height), ptr(out), stream_handle(data.device)),
               "sx_gradient_magnitude")
    return IntervalField(interval_set=field.interval_set, values=like(field.values, out),
                         interval_cell_offsets=field.interval_cell_offsets)


def _threshold_set(data: torch.Tensor, width: int, height: int, threshold: float, gradient: bool, kind) -> IntervalSet:
    thr = float(np.float32(threshold))
    b, e, off = _core.threshold_rle(data, int(width), int(height), thr, gradient, data.device)
    rows = torch.arange(int(height), dtype=I32, device=data.device)
    return IntervalSet._trusted(like(kind, b), like(kind, e), like(kind, off), like(kind, rows), int(height))


def intervals_above_threshold_interval_field(field: IntervalField, *, width: int, height: int, threshold: float
                                             ) -> IntervalSet:
    """Runs of ``value >= threshold`` per row, rows ``arange(height)`` (``regrid.py:277-333``)."""
    data = _grid_values(field, width, height, check_rows=False)
    return _threshold_set(data, width, height, threshold, False, field.values)


def gradient_tag_threshold_interval_field(field: IntervalField, *, width: int, height: int, threshold: float,
                                          epsilon: float = 1e-8) -> IntervalSet:
    """Runs of ``|grad u| >= max(threshold, epsilon)``, fused in one kernel (``regrid.py:336-350``)."""
    data = _grid_values(field, width, height, check_rows=True)
    return _threshold_set(data, width, height, max(float(threshold), float(epsilon)), True, field.values)


def gradient_tag_set(field: IntervalField, *, width: int, height: int, frac_high: float, epsilon: float = 1e-8
                     ) -> IntervalSet:
    """Tag the top ``frac_high`` fraction of the values above ``epsilon`` (``regrid.py:353-380``)."""
    frac_high = float(max(0.0, min(1.0, frac_high)))
    if frac_high <= 0.0:
        return _empty_interval_set(height)
    values = _t(field.values).to(torch.float32)
    positive = values[values > float(np.float32(epsilon))]
    if positive.numel() == 0:
        return _empty_interval_set(height)
    count = int(np.ceil(positive.numel() * frac_high))
    count = max(1, min(int(positive.numel()), count))
    idx = int(positive.numel()) - count
    threshold = float(torch.kthvalue(positive, idx + 1).values.item())
    return intervals_above_threshold_interval_field(field, width=width, height=height,
                                                    threshold=max(threshold, float(epsilon)))


def gradient_tag_threshold_set(field: IntervalField, *, width: int, height: int, threshold: float,
                               epsilon: float = 1e-8) -> IntervalSet:
    """Runs of ``value >= max(threshold, epsilon)`` (``regrid.py:383-401``)."""
    return intervals_above_threshold_interval_field(field, width=width, height=height,
                                                    threshold=max(float(threshold), float(epsilon)))


def enforce_two_level_grading_set(refine_set: IntervalSet, *, padding: int = 1, mode: str = "von_neumann",
                                  width: int, height: int) -> IntervalSet:
    """2:1 grading by dilation, clipped to the domain (``regrid.py:404-442``).

    ``moore`` dilates the box; ``von_neumann`` takes the union of the
    horizontal and vertical dilations.  ``padding <= 0`` returns the input.
    """
    padding = int(padding)
    if padding <= 0:
        return refine_set
    if mode not in {"von_neumann", "moore"}:
        raise ValueError("mode must be 'von_neumann' or 'moore'")
    if mode == "moore":
        expanded = dilate_interval_set(refine_set, halo_x=padding, halo_y=padding)
    else:
        horiz = dilate_interval_set(refine_set, halo_x=padding, halo_y=0)
        vert = dilate_interval_set(refine_set, halo_x=0, halo_y=padding)
        expanded = evaluate(make_union(make_input(horiz), make_input(vert)))
    expanded = clip_interval_set(expanded, width=width, height=height)
    base = clip_interval_set(refine_set, width=width, height=height)
    union = evaluate(make_union(make_input(base), make_input(expanded)))
    return clip_interval_set(union, width=width, height=height)


__all__ = [
    "gradient_magnitude_interval_field",
    "intervals_above_threshold_interval_field",
    "gradient_tag_threshold_interval_field",
    "gradient_tag_set",
    "gradient_tag_threshold_set",
    "enforce_two_level_grading_set",
]
