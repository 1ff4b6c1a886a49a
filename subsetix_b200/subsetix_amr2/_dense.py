"""Whole-grid kernels for the two-level wrappers (``api`` and ``runner``).

The reference's Samurai-style wrappers keep both levels as whole
rectangles (``subsetix_amr2/api.py:141-190``).  On a whole rectangle the
interval kernels of a regrid, a synchronisation and an upwind step reduce to
dense ones, which this module calls through the C ABI:

* ``regrid``: gradient tag and 2:1 grading straight into int8 action bytes
  (``sx_amr_regrid_full``), the same cell set as the reference's
  gradient -> threshold -> grading interval pipeline;
* ``sync``: restriction into REFINE coarse cells and injection into the
  fine blocks of the others (``sx_amr_sync_full``), as
  ``synchronize_interval_fields(..., reducer="mean", copy=False)``;
* ``upwind``: one first-order upwind step with zero exterior
  (``sx_upwind_full``), as ``step_upwind_interval``.

Every helper takes ``[rows, cols]`` tensors and launches on the current
stream without host synchronisation.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .. import _lib
from .._runtime import ptr, stream_handle
from ..subsetix_cupy.expressions import _t
from ..subsetix_cupy.interval_field import IntervalField

_MODE_CODES = {"von_neumann": 0, "moore": 1}


def _code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.SX_F32
    if t.dtype == torch.float64:
        return _lib.SX_F64
    raise TypeError(f"whole-grid kernels take float32 or float64 values, not {t.dtype}")


def grid_values(field: IntervalField, width: int, height: int) -> Optional[torch.Tensor]:
    """``field``'s values as a ``[height, width]`` float tensor when the field is the whole grid, else None.

    Only sets made by ``full_interval_set`` (which carry a marker) qualify,
    so the test costs no device work.
    """
    if not isinstance(field, IntervalField):
        return None
    s = field.interval_set
    if getattr(s, "_full_width", None) != int(width) or s.row_count != int(height):
        return None
    v = _t(field.values)
    if v.dtype not in (torch.float32, torch.float64) or v.numel() != width * height or not v.is_contiguous():
        return None
    return v.view(height, width)


def regrid(coarse: torch.Tensor, actions: torch.Tensor, *, threshold: float, epsilon: float, padding: int,
           mode: str) -> None:
    """Action bytes of the refine region: cells with gradient >= max(threshold, epsilon), graded by ``padding``."""
    H, W = coarse.shape
    tags = torch.empty((H, W), dtype=torch.uint8, device=coarse.device)
    thr = float(np.float32(max(float(threshold), float(epsilon))))
    lib = _lib.load()
    _lib.check(lib.sx_amr_regrid_full(_code(coarse), ptr(coarse), ptr(tags), ptr(actions), W, H, 1, thr,
                                      max(int(padding), 0), _MODE_CODES[mode], stream_handle(coarse.device)),
               "sx_amr_regrid_full")


def sync(coarse: torch.Tensor, fine: torch.Tensor, actions: Optional[torch.Tensor], ratio: int) -> None:
    """Restrict fine blocks into REFINE coarse cells, inject the other coarse cells; ``actions=None`` injects all."""
    H, W = coarse.shape
    if actions is None:
        actions = torch.zeros((H, W), dtype=torch.int8, device=coarse.device)
    lib = _lib.load()
    _lib.check(lib.sx_amr_sync_full(_code(coarse), ptr(coarse), ptr(fine), ptr(actions), W, H, 1, int(ratio),
                                    stream_handle(coarse.device)), "sx_amr_sync_full")


def upwind(values: torch.Tensor, out: torch.Tensor, *, a: float, b: float, dt: float, dx: float, dy: float) -> None:
    """``out`` = one upwind step of ``values`` (distinct buffers), zero outside the grid."""
    H, W = values.shape
    lib = _lib.load()
    _lib.check(lib.sx_upwind_full(_code(values), ptr(values), ptr(out), W, H, 1, float(a), float(b), float(dt),
                                  float(dx), float(dy), stream_handle(values.device)), "sx_upwind_full")
