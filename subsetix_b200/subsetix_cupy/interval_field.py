"""Interval fields: one value per active cell (drop-in for ``subsetix_cupy.interval_field``).

Names and behaviour follow ``subsetix_cupy/interval_field.py`` of the
reference.  Cell offsets come from ``sx_cell_offsets``, a single-pass
device scan that also returns the cell total.  Cell lookups run in
``sx_locate_cells``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Optional

import numpy as np
import torch

from .. import _core
from .._runtime import is_cupy, like, to_tensor
from .expressions import IntervalSet, _t

I32 = torch.int32

_TORCH_DTYPES = {
    np.dtype(np.float32): torch.float32,
    np.dtype(np.float64): torch.float64,
    np.dtype(np.int8): torch.int8,
    np.dtype(np.uint8): torch.uint8,
    np.dtype(np.int16): torch.int16,
    np.dtype(np.int32): torch.int32,
    np.dtype(np.int64): torch.int64,
    np.dtype(np.bool_): torch.bool,
    np.dtype(np.float16): torch.float16,
}


def torch_dtype(dtype) -> torch.dtype:
    """torch dtype for a NumPy/CuPy/torch dtype specification."""
    if isinstance(dtype, torch.dtype):
        return dtype
    return _TORCH_DTYPES[np.dtype(dtype)]


@dataclass(frozen=True)
class IntervalField:
    """Values attached to the cells of an :class:`IntervalSet`, stored row by row.

    ``interval_cell_offsets`` (int32, ``interval_count + 1`` entries) gives
    the first value index of each interval (``interval_field.py:19-43``).
    """

    interval_set: IntervalSet
    values: Any
    interval_cell_offsets: Any

    @property
    def cell_count(self) -> int:
        off = self.interval_cell_offsets
        if int(off.shape[0]) == 0:
            return 0
        return int(_t(off)[-1].item())


def _fill_dtype(fill_value, dtype) -> torch.dtype:
    if dtype is not None:
        return torch_dtype(dtype)
    return torch_dtype(np.asarray(fill_value).dtype)


def create_interval_field(interval_set: IntervalSet, fill_value: float = 0.0, *, dtype: Any | None = None
                          ) -> IntervalField:
    """Field on ``interval_set`` filled with ``fill_value`` (``interval_field.py:46-89``).

    With ``dtype`` None the dtype is inferred from ``fill_value`` as NumPy
    does (a Python float gives float64).
    """
    b = interval_set.begin
    if int(np.prod(b.shape)) != int(np.prod(interval_set.end.shape)):
        raise ValueError("IntervalSet begin/end size mismatch")
    bt = _t(b)
    device = _t(interval_set.row_offsets).device
    if bt.numel() == 0:
        off = torch.zeros(1, dtype=I32, device=device)
        total = 0
    else:
        off, total = _core.cell_offsets(bt, _t(interval_set.end), device)
    values = torch.full((total,), fill_value, dtype=_fill_dtype(fill_value, dtype), device=device)
    return IntervalField(interval_set=interval_set, values=like(b, values), interval_cell_offsets=like(b, off))


def _locate_interval(interval_set: IntervalSet, row: int, x: int) -> Optional[int]:
    """Index of the interval holding (row, x), None when inactive (``interval_field.py:92-117``)."""
    rows = _t(interval_set.rows)
    if rows.numel() == 0:
        raise IndexError("row out of range")
    q_r = torch.tensor([int(row)], dtype=I32, device=rows.device)
    q_c = torch.tensor([int(x)], dtype=I32, device=rows.device)
    pos = int(torch.searchsorted(rows, q_r).item())
    if pos >= rows.numel() or int(rows[pos].item()) != int(row):
        raise IndexError("row out of range")
    off = _t(interval_set.row_offsets)
    start, stop = int(off[pos].item()), int(off[pos + 1].item())
    if start == stop:
        return None
    b = _t(interval_set.begin)[start:stop]
    e = _t(interval_set.end)[start:stop]
    hit = torch.nonzero((q_c >= b) & (q_c < e))
    if hit.numel() == 0:
        return None
    return start + int(hit[0, 0].item())


def set_cell(field: IntervalField, row: int, x: int, value: float) -> bool:
    """Write the cell (row, x); False when the cell is inactive (``interval_field.py:120-137``)."""
    idx = _locate_interval(field.interval_set, row, x)
    if idx is None:
        return False
    base = int(_t(field.interval_cell_offsets)[idx].item())
    local = int(x) - int(_t(field.interval_set.begin)[idx].item())
    vi = base + local
    vals = _t(field.values)
    if vi < 0 or vi >= vals.numel():
        return False
    vals[vi] = value
    return True


def get_cell(field: IntervalField, row: int, x: int):
    """Value of the cell (row, x), None when inactive (``interval_field.py:140-159``)."""
    idx = _locate_interval(field.interval_set, row, x)
    if idx is None:
        return None
    base = int(_t(field.interval_cell_offsets)[idx].item())
    local = int(x) - int(_t(field.interval_set.begin)[idx].item())
    vi = base + local
    vals = field.values
    if vi < 0 or vi >= int(np.prod(vals.shape)):
        return None
    return vals[vi]


def locate_interval_cells(field: IntervalField, rows: Any, cols: Any, *, out: Any | None = None):
    """Global interval index per (row, col) query, -1 when inactive (``interval_field.py:247-297``)."""
    from .. import _lib
    from .._runtime import ptr, stream_handle

    s = field.interval_set
    device = _t(s.row_offsets).device
    r = to_tensor(rows, dtype=I32, device=device)
    c = to_tensor(cols, dtype=I32, device=device)
    if tuple(r.shape) != tuple(c.shape):
        raise ValueError("rows and cols must share the same shape")
    fr, fc = r.reshape(-1).contiguous(), c.reshape(-1).contiguous()
    q = int(fr.numel())
    if out is None:
        o = torch.empty(q, dtype=I32, device=device)
    else:
        o = to_tensor(out, dtype=I32, device=device)
        if o.numel() != q:
            raise ValueError("out array must match query size")
    if q:
        lib = _lib.load()
        _lib.check(lib.sx_locate_cells(ptr(_t(s.rows)), ptr(_t(s.row_offsets)), ptr(_t(s.begin)), ptr(_t(s.end)),
                                       int(_t(s.rows).numel()), ptr(fr), ptr(fc), q, ptr(o), stream_handle(device)),
                   "sx_locate_cells")
    kind = rows if is_cupy(rows) else (out if out is not None else None)
    return like(kind, o.reshape(r.shape))


__all__ = ["IntervalField", "create_interval_field", "get_cell", "set_cell", "locate_interval_cells"]
