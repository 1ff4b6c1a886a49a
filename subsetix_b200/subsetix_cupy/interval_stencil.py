"""First-order upwind step on interval fields (drop-in for ``subsetix_cupy.interval_stencil``).

Arguments, checks and results follow ``subsetix_cupy/interval_stencil.py``
of the reference.  On geometry whose rows are sorted and disjoint (the
usual case, checked once per set) the chunked kernel ``sx_upwind_chunked``
runs: warps take chunks of 128 cells of one interval in four coalesced
sub-rounds, exchange left/right neighbours by shuffles and find the cells
above and below through a per-cell neighbour table built with the plan.  Other geometry takes ``sx_upwind``, which assigns 256 consecutive
cells to each block and searches every neighbour.  Both give the same
values.  Float32 is the
reference's arithmetic.  Float64 values run the same formula in double
precision (an addition of this package).
"""

from __future__ import annotations

import weakref
from typing import Any, Optional

import torch

from .. import _core, _lib
from .._runtime import like, to_tensor
from .expressions import _t
from .interval_field import IntervalField

I32 = torch.int32


class _Geometry:
    """Per-set data the stencil needs: row lookup and row-shape flags.

    Cached on the set object, so repeated steps on one geometry pay for the
    lookup (and its synchronising range check) once.
    """

    __slots__ = ("height", "lookup", "direct", "chunk_off", "chunks", "cell_off", "table", "_seen")

    def __init__(self, height: int, lookup: torch.Tensor, direct: bool, chunk_off=None, chunks: int = 0,
                 cell_off=None, table=None):
        self.height = height
        self.lookup = lookup
        self.direct = direct
        self.chunk_off = chunk_off
        self.chunks = chunks
        self.cell_off = cell_off
        self.table = table
        self._seen = None

    def canonical(self, cell_off: torch.Tensor) -> bool:
        """Whether ``cell_off`` is the prefix sum of the interval lengths.

        The chunk plan holds value indices taken from that prefix sum, so the
        chunked kernel serves only fields laid out that way.  The answer for
        one offsets tensor is kept until the tensor is modified in place.
        """
        seen = self._seen
        if seen is not None and seen[0]() is cell_off and seen[1] == cell_off._version:
            return seen[2]
        ok = cell_off.data_ptr() == self.cell_off.data_ptr() or bool(torch.equal(cell_off, self.cell_off))
        try:
            self._seen = (weakref.ref(cell_off), cell_off._version, ok)
        except TypeError:  # pragma: no cover - tensors that refuse weak references
            self._seen = None
        return ok


def _geometry(interval_set, height: int) -> _Geometry:
    cache = getattr(interval_set, "_sx_stencil", None)
    if cache is not None and cache.height == height:
        return cache
    rows = _t(interval_set.rows)
    device = _t(interval_set.row_offsets).device
    lookup, bad = _core.row_lookup(rows, height, device)
    if bad:
        # The reference's lookup scatter wraps rows outside [0, height)
        # (interval_stencil.py:183-191); they are rejected here.
        raise ValueError("interval_set rows exceed provided height")
    flags = _core.check_rows(_t(interval_set.begin), _t(interval_set.end), _t(interval_set.row_offsets), device)
    direct = not (flags & (_lib.ROWS_UNSORTED_BEGIN | _lib.ROWS_OVERLAP | _lib.ROWS_EMPTY))
    chunk_off, chunks, coff, table = (None, 0, None, None)
    if direct:
        b, e = _t(interval_set.begin), _t(interval_set.end)
        coff, cells = _core.cell_offsets(b, e, device)
        chunk_off, chunks = _core.upwind_plan(rows, _t(interval_set.row_offsets), b, e, coff, lookup, height, device)
        table = _core.upwind_table(b, e, coff, chunk_off, chunks, cells, device)
    geo = _Geometry(height, lookup, direct, chunk_off, chunks, coff, table)
    try:
        object.__setattr__(interval_set, "_sx_stencil", geo)
    except Exception:  # pragma: no cover - sets that refuse attributes
        pass
    return geo


def step_upwind_interval(field: IntervalField, *, width: int, height: int, a: float, b: float, dt: float, dx: float,
                         dy: float, out: Any | None = None, row_ids: Any | None = None):
    """One upwind step with zero exterior; returns ``out`` (``interval_stencil.py:126-219``).

    Values are computed in float32, as in the reference, unless the field
    holds float64, which runs the FP64 kernel.
    """
    width = int(width)
    height = int(height)
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    s = field.interval_set
    device = _t(s.row_offsets).device
    begin = _t(s.begin)
    cell_off = _t(field.interval_cell_offsets)
    vals = _t(field.values)
    dtype = torch.float64 if vals.dtype == torch.float64 else torch.float32
    if vals.dtype != dtype:
        vals = vals.to(dtype)
    n = int(begin.numel())
    if int(cell_off.numel()) != n + 1:
        raise ValueError("interval_cell_offsets must have length interval_count + 1")
    if out is None:
        out_t = torch.empty(vals.shape, dtype=dtype, device=device)
        kind = field.values
    else:
        out_t = to_tensor(out)
        if out_t.dtype != dtype:
            raise TypeError("out must be float32" if dtype == torch.float32 else "out must be float64")
        if tuple(out_t.shape) != tuple(vals.shape):
            raise ValueError("out must match field values shape")
        kind = out
    if n == 0:
        out_t.fill_(0.0)
        return out if out is not None else like(kind, out_t)
    rid = None
    if row_ids is not None:
        rid = to_tensor(row_ids, dtype=I32, device=device).reshape(-1)
        if int(rid.numel()) != n:
            raise ValueError("row_ids must have one entry per interval")
    geo = _geometry(s, height)
    if rid is not None:
        if bool(((rid < 0) | (rid >= height)).any()) or int(geo.lookup[rid.long()].min().item()) < 0:
            raise ValueError("interval_set rows exceed provided height")
    vals = vals.contiguous()
    if (geo.chunk_off is not None and rid is None and out_t.data_ptr() != vals.data_ptr()
            and geo.canonical(cell_off)):
        # fixed geometry with sorted, disjoint rows and packed values: the chunked kernel (same results)
        _core.upwind_chunked(_t(s.row_offsets), begin, _t(s.end), cell_off, geo.chunk_off, geo.chunks, geo.lookup, vals,
                             out_t, width, height, a, b, dt, dx, dy, device, table=geo.table)
    else:
        _core.upwind(_t(s.rows), _t(s.row_offsets), begin, _t(s.end), cell_off, int(vals.numel()), geo.lookup, vals,
                     out_t, width, height, a, b, dt, dx, dy, geo.direct and rid is None, device, row_ids=rid)
    return out if out is not None else like(kind, out_t)


def step_upwind_interval_field(field: IntervalField, *, width: int, height: int, a: float, b: float, dt: float,
                               dx: float, dy: float, row_ids: Any | None = None) -> IntervalField:
    """:func:`step_upwind_interval` wrapped in a new field (``interval_stencil.py:222-251``)."""
    values = step_upwind_interval(field, width=width, height=height, a=a, b=b, dt=dt, dx=dx, dy=dy, row_ids=row_ids)
    return IntervalField(interval_set=field.interval_set, values=values,
                         interval_cell_offsets=field.interval_cell_offsets)


__all__ = ["step_upwind_interval", "step_upwind_interval_field"]
