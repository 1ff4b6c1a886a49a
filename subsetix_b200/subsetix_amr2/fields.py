"""Field transfers for two-level AMR (drop-in for ``subsetix_amr2.fields``).

Names, arguments and exceptions follow ``subsetix_amr2/fields.py`` of the
reference.  Subset copies run ``sx_subset_rows`` (superset row of each
subset interval, with the containment check) and ``sx_subset_copy`` (one
warp per subset interval).  Value runs for the action field come from
``sx_value_runs`` (one warp per interval, ballot-based run detection).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum
from typing import Dict, Optional

import numpy as np
import torch

from .. import _core, _lib
from .._runtime import like, ptr, stream_handle
from ..subsetix_cupy.expressions import (
    IntervalSet,
    _t,
    evaluate,
    make_difference,
    make_input,
    make_intersection,
)
from ..subsetix_cupy.interval_field import IntervalField, create_interval_field
from ..subsetix_cupy.morphology import full_interval_set
from ..subsetix_cupy.multilevel import prolong_field, restrict_field, prolong_set

I32 = torch.int32

_VALUE_TYPES = {
    torch.float32: (_lib.SX_F32, np.float32),
    torch.float64: (_lib.SX_F64, np.float64),
    torch.int8: (2, np.int8),
    torch.uint8: (2, np.uint8),
    torch.bool: (2, np.uint8),
    torch.int32: (3, np.int32),
    torch.int64: (4, np.int64),
}
_SUBSET_DTYPES = (torch.float32, torch.float64, torch.int8, torch.int32, torch.int64, torch.bool)


def _interval_row_ids(interval_set: IntervalSet):
    return interval_set.interval_rows()


def _empty_interval_like(interval_set: IntervalSet) -> IntervalSet:
    if not isinstance(interval_set, IntervalSet):
        raise TypeError("interval_set must be an IntervalSet")
    rows = _t(interval_set.rows).clone()
    z = torch.zeros(0, dtype=I32, device=rows.device)
    off = torch.zeros(interval_set.row_count + 1, dtype=I32, device=rows.device)
    k = interval_set.begin
    return IntervalSet._trusted(like(k, z), like(k, z.clone()), like(k, off), like(k, rows))


def _interval_field_value_intervals(field: IntervalField, target) -> IntervalSet:
    """Runs of cells equal to ``target`` inside each interval; all rows kept (``fields.py:39-100``)."""
    s = field.interval_set
    vals = _t(field.values)
    if vals.numel() == 0:
        return _empty_interval_like(s)
    code, npt = _VALUE_TYPES[vals.dtype]
    n = int(s.begin.shape[0])
    if n == 0 or s.row_count == 0:
        return _empty_interval_like(s)
    device = vals.device
    lib = _lib.load()
    coff = _t(field.interval_cell_offsets)
    tgt = np.array([target], dtype=npt)
    counts = _core.empty_i32(n, device)
    st = stream_handle(device)
    _lib.check(lib.sx_value_runs(code, ptr(vals), ptr(coff), n, tgt.ctypes.data, ptr(counts), None, None, None, None,
                                 st), "sx_value_runs(count)")
    run_off, total = _core.scan(counts, device)
    if total == 0:
        return _empty_interval_like(s)
    ob = _core.empty_i32(total, device)
    oe = _core.empty_i32(total, device)
    _lib.check(lib.sx_value_runs(code, ptr(vals), ptr(coff), n, tgt.ctypes.data, None, ptr(run_off), ptr(_t(s.begin)),
                                 ptr(ob), ptr(oe), st), "sx_value_runs(write)")
    R = s.row_count
    off = _core.empty_i32(R + 1, device)
    _lib.check(lib.sx_gather_i32(ptr(_t(s.row_offsets)), R + 1, ptr(run_off), ptr(off), st), "sx_gather_i32")
    k = s.begin
    return IntervalSet._trusted(like(k, ob), like(k, oe), like(k, off), like(k, _t(s.rows).clone()))


def _subset_positions(subset: IntervalSet, superset: IntervalSet, what: str):
    n = int(subset.begin.shape[0])
    device = _t(subset.row_offsets).device
    sup_rows = _t(superset.rows)
    if n and sup_rows.numel() == 0:
        raise IndexError("cannot do a non-empty take from an empty axes.")
    pos, missing = _core.subset_rows(_t(subset.row_offsets), _t(subset.rows), n, sup_rows, device)
    if missing:
        raise ValueError(f"subset rows must be contained within the {what} field")
    return pos


def _check_subset_dtype(values) -> None:
    if _t(values).dtype not in _SUBSET_DTYPES:
        raise TypeError(f"interval subset kernels do not support dtype {values.dtype}")


def _gather_subset_into(field: IntervalField, subset_field: IntervalField) -> None:
    n = int(subset_field.interval_set.begin.shape[0])
    if n == 0:
        return
    _check_subset_dtype(subset_field.values)
    pos = _subset_positions(subset_field.interval_set, field.interval_set, "source")
    sub, sup = subset_field.interval_set, field.interval_set
    _core.subset_copy(False, pos, (_t(sub.begin), _t(sub.end), _t(subset_field.interval_cell_offsets)),
                      (_t(sup.row_offsets), _t(sup.begin), _t(sup.end), _t(field.interval_cell_offsets)),
                      _t(subset_field.values), _t(field.values).to(_t(subset_field.values).dtype),
                      _t(sub.row_offsets).device)


def _scatter_subset_from(subset_field: IntervalField, field: IntervalField) -> None:
    n = int(subset_field.interval_set.begin.shape[0])
    if n == 0:
        return
    _check_subset_dtype(subset_field.values)
    dst = _t(field.values)
    src = _t(subset_field.values)
    if src.dtype != dst.dtype:
        src = src.to(dst.dtype)
    pos = _subset_positions(subset_field.interval_set, field.interval_set, "destination")
    sub, sup = subset_field.interval_set, field.interval_set
    _core.subset_copy(True, pos, (_t(sub.begin), _t(sub.end), _t(subset_field.interval_cell_offsets)),
                      (_t(sup.row_offsets), _t(sup.begin), _t(sup.end), _t(field.interval_cell_offsets)),
                      src, dst, dst.device)


def gather_interval_subset(field: IntervalField, subset: IntervalSet) -> IntervalField:
    """New field on ``subset`` holding ``field``'s values there (``fields.py:372-385``)."""
    if not isinstance(field, IntervalField):
        raise TypeError("field must be an IntervalField")
    if not isinstance(subset, IntervalSet):
        raise TypeError("subset must be an IntervalSet")
    subset_field = create_interval_field(subset, fill_value=0.0, dtype=_t(field.values).dtype)
    _gather_subset_into(field, subset_field)
    return subset_field


def scatter_interval_subset(field: IntervalField, subset_field: IntervalField) -> None:
    """Write ``subset_field``'s values into ``field`` at the same coordinates (``fields.py:388-399``)."""
    if not isinstance(field, IntervalField):
        raise TypeError("field must be an IntervalField")
    if not isinstance(subset_field, IntervalField):
        raise TypeError("subset_field must be an IntervalField")
    _scatter_subset_from(subset_field, field)


def clone_interval_field(field: IntervalField) -> IntervalField:
    if not isinstance(field, IntervalField):
        raise TypeError("field must be an IntervalField")
    return IntervalField(interval_set=field.interval_set, values=like(field.values, _t(field.values).clone()),
                         interval_cell_offsets=field.interval_cell_offsets)


class Action(IntEnum):
    COARSEN = -1
    KEEP = 0
    REFINE = 1


_FULL_ACTION_INTERVAL_CACHE: Dict[tuple, IntervalSet] = {}


def _full_action_interval_set(width: int, height: int) -> IntervalSet:
    key = (height, width, torch.cuda.current_device())
    cached = _FULL_ACTION_INTERVAL_CACHE.get(key)
    if cached is None:
        cached = full_interval_set(width, height)
        _FULL_ACTION_INTERVAL_CACHE[key] = cached
    return cached


@dataclass
class ActionField:
    """int8 action per coarse cell over the full domain (``fields.py:443-569``).

    The refine set, its prolongation and the coarse-only set are cached
    until the actions change.
    """

    field: IntervalField
    ratio: int
    width: int
    height: int
    _refine_set_cache: Optional[IntervalSet] = None
    _fine_set_cache: Optional[IntervalSet] = None
    _coarse_only_cache: Optional[IntervalSet] = None

    @classmethod
    def from_interval_set(cls, interval_set: IntervalSet, *, width: int, height: int, ratio: int,
                          default: Action = Action.KEEP) -> "ActionField":
        if not isinstance(interval_set, IntervalSet):
            raise TypeError("interval_set must be an IntervalSet")
        w, h = int(width), int(height)
        if h <= 0 or w <= 0:
            raise ValueError("width and height must be positive")
        if interval_set.row_count != h:
            raise ValueError("interval_set row count must match height")
        rows = _t(interval_set.rows)
        if rows.numel() != h:
            raise ValueError("interval_set must provide exactly one row per coarse index")
        if getattr(interval_set, "_dense_rows", None) != h:
            if not bool(torch.equal(rows, torch.arange(h, dtype=I32, device=rows.device))):
                raise ValueError("interval_set row ids must equal the coarse domain [0, height)")
        field = create_interval_field(interval_set, fill_value=int(default), dtype=np.int8)
        if int(field.values.shape[0]) != w * h:
            raise ValueError("interval_set must cover exactly width * height cells")
        action = cls(field=field, ratio=int(ratio), width=w, height=h)
        action._refine_set_cache = _empty_interval_like(interval_set)
        return action

    @classmethod
    def full_grid(cls, height: int, width: int, ratio: int, *, default: Action = Action.KEEP) -> "ActionField":
        h, w = int(height), int(width)
        if h <= 0 or w <= 0:
            raise ValueError("height and width must be positive")
        return cls.from_interval_set(_full_action_interval_set(w, h), width=w, height=h, ratio=ratio, default=default)

    def _refresh_from_values(self) -> None:
        self._refine_set_cache = _interval_field_value_intervals(self.field, int(Action.REFINE))
        self._fine_set_cache = None
        self._coarse_only_cache = None

    def set_from_interval_set(self, refine_set: IntervalSet) -> None:
        """Mark ``refine_set`` (which must lie in the domain) REFINE, everything else KEEP."""
        if not isinstance(refine_set, IntervalSet):
            raise TypeError("refine_set must be an IntervalSet")
        domain = self.field.interval_set
        vals = _t(self.field.values)
        if int(refine_set.begin.shape[0]) == 0:
            vals.fill_(int(Action.KEEP))
            self._refine_set_cache = _empty_interval_like(domain)
            self._fine_set_cache = None
            self._coarse_only_cache = None
            return
        outside = evaluate(make_difference(make_input(refine_set), make_input(domain)))
        if int(outside.begin.shape[0]) != 0:
            raise ValueError("refine_set must be contained within the action domain")
        aligned = evaluate(make_intersection(make_input(refine_set), make_input(domain)))
        vals.fill_(int(Action.KEEP))
        subset = create_interval_field(aligned, fill_value=int(Action.REFINE), dtype=np.int8)
        scatter_interval_subset(self.field, subset)
        self._refine_set_cache = aligned
        self._fine_set_cache = None
        self._coarse_only_cache = None

    def refine_set(self) -> IntervalSet:
        if self._refine_set_cache is None:
            self._refresh_from_values()
        return self._refine_set_cache

    def fine_set(self) -> IntervalSet:
        if self._fine_set_cache is None:
            self._fine_set_cache = prolong_set(self.refine_set(), int(self.ratio))
        return self._fine_set_cache

    def coarse_only_set(self) -> IntervalSet:
        if self._coarse_only_cache is None:
            self._coarse_only_cache = evaluate(make_difference(make_input(self.field.interval_set),
                                                               make_input(self.refine_set())))
        return self._coarse_only_cache

    def coarse_interval_set(self) -> IntervalSet:
        return self.field.interval_set

    def values(self):
        return self.field.values


def synchronize_interval_fields(coarse: IntervalField, fine: IntervalField, actions: ActionField, *, ratio: int,
                                reducer: str = "mean", fill_fine_outside: bool = True, copy: bool = True):
    """coarse[refine] <- restrict(fine)[refine]; fine[prolong(coarse_only)] <- prolong(coarse[coarse_only]).

    Follows ``fields.py:570-612``; with ``copy=False`` the fields are
    updated in place.  Float32 fields as in the reference; float64 fields
    (both levels) take the FP64 kernels.
    """
    if not isinstance(coarse, IntervalField):
        raise TypeError("coarse must be an IntervalField")
    if not isinstance(fine, IntervalField):
        raise TypeError("fine must be an IntervalField")
    if not isinstance(actions, ActionField):
        raise TypeError("actions must be an ActionField")
    if int(actions.ratio) != int(ratio):
        raise ValueError("ratio argument must match ActionField ratio")
    cd, fd = _t(coarse.values).dtype, _t(fine.values).dtype
    if not ((cd == torch.float32 and fd == torch.float32) or (cd == torch.float64 and fd == torch.float64)):
        raise TypeError("coarse and fine interval fields must use float32 values")
    coarse_target = clone_interval_field(coarse) if copy else coarse
    fine_target = clone_interval_field(fine) if copy else fine
    dtype = np.float64 if cd == torch.float64 else np.float32
    restricted = restrict_field(fine, ratio, reducer=reducer, dtype=dtype)
    refine_set = actions.refine_set()
    if int(refine_set.begin.shape[0]) != 0:
        scatter_interval_subset(coarse_target, gather_interval_subset(restricted, refine_set))
    if fill_fine_outside:
        coarse_only = actions.coarse_only_set()
        if int(coarse_only.begin.shape[0]) != 0:
            coarse_subset = gather_interval_subset(coarse_target, coarse_only)
            fine_subset = prolong_field(coarse_subset, ratio, dtype=dtype)
            if int(fine_subset.values.shape[0]) != 0:
                scatter_interval_subset(fine_target, fine_subset)
    return coarse_target, fine_target


__all__ = [
    "Action",
    "ActionField",
    "clone_interval_field",
    "gather_interval_subset",
    "scatter_interval_subset",
    "synchronize_interval_fields",
]
