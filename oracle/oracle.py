"""CPU oracle for the interval-set AMR hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it.  The product package ``subsetix_b200`` never imports it.

It restates the reference's host orchestration in NumPy.  Each function
gives the file and line of the reference code it follows.  The per-row
sweeps (set operations, merges, field transfers, upwind, threshold
run-length encoding, subset copies) run in ``sx_oracle.c``, loaded through
ctypes.  That library is built by ``oracle/build_oracle.py``.

Sets are :class:`ISet` tuples of int32 NumPy arrays ``(begin, end,
row_offsets, rows)``.  They have the same layout and invariants as the
reference's ``IntervalSet`` (``subsetix_cupy/expressions.py:144-227``).

Parity is pinned in two ways.  ``tests/golden/*.npz`` holds outputs of the
reference package itself, produced by ``tests/golden/make_golden.py``.  The
oracle tests also restate the reference's unit-test golden vectors.
"""

from __future__ import annotations

import ctypes
import math
import os
from typing import Callable, Dict, List, NamedTuple, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsx_oracle.so")
_lib = None

I32 = np.int32


def lib():
    """Load (building on first use if needed) the C half of the oracle."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from . import build_oracle  # type: ignore

            build_oracle.build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_threads.restype = ctypes.c_int
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def threads() -> int:
    return int(lib().orc_threads())


class ISet(NamedTuple):
    begin: np.ndarray
    end: np.ndarray
    row_offsets: np.ndarray
    rows: np.ndarray

    @property
    def row_count(self) -> int:
        return int(self.row_offsets.size - 1)

    @property
    def size(self) -> int:
        return int(self.begin.size)


def make(begin, end, row_offsets, rows=None) -> ISet:
    """``build_interval_set`` equivalent (expressions.py:413-443)."""
    off = np.asarray(row_offsets, dtype=I32)
    b = np.asarray(begin, dtype=I32).reshape(-1)
    e = np.asarray(end, dtype=I32).reshape(-1)
    if int(off[-1]) != b.size:
        raise ValueError("row_offsets final entry must equal the interval count")
    r = np.arange(off.size - 1, dtype=I32) if rows is None else np.asarray(rows, dtype=I32)
    return validate(ISet(b, e, off, r))


def validate(s: ISet) -> ISet:
    """``IntervalSet.__post_init__`` checks (expressions.py:166-227)."""
    if s.begin.shape != s.end.shape:
        raise ValueError("begin and end must share the same shape")
    if s.row_offsets.ndim != 1:
        raise ValueError("row_offsets must be one-dimensional")
    if int(s.row_offsets[0]) != 0:
        raise ValueError("row_offsets must start at zero")
    if int(s.row_offsets[-1]) != s.begin.size:
        raise ValueError("row_offsets last entry must match interval count")
    if s.rows.ndim != 1:
        raise ValueError("rows must be one-dimensional")
    if s.rows.size != s.row_offsets.size - 1:
        raise ValueError("rows length must match row_offsets size - 1")
    if s.rows.size > 1 and not bool(np.all(np.diff(s.rows.astype(np.int64)) > 0)):
        raise ValueError("rows must be strictly increasing")
    return s


def empty(rows: np.ndarray) -> ISet:
    rows = np.asarray(rows, dtype=I32)
    z = np.zeros(0, I32)
    return ISet(z, z.copy(), np.zeros(rows.size + 1, I32), rows)


def interval_rows(s: ISet) -> np.ndarray:
    """Row id of every interval (expressions.py:236-249)."""
    if s.begin.size == 0 or s.row_offsets.size <= 1:
        return np.zeros(0, I32)
    counts = np.diff(s.row_offsets.astype(np.int64))
    return np.repeat(s.rows, counts).astype(I32)


def interval_row_ordinals(s: ISet) -> np.ndarray:
    """Row ordinal of every interval (multilevel.py:154-166)."""
    if s.begin.size == 0 or s.row_offsets.size <= 1:
        return np.zeros(0, I32)
    counts = np.diff(s.row_offsets.astype(np.int64))
    return np.repeat(np.arange(s.row_count, dtype=I32), counts)


# ---------------------------------------------------------------------------
# Row alignment and binary operations (expressions.py:58-141, 446-528)
# ---------------------------------------------------------------------------

def reindex(s: ISet, rows_out: np.ndarray) -> ISet:
    """Re-express ``s`` on the row set ``rows_out`` (expressions.py:58-128).

    Intervals whose row is in ``rows_out`` keep their order.  Rows of
    ``rows_out`` that ``s`` lacks become empty rows.
    """
    rows_out = np.asarray(rows_out, dtype=I32)
    if rows_out.size == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(1, I32), rows_out)
    if s.rows.size == rows_out.size and np.array_equal(s.rows, rows_out):
        return ISet(s.begin, s.end, s.row_offsets, rows_out)
    per = interval_rows(s)
    if per.size == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(rows_out.size + 1, I32), rows_out)
    pos = np.searchsorted(rows_out, per)
    valid = pos < rows_out.size
    idx = np.nonzero(valid)[0]
    match = rows_out[pos[valid]] == per[valid]
    idx = idx[match]
    tpos = pos[valid][match]
    if idx.size == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(rows_out.size + 1, I32), rows_out)
    order = np.lexsort((idx, tpos))
    idx, tpos = idx[order], tpos[order]
    counts = np.bincount(tpos, minlength=rows_out.size)
    off = np.zeros(rows_out.size + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return ISet(s.begin[idx].astype(I32), s.end[idx].astype(I32), off.astype(I32), rows_out)


def align(lhs: ISet, rhs: ISet) -> Tuple[ISet, ISet, np.ndarray]:
    """Put both operands on ``union1d`` of their rows (expressions.py:131-141)."""
    if lhs.rows.size == rhs.rows.size and (lhs.rows.size == 0 or np.array_equal(lhs.rows, rhs.rows)):
        return lhs, rhs, lhs.rows
    rows_out = np.union1d(lhs.rows, rhs.rows).astype(I32)
    return reindex(lhs, rows_out), reindex(rhs, rows_out), rows_out


_OPS = {"union": 0, "intersection": 1, "difference": 2}


def apply_binary(lhs: ISet, rhs: ISet, mode: str) -> ISet:
    """One binary op: align, count, prefix sum, write (expressions.py:446-528)."""
    la, ra, rows_out = align(lhs, rhs)
    rows_out = np.asarray(rows_out, I32)
    R = la.row_offsets.size - 1
    if R == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(1, I32), rows_out)
    op = _OPS[mode]
    L = lib()
    counts = np.empty(R, I32)
    args = (_p(la.begin), _p(la.end), _p(la.row_offsets), _p(ra.begin), _p(ra.end), _p(ra.row_offsets))
    L.orc_setop_count(ctypes.c_int(op), ctypes.c_int64(R), *args, _p(counts))
    off = np.zeros(R + 1, I32)
    np.cumsum(counts, dtype=I32, out=off[1:])
    total = int(off[-1])
    if total == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), off, rows_out)
    ob = np.empty(total, I32)
    oe = np.empty(total, I32)
    L.orc_setop_write(ctypes.c_int(op), ctypes.c_int64(R), *args, _p(off), _p(ob), _p(oe))
    return ISet(ob, oe, off, rows_out)


def union(a, b): return apply_binary(a, b, "union")
def intersection(a, b): return apply_binary(a, b, "intersection")
def difference(a, b): return apply_binary(a, b, "difference")


def symmetric_difference(a: ISet, b: ISet) -> ISet:
    """(A \\ B) | (B \\ A), as make_symmetric_difference does (expressions.py:380-388)."""
    return union(difference(a, b), difference(b, a))


def complement(universe: ISet, subset: ISet) -> ISet:
    """universe \\ subset (expressions.py:391-399)."""
    return difference(universe, subset)


BINARY: Dict[str, Callable[[ISet, ISet], ISet]] = {
    "union": union,
    "intersection": intersection,
    "difference": difference,
    "symmetric_difference": symmetric_difference,
    "complement": complement,
}


def evaluate(spec, leaves: Dict[str, ISet]) -> ISet:
    """Evaluate a nested tuple ``(op, lhs, rhs)`` over named leaves, lhs first (expressions.py:357-360)."""
    if isinstance(spec, str):
        return leaves[spec]
    return BINARY[spec[0]](evaluate(spec[1], leaves), evaluate(spec[2], leaves))


# ---------------------------------------------------------------------------
# Morphology (morphology.py)
# ---------------------------------------------------------------------------

def build_from_rows(rows, begin, end, rows_hint=None) -> ISet:
    """Sort by (row, begin), group rows, merge touching runs (morphology.py:21-107)."""
    rows = np.asarray(rows, I32)
    begin = np.asarray(begin, I32)
    end = np.asarray(end, I32)
    if begin.size == 0:
        if rows_hint is not None:
            rows_out = np.unique(np.asarray(rows_hint, I32))
            return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(rows_out.size + 1, I32), rows_out.astype(I32))
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(1, I32), np.zeros(0, I32))
    order = np.lexsort((begin, rows))
    rs, bs, es = rows[order], begin[order], end[order]
    uniq, inverse = np.unique(rs, return_inverse=True)
    rows_out = np.union1d(np.unique(np.asarray(rows_hint, I32)), uniq) if rows_hint is not None else uniq
    rows_out = rows_out.astype(I32)
    R = rows_out.size
    counts_full = np.zeros(R, np.int64)
    counts_full[np.searchsorted(rows_out, uniq)] = np.bincount(inverse, minlength=uniq.size)
    raw_off = np.zeros(R + 1, I32)
    np.cumsum(counts_full, dtype=I32, out=raw_off[1:])
    L = lib()
    counts = np.empty(R, I32)
    bs = np.ascontiguousarray(bs, I32)
    es = np.ascontiguousarray(es, I32)
    L.orc_merge_rows(ctypes.c_int64(R), _p(bs), _p(es), _p(raw_off), None, _p(counts), None, None)
    off = np.zeros(R + 1, I32)
    np.cumsum(counts, dtype=I32, out=off[1:])
    total = int(off[-1])
    if total == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), off, rows_out)
    ob = np.empty(total, I32)
    oe = np.empty(total, I32)
    L.orc_merge_rows(ctypes.c_int64(R), _p(bs), _p(es), _p(raw_off), _p(off), None, _p(ob), _p(oe))
    return ISet(ob, oe, off, rows_out)


def copy(s: ISet) -> ISet:
    return ISet(s.begin.copy(), s.end.copy(), s.row_offsets.copy(), s.rows.copy())


def dilate(s: ISet, halo_x: int = 1, halo_y: int = 1) -> ISet:
    """Box dilation, unbounded (morphology.py:211-265)."""
    if halo_x < 0 or halo_y < 0:
        raise ValueError("halo_x and halo_y must be non-negative")
    if halo_x == 0 and halo_y == 0:
        return copy(s)
    b = s.begin.astype(I32)
    e = s.end.astype(I32)
    per = interval_rows(s)
    if halo_x > 0:
        b = (b - halo_x).astype(I32)
        e = (e + halo_x).astype(I32)
    if per.size == 0:
        rows_arr = s.rows if s.row_count > 0 else np.zeros(0, I32)
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(s.row_count + 1, I32), rows_arr)
    if halo_y == 0:
        return build_from_rows(per, b, e, rows_hint=s.rows)
    shifts = np.arange(-halo_y, halo_y + 1, dtype=I32)
    rows_all = (per[:, None] + shifts[None, :]).reshape(-1)
    return build_from_rows(rows_all, np.repeat(b, shifts.size), np.repeat(e, shifts.size))


def full(width: int, height: int) -> ISet:
    """Full rectangle [0, width) x [0, height) (morphology.py:344-358)."""
    if height <= 0 or width <= 0:
        z = np.zeros(0, I32)
        return ISet(z, z.copy(), np.zeros(1, I32), z.copy())
    return ISet(np.zeros(height, I32), np.full(height, width, I32), np.arange(height + 1, dtype=I32),
                np.arange(height, dtype=I32))


def clip(s: ISet, width: int, height: int) -> ISet:
    """Clip to [0, width) x [0, height) with dense rows (morphology.py:268-319)."""
    if width <= 0:
        raise ValueError("width must be positive")
    if height < 0:
        raise ValueError("height must be non-negative")
    clipped = intersection(full(width, height), s)

    def dense_empty():
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(height + 1, I32), np.arange(height, dtype=I32))

    if clipped.begin.size == 0:
        return dense_empty()
    rows = interval_rows(clipped)
    if rows.size == 0:
        return dense_empty()
    mask = (rows >= 0) & (rows < height)
    rows, b, e = rows[mask], clipped.begin[mask], clipped.end[mask]
    if rows.size == 0:
        return dense_empty()
    return build_from_rows(rows, b, e, rows_hint=np.arange(height, dtype=I32))


def ghost_zones(s: ISet, halo_x: int = 1, halo_y: int = 1, *, width: int, height: Optional[int] = None) -> ISet:
    """clip(dilate(S)) \\ clip(S) (morphology.py:322-341)."""
    if height is None:
        height = s.row_offsets.size - 1
    return copy(difference(clip(dilate(s, halo_x, halo_y), width, height), clip(s, width, height)))


def erode(s: ISet, halo_x: int = 1, halo_y: int = 1, *, width: int, height: Optional[int] = None) -> ISet:
    """U \\ clip(dilate(U \\ clip(S))) with U the domain (morphology.py:361-386)."""
    if height is None:
        height = s.row_offsets.size - 1
    if width <= 0 or height < 0:
        raise ValueError("width must be positive and height must be non-negative")
    base = clip(s, width, height)
    universe = full(width, height)
    comp = difference(universe, base)
    dil = clip(dilate(comp, halo_x, halo_y), width, height)
    return copy(difference(universe, dil))


# ---------------------------------------------------------------------------
# Multilevel sets and fields (multilevel.py, interval_field.py)
# ---------------------------------------------------------------------------

def prolong_set_impl(s: ISet, ratio: int) -> Tuple[ISet, np.ndarray]:
    """Scale by ``ratio``; only occupied rows are kept (multilevel.py:213-264)."""
    if ratio < 1:
        raise ValueError("ratio must be >= 1")
    if ratio == 1:
        return s, np.arange(s.begin.size, dtype=I32)
    R = s.row_count
    rv = np.arange(ratio, dtype=I32)
    if R == 0 or s.begin.size == 0:
        fine_rows = (s.rows[:, None] * ratio + rv[None, :]).reshape(-1) if R > 0 else np.zeros(0, I32)
        rows_out = np.sort(fine_rows).astype(I32)
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(rows_out.size + 1, I32), rows_out), np.zeros(0, I32)
    n = s.begin.size
    sb = (s.begin * ratio).astype(I32)
    se = (s.end * ratio).astype(I32)
    base = np.repeat(np.arange(n, dtype=I32), ratio)
    frows = (interval_rows(s)[:, None] * ratio + rv[None, :]).reshape(-1).astype(I32)
    rb = np.repeat(sb, ratio)
    re = np.repeat(se, ratio)
    order = np.lexsort((rb, frows))
    frows_s, b_s, e_s, base_s = frows[order], rb[order], re[order], base[order]
    rows_out = np.unique(frows_s).astype(I32)
    pos = np.searchsorted(rows_out, frows_s, side="left")
    counts = np.bincount(pos, minlength=rows_out.size)
    off = np.zeros(rows_out.size + 1, I32)
    np.cumsum(counts, dtype=I32, out=off[1:])
    return ISet(b_s.astype(I32), e_s.astype(I32), off, rows_out), base_s.astype(I32)


def prolong_set(s: ISet, ratio: int) -> ISet:
    return prolong_set_impl(s, ratio)[0]


def restrict_set(s: ISet, ratio: int) -> ISet:
    """Floor/ceil coarsening, then sort and merge (multilevel.py:272-362)."""
    if ratio < 1:
        raise ValueError("ratio must be >= 1")
    R = s.row_count
    if R == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(1, I32), np.zeros(0, I32))
    if s.begin.size == 0:
        cr = np.unique(s.rows // ratio).astype(I32)
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(cr.size + 1, I32), cr)
    crows = (interval_rows(s) // ratio).astype(I32)
    cb = (s.begin // ratio).astype(I32)
    ce = ((s.end + ratio - 1) // ratio).astype(I32)
    mask = ce > cb
    if not bool(mask.any()):
        cr = np.unique(crows).astype(I32)
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(cr.size + 1, I32), cr)
    crows, cb, ce = crows[mask], cb[mask], ce[mask]
    order = np.lexsort((cb, crows))
    crows, cb, ce = crows[order], np.ascontiguousarray(cb[order]), np.ascontiguousarray(ce[order])
    rows_out = np.unique(crows).astype(I32)
    pos = np.searchsorted(rows_out, crows, side="left")
    raw = np.zeros(rows_out.size + 1, I32)
    np.cumsum(np.bincount(pos, minlength=rows_out.size), dtype=I32, out=raw[1:])
    L = lib()
    counts = np.empty(rows_out.size, I32)
    L.orc_merge_rows(ctypes.c_int64(rows_out.size), _p(cb), _p(ce), _p(raw), None, _p(counts), None, None)
    off = np.zeros(rows_out.size + 1, I32)
    np.cumsum(counts, dtype=I32, out=off[1:])
    total = int(off[-1])
    if total == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), off, rows_out)
    ob = np.empty(total, I32)
    oe = np.empty(total, I32)
    L.orc_merge_rows(ctypes.c_int64(rows_out.size), _p(cb), _p(ce), _p(raw), _p(off), None, _p(ob), _p(oe))
    return ISet(ob, oe, off, rows_out)


def cell_offsets(s: ISet) -> np.ndarray:
    """int32 prefix sum of interval lengths (interval_field.py:67-73)."""
    off = np.zeros(s.begin.size + 1, I32)
    if s.begin.size:
        np.cumsum((s.end - s.begin).astype(I32), dtype=I32, out=off[1:])
    return off


def coarse_to_fine_indices(coarse: ISet, fine: ISet, ratio: int) -> np.ndarray:
    """Fine interval index of each (coarse interval, sub-row) (multilevel.py:169-210).

    Out-of-range positions wrap around, as device-array fancy indexing does
    in the reference.  A misaligned fine set therefore fails the same
    equality checks and raises the same ``ValueError``.
    """
    if ratio < 1:
        raise ValueError("ratio must be >= 1")
    crows, frows = coarse.rows, fine.rows
    if crows.size == 0:
        return np.zeros(0, I32)
    expected = (crows[:, None].astype(np.int64) * ratio + np.arange(ratio)[None, :]).reshape(-1)
    if frows.size != expected.size:
        raise ValueError("fine set row count does not match coarse x ratio")
    if bool(np.any(frows != expected)):
        raise ValueError("fine set rows do not align with refinement ratio")
    n = coarse.begin.size
    if n == 0:
        return np.zeros(0, I32)
    ords = interval_row_ordinals(coarse)
    ordinal = np.arange(n, dtype=np.int64) - coarse.row_offsets[ords]
    actual = crows[ords].astype(np.int64)
    fvals = actual[:, None] * ratio + np.arange(ratio)[None, :]
    fords = np.searchsorted(frows, fvals, side="left").reshape(-1)
    wrapped = fords % frows.size
    if bool(np.any(frows[wrapped] != fvals.reshape(-1))):
        raise ValueError("fine row ids missing expected refinement entries")
    foff = fine.row_offsets.astype(np.int64)
    idx = foff[fords % foff.size] + np.repeat(ordinal, ratio)
    return idx.astype(I32)


class Field(NamedTuple):
    iset: ISet
    values: np.ndarray
    offsets: np.ndarray


def create_field(s: ISet, fill=0.0, dtype=np.float32) -> Field:
    off = cell_offsets(s)
    return Field(s, np.full(int(off[-1]), fill, dtype=dtype), off)


def prolong_field(f: Field, ratio: int, dtype=np.float32) -> Field:
    """Fine field by injection on the prolonged set (multilevel.py:365-407).

    ``dtype`` float32 is the reference.  float64 is the new FP64 path with
    the same structure.
    """
    if ratio < 1:
        raise ValueError("ratio must be >= 1")
    fine_set, _ = prolong_set_impl(f.iset, ratio)
    out = create_field(fine_set, 0.0, dtype)
    if out.values.size == 0 or f.values.size == 0:
        return out
    if ratio == 1:
        out.values[...] = f.values.astype(dtype)
        return out
    n = f.iset.begin.size
    if n == 0:
        return out
    fidx = coarse_to_fine_indices(f.iset, fine_set, ratio)
    src = np.ascontiguousarray(f.values.astype(dtype))
    fn = lib().orc_prolong_field_f32 if dtype == np.float32 else lib().orc_prolong_field_f64
    fn(ctypes.c_int64(n), ctypes.c_int(ratio), _p(f.offsets), _p(out.offsets), _p(fidx), _p(src), _p(out.values))
    return out


_REDUCERS = {"mean": 0, "sum": 1, "min": 2, "max": 3}


def restrict_field(f: Field, ratio: int, reducer: str = "mean", dtype=np.float32) -> Field:
    """Block reduction onto ``restrict_set`` of the fine set (multilevel.py:410-479)."""
    coarse_set = restrict_set(f.iset, ratio)
    out = create_field(coarse_set, 0.0, dtype)
    if f.values.size == 0 or out.values.size == 0:
        return out
    if ratio <= 0:
        raise ValueError("ratio must be >= 1")
    if ratio == 1:
        # the reference raises NameError here (multilevel.py:421-423)
        raise NameError("name 'target_dtype' is not defined")
    code = _REDUCERS.get(reducer)
    if code is None:
        raise ValueError(f"unsupported reducer '{reducer}'")
    n = coarse_set.begin.size
    if n == 0:
        return out
    fidx = coarse_to_fine_indices(coarse_set, f.iset, ratio)
    if fidx.size != n * ratio:
        raise ValueError("interval mapping mismatch for restriction")
    exp_b = np.repeat(coarse_set.begin.astype(np.int64) * ratio, ratio)
    exp_e = np.repeat(coarse_set.end.astype(np.int64) * ratio, ratio)
    nf = f.iset.begin.size
    wrapped = fidx % nf if nf else fidx
    if bool(np.any(f.iset.begin[wrapped] != exp_b)) or bool(np.any(f.iset.end[wrapped] != exp_e)):
        raise ValueError("fine field is not aligned with coarse geometry for restriction")
    src = np.ascontiguousarray(f.values.astype(dtype))
    if dtype == np.float32:
        norm = ctypes.c_float(np.float32(1.0 / (ratio * ratio)) if code == 0 else np.float32(1.0))
        fn = lib().orc_restrict_field_f32
    else:
        norm = ctypes.c_double(1.0 / (ratio * ratio) if code == 0 else 1.0)
        fn = lib().orc_restrict_field_f64
    fn(ctypes.c_int64(n), ctypes.c_int(ratio), ctypes.c_int(code), norm, _p(out.offsets), _p(f.offsets),
       _p(fidx), _p(src), _p(out.values))
    return out


# ---------------------------------------------------------------------------
# Upwind (interval_stencil.py:126-219)
# ---------------------------------------------------------------------------

def upwind(f: Field, *, width: int, height: int, a: float, b: float, dt: float, dx: float, dy: float,
           dtype=np.float32) -> np.ndarray:
    """One first-order upwind step with zero exterior.

    ``dtype`` float32 follows the reference, which casts every parameter to
    float32.  float64 is the new FP64 oracle.
    """
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    s = f.iset
    vals = np.ascontiguousarray(f.values.astype(dtype))
    out = np.empty_like(vals)
    n = s.begin.size
    if n == 0:
        out.fill(0)
        return out
    row_ids = interval_rows(s)
    # Rows must lie in [0, height).  The reference builds its row lookup by
    # fancy-index assignment, which on the device wraps out-of-range rows
    # instead of rejecting them (interval_stencil.py:183-191); that case is
    # rejected here.
    if s.rows.size and (int(s.rows.min()) < 0 or int(s.rows.max()) >= height):
        raise ValueError("interval_set rows exceed provided height")
    lookup = np.full(height, -1, I32)
    if s.rows.size:
        lookup[s.rows] = np.arange(s.rows.size, dtype=I32)
    ords = lookup[row_ids]
    if int(ords.min()) < 0:
        raise ValueError("interval_set rows exceed provided height")
    ct = ctypes.c_float if dtype == np.float32 else ctypes.c_double
    fn = lib().orc_upwind_f32 if dtype == np.float32 else lib().orc_upwind_f64
    cast = np.float32 if dtype == np.float32 else np.float64
    fn(ctypes.c_int64(n), _p(row_ids), _p(s.begin), _p(s.end), _p(s.row_offsets), _p(f.offsets), _p(ords),
       _p(lookup), _p(vals), _p(out), ctypes.c_int(width), ctypes.c_int(height),
       ct(cast(a)), ct(cast(b)), ct(cast(dt)), ct(cast(dx)), ct(cast(dy)))
    return out


# ---------------------------------------------------------------------------
# Regrid (subsetix_amr2/regrid.py)
# ---------------------------------------------------------------------------

def gradient_magnitude(values: np.ndarray, width: int, height: int) -> np.ndarray:
    """regrid.py:233-274 on a full grid field."""
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    data = np.ascontiguousarray(values.astype(np.float32))
    if data.size != width * height:
        raise ValueError("field cell count mismatch with width/height")
    out = np.empty_like(data)
    lib().orc_gradient_f32(_p(data), ctypes.c_int(width), ctypes.c_int(height), _p(out))
    return out


def threshold_intervals(values: np.ndarray, width: int, height: int, threshold: float) -> ISet:
    """Rows of ``values >= threshold`` as intervals, rows = arange(height) (regrid.py:277-333)."""
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    data = np.ascontiguousarray(values.astype(np.float32))
    if data.size != width * height:
        raise ValueError("field cell count mismatch with width/height")
    L = lib()
    counts = np.empty(height, I32)
    thr = ctypes.c_float(np.float32(threshold))
    L.orc_threshold_rle(_p(data), ctypes.c_int(width), ctypes.c_int(height), thr, None, _p(counts), None, None)
    off = np.zeros(height + 1, I32)
    np.cumsum(counts, dtype=I32, out=off[1:])
    total = int(off[-1])
    ob = np.empty(total, I32)
    oe = np.empty(total, I32)
    if total:
        L.orc_threshold_rle(_p(data), ctypes.c_int(width), ctypes.c_int(height), thr, _p(off), None, _p(ob), _p(oe))
    return ISet(ob, oe, off, np.arange(height, dtype=I32))


def gradient_tag_threshold(values, width, height, threshold, epsilon=1e-8) -> ISet:
    """regrid.py:336-350."""
    return threshold_intervals(gradient_magnitude(values, width, height), width, height,
                               max(float(threshold), float(epsilon)))


def gradient_tag_set(values, width, height, frac_high, epsilon=1e-8) -> ISet:
    """Runs of the top ``frac_high`` fraction of the positive values (regrid.py:353-383).

    The threshold is the value of rank ``n - ceil(n * frac)`` among the
    ``n`` values above ``epsilon`` (a k-th order statistic, the same for any
    partition algorithm); cells with ``value >= max(threshold, epsilon)`` are
    tagged.
    """
    frac = float(max(0.0, min(1.0, frac_high)))
    if frac <= 0.0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(height + 1, I32), np.arange(height, dtype=I32))
    v = np.asarray(values, np.float32).reshape(-1)
    pos = v[v > np.float32(epsilon)]
    if pos.size == 0:
        return ISet(np.zeros(0, I32), np.zeros(0, I32), np.zeros(height + 1, I32), np.arange(height, dtype=I32))
    count = max(1, min(int(pos.size), int(np.ceil(pos.size * frac))))
    idx = int(pos.size) - count
    thr = float(np.partition(pos, idx)[idx])
    return threshold_intervals(v, width, height, max(thr, float(epsilon)))


def grading(refine: ISet, padding: int = 1, mode: str = "von_neumann", *, width: int, height: int) -> ISet:
    """Two-level grading dilation (regrid.py:404-442)."""
    padding = int(padding)
    if padding <= 0:
        return refine
    if mode not in {"von_neumann", "moore"}:
        raise ValueError("mode must be 'von_neumann' or 'moore'")
    if mode == "moore":
        expanded = dilate(refine, padding, padding)
    else:
        expanded = union(dilate(refine, padding, 0), dilate(refine, 0, padding))
    expanded = clip(expanded, width, height)
    base = clip(refine, width, height)
    return clip(union(base, expanded), width, height)


# ---------------------------------------------------------------------------
# Fields synchronisation (subsetix_amr2/fields.py)
# ---------------------------------------------------------------------------

def subset_copy(direction: str, super_f: Field, sub_f: Field) -> None:
    """Gather (super -> sub) or scatter (sub -> super) by coordinates (fields.py:302-385)."""
    n = sub_f.iset.begin.size
    if n == 0:
        return
    sub_rows = interval_rows(sub_f.iset)
    super_rows = super_f.iset.rows
    pos = np.searchsorted(super_rows, sub_rows, side="left")
    wrapped = pos % super_rows.size if super_rows.size else pos
    if super_rows.size == 0 or bool(np.any(super_rows[wrapped] != sub_rows)):
        which = "source" if direction == "gather" else "destination"
        raise ValueError(f"subset rows must be contained within the {which} field")
    pos = pos.astype(I32)
    es = sub_f.values.dtype.itemsize
    lib().orc_subset_copy(ctypes.c_int(0 if direction == "gather" else 1), ctypes.c_int64(n), ctypes.c_int(es),
                          _p(pos), _p(sub_f.iset.begin), _p(sub_f.iset.end), _p(sub_f.offsets),
                          _p(super_f.iset.row_offsets), _p(super_f.iset.begin), _p(super_f.iset.end),
                          _p(super_f.offsets), ctypes.c_int32(super_f.iset.row_count),
                          _p(sub_f.values), _p(super_f.values))


def gather_subset(super_f: Field, subset: ISet) -> Field:
    out = create_field(subset, 0, super_f.values.dtype)
    subset_copy("gather", super_f, out)
    return out


def scatter_subset(super_f: Field, sub_f: Field) -> None:
    subset_copy("scatter", super_f, sub_f)


def value_intervals(f: Field, target) -> ISet:
    """Runs of cells equal to ``target`` inside each interval (fields.py:41-100)."""
    s = f.iset
    total = f.values.size
    if total == 0:
        return empty(s.rows.copy())
    match = f.values == f.values.dtype.type(target)
    if not bool(match.any()):
        return empty(s.rows.copy())
    off = f.offsets
    idx_of = np.repeat(np.arange(s.begin.size), np.diff(off.astype(np.int64)))
    local = np.arange(total) - off[idx_of]
    cols = s.begin[idx_of] + local
    rows_c = interval_rows(s)[idx_of]
    prev = np.zeros(total, bool)
    prev[1:] = match[:-1]
    prev[off[:-1][off[:-1] < total]] = False
    start = match & ~prev
    nxt = np.zeros(total, bool)
    nxt[:-1] = match[1:]
    ends_idx = off[1:] - 1
    nxt[ends_idx[(ends_idx >= 0) & (ends_idx < total)]] = False
    stop = match & ~nxt
    si = np.nonzero(start)[0]
    ei = np.nonzero(stop)[0]
    if si.size == 0:
        return empty(s.rows.copy())
    rpos = np.searchsorted(s.rows, rows_c[si], side="left")
    cnt = np.bincount(rpos, minlength=s.rows.size)
    roff = np.zeros(s.rows.size + 1, I32)
    np.cumsum(cnt, dtype=I32, out=roff[1:])
    return ISet(cols[si].astype(I32), (cols[ei] + 1).astype(I32), roff, s.rows.copy())


class Actions:
    """ActionField equivalent over a full coarse grid (fields.py:443-569)."""

    def __init__(self, width: int, height: int, ratio: int):
        self.width, self.height, self.ratio = int(width), int(height), int(ratio)
        self.domain = full(width, height)
        self.field = create_field(self.domain, 0, np.int8)
        self.refine = empty(self.domain.rows.copy())

    def set_from(self, refine: ISet) -> None:
        if refine.begin.size == 0:
            self.field.values.fill(0)
            self.refine = empty(self.domain.rows.copy())
            return
        outside = difference(refine, self.domain)
        if outside.begin.size != 0:
            raise ValueError("refine_set must be contained within the action domain")
        aligned = intersection(refine, self.domain)
        self.field.values.fill(0)
        scatter_subset(self.field, create_field(aligned, 1, np.int8))
        self.refine = aligned

    def fine_set(self) -> ISet:
        return prolong_set(self.refine, self.ratio)

    def coarse_only(self) -> ISet:
        return difference(self.domain, self.refine)


def synchronize(coarse: Field, fine: Field, actions: Actions, ratio: int, dtype=np.float32,
                coarse_only: Optional[ISet] = None) -> None:
    """In-place coarse/fine sync with the mean reducer (fields.py:570-612, copy=False)."""
    restricted = restrict_field(fine, ratio, "mean", dtype)
    if actions.refine.begin.size != 0:
        scatter_subset(coarse, gather_subset(restricted, actions.refine))
    co = actions.coarse_only() if coarse_only is None else coarse_only
    if co.begin.size != 0:
        sub = gather_subset(coarse, co)
        fsub = prolong_field(sub, ratio, dtype)
        if fsub.values.size != 0:
            scatter_subset(fine, fsub)


class AMR2:
    """AMR2Simulation restated (simulation.py:275-489), FP32 or FP64 storage."""

    def __init__(self, resolution: int, velocity, cfl: float = 0.9, threshold: float = 0.05,
                 grading_pad: int = 1, mode: str = "von_neumann", ratio: int = 2, dtype=np.float32):
        self.W = self.H = int(resolution)
        self.ratio = int(ratio)
        self.velocity = (float(velocity[0]), float(velocity[1]))
        self.threshold, self.pad, self.mode = float(threshold), int(grading_pad), mode
        self.dtype = dtype
        self.dxc = 1.0 / self.W
        self.dyc = 1.0 / self.H
        self.dxf = self.dxc / ratio
        self.dyf = self.dyc / ratio
        denom = abs(self.velocity[0]) / self.dxf + abs(self.velocity[1]) / self.dyf
        self.dt = cfl / denom if denom > 0 else 0.0
        self.step = 0
        self.time = 0.0

    def refine_from(self, coarse: Field) -> ISet:
        tags = gradient_tag_threshold(coarse.values, self.W, self.H, self.threshold)
        return grading(tags, self.pad, self.mode, width=self.W, height=self.H)

    def init(self, coarse_values: np.ndarray) -> None:
        dom = full(self.W, self.H)
        self.coarse = Field(dom, np.asarray(coarse_values, self.dtype).reshape(-1).copy(), cell_offsets(dom))
        self.actions = Actions(self.W, self.H, self.ratio)
        self.actions.set_from(self.refine_from(self.coarse))
        self.coarse_only = self.actions.coarse_only()
        self.fine = prolong_field(self.coarse, self.ratio, self.dtype)

    def _sync(self):
        synchronize(self.coarse, self.fine, self.actions, self.ratio, self.dtype, self.coarse_only)

    def run(self, steps: int, regrid_every: int = 1) -> None:
        period = max(1, int(regrid_every))
        a, b = self.velocity
        for _ in range(int(steps)):
            self._sync()
            if self.step % period == 0:
                self.actions.set_from(self.refine_from(self.coarse))
                self.coarse_only = self.actions.coarse_only()
            cv = upwind(self.coarse, width=self.W, height=self.H, a=a, b=b, dt=self.dt, dx=self.dxc, dy=self.dyc,
                        dtype=self.dtype)
            fv = upwind(self.fine, width=self.W * self.ratio, height=self.H * self.ratio, a=a, b=b, dt=self.dt,
                        dx=self.dxf, dy=self.dyf, dtype=self.dtype)
            self.coarse = Field(self.coarse.iset, cv, self.coarse.offsets)
            self.fine = Field(self.fine.iset, fv, self.fine.offsets)
            self._sync()
            self.step += 1
            self.time += self.dt


# ---------------------------------------------------------------------------
# Dense-mask oracle (canonical inputs only)
# ---------------------------------------------------------------------------

def to_cells(s: ISet) -> set:
    cells = set()
    for ordinal, row in enumerate(s.rows.tolist()):
        for i in range(int(s.row_offsets[ordinal]), int(s.row_offsets[ordinal + 1])):
            cells.update((row, c) for c in range(int(s.begin[i]), int(s.end[i])))
    return cells


def mass_kahan(values: np.ndarray, cell_area: float) -> float:
    """Compensated (Neumaier) sum of ``values * cell_area`` in float64."""
    s = 0.0
    c = 0.0
    for v in np.asarray(values, dtype=np.float64).tolist():
        t = s + v
        if abs(s) >= abs(v):
            c += (s - t) + v
        else:
            c += (v - t) + s
        s = t
    return (s + c) * cell_area
