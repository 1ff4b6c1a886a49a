"""Morphology on interval sets (drop-in for ``subsetix_cupy.morphology``).

Names, arguments, results and exceptions follow the reference module
(``subsetix_cupy/morphology.py``).  The compute path is new:

* Dilation does not build ``(2*halo_y + 1) * n`` candidate intervals and
  sort them.  The occupied rows are shifted by every ``dy`` and aligned on
  the device (``sx_align_rows``).  Then one union-mode row sweep
  (``sx_bool_eval``, ``SX_MODE_UNION``) merges the widened intervals of up to
  9 shifted copies per launch.  Larger ``halo_y`` chains sweeps of at most 9
  copies each; box dilation composes exactly.
* Clipping is one fused intersection with the domain rectangle on dense
  rows.
* Inputs outside the sweeps' contract (empty, unsorted or overlapping
  intervals) are detected on the device.  They then take the reference's
  sort-and-merge construction, :func:`_build_interval_set_from_rows`, which
  runs as a device sort plus this package's row-merge kernel.
"""

from __future__ import annotations

from numbers import Integral
from typing import Optional

import torch

from .. import _core, _lib
from .expressions import (
    CuPyWorkspace,
    IntervalSet,
    _dense_key,
    _t,
    evaluate,
    make_difference,
    make_input,
    make_intersection,
)
from .._runtime import like

I32 = torch.int32
_MAX_SHIFTS = 9  # leaves per union sweep


def _kind(s: IntervalSet):
    return s.begin


def _empty_set(device, rows: Optional[torch.Tensor] = None, kind=None) -> IntervalSet:
    z = torch.zeros(0, dtype=I32, device=device)
    r = z.clone() if rows is None else rows
    off = torch.zeros(int(r.numel()) + 1, dtype=I32, device=device)
    return IntervalSet._trusted(like(kind, z), like(kind, z.clone()), like(kind, off), like(kind, r))


def _wrap(kind, b, e, off, rows, dense=None) -> IntervalSet:
    return IntervalSet._trusted(like(kind, b), like(kind, e), like(kind, off), like(kind, rows), dense)


def _build_interval_set_from_rows(rows, begin, end, *, rows_hint=None, kind=None) -> IntervalSet:
    """Sort by (row, begin), group rows (with ``rows_hint``), merge (``morphology.py:21-105``).

    The lexicographic sort is a stable device sort of one 64-bit key, which
    orders ties the same way as the reference's ``lexsort``.  The output rows
    are the device row union (``sx_align_rows``), and the merge is
    ``sx_merge_rows`` (the reference's merge kernels).
    """
    b = _t(begin).to(I32)
    device = b.device
    e = _t(end).to(I32)
    kind = begin if kind is None else kind
    if b.numel() == 0:
        if rows_hint is not None:
            rows_out = torch.unique(_t(rows_hint).to(device=device, dtype=I32))
            return _empty_set(device, rows_out.to(I32), kind)
        return _empty_set(device, None, kind)
    r = _t(rows).to(device=device, dtype=I32)
    key = (r.to(torch.int64) << 32) | (b.to(torch.int64) + (1 << 31))
    order = torch.sort(key, stable=True).indices
    r_s, b_s, e_s = r[order], b[order], e[order]
    n = int(r_s.numel())
    ident = torch.arange(n + 1, dtype=I32, device=device)
    lists = [(r_s, ident, 0, False)]
    ends = [r_s[0:1], r_s[-1:]]
    if rows_hint is not None:
        hint = _t(rows_hint).to(device=device, dtype=I32).reshape(-1)
        if hint.numel():
            lists.append((hint, None, 0, False))
            ends += [hint.min().reshape(1), hint.max().reshape(1)]
    host = torch.cat(ends).cpu()
    lo, hi = int(host.min()), int(host.max())
    rows_out, offs = _core.align_rows(lists, lo, hi, device, [True] + [False] * (len(lists) - 1))
    ob, oe, off = _core.merge_rows(b_s, e_s, offs[0], device)
    return _wrap(kind, ob, oe, off, rows_out)


def _compact_interval_set(interval_set: IntervalSet) -> IntervalSet:
    """Occupied rows only, touching and overlapping intervals merged (``morphology.py:108-110``)."""
    s = interval_set
    device = _t(s.row_offsets).device
    n = int(s.begin.shape[0])
    if n == 0:
        return _empty_set(device, None, s.begin)
    out = _union_sweep(s, [0], 0, skip_empty=True)
    if out is not None:
        return out
    return _build_interval_set_from_rows(s.interval_rows(), s.begin, s.end, kind=s.begin)


def _union_sweep(s: IntervalSet, shifts, widen: int, skip_empty: bool) -> Optional[IntervalSet]:
    """Merged union of ``s`` shifted by each row offset in ``shifts`` and widened by ``widen``.

    Output rows: the shifted occupied rows (``skip_empty``) or, with the
    single shift 0 and ``skip_empty`` False, the rows of ``s``.  Returns None
    when the input is outside the union sweep's contract.
    """
    device = _t(s.row_offsets).device
    b, e = _t(s.begin), _t(s.end)
    rows, off = _t(s.rows), _t(s.row_offsets)
    dense = None
    if not skip_empty and list(shifts) == [0]:
        rows_out, offs = rows, [off]
        dense = _dense_key(s)
    else:
        host = torch.cat([rows[0:1], rows[-1:]]).cpu()
        lo, hi = int(host[0]) + min(shifts), int(host[1]) + max(shifts)
        lists = [(rows, off, dy, skip_empty) for dy in shifts]
        rows_out, offs = _core.align_rows(lists, lo, hi, device, [True] * len(lists))
    R = int(rows_out.numel())
    if R == 0:
        return _empty_set(device, rows_out, s.begin)
    leaves = [(b, e, o, widen) for o in offs]
    ob, oe, ooff, total, flags = _core.bool_eval(leaves, R, [0] * 8, _lib.MODE_UNION, device)
    if flags & _lib.FLAG_CONTRACT:
        return None
    if flags & (_lib.FLAG_CAPACITY | _lib.FLAG_TIMEOUT):
        raise _lib.SubsetixError(f"union sweep failed (flags={flags})")
    return _wrap(s.begin, ob[:total].clone(), oe[:total].clone(), ooff, rows_out, dense)


def translate_interval_set(interval_set: IntervalSet, dx: int = 0, dy: int = 0) -> IntervalSet:
    """Shift every interval by ``dx`` and every row by ``dy`` (``morphology.py:113-137``)."""
    if not isinstance(dx, Integral) or not isinstance(dy, Integral):
        raise TypeError("dx and dy must be integers")
    dx, dy = int(dx), int(dy)
    s = interval_set
    if dx == 0 and dy == 0:
        return s.copy()
    b = _t(s.begin).clone()
    e = _t(s.end).clone()
    if dx:
        b += dx
        e += dx
    rows = _t(s.rows).clone()
    if dy and rows.numel() > 0:
        rows += dy
    return IntervalSet(like(s.begin, b), like(s.begin, e), like(s.begin, _t(s.row_offsets).clone()),
                       like(s.begin, rows))


def _check_direction(dx, dy) -> None:
    if not isinstance(dx, Integral) or not isinstance(dy, Integral):
        raise TypeError("dx and dy must be integers")
    if dx == 0 and dy == 0:
        raise ValueError("direction (dx, dy) must be non-zero")


def interior_for_direction(interval_set: IntervalSet, dx: int, dy: int, *,
                           workspace: Optional[CuPyWorkspace] = None) -> IntervalSet:
    """Cells whose neighbour at ``(dx, dy)`` is also in the set (``morphology.py:140-161``)."""
    _check_direction(dx, dy)
    neighbour = translate_interval_set(interval_set, dx=-int(dx), dy=-int(dy))
    interior = evaluate(make_intersection(make_input(interval_set), make_input(neighbour)), workspace=workspace)
    return _compact_interval_set(interior).copy()


def boundary_for_direction(interval_set: IntervalSet, dx: int, dy: int, *,
                           workspace: Optional[CuPyWorkspace] = None) -> IntervalSet:
    """Cells lacking a neighbour at ``(dx, dy)`` (``morphology.py:164-183``)."""
    _check_direction(dx, dy)
    interior = interior_for_direction(interval_set, dx=dx, dy=dy, workspace=workspace)
    boundary = evaluate(make_difference(make_input(interval_set), make_input(interior)), workspace=workspace)
    return _compact_interval_set(boundary).copy()


def boundary_layer(interval_set: IntervalSet, *, workspace: Optional[CuPyWorkspace] = None) -> IntervalSet:
    """Cells missing at least one axial neighbour (``morphology.py:186-208``)."""
    interior = interval_set
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        neighbour = translate_interval_set(interval_set, dx=-dx, dy=-dy)
        interior = evaluate(make_intersection(make_input(interior), make_input(neighbour)), workspace=workspace)
    interior_compact = _compact_interval_set(interior)
    boundary = evaluate(make_difference(make_input(interval_set), make_input(interior_compact)), workspace=workspace)
    return _compact_interval_set(boundary).copy()


def _dilate_reference_order(s: IntervalSet, halo_x: int, halo_y: int) -> IntervalSet:
    """Candidate intervals plus sort-and-merge, as the reference builds them (``morphology.py:211-248``)."""
    b = _t(s.begin).to(I32)
    e = _t(s.end).to(I32)
    per = _t(s.interval_rows())
    if halo_x > 0:
        b = b - halo_x
        e = e + halo_x
    if halo_y == 0:
        return _build_interval_set_from_rows(per, b, e, rows_hint=_t(s.rows), kind=s.begin).copy()
    shifts = torch.arange(-halo_y, halo_y + 1, dtype=I32, device=b.device)
    rows_all = (per[:, None] + shifts[None, :]).reshape(-1)
    k = int(shifts.numel())
    return _build_interval_set_from_rows(rows_all, b.repeat_interleave(k), e.repeat_interleave(k),
                                         kind=s.begin).copy()


def _dilate_unbounded(s: IntervalSet, halo_x: int, halo_y: int) -> IntervalSet:
    if halo_x == 0 and halo_y == 0:
        return s.copy()
    device = _t(s.row_offsets).device
    if int(s.begin.shape[0]) == 0:
        R = s.row_count
        rows = _t(s.rows) if R > 0 else torch.zeros(0, dtype=I32, device=device)
        return _empty_set(device, rows.clone(), s.begin)
    if halo_y == 0:
        out = _union_sweep(s, [0], halo_x, skip_empty=False)
        return out if out is not None else _dilate_reference_order(s, halo_x, 0)
    step = min(halo_y, (_MAX_SHIFTS - 1) // 2)
    out = _union_sweep(s, list(range(-step, step + 1)), halo_x, skip_empty=True)
    if out is None:
        return _dilate_reference_order(s, halo_x, halo_y)
    rest = halo_y - step
    while rest > 0:
        step = min(rest, (_MAX_SHIFTS - 1) // 2)
        out = _union_sweep(out, list(range(-step, step + 1)), 0, skip_empty=True)
        rest -= step
    return out


def dilate_interval_set(interval_set: IntervalSet, halo_x: int = 1, halo_y: int = 1) -> IntervalSet:
    """Box dilation by ``halo_x`` columns and ``halo_y`` rows, unbounded (``morphology.py:251-265``)."""
    if halo_x < 0 or halo_y < 0:
        raise ValueError("halo_x and halo_y must be non-negative")
    return _dilate_unbounded(interval_set, int(halo_x), int(halo_y))


def full_interval_set(width: int, height: int) -> IntervalSet:
    """The rectangle [0, width) x [0, height) (``morphology.py:344-358``)."""
    from .._runtime import current_device

    device = current_device()
    if height <= 0 or width <= 0:
        z = torch.zeros(0, dtype=I32, device=device)
        return IntervalSet._trusted(z, z.clone(), torch.zeros(1, dtype=I32, device=device), z.clone())
    h = int(height)
    s = IntervalSet._trusted(torch.zeros(h, dtype=I32, device=device),
                             torch.full((h,), int(width), dtype=I32, device=device),
                             torch.arange(h + 1, dtype=I32, device=device),
                             torch.arange(h, dtype=I32, device=device), h)
    # Marks the set as the whole rectangle, so whole-grid fast paths need no device check.
    object.__setattr__(s, "_full_width", int(width))
    return s


def _dense_empty(height: int, device, kind) -> IntervalSet:
    z = torch.zeros(0, dtype=I32, device=device)
    return _wrap(kind, z, z.clone(), torch.zeros(height + 1, dtype=I32, device=device),
                 torch.arange(height, dtype=I32, device=device), height)


def clip_interval_set(interval_set: IntervalSet, *, width: int, height: int) -> IntervalSet:
    """Intersection with [0, width) x [0, height) on dense rows ``arange(height)`` (``morphology.py:268-319``).

    One fused intersection sweep over the domain's rows.  Inputs outside the
    sweep's contract take the reference's order: the exact intersection
    kernel, then the sort-and-merge construction.
    """
    if width <= 0:
        raise ValueError("width must be positive")
    if height < 0:
        raise ValueError("height must be non-negative")
    s = interval_set
    device = _t(s.row_offsets).device
    H, W = int(height), int(width)
    kind = s.begin
    if H == 0 or int(s.begin.shape[0]) == 0 or s.row_count == 0:
        return _dense_empty(H, device, kind)
    dom_rows = torch.arange(H, dtype=I32, device=device)
    dom_off = torch.arange(H + 1, dtype=I32, device=device)
    dom_b = torch.zeros(H, dtype=I32, device=device)
    dom_e = torch.full((H,), W, dtype=I32, device=device)
    _, offs = _core.align_rows([(dom_rows, dom_off, 0, False), (_t(s.rows), _t(s.row_offsets), 0, False)], 0, H - 1,
                               device, [False, True])
    s_off = offs[1]
    table = [0b1000] + [0] * 7
    ob, oe, ooff, total, flags = _core.bool_eval([(dom_b, dom_e, dom_off, 0), (_t(s.begin), _t(s.end), s_off, 0)], H,
                                                 table, _lib.MODE_TABLE, device)
    if not flags & (_lib.FLAG_CONTRACT | _lib.FLAG_LONG_TILE):
        if flags & (_lib.FLAG_CAPACITY | _lib.FLAG_TIMEOUT):
            raise _lib.SubsetixError(f"clip sweep failed (flags={flags})")
        if total == 0:
            return _dense_empty(H, device, kind)
        return _wrap(kind, ob[:total].clone(), oe[:total].clone(), ooff, dom_rows, H)
    cb, ce, coff = _core.exact_setop(_core.OP_INTERSECTION, (dom_b, dom_e, dom_off), (_t(s.begin), _t(s.end), s_off),
                                     H, device)
    if cb.numel() == 0:
        return _dense_empty(H, device, kind)
    per = torch.repeat_interleave(dom_rows, (coff[1:] - coff[:-1]).to(torch.int64), output_size=int(cb.numel()))
    return _build_interval_set_from_rows(per, cb, ce, rows_hint=dom_rows, kind=kind)


def ghost_zones(interval_set: IntervalSet, halo_x: int = 1, halo_y: int = 1, *, width: int,
                height: Optional[int] = None) -> IntervalSet:
    """clip(dilate(S)) minus clip(S) (``morphology.py:322-341``)."""
    if height is None:
        height = int(interval_set.row_offsets.shape[0]) - 1
    dilated = dilate_interval_set(interval_set, halo_x=halo_x, halo_y=halo_y)
    clipped = clip_interval_set(dilated, width=width, height=height)
    base = clip_interval_set(interval_set, width=width, height=height)
    return evaluate(make_difference(make_input(clipped), make_input(base))).copy()


def erode_interval_set(interval_set: IntervalSet, halo_x: int = 1, halo_y: int = 1, *, width: int,
                       height: Optional[int] = None) -> IntervalSet:
    """U minus clip(dilate(U minus clip(S))), U the domain (``morphology.py:361-386``)."""
    if height is None:
        height = int(interval_set.row_offsets.shape[0]) - 1
    if width <= 0 or height < 0:
        raise ValueError("width must be positive and height must be non-negative")
    base = clip_interval_set(interval_set, width=width, height=height)
    universe = full_interval_set(width, height)
    complement = evaluate(make_difference(make_input(universe), make_input(base)))
    dilated = dilate_interval_set(complement, halo_x=halo_x, halo_y=halo_y)
    dilated_clipped = clip_interval_set(dilated, width=width, height=height)
    return evaluate(make_difference(make_input(universe), make_input(dilated_clipped))).copy()


__all__ = [
    "translate_interval_set",
    "interior_for_direction",
    "boundary_for_direction",
    "boundary_layer",
    "dilate_interval_set",
    "erode_interval_set",
    "full_interval_set",
    "ghost_zones",
    "clip_interval_set",
]
