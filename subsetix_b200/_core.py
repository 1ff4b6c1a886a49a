"""Device-level building blocks over torch tensors, each one C-ABI call.

Everything here takes and returns int32 CUDA tensors and enqueues work on
the current torch stream.  Functions whose output size depends on the data
read one small ``result`` pair back from the device.  The reference API
returns sized arrays, so it synchronises at the same points
(``subsetix_cupy/expressions.py:503``).
"""

from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import torch

from . import _lib
from ._runtime import ptr, read_pair, stream_handle, workspace

I32 = torch.int32

OP_UNION, OP_INTERSECTION, OP_DIFFERENCE = 0, 1, 2

# Launch tuning for the row sweep (sx_tuning).  Empty means automatic.  The
# autotuner (subsetix_b200/autotune.py) fills it per workload.
TUNING: dict = {}


def empty_i32(n: int, device) -> torch.Tensor:
    return torch.empty(max(int(n), 0), dtype=I32, device=device)


def bool_eval(leaves: Sequence[Tuple[torch.Tensor, torch.Tensor, torch.Tensor, int]], rows: int, table: Sequence[int],
              mode: int, device, out: Optional[Tuple[torch.Tensor, torch.Tensor]] = None):
    """Run the row sweep (sx_bool_eval) and read back its result pair.

    ``leaves`` are ``(begin, end, aligned_offsets, widen)`` tuples; ``mode``
    is ``_lib.MODE_TABLE`` (truth table over canonical leaves) or
    ``_lib.MODE_UNION`` (merged union of widened leaves).  Returns
    ``(begin, end, offsets, total, flags)``; begin and end are capacity
    buffers to be sliced to ``total``.
    """
    ob, oe, ooff, result = bool_eval_async(leaves, rows, table, mode, device, out)
    if result is None:
        return ob, oe, ooff, 0, 0
    total, flags = read_pair(result)
    return ob, oe, ooff, total, flags


def bool_eval_async(leaves: Sequence[Tuple[torch.Tensor, torch.Tensor, torch.Tensor, int]], rows: int,
                    table: Sequence[int], mode: int, device, out: Optional[Tuple[torch.Tensor, torch.Tensor]] = None,
                    result: Optional[torch.Tensor] = None, offsets: Optional[torch.Tensor] = None,
                    tuning: Optional[dict] = None):
    """Enqueue the row sweep without waiting.

    Returns ``(begin, end, offsets, result)``; ``result`` is the device pair
    ``(total, flags)``, or None when there are no rows.
    """
    lib = _lib.load()
    k = len(leaves)
    sizes = [int(b.numel()) for b, _, _, _ in leaves]
    cap = max(1, sum(sizes))
    if out is None:
        ob = empty_i32(cap, device)
        oe = empty_i32(cap, device)
    else:
        ob, oe = out
        if ob.numel() < cap or oe.numel() < cap:
            raise ValueError("output buffers below the required capacity")
    ooff = empty_i32(rows + 1, device) if offsets is None else offsets
    if rows == 0:
        ooff.zero_()
        return ob, oe, ooff, None
    if result is None:
        result = empty_i32(2, device)
    arr = (_lib.SxLeaf * k)()
    for i, (b, e, off, widen) in enumerate(leaves):
        arr[i].begin = ptr(b)
        arr[i].end = ptr(e)
        arr[i].row_offsets = ptr(off)
        arr[i].widen = int(widen)
    tab = (ctypes.c_uint32 * 8)(*[int(x) & 0xFFFFFFFF for x in (list(table) + [0] * 8)[:8]])
    wsp, wsn = workspace(device, lib.sx_bool_workspace_bytes(int(rows)))
    t = TUNING if tuning is None else tuning
    tun = _lib.SxTuning(int(t.get("kernel", 0)), int(t.get("blocks_per_sm", 0)), int(t.get("staging_cap", 0)))
    rc = lib.sx_bool_eval(arr, k, int(rows), tab, int(mode), ptr(ob), ptr(oe), ptr(ooff), cap, ptr(result), wsp, wsn,
                          ctypes.byref(tun), stream_handle(device))
    _lib.check(rc, "sx_bool_eval")
    return ob, oe, ooff, result


def scan(counts: torch.Tensor, device) -> Tuple[torch.Tensor, int]:
    """Exclusive prefix sum: ``(offsets[n + 1], total)`` (synchronising)."""
    lib = _lib.load()
    n = int(counts.numel())
    out = empty_i32(n + 1, device)
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_scan_workspace_bytes(n))
    rc = lib.sx_scan_i32(ptr(counts), n, ptr(out), ptr(result), wsp, wsn, stream_handle(device))
    _lib.check(rc, "sx_scan_i32")
    total, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_scan_i32: look-back wait timed out")
    return out, total


def exact_setop(op: int, lhs, rhs, rows: int, device):
    """Reference-order binary op on aligned operands.  Returns ``(begin, end, offsets)``."""
    lib = _lib.load()
    lb, le, loff = lhs
    rb, re, roff = rhs
    if rows == 0:
        return empty_i32(0, device), empty_i32(0, device), torch.zeros(1, dtype=I32, device=device)
    counts = empty_i32(rows, device)
    s = stream_handle(device)
    rc = lib.sx_exact_setop(op, rows, ptr(lb), ptr(le), ptr(loff), ptr(rb), ptr(re), ptr(roff), ptr(counts), None,
                            None, None, s)
    _lib.check(rc, "sx_exact_setop(count)")
    off, total = scan(counts, device)
    ob = empty_i32(total, device)
    oe = empty_i32(total, device)
    if total:
        rc = lib.sx_exact_setop(op, rows, ptr(lb), ptr(le), ptr(loff), ptr(rb), ptr(re), ptr(roff), None, ptr(off),
                                ptr(ob), ptr(oe), s)
        _lib.check(rc, "sx_exact_setop(write)")
    return ob, oe, off


def merge_rows(begin: torch.Tensor, end: torch.Tensor, offsets: torch.Tensor, device):
    """Run merge of begin-sorted rows (kernels.py:292-381).  Returns ``(begin, end, offsets)``."""
    lib = _lib.load()
    rows = int(offsets.numel()) - 1
    if rows <= 0:
        return empty_i32(0, device), empty_i32(0, device), torch.zeros(max(rows, 0) + 1, dtype=I32, device=device)
    counts = empty_i32(rows, device)
    s = stream_handle(device)
    _lib.check(lib.sx_merge_rows(rows, ptr(begin), ptr(end), ptr(offsets), ptr(counts), None, None, None, s),
               "sx_merge_rows(count)")
    off, total = scan(counts, device)
    ob = empty_i32(total, device)
    oe = empty_i32(total, device)
    if total:
        _lib.check(lib.sx_merge_rows(rows, ptr(begin), ptr(end), ptr(offsets), None, ptr(off), ptr(ob), ptr(oe), s),
                   "sx_merge_rows(write)")
    return ob, oe, off


def align_rows(lists: Sequence[Tuple[torch.Tensor, torch.Tensor, int, bool]], row_min: int, row_max: int, device,
               want_offsets: Sequence[bool]) -> Tuple[torch.Tensor, List[Optional[torch.Tensor]]]:
    """Sorted union of ``rows + shift`` over the lists, plus aligned offsets.

    ``lists`` holds ``(rows, offsets, shift, skip_empty)`` tuples.  Returns
    ``(rows_out, [aligned offsets or None])``.  This call synchronises.
    """
    lib = _lib.load()
    k = len(lists)
    cap = 0
    for rows, _, _, _ in lists:
        cap += int(rows.numel())
    span = int(row_max) - int(row_min) + 1
    cap = max(1, min(cap, max(span, 1)))
    rows_out = empty_i32(cap, device)
    aligned = [empty_i32(cap + 1, device) if w else None for w in want_offsets]
    arr = (_lib.SxRowList * k)()
    for i, (rows, off, shift, skip) in enumerate(lists):
        arr[i].rows = ptr(rows)
        arr[i].row_offsets = ptr(off)
        arr[i].count = int(rows.numel())
        arr[i].shift = int(shift)
        arr[i].skip_empty = 1 if skip else 0
    aptrs = (ctypes.c_void_p * k)(*[ptr(a) if a is not None else None for a in aligned])
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_align_workspace_bytes(int(row_min), int(row_max)))
    rc = lib.sx_align_rows(arr, k, int(row_min), int(row_max), ptr(rows_out), cap, aptrs, ptr(result), wsp, wsn,
                           stream_handle(device))
    _lib.check(rc, "sx_align_rows")
    n, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_align_rows: look-back wait timed out")
    return rows_out[:n], [a[: n + 1] if a is not None else None for a in aligned]
