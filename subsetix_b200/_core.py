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

# Launch tuning for the row sweep (sx_tuning).  TUNING, when not empty,
# applies to every evaluation.  TUNED maps a workload key (workload_key) to
# the launch shape the autotuner (subsetix_b200/autotune.py) found fastest for
# that kind of workload; buffer sizes are still taken from each evaluation's
# own largest tile.  Neither ever changes results.
TUNING: dict = {}
TUNED: dict = {}


def workload_key(sizes: Sequence[int], rows: int) -> str:
    """Bucket of a set-algebra workload: leaf count, log2 rows, log2 mean boundaries per 32-row tile."""
    import math

    tiles = max(1, (int(rows) + 31) // 32)
    per_tile = 2 * sum(int(s) for s in sizes) / tiles
    return f"k{len(sizes)}-r{int(math.log2(max(rows, 1)))}-t{int(math.log2(max(per_tile, 1.0)))}"


def empty_i32(n: int, device) -> torch.Tensor:
    return torch.empty(max(int(n), 0), dtype=I32, device=device)


def tile_stats(leaves, rows: int, device, tile_rows_a: int = 8, tile_rows_b: int = 32):
    """``(largest a-row tile, largest b-row tile, largest a-row tile span)`` in boundaries and coordinates.

    One launch of ``sx_tile_boundaries_max`` and one read-back.
    """
    if rows <= 0 or any(len(leaf) > 5 and leaf[5] is not None for leaf in leaves):
        return 0, 0, 0  # no rows, or explicit row ranges (the union sweep has no tiles)
    lib = _lib.load()
    arr = (_lib.SxLeaf * len(leaves))()
    for i, leaf in enumerate(leaves):
        arr[i].begin = ptr(leaf[0])
        arr[i].end = ptr(leaf[1])
        arr[i].row_offsets = ptr(leaf[2])
    out = empty_i32(3, device)
    _lib.check(lib.sx_tile_boundaries_max(arr, len(leaves), int(rows), int(tile_rows_a), int(tile_rows_b), ptr(out),
                                          stream_handle(device)), "sx_tile_boundaries_max")
    a, b, span = (int(x) for x in out.tolist())
    return a, b, span


def max_tile_boundaries(leaves, rows: int, device, tile_rows=32):
    """Largest number of leaf boundaries in one tile of ``tile_rows`` aligned rows (one synchronisation).

    ``tile_rows`` may be a pair of tile heights; the result is then a list
    with one maximum per height, from the same launch and read-back.
    """
    heights = list(tile_rows) if isinstance(tile_rows, (tuple, list)) else [tile_rows, tile_rows]
    a, b, _ = tile_stats(leaves, rows, device, heights[0], heights[1])
    return [a, b] if isinstance(tile_rows, (tuple, list)) else a


def _default_keys(leaves, rows: int, tile_rows: int = 32) -> int:
    tiles = max(1, (rows + tile_rows - 1) // tile_rows)
    avg = 2 * sum(int(leaf[0].numel()) for leaf in leaves) // tiles
    return avg + avg // 4 + 64


def auto_tuning(leaves, rows: int, device) -> dict:
    """The automatic launch shape of a truth-table sweep (one launch and one read-back, two when rows are skewed).

    Even rows (the largest 8-row tile within 3x the mean plus 256
    boundaries): the row-lane sweep on 16-row tiles, two lanes per row, when
    every such tile spans at most 65534 columns (16-bit coordinates), else
    8-row warp tiles with 32-bit keys; buffers are sized for the largest tile,
    so no tile leaves the staged sweep.  Skewed rows: 32-row block tiles
    sized for their largest tile, which evens out the load.
    """
    need16, need8, span16 = tile_stats(leaves, rows, device, 16, 8)
    mean8 = 2 * sum(int(leaf[0].numel()) for leaf in leaves) / max(1, (rows + 7) // 8)
    if need8 <= 3 * mean8 + 256:
        if span16 <= 65534:
            return {"kernel": 7, "staging_cap": min(need16, 25000), "tile_rows": 16, "warps": 2}
        return {"kernel": 5, "staging_cap": min(need8, 25000), "tile_rows": 8, "warps": 2}
    need32 = max_tile_boundaries(leaves, rows, device, tile_rows=32)
    return {"kernel": 4, "staging_cap": min(need32, 25000), "tile_rows": 32, "warps": 4}


def bool_eval(leaves: Sequence[Tuple[torch.Tensor, torch.Tensor, torch.Tensor, int]], rows: int, table: Sequence[int],
              mode: int, device, out: Optional[Tuple[torch.Tensor, torch.Tensor]] = None):
    """Run the row sweep (sx_bool_eval) and read back its result pair.

    ``leaves`` are ``(begin, end, aligned_offsets, widen[, scale[, row_ends]])``
    tuples; ``mode``
    is ``_lib.MODE_TABLE`` (truth table over canonical leaves) or
    ``_lib.MODE_UNION`` (merged union of widened leaves).  Returns
    ``(begin, end, offsets, total, flags)``; begin and end are capacity
    buffers to be sliced to ``total``.
    """
    tuning = None
    tuned = TUNED.get(workload_key([int(leaf[0].numel()) for leaf in leaves], rows)) if TUNED else None
    if mode == _lib.MODE_TABLE and not TUNING and rows > 0 and tuned is not None:
        tuning = dict(tuned)
        if tuning.get("kernel") in (3, 4, 5, 6, 7):
            tr = int(tuning.get("tile_rows", 0)) or {5: 8, 6: 8, 7: 16}.get(tuning["kernel"], 32)
            tuning["staging_cap"] = min(max_tile_boundaries(leaves, rows, device, tile_rows=tr), 25000)
    elif mode == _lib.MODE_TABLE and not TUNING and rows > 0:
        tuning = auto_tuning(leaves, rows, device)
    ob, oe, ooff, result = bool_eval_async(leaves, rows, table, mode, device, out, tuning=tuning)
    if result is None:
        return ob, oe, ooff, 0, 0
    total, flags = read_pair(result)
    return ob, oe, ooff, total, flags


def bool_eval_async(leaves: Sequence[Tuple[torch.Tensor, torch.Tensor, torch.Tensor, int]], rows: int,
                    table: Sequence[int], mode: int, device, out: Optional[Tuple[torch.Tensor, torch.Tensor]] = None,
                    result: Optional[torch.Tensor] = None, offsets: Optional[torch.Tensor] = None,
                    tuning: Optional[dict] = None, scratch: Optional[torch.Tensor] = None):
    """Enqueue the row sweep without waiting.

    Returns ``(begin, end, offsets, result)``; ``result`` is the device pair
    ``(total, flags)``, or None when there are no rows.  ``scratch`` (bytes,
    at least ``sx_bool_workspace_bytes(rows)``) replaces the per-stream
    workspace, for launches captured in a graph.
    """
    lib = _lib.load()
    k = len(leaves)
    sizes = [int(leaf[0].numel()) for leaf in leaves]
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
    for i, leaf in enumerate(leaves):
        b, e, off, widen = leaf[:4]
        scale = leaf[4] if len(leaf) > 4 else 0
        ends = leaf[5] if len(leaf) > 5 else None
        arr[i].begin = ptr(b)
        arr[i].end = ptr(e)
        arr[i].row_offsets = ptr(off)
        arr[i].row_ends = ptr(ends)
        arr[i].widen = int(widen)
        arr[i].scale = int(scale)
    tab = (ctypes.c_uint32 * 8)(*[int(x) & 0xFFFFFFFF for x in (list(table) + [0] * 8)[:8]])
    if scratch is None:
        wsp, wsn = workspace(device, lib.sx_bool_workspace_bytes(int(rows)))
    else:
        if int(scratch.numel()) < int(lib.sx_bool_workspace_bytes(int(rows))):
            raise ValueError("scratch below sx_bool_workspace_bytes(rows)")
        wsp, wsn = scratch.data_ptr(), int(scratch.numel())
    t = TUNING if tuning is None else tuning
    tun = _lib.SxTuning(int(t.get("kernel", 0)), int(t.get("blocks_per_sm", 0)), int(t.get("staging_cap", 0)),
                        int(t.get("warps", 0)), int(t.get("tile_rows", 0)), int(t.get("wait_limit", 0)),
                        int(t.get("withhold_tile", 0)))
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


def align_rows(lists: Sequence[tuple], row_min: int, row_max: int, device, want_offsets: Sequence[bool],
               want_ends: Optional[Sequence[bool]] = None):
    """Sorted union of ``floor((rows + shift) / div)`` over the lists, plus aligned offsets.

    ``lists`` holds ``(rows, offsets, shift, skip_empty[, div, phase])``
    tuples.  Returns ``(rows_out, [aligned offsets or None])``, or with
    ``want_ends`` ``(rows_out, [starts or None], [stops or None])``.  This
    call synchronises.
    """
    lib = _lib.load()
    k = len(lists)
    cap = 0
    for item in lists:
        cap += int(item[0].numel())
    span = int(row_max) - int(row_min) + 1
    cap = max(1, min(cap, max(span, 1)))
    rows_out = empty_i32(cap, device)
    aligned = [empty_i32(cap + 1, device) if w else None for w in want_offsets]
    ends = [empty_i32(cap, device) if w else None for w in (want_ends or [False] * k)]
    arr = (_lib.SxRowList * k)()
    for i, item in enumerate(lists):
        rows, off, shift, skip = item[:4]
        arr[i].rows = ptr(rows)
        arr[i].row_offsets = ptr(off)
        arr[i].count = int(rows.numel())
        arr[i].shift = int(shift)
        arr[i].skip_empty = 1 if skip else 0
        arr[i].div = int(item[4]) if len(item) > 4 else 1
        arr[i].phase = int(item[5]) if len(item) > 5 else 0
    aptrs = (ctypes.c_void_p * k)(*[ptr(a) if a is not None else None for a in aligned])
    eptrs = (ctypes.c_void_p * k)(*[ptr(a) if a is not None else None for a in ends])
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_align_workspace_bytes(int(row_min), int(row_max)))
    rc = lib.sx_align_rows(arr, k, int(row_min), int(row_max), ptr(rows_out), cap, aptrs,
                           eptrs if want_ends else None, ptr(result), wsp, wsn, stream_handle(device))
    _lib.check(rc, "sx_align_rows")
    n, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_align_rows: look-back wait timed out")
    starts = [a[: n + 1] if a is not None else None for a in aligned]
    if want_ends:
        return rows_out[:n], starts, [a[:n] if a is not None else None for a in ends]
    return rows_out[:n], starts


# ---------------------------------------------------------------------------
# Interval fields and multilevel kernels
# ---------------------------------------------------------------------------

def _flag_word(device) -> torch.Tensor:
    return empty_i32(1, device)


def check_rows(begin: torch.Tensor, end: torch.Tensor, offsets: torch.Tensor, device, sync: bool = True):
    """OR of ``_lib.ROWS_*`` bits over adjacent interval pairs (sx_check_rows)."""
    lib = _lib.load()
    flags = _flag_word(device)
    rows = int(offsets.numel()) - 1
    _lib.check(lib.sx_check_rows(ptr(begin), ptr(end), ptr(offsets), max(rows, 0), int(begin.numel()), ptr(flags),
                                 stream_handle(device)), "sx_check_rows")
    return int(flags.item()) if sync else flags


def cell_offsets(begin: torch.Tensor, end: torch.Tensor, device, sync: bool = True):
    """int32 exclusive scan of interval lengths.  Returns ``(offsets, total)``."""
    lib = _lib.load()
    n = int(begin.numel())
    out = empty_i32(n + 1, device)
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_scan_workspace_bytes(n))
    _lib.check(lib.sx_cell_offsets(ptr(begin), ptr(end), n, ptr(out), ptr(result), wsp, wsn, stream_handle(device)),
               "sx_cell_offsets")
    if not sync:
        return out, result
    total, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_cell_offsets: look-back wait timed out")
    return out, total


def prolong_set(rows: torch.Tensor, offsets: torch.Tensor, begin: torch.Tensor, end: torch.Tensor, ratio: int,
                device):
    """sx_prolong_set.  Returns ``(rows_out, offsets_out, begin, end, unsorted)`` sized to the output."""
    lib = _lib.load()
    R = int(rows.numel())
    n = int(begin.numel())
    rows_out = empty_i32(R * ratio, device)
    off_out = empty_i32(R * ratio + 1, device)
    ob = empty_i32(n * ratio, device)
    oe = empty_i32(n * ratio, device)
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_prolong_set_workspace_bytes(R))
    _lib.check(lib.sx_prolong_set(ptr(rows), ptr(offsets), ptr(begin), ptr(end), R, n, int(ratio), ptr(rows_out),
                                  ptr(off_out), ptr(ob), ptr(oe), ptr(result), wsp, wsn, stream_handle(device)),
               "sx_prolong_set")
    occupied, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_prolong_set: look-back wait timed out")
    m = occupied * ratio
    return rows_out[:m], off_out[: m + 1], ob, oe, bool(flags & 1)


def _dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.SX_F32
    if t.dtype == torch.float64:
        return _lib.SX_F64
    raise TypeError(f"field values must be float32 or float64, got {t.dtype}")


def prolong_field(coarse_offsets, coarse_cell_offsets, n: int, fine_offsets, fine_cell_offsets, ratio: int,
                  coarse_values, fine_values, device):
    lib = _lib.load()
    rows = int(coarse_offsets.numel()) - 1
    _lib.check(lib.sx_prolong_field(_dtype_code(coarse_values), ptr(coarse_offsets), rows, ptr(coarse_cell_offsets),
                                    int(n), ptr(fine_offsets), ptr(fine_cell_offsets), int(ratio), ptr(coarse_values),
                                    ptr(fine_values), stream_handle(device)), "sx_prolong_field")


def coarse_fine_check(coarse, fine, ratio: int, device, sync: bool = True):
    """Flags of sx_coarse_fine_check.  ``coarse``/``fine`` are ``(rows, offsets, begin, end)``."""
    lib = _lib.load()
    cr, coff, cb, ce = coarse
    fr, foff, fb, fe = fine
    flags = _flag_word(device)
    _lib.check(lib.sx_coarse_fine_check(ptr(cr), int(cr.numel()), ptr(coff), ptr(cb), ptr(ce), int(cb.numel()),
                                        ptr(fr), int(fr.numel()), ptr(foff), ptr(fb), ptr(fe), int(fb.numel()),
                                        int(ratio), ptr(flags), stream_handle(device)), "sx_coarse_fine_check")
    return int(flags.item()) if sync else flags


def restrict_field(coarse_offsets, coarse_cell_offsets, coarse_n: int, fine_offsets, fine_cell_offsets, ratio: int,
                   reducer: int, fine_values, coarse_values, device):
    lib = _lib.load()
    rows = int(coarse_offsets.numel()) - 1
    _lib.check(lib.sx_restrict_field(_dtype_code(fine_values), ptr(coarse_offsets), rows, ptr(coarse_cell_offsets),
                                     int(coarse_n), ptr(fine_offsets), ptr(fine_cell_offsets), int(ratio),
                                     int(reducer), ptr(fine_values), ptr(coarse_values), stream_handle(device)),
               "sx_restrict_field")


def subset_rows(sub_offsets, sub_rows, sub_n: int, sup_rows, device, sync: bool = True):
    """Superset row ordinal per subset interval.  Returns ``(pos, missing)``."""
    lib = _lib.load()
    pos = empty_i32(sub_n, device)
    flags = _flag_word(device)
    _lib.check(lib.sx_subset_rows(ptr(sub_offsets), ptr(sub_rows), int(sub_rows.numel()), int(sub_n), ptr(sup_rows),
                                  int(sup_rows.numel()), ptr(pos), ptr(flags), stream_handle(device)),
               "sx_subset_rows")
    return pos, (bool(flags.item()) if sync else flags)


def subset_copy(scatter: bool, pos, sub, sup, sub_values, sup_values, device):
    """sx_subset_copy.  ``sub`` = ``(begin, end, cell_offsets)``; ``sup`` = ``(offsets, begin, end, cell_offsets)``."""
    lib = _lib.load()
    sb, se, scoff = sub
    uoff, ub, ue, ucoff = sup
    _lib.check(lib.sx_subset_copy(1 if scatter else 0, int(sb.numel()), ptr(pos), ptr(sb), ptr(se), ptr(scoff),
                                  ptr(uoff), ptr(ub), ptr(ue), ptr(ucoff), int(uoff.numel()) - 1, ptr(sub_values),
                                  ptr(sup_values), int(sub_values.element_size()), stream_handle(device)),
               "sx_subset_copy")


def row_lookup(rows, height: int, device, sync: bool = True):
    """Row ordinal per row id in [0, height) (-1 when absent).  Returns ``(lookup, out_of_range)``."""
    lib = _lib.load()
    lookup = empty_i32(height, device)
    flags = _flag_word(device)
    _lib.check(lib.sx_row_lookup(ptr(rows), int(rows.numel()), int(height), ptr(lookup), ptr(flags),
                                 stream_handle(device)), "sx_row_lookup")
    return lookup, (bool(flags.item()) if sync else flags)


def upwind(rows, offsets, begin, end, cell_offs, cells: int, lookup, values, out, width: int, height: int, a, b, dt,
           dx, dy, direct: bool, device, row_ids=None):
    lib = _lib.load()
    _lib.check(lib.sx_upwind(_dtype_code(values), ptr(rows), ptr(row_ids), ptr(offsets), int(rows.numel()), ptr(begin),
                             ptr(end), ptr(cell_offs), int(begin.numel()), int(cells), ptr(lookup), ptr(values),
                             ptr(out), int(width), int(height), float(a), float(b), float(dt), float(dx), float(dy),
                             1 if direct else 0, stream_handle(device)), "sx_upwind")


def upwind_plan(rows, offsets, begin, end, cell_offs, lookup, height: int, device):
    """Plan of sx_upwind_chunked for a fixed geometry: ``(chunk_info, chunks)`` (one synchronisation)."""
    lib = _lib.load()
    n = int(begin.numel())
    chunk_off = empty_i32(n + 1, device)
    result = empty_i32(2, device)
    wsp, wsn = workspace(device, lib.sx_scan_workspace_bytes(n))
    s = stream_handle(device)
    _lib.check(lib.sx_upwind_plan(ptr(begin), ptr(end), n, ptr(chunk_off), ptr(result), wsp, wsn, s),
               "sx_upwind_plan")
    chunks, flags = read_pair(result)
    if flags & _lib.FLAG_TIMEOUT:
        raise _lib.SubsetixError("sx_upwind_plan: look-back wait timed out")
    info = empty_i32(16 * max(chunks, 1), device)
    _lib.check(lib.sx_upwind_plan_fill(ptr(rows), ptr(offsets), int(rows.numel()), ptr(begin), ptr(end),
                                       ptr(cell_offs), n, ptr(chunk_off), chunks, ptr(lookup), int(height), ptr(info),
                                       s), "sx_upwind_plan_fill")
    return info, chunks


def upwind_table(begin, end, cell_offs, chunk_info, chunks: int, cells: int, device):
    """Neighbour table of a chunk plan (uint16 per cell; one synchronisation)."""
    lib = _lib.load()
    table = torch.empty(max(int(cells), 1), dtype=torch.int16, device=device)
    status = empty_i32(1, device)
    _lib.check(lib.sx_upwind_plan_table(ptr(begin), ptr(end), ptr(cell_offs), ptr(chunk_info), int(chunks), ptr(table),
                                        ptr(status), stream_handle(device)), "sx_upwind_plan_table")
    if int(status.item()):
        raise _lib.SubsetixError("sx_upwind_plan_table: cell offsets are not the packed prefix sum")
    return table


def upwind_chunked(offsets, begin, end, cell_offs, chunk_info, chunks: int, lookup, values, out, width: int,
                   height: int, a, b, dt, dx, dy, device, table=None):
    lib = _lib.load()
    _lib.check(lib.sx_upwind_chunked(_dtype_code(values), ptr(offsets), ptr(begin), ptr(end), ptr(cell_offs),
                                     ptr(chunk_info), int(chunks), ptr(lookup), ptr(table), ptr(values), ptr(out),
                                     int(width), int(height), float(a), float(b), float(dt), float(dx), float(dy),
                                     stream_handle(device)), "sx_upwind_chunked")


def threshold_rle(values, width: int, height: int, threshold: float, gradient: bool, device):
    """Runs of value >= threshold per row of a full grid.  Returns ``(begin, end, offsets)`` (synchronising)."""
    lib = _lib.load()
    counts = empty_i32(height, device)
    s = stream_handle(device)
    _lib.check(lib.sx_threshold_rle(ptr(values), int(width), int(height), float(threshold), 1 if gradient else 0,
                                    ptr(counts), None, None, None, s), "sx_threshold_rle(count)")
    off, total = scan(counts, device)
    ob = empty_i32(total, device)
    oe = empty_i32(total, device)
    if total:
        _lib.check(lib.sx_threshold_rle(ptr(values), int(width), int(height), float(threshold), 1 if gradient else 0,
                                        None, ptr(off), ptr(ob), ptr(oe), s), "sx_threshold_rle(write)")
    return ob, oe, off


def mass_integral(values, scale: float, device, out: Optional[torch.Tensor] = None, parts: int = 592):
    """Compensated FP64 sum times ``scale`` into a device scalar (no synchronisation)."""
    lib = _lib.load()
    if out is None:
        out = torch.empty(1, dtype=torch.float64, device=device)
    part = torch.empty(2 * parts, dtype=torch.float64, device=device)
    _lib.check(lib.sx_mass_integral(_dtype_code(values), ptr(values), int(values.numel()), float(scale), ptr(part),
                                    int(parts), ptr(out), stream_handle(device)), "sx_mass_integral")
    return out
