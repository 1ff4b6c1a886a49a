"""Launch autotuner for the row-sweep set algebra (sx_bool_eval).

The candidates are the kernel kinds of ``sx_tuning``: the row-lane sweep
(16-row tiles with two lanes per row, 32-row tiles with one), the warp-tile
segmented sweep (8-row tiles, 32-bit and 16-bit keys) with several warps
per block, the block-tile
segmented sweep (32-row tiles) with two block sizes, the merge-path tile
kernel with two key capacities per tile, and the one-lane-per-row sweep
with several residency caps.  Each candidate is timed with CUDA events on the
caller's workload; the fastest is cached under a key of the workload's
shape (leaf count, row count, mean boundaries per 32-row tile, bucketed by
powers of two) and installed in ``_core.TUNED`` under that key, so later
evaluations of that kind of workload use its kernel and block shape (with
buffers sized for their own largest tile).  Results never depend on the
tuning; only speed does.
"""

from __future__ import annotations

import json
import math
import os
from typing import Dict, List, Optional, Sequence

import torch

from . import _core, _lib

_CACHE: Dict[str, dict] = {}


workload_key = _core.workload_key


def candidates(sizes: Sequence[int], rows: int, largest_tile: int = 0, largest_eighth_tile: int = 0,
               largest_half_tile: int = 0) -> List[dict]:
    tiles = max(1, (int(rows) + 31) // 32)
    avg = 2 * sum(int(s) for s in sizes) / tiles
    out = []
    # buffers for the largest tile when it is known (every tile then stays staged, and no slice is larger than
    # needed), else 1.25x the mean tile
    cap16 = min(int(largest_half_tile) or int(avg / 2 * 1.25 + 64), 25000)
    for w in (1, 2, 4):
        out.append({"kernel": 7, "staging_cap": cap16, "warps": w, "tile_rows": 16})
    out.append({"kernel": 7, "staging_cap": min(int(largest_tile) or int(avg * 1.25 + 64), 25000), "warps": 1,
                "tile_rows": 32})
    cap8 = min(int(largest_eighth_tile) or int(avg / 4 * 1.25 + 64), 25000)
    for w in (2, 4, 8):
        out.append({"kernel": 5, "staging_cap": cap8, "warps": w, "tile_rows": 8})
    for w in (2, 4, 8):
        out.append({"kernel": 6, "staging_cap": cap8, "warps": w, "tile_rows": 8})
    cap = min(int(largest_tile) or int(avg * 1.25 + 256), 25000)
    for w in (4, 8):
        out.append({"kernel": 4, "staging_cap": cap, "warps": w, "tile_rows": 32})
    for f in (1.25, 2.0):
        out.append({"kernel": 3, "staging_cap": int(avg * f + 256)})
    for b in (3, 5, 8):
        out.append({"kernel": 1, "blocks_per_sm": b})
    return out


def tune_bool_eval(leaves, rows: int, table: Sequence[int], device, *, mode: int = _lib.MODE_TABLE,
                   repeats: int = 5, install: bool = True, cache_path: Optional[str] = None) -> dict:
    """Time every candidate on ``leaves`` and return (and install) the fastest tuning."""
    sizes = [int(leaf[0].numel()) for leaf in leaves]
    key = workload_key(sizes, rows)
    if key in _CACHE:
        best = _CACHE[key]
    else:
        cap = max(1, sum(sizes))
        ob = torch.empty(cap, dtype=torch.int32, device=device)
        oe = torch.empty(cap, dtype=torch.int32, device=device)
        off = torch.empty(rows + 1, dtype=torch.int32, device=device)
        res = torch.empty(2, dtype=torch.int32, device=device)
        stream = torch.cuda.current_stream(device)
        timings = []
        table_mode = mode == _lib.MODE_TABLE
        largest, eighth = _core.max_tile_boundaries(leaves, rows, device, tile_rows=(32, 8)) if table_mode else (0, 0)
        half = _core.max_tile_boundaries(leaves, rows, device, tile_rows=16) if table_mode else 0
        for cand in candidates(sizes, rows, largest, eighth, half):
            def launch():
                _core.bool_eval_async(leaves, rows, table, mode, device, out=(ob, oe), result=res, offsets=off,
                                      tuning=cand)
            launch()
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(repeats):
                launch()
            e1.record(stream)
            torch.cuda.synchronize(device)
            timings.append((e0.elapsed_time(e1) / repeats, cand))
        ms, best = min(timings, key=lambda t: t[0])
        best = dict(best, ms=ms, key=key)
        _CACHE[key] = best
        if cache_path:
            data = {}
            if os.path.exists(cache_path):
                with open(cache_path) as f:
                    data = json.load(f)
            data[key] = best
            with open(cache_path, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
    if install:
        _core.TUNED[key] = {k: v for k, v in best.items() if k in ("kernel", "blocks_per_sm", "warps", "tile_rows")}
    return best


def load_cache(path: str) -> None:
    """Merge a saved cache file into the in-memory cache."""
    with open(path) as f:
        _CACHE.update(json.load(f))


__all__ = ["tune_bool_eval", "candidates", "workload_key", "load_cache"]
