"""Seeded synthetic interval geometry for the benchmark and parity workloads.

Every generator returns host NumPy arrays ``(begin, end, row_offsets, rows)``
in the CSR interval layout: int32 throughout, half-open ``[begin, end)``,
sorted and disjoint inside each row.  All randomness comes from
``numpy.random.default_rng(seed)``.  Geometric draws use support
``{1, 2, ...}``, so every interval is non-empty and every gap is at least one
cell.  The sets are therefore canonical: no two intervals in a row touch.

Workloads:

* :func:`random_rows_set` — 256x256 rows with ``min(Poisson(4), 8)``
  intervals per row.  Gaps are Geom(mean 8) and lengths Geom(mean 12),
  starting at x = 0 and clipped to the width.
* :func:`disk_set`, :func:`annulus_set`, :func:`checkerboard_set` and
  :func:`circles_set` — the 4096x4096 shapes.  A cell ``(x, y)`` is inside a
  round shape when its centre ``(x + 0.5, y + 0.5)`` lies within the radius.
* :func:`stack_rows` — places copies of a set on disjoint row bands, each
  copy shifted in x.  One launch can then process many copies; this is the
  batched variant of the shape workload.
* :func:`batched_uneven_sets` — 256 independent sets.  Sides are drawn
  log-uniform in [128, 4096], and the interval count per row is
  ``min(round(LogNormal(1.5, 1.0)), side // 2)``.  The intervals pair up
  ``2k`` distinct sorted points in ``[0, side]``.
"""

from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

HostSet = Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]


def _pack(row_lists: Sequence[Tuple[np.ndarray, np.ndarray]], rows: np.ndarray | None = None) -> HostSet:
    counts = np.array([len(b) for b, _ in row_lists], dtype=np.int64)
    offsets = np.zeros(len(row_lists) + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    if len(row_lists):
        begin = np.concatenate([np.asarray(b, dtype=np.int64) for b, _ in row_lists]) if offsets[-1] else np.zeros(0, np.int64)
        end = np.concatenate([np.asarray(e, dtype=np.int64) for _, e in row_lists]) if offsets[-1] else np.zeros(0, np.int64)
    else:
        begin = np.zeros(0, np.int64)
        end = np.zeros(0, np.int64)
    if rows is None:
        rows = np.arange(len(row_lists), dtype=np.int64)
    return (begin.astype(np.int32), end.astype(np.int32), offsets.astype(np.int32), np.asarray(rows, dtype=np.int32))


def mask_to_set(mask: np.ndarray, x_offset: int = 0) -> HostSet:
    """Run-length encode a dense boolean mask ``[height, width]`` row by row."""

    mask = np.asarray(mask, dtype=bool)
    height, width = mask.shape
    padded = np.zeros((height, width + 2), dtype=np.int8)
    padded[:, 1:-1] = mask
    diff = np.diff(padded, axis=1)
    starts_r, starts_c = np.nonzero(diff == 1)
    ends_r, ends_c = np.nonzero(diff == -1)
    counts = np.bincount(starts_r, minlength=height)
    offsets = np.zeros(height + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])
    begin = (starts_c + x_offset).astype(np.int32)
    end = (ends_c + x_offset).astype(np.int32)
    return begin, end, offsets.astype(np.int32), np.arange(height, dtype=np.int32)


def set_to_mask(host_set: HostSet, width: int, height: int, x_offset: int = 0) -> np.ndarray:
    """Dense boolean mask of a set whose rows are ``0..height-1`` (cells outside are ignored)."""

    begin, end, offsets, rows = host_set
    mask = np.zeros((height, width), dtype=bool)
    for ordinal, row in enumerate(rows):
        if row < 0 or row >= height:
            continue
        for idx in range(offsets[ordinal], offsets[ordinal + 1]):
            b = max(int(begin[idx]) - x_offset, 0)
            e = min(int(end[idx]) - x_offset, width)
            if e > b:
                mask[row, b:e] = True
    return mask


def random_rows_set(seed: int, width: int = 256, height: int = 256,
                    mean_count: float = 4.0, max_count: int = 8,
                    mean_gap: float = 8.0, mean_length: float = 12.0) -> HostSet:
    rng = np.random.default_rng(seed)
    rows: List[Tuple[List[int], List[int]]] = []
    for _ in range(height):
        k = min(int(rng.poisson(mean_count)), max_count)
        x = 0
        b_row: List[int] = []
        e_row: List[int] = []
        for _ in range(k):
            gap = int(rng.geometric(1.0 / mean_gap))
            length = int(rng.geometric(1.0 / mean_length))
            x += gap
            b = x
            x += length
            if b >= width:
                break
            b_row.append(b)
            e_row.append(min(x, width))
        rows.append((b_row, e_row))
    return _pack(rows)


def _round_mask(width: int, height: int, cx: float, cy: float, r_out: float, r_in: float | None = None) -> np.ndarray:
    ys = (np.arange(height, dtype=np.float64) + 0.5 - cy)[:, None]
    xs = (np.arange(width, dtype=np.float64) + 0.5 - cx)[None, :]
    d2 = xs * xs + ys * ys
    mask = d2 <= r_out * r_out
    if r_in is not None:
        mask &= d2 > r_in * r_in
    return mask


def disk_set(size: int = 4096, radius: float = 1500.0) -> HostSet:
    c = size / 2.0
    return mask_to_set(_round_mask(size, size, c, c, radius))


def annulus_set(size: int = 4096, r_in: float = 800.0, r_out: float = 1200.0) -> HostSet:
    c = size / 2.0
    return mask_to_set(_round_mask(size, size, c, c, r_out, r_in))


def checkerboard_set(size: int = 4096, period: int = 64, shift_x: int = 0) -> HostSet:
    xs = np.arange(size)[None, :] + shift_x
    ys = np.arange(size)[:, None]
    mask = ((xs // period) + (ys // period)) % 2 == 0
    return mask_to_set(mask)


def circles_set(size: int = 4096, count: int = 200, seed: int = 2,
                r_min: float = 20.0, r_max: float = 200.0) -> HostSet:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, float(size), size=(count, 2))
    radii = rng.uniform(r_min, r_max, size=count)
    mask = np.zeros((size, size), dtype=bool)
    for (cx, cy), r in zip(centres, radii):
        y0 = max(int(np.floor(cy - r)) - 1, 0)
        y1 = min(int(np.ceil(cy + r)) + 1, size)
        x0 = max(int(np.floor(cx - r)) - 1, 0)
        x1 = min(int(np.ceil(cx + r)) + 1, size)
        if y0 >= y1 or x0 >= x1:
            continue
        ys = (np.arange(y0, y1, dtype=np.float64) + 0.5 - cy)[:, None]
        xs = (np.arange(x0, x1, dtype=np.float64) + 0.5 - cx)[None, :]
        mask[y0:y1, x0:x1] |= (xs * xs + ys * ys) <= r * r
    return mask_to_set(mask)


def shape_operands(size: int = 4096) -> List[HostSet]:
    """Operands A..E of ``((A | B) - (C & D)) ^ E`` on the 4096x4096 shapes.

    A is the disk (r=1500), B the annulus (800-1200), C the 64-px
    checkerboard, D the union of 200 seeded circles and E the checkerboard
    shifted by 32 px in x.
    """

    scale = size / 4096.0
    return [
        disk_set(size, 1500.0 * scale),
        annulus_set(size, 800.0 * scale, 1200.0 * scale),
        checkerboard_set(size, max(1, int(64 * scale))),
        circles_set(size, 200, 2, 20.0 * scale, 200.0 * scale),
        checkerboard_set(size, max(1, int(64 * scale)), shift_x=max(1, int(32 * scale))),
    ]


def stack_rows(host_set: HostSet, copies: int, row_stride: int, shift_step: int = 37, shift_mod: int = 128,
               first: int = 0) -> HostSet:
    """Stack ``copies`` x-shifted copies of a set on disjoint row bands.

    Copy ``k`` (counted from ``first``, so batches split across ranks stay
    distinct) moves its rows by ``(k - first) * row_stride`` and its columns
    by ``(k * shift_step) % shift_mod - shift_mod // 2``.
    """

    begin, end, offsets, rows = host_set
    n = int(offsets[-1])
    r = int(rows.size)
    shifts = ((np.arange(copies, dtype=np.int64) + first) * shift_step) % shift_mod - shift_mod // 2
    b = (begin[None, :].astype(np.int64) + shifts[:, None]).reshape(-1)
    e = (end[None, :].astype(np.int64) + shifts[:, None]).reshape(-1)
    counts = np.diff(offsets.astype(np.int64))
    all_counts = np.tile(counts, copies)
    off = np.zeros(copies * r + 1, dtype=np.int64)
    np.cumsum(all_counts, out=off[1:])
    rows_all = (rows[None, :].astype(np.int64) + np.arange(copies, dtype=np.int64)[:, None] * row_stride).reshape(-1)
    assert off[-1] == n * copies
    return b.astype(np.int32), e.astype(np.int32), off.astype(np.int32), rows_all.astype(np.int32)


def _uneven_rows(rng: np.random.Generator, side: int, mu: float, sigma: float) -> HostSet:
    rows: List[Tuple[np.ndarray, np.ndarray]] = []
    for _ in range(side):
        k = int(round(float(rng.lognormal(mu, sigma))))
        k = min(k, side // 2)
        if k <= 0:
            rows.append((np.zeros(0, np.int64), np.zeros(0, np.int64)))
            continue
        pts = np.sort(rng.choice(side + 1, size=2 * k, replace=False))
        rows.append((pts[0::2], pts[1::2]))
    return _pack(rows)


def batched_uneven_sets(count: int = 256, seed: int = 3, side_seed: int = 3,
                        side_lo: int = 128, side_hi: int = 4096,
                        mu: float = 1.5, sigma: float = 1.0) -> Tuple[List[int], List[HostSet]]:
    """``count`` independent sets with log-uniform sides; returns ``(sides, sets)``."""

    side_rng = np.random.default_rng(side_seed)
    sides = [int(round(float(np.exp(side_rng.uniform(np.log(side_lo), np.log(side_hi)))))) for _ in range(count)]
    rng = np.random.default_rng(seed)
    return sides, [_uneven_rows(rng, s, mu, sigma) for s in sides]


def concat_sets(sets: Sequence[HostSet], row_strides: Sequence[int]) -> HostSet:
    """Concatenate sets onto disjoint row bands (set ``i`` starts at row ``sum(row_strides[:i])``)."""

    begins, ends, counts, rows_list = [], [], [], []
    base = 0
    for (b, e, off, rows), stride in zip(sets, row_strides):
        begins.append(b)
        ends.append(e)
        counts.append(np.diff(off.astype(np.int64)))
        rows_list.append(rows.astype(np.int64) + base)
        base += int(stride)
    cnt = np.concatenate(counts) if counts else np.zeros(0, np.int64)
    off = np.zeros(cnt.size + 1, dtype=np.int64)
    np.cumsum(cnt, out=off[1:])
    return (np.concatenate(begins).astype(np.int32) if begins else np.zeros(0, np.int32),
            np.concatenate(ends).astype(np.int32) if ends else np.zeros(0, np.int32),
            off.astype(np.int32),
            np.concatenate(rows_list).astype(np.int32) if rows_list else np.zeros(0, np.int32))


def disk_rows(size: int, radius: float, cx: float | None = None, cy: float | None = None) -> HostSet:
    """Disk of cells whose centres lie within ``radius`` of ``(cx, cy)`` (cell units), built row by row.

    Rows that the disk misses are left out; each kept row holds one interval.
    """
    cx = size / 2.0 if cx is None else cx
    cy = size / 2.0 if cy is None else cy
    ys = np.arange(size, dtype=np.float64)
    dy = ys + 0.5 - cy
    inside = dy * dy <= radius * radius
    hw = np.sqrt(np.maximum(radius * radius - dy * dy, 0.0))
    x0 = np.maximum(np.ceil(cx - hw - 0.5), 0).astype(np.int64)
    x1 = np.minimum(np.floor(cx + hw - 0.5), size - 1).astype(np.int64) + 1
    keep = inside & (x1 > x0)
    rows = np.nonzero(keep)[0]
    off = np.arange(rows.size + 1, dtype=np.int64)
    return x0[keep].astype(np.int32), x1[keep].astype(np.int32), off.astype(np.int32), rows.astype(np.int32)


def prolong_rows(s: HostSet, ratio: int) -> HostSet:
    """``[b r, e r)`` on rows ``y r .. y r + r - 1`` for every row ``y`` of ``s`` (the set prolongation)."""
    b, e, off, rows = s
    r = int(ratio)
    counts = np.diff(off.astype(np.int64))
    fb, fe, frows, fcounts = [], [], [], []
    for k, y in enumerate(rows):
        lo, hi = int(off[k]), int(off[k + 1])
        for d in range(r):
            fb.append(b[lo:hi].astype(np.int64) * r)
            fe.append(e[lo:hi].astype(np.int64) * r)
            frows.append(int(y) * r + d)
            fcounts.append(int(counts[k]))
    fo = np.zeros(len(fcounts) + 1, np.int64)
    np.cumsum(fcounts, out=fo[1:])
    cat = (lambda xs: np.concatenate(xs) if xs else np.zeros(0, np.int64))
    return (cat(fb).astype(np.int32), cat(fe).astype(np.int32), fo.astype(np.int32),
            np.asarray(frows, np.int64).astype(np.int32))


def nested_disk_levels(base: int, radii: Sequence[float], ratio: int = 2) -> List[HostSet]:
    """Levels of a nested hierarchy: the whole ``base x base`` grid, then one disk per radius.

    Level ``k >= 1`` is the disk of radius ``radii[k-1]`` (a fraction of the
    domain side, centred) rasterised on level ``k-1``'s grid and prolonged by
    ``ratio``, so that every coarse cell under it has all its children in it.
    """
    full = (np.zeros(base, np.int32), np.full(base, base, np.int32), np.arange(base + 1, dtype=np.int32),
            np.arange(base, dtype=np.int32))
    levels = [full]
    n = base
    for rad in radii:
        levels.append(prolong_rows(disk_rows(n, rad * n), ratio))
        n *= ratio
    return levels
