"""Helpers shared by the GPU parity tests."""

from __future__ import annotations

import numpy as np
import torch

from oracle import oracle as O


def host(s):
    """(begin, end, row_offsets, rows) of a device IntervalSet as NumPy int32 arrays."""
    return tuple(np.asarray(torch.as_tensor(x).cpu().numpy(), dtype=np.int32)
                 for x in (s.begin, s.end, s.row_offsets, s.rows))


def dev_set(h, device="cuda"):
    from subsetix_b200.subsetix_cupy.expressions import IntervalSet

    b, e, off, rows = [torch.as_tensor(np.asarray(a, dtype=np.int32), device=device) for a in h]
    return IntervalSet(begin=b, end=e, row_offsets=off, rows=rows)


def assert_same(actual, expected, msg=""):
    a = host(actual) if not isinstance(actual, tuple) else actual
    for name, x, y in zip(("begin", "end", "row_offsets", "rows"), a, expected):
        np.testing.assert_array_equal(np.asarray(x), np.asarray(y), err_msg=f"{msg} {name}")


def iset(h):
    return O.ISet(*[np.asarray(a, dtype=np.int32) for a in h])


def rand_set(height, mean_count, seed, row_stride=1, min_per_row=0, max_col=None, touching=False, row0=-3):
    """Seeded random set: rows ``row0 + k * row_stride``, sorted intervals per row.

    ``touching`` lets neighbouring intervals share an end point (gap 0) now
    and then; ``max_col`` keeps every interval inside ``[0, max_col)``.
    """
    rng = np.random.default_rng(seed)
    begins, ends, counts = [], [], []
    for _ in range(height):
        k = max(int(rng.poisson(mean_count)), min_per_row)
        x = int(rng.integers(-5, 5)) if max_col is None else 0
        row_b, row_e = [], []
        for _ in range(k):
            gap = int(rng.geometric(0.2)) - (1 if touching and rng.random() < 0.3 else 0)
            length = int(rng.geometric(0.1))
            b = x + max(gap, 0 if touching else 1)
            e = b + length
            if max_col is not None and e > max_col:
                break
            row_b.append(b)
            row_e.append(e)
            x = e
        begins += row_b
        ends += row_e
        counts.append(len(row_b))
    off = np.zeros(height + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    rows = row0 + row_stride * np.arange(height)
    return (np.asarray(begins, np.int32), np.asarray(ends, np.int32), off.astype(np.int32), rows.astype(np.int32))
