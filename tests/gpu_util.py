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
