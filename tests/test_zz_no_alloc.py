"""The allocation-free entry point against the regular one.

sx_bool_eval_static serves callers that cannot allocate device memory
(a host that owns the device heap, or a loop that cannot pay for
cudaMalloc's synchronisation).  It keeps its look-back scratch in a fixed
array inside the library instead of a caller workspace.  Its results must
equal sx_bool_eval's, bit for bit, on two consecutive calls: the second call
reuses the array the first one left behind.

The file name makes pytest collect it last, so a run that stops at the
first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest
import torch

from subsetix_b200 import _core, _lib
from subsetix_b200._runtime import ptr, stream_handle

pytestmark = pytest.mark.gpu


def _random_rows(rng, rows, mean):
    begins, ends, off = [], [], [0]
    for _ in range(rows):
        x = int(rng.integers(-50, 50))
        for _ in range(int(rng.poisson(mean))):
            x += int(rng.geometric(1 / 5.0))
            begins.append(x)
            x += int(rng.geometric(1 / 7.0))
            ends.append(x)
        off.append(len(begins))
    return [np.asarray(a, np.int32) for a in (begins, ends, off)]


def _leaves(device, seed):
    rng = np.random.default_rng(seed)
    rows = 5000
    return rows, [tuple(torch.as_tensor(a, device=device) for a in _random_rows(rng, rows, m)) for m in (3, 6, 9)]


# ((A | B) - C) as a truth table over bits (A=1, B=2, C=4)
TABLE = [sum(1 << s for s in range(8) if ((s & 1) or (s & 2)) and not (s & 4))] + [0] * 7


def _static_call(lib, leaves, rows, device):
    k = len(leaves)
    arr = (_lib.SxLeaf * k)()
    for i, (b, e, off) in enumerate(leaves):
        arr[i].begin, arr[i].end, arr[i].row_offsets, arr[i].widen = ptr(b), ptr(e), ptr(off), 0
    cap = max(1, sum(int(b.numel()) for b, _, _ in leaves))
    ob = torch.full((cap,), -7, dtype=torch.int32, device=device)
    oe = torch.full((cap,), -7, dtype=torch.int32, device=device)
    ooff = torch.full((rows + 1,), -7, dtype=torch.int32, device=device)
    result = torch.full((2,), -7, dtype=torch.int32, device=device)
    tab = (ctypes.c_uint32 * 8)(*TABLE)
    rc = lib.sx_bool_eval_static(arr, k, rows, tab, _lib.MODE_TABLE, ptr(ob), ptr(oe), ptr(ooff), cap, ptr(result),
                                 stream_handle(device))
    assert rc == _lib.SX_OK, _lib.last_error()
    total, flags = (int(x) for x in result.cpu())
    return ob[:total].cpu(), oe[:total].cpu(), ooff.cpu(), flags


def test_static_scratch_matches_workspace_entry_point(cuda_device):
    lib = _lib.load()
    rows, leaves = _leaves(cuda_device, 11)
    specs = [(b, e, off, 0) for b, e, off in leaves]
    ob, oe, ooff, total, flags = _core.bool_eval(specs, rows, TABLE, _lib.MODE_TABLE, cuda_device)
    assert flags == 0
    want = (ob[:total].cpu(), oe[:total].cpu(), ooff.cpu())
    for _ in range(2):  # the second call reuses the scratch left by the first
        got_b, got_e, got_off, got_flags = _static_call(lib, leaves, rows, cuda_device)
        assert got_flags == 0
        assert torch.equal(got_b, want[0])
        assert torch.equal(got_e, want[1])
        assert torch.equal(got_off, want[2])


def test_static_scratch_rejects_oversized_input(cuda_device):
    lib = _lib.load()
    arr = (_lib.SxLeaf * 1)()
    tab = (ctypes.c_uint32 * 8)(*TABLE)
    rc = lib.sx_bool_eval_static(arr, 1, 3944449, tab, _lib.MODE_TABLE, None, None, None, 0, None,
                                 stream_handle(cuda_device))
    assert rc == _lib.SX_ERR_CAPACITY
    assert "3944448" in _lib.last_error()


def _sparse_rows(rng, rows, mean):
    """Vectorised random rows: Poisson(mean) intervals per row, gaps and lengths of at least one cell."""
    counts = rng.poisson(mean, rows)
    n = int(counts.sum())
    off = np.zeros(rows + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    steps = rng.geometric(1 / 4.0, size=2 * n).reshape(n, 2)
    row_of = np.repeat(np.arange(rows), counts)
    # positions restart at every row: cumulative sums within each row
    flat = steps.reshape(-1).cumsum()
    start_of_row = np.zeros(rows, np.int64)
    first = off[:-1][counts > 0]
    base = np.where(first > 0, flat[2 * first - 1], 0)
    start_of_row[counts > 0] = base
    pos = flat - np.repeat(start_of_row[row_of], 2)
    b = pos[0::2].astype(np.int32)
    e = pos[1::2].astype(np.int32)
    return b, e, off.astype(np.int32)


def test_static_scratch_large_input_takes_32_row_tiles(cuda_device):
    """Above about a million rows the built-in array holds only 32-row tiles' look-back state."""
    lib = _lib.load()
    rng = np.random.default_rng(21)
    rows = 1_100_000
    leaves = [tuple(torch.as_tensor(a, device=cuda_device) for a in _sparse_rows(rng, rows, m)) for m in (0.6, 1.0, 1.4)]
    specs = [(b, e, off, 0) for b, e, off in leaves]
    ob, oe, ooff, total, flags = _core.bool_eval(specs, rows, TABLE, _lib.MODE_TABLE, cuda_device)
    assert flags == 0
    for _ in range(2):
        got_b, got_e, got_off, got_flags = _static_call(lib, leaves, rows, cuda_device)
        assert got_flags == 0
        assert torch.equal(got_b, ob[:total].cpu())
        assert torch.equal(got_e, oe[:total].cpu())
        assert torch.equal(got_off, ooff.cpu())


def test_static_scratch_union_mode(cuda_device):
    """The merged union of widened leaves (the dilation sweep) through the static entry point."""
    lib = _lib.load()
    rows, leaves = _leaves(cuda_device, 13)
    arr = (_lib.SxLeaf * len(leaves))()
    for i, (b, e, off) in enumerate(leaves):
        arr[i].begin, arr[i].end, arr[i].row_offsets, arr[i].widen = ptr(b), ptr(e), ptr(off), i
    specs = [(b, e, off, i) for i, (b, e, off) in enumerate(leaves)]
    ob, oe, ooff, total, flags = _core.bool_eval(specs, rows, [0] * 8, _lib.MODE_UNION, cuda_device)
    assert flags == 0
    cap = max(1, sum(int(b.numel()) for b, _, _ in leaves))
    for _ in range(2):
        sb = torch.full((cap,), -7, dtype=torch.int32, device=cuda_device)
        se = torch.full((cap,), -7, dtype=torch.int32, device=cuda_device)
        soff = torch.full((rows + 1,), -7, dtype=torch.int32, device=cuda_device)
        res = torch.full((2,), -7, dtype=torch.int32, device=cuda_device)
        tab = (ctypes.c_uint32 * 8)(*([0] * 8))
        rc = lib.sx_bool_eval_static(arr, len(leaves), rows, tab, _lib.MODE_UNION, ptr(sb), ptr(se), ptr(soff), cap,
                                     ptr(res), stream_handle(cuda_device))
        assert rc == _lib.SX_OK, _lib.last_error()
        n, f = (int(x) for x in res.cpu())
        assert f == 0 and n == total
        assert torch.equal(sb[:n].cpu(), ob[:total].cpu())
        assert torch.equal(se[:n].cpu(), oe[:total].cpu())
        assert torch.equal(soff.cpu(), ooff.cpu())
