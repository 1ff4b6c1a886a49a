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
