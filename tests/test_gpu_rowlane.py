"""The row-lane sweep (sx_tuning kernel 7) against the oracle and a dense-mask check.

One lane sweeps one row of a 32-row tile over 16-bit coordinates staged in
shared memory.  Its outputs must be bit-exact: expressions against the
oracle, arbitrary truth tables over one to eight leaves against dense
boolean masks of every row, tiles too wide for 16 bits (the global-memory
sweep of the same launch) and tiles above the staging capacity equal to the
staged ones, and inputs outside the contract (empty, touching, overlapping
or unsorted intervals) reported with SX_FLAG_CONTRACT.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from subsetix_b200 import _core, _lib, synth
from tests.gpu_util import assert_same, dev_set, iset

pytestmark = pytest.mark.gpu

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")


def _rows(rng, rows, mean, x0=0, spread=0, gap=6.0, length=9.0):
    """Canonical rows: Poisson(mean) intervals per row from x0 + U[0, spread), geometric gaps and lengths >= 1."""
    begins, ends, off = [], [], [0]
    for _ in range(rows):
        x = x0 + (int(rng.integers(0, spread)) if spread > 0 else 0)
        for _ in range(int(rng.poisson(mean))):
            x += int(rng.geometric(1 / gap))
            begins.append(x)
            x += int(rng.geometric(1 / length))
            ends.append(x)
        off.append(len(begins))
    return [np.asarray(a, np.int32) for a in (begins, ends, off)]


def _masks(leaf, rows, x0, width):
    b, e, off = leaf
    m = np.zeros((rows, width), bool)
    for r in range(rows):
        for j in range(off[r], off[r + 1]):
            m[r, b[j] - x0:e[j] - x0] = True
    return m


def _runs(mask, x0):
    """Maximal runs of every row of a boolean mask: (begin, end, row_offsets)."""
    rows, width = mask.shape
    pad = np.zeros((rows, width + 2), np.int8)
    pad[:, 1:-1] = mask
    d = np.diff(pad, axis=1)
    rb, cb = np.nonzero(d == 1)
    re_, ce = np.nonzero(d == -1)
    off = np.zeros(rows + 1, np.int64)
    np.add.at(off, rb + 1, 1)
    return (cb + x0).astype(np.int32), (ce + x0).astype(np.int32), np.cumsum(off).astype(np.int32)


def _table_eval(leaves, rows, table, tuning, device):
    d = [tuple(torch.as_tensor(a, device=device) for a in leaf) + (0,) for leaf in leaves]
    saved = dict(_core.TUNING)
    try:
        _core.TUNING.clear()
        _core.TUNING.update(tuning)
        ob, oe, ooff, total, flags = _core.bool_eval(d, rows, table, _lib.MODE_TABLE, device)
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)
    return ob[:total].cpu().numpy(), oe[:total].cpu().numpy(), ooff.cpu().numpy(), flags


def _random_table(rng, k):
    """A truth table over k leaves with f(empty) = 0, as 8 words."""
    bits = rng.integers(0, 2, 1 << k)
    bits[0] = 0
    words = [0] * 8
    for s, v in enumerate(bits):
        if v:
            words[s >> 5] |= 1 << (s & 31)
    return words, bits


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("tuning", [{"kernel": 7}, {"kernel": 7, "tile_rows": 32}, {"kernel": 7, "tile_rows": 8},
                                    {"kernel": 7, "staging_cap": 64, "warps": 3}])
def test_random_truth_tables_against_dense_masks(cuda_device, k, tuning):
    rng = np.random.default_rng(100 + k)
    rows, x0, width = 203, -40, 1400  # a partial last tile of 11 rows
    leaves = [_rows(rng, rows, float(rng.uniform(0.3, 9.0)), x0=x0, spread=30, gap=5.0 + l, length=4.0 + 2 * l)
              for l in range(k)]
    width = max(width, max(int(leaf[1].max(initial=x0)) - x0 + 1 for leaf in leaves))
    words, bits = _random_table(rng, k)
    masks = [_masks(leaf, rows, x0, width) for leaf in leaves]
    state = sum(m.astype(np.int64) << l for l, m in enumerate(masks))
    want = _runs(bits[state].astype(bool), x0)
    got_b, got_e, got_off, flags = _table_eval(leaves, rows, words, tuning, cuda_device)
    assert flags == 0
    np.testing.assert_array_equal(got_b, want[0])
    np.testing.assert_array_equal(got_e, want[1])
    np.testing.assert_array_equal(got_off, want[2])


@pytest.mark.parametrize("tuning", [{"kernel": 7}, {"kernel": 7, "warps": 1}, {"kernel": 7, "staging_cap": 200},
                                    {"kernel": 7, "tile_rows": 32, "warps": 1}, {"kernel": 7, "tile_rows": 8, "warps": 4}])
def test_shape_expression_against_oracle(cuda_device, tuning):
    ops = synth.shape_operands(1024)
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", ops)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", ops)}
    spec = ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E")
    expr = sc.make_symmetric_difference(
        sc.make_difference(sc.make_union(sc.make_input(leaves_d["A"]), sc.make_input(leaves_d["B"])),
                           sc.make_intersection(sc.make_input(leaves_d["C"]), sc.make_input(leaves_d["D"]))),
        sc.make_input(leaves_d["E"]))
    saved = dict(_core.TUNING)
    try:
        _core.TUNING.clear()
        _core.TUNING.update(tuning)
        got = sc.evaluate(expr)
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)
    assert_same(got, O.evaluate(spec, leaves_h), str(tuning))


def _mix(wide, narrow, rows):
    """Rows of ``wide`` in odd 32-row tiles, rows of ``narrow`` in even ones."""
    parts = []
    for r in range(rows):
        b, e, off = wide if (r // 32) % 2 else narrow
        parts.append((b[off[r]:off[r + 1]], e[off[r]:off[r + 1]]))
    return (np.concatenate([p[0] for p in parts]).astype(np.int32),
            np.concatenate([p[1] for p in parts]).astype(np.int32),
            np.concatenate([[0], np.cumsum([len(p[0]) for p in parts])]).astype(np.int32))


def test_wide_tiles_take_the_global_sweep(cuda_device):
    """Tiles spanning more than 65534 columns sweep global memory in the same launch: same results."""
    rng = np.random.default_rng(7)
    rows = 130  # tiles 1 and 3 wide, tiles 0, 2 and 4 (two rows) narrow
    wide = [_rows(rng, rows, 4.0, x0=-2_000_000, spread=4_000_000, gap=3000.0, length=5000.0) for _ in range(2)]
    narrow = [_rows(rng, rows, 6.0, x0=10, spread=50) for _ in range(2)]
    a, b = _mix(wide[0], narrow[0], rows), _mix(wide[1], narrow[1], rows)
    table = [0b0110] + [0] * 7  # xor
    for tr in (8, 16, 32):
        got = _table_eval([a, b], rows, table, {"kernel": 7, "tile_rows": tr}, cuda_device)
        assert got[3] == 0
        _check_xor(got, a, b, rows)


def _check_xor(got, a, b, rows):
    ids = np.arange(rows, dtype=np.int32)
    want = O.symmetric_difference(O.ISet(a[0], a[1], a[2], ids), O.ISet(b[0], b[1], b[2], ids))
    np.testing.assert_array_equal(got[0], want.begin)
    np.testing.assert_array_equal(got[1], want.end)
    np.testing.assert_array_equal(got[2], want.row_offsets)


def test_empty_rows_and_empty_leaves(cuda_device):
    rng = np.random.default_rng(3)
    rows = 97
    a = _rows(rng, rows, 0.4, spread=100)
    empty = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(rows + 1, np.int32))
    for table in ([0b10] + [0] * 7, [0b1110] + [0] * 7, [0b1000] + [0] * 7):
        ref = _table_eval([a, empty], rows, table, {"kernel": 5}, cuda_device)
        for tr in (8, 16, 32):
            got = _table_eval([a, empty], rows, table, {"kernel": 7, "tile_rows": tr}, cuda_device)
            assert got[3] == 0
            for x, y in zip(got[:3], ref[:3]):
                np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("tile_rows", [8, 16, 32])
@pytest.mark.parametrize("case", ["empty", "touching", "overlap", "unsorted", "offsets"])
def test_contract_violations_are_flagged(cuda_device, case, tile_rows):
    rng = np.random.default_rng(5)
    rows = 70
    b, e, off = _rows(rng, rows, 5.0, spread=20)
    b, e, off = b.copy(), e.copy(), off.copy()
    r = next(r for r in range(32, 64) if off[r + 1] - off[r] >= 3)  # a row of tile 1
    j = int(off[r]) + 1  # an interval in the middle of it
    if case == "empty":
        e[j] = b[j]
    elif case == "touching":
        b[j] = e[j - 1]
    elif case == "overlap":
        b[j] = e[j - 1] - 1
    elif case == "unsorted":
        b[j], e[j], b[j + 1], e[j + 1] = b[j + 1], e[j + 1], b[j], e[j]
    else:
        off[r + 1] = off[r] - 1
    other = _rows(rng, rows, 3.0, spread=20)
    _, _, _, flags = _table_eval([(b, e, off), other], rows, [0b1110] + [0] * 7,
                                 {"kernel": 7, "tile_rows": tile_rows}, cuda_device)
    assert flags & _lib.FLAG_CONTRACT, case


def test_tuning_rejects_other_tile_heights(cuda_device):
    leaf = tuple(torch.as_tensor(a, device=cuda_device) for a in _rows(np.random.default_rng(1), 40, 2.0)) + (0,)
    saved = dict(_core.TUNING)
    try:
        _core.TUNING.clear()
        _core.TUNING.update({"kernel": 7, "tile_rows": 12})
        with pytest.raises(ValueError, match="32 rows"):
            _core.bool_eval([leaf], 40, [0b10] + [0] * 7, _lib.MODE_TABLE, cuda_device)
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)


@pytest.mark.parametrize("x0", [2**31 - 70000, -2**31 + 5])
def test_coordinates_next_to_the_int32_limits(cuda_device, x0):
    """Narrow tiles (staged, 16-bit offsets from the tile's xmin) whose coordinates lie next to INT_MAX or INT_MIN."""
    rng = np.random.default_rng(17)
    rows = 80
    leaves = [_rows(rng, rows, 6.0, x0=x0, spread=200, gap=7.0 + l, length=5.0 + l) for l in range(3)]
    assert all(int(leaf[1].max()) < 2**31 - 1 for leaf in leaves)
    words = [sum(1 << s for s in range(8) if (s & 1) and not (s & 4)) | (1 << 2)] + [0] * 7  # (A - C) | (B alone)
    bits = np.array([(words[0] >> s) & 1 for s in range(8)])
    width = max(int(leaf[1].max()) - x0 + 1 for leaf in leaves)
    masks = [_masks(leaf, rows, x0, width) for leaf in leaves]
    state = sum(m.astype(np.int64) << l for l, m in enumerate(masks))
    want = _runs(bits[state].astype(bool), 0)
    for tr in (8, 16, 32):
        got_b, got_e, got_off, flags = _table_eval(leaves, rows, words, {"kernel": 7, "tile_rows": tr}, cuda_device)
        assert flags == 0
        np.testing.assert_array_equal(got_b.astype(np.int64) - x0, want[0])
        np.testing.assert_array_equal(got_e.astype(np.int64) - x0, want[1])
        np.testing.assert_array_equal(got_off, want[2])
