"""Set algebra on the GPU against the reference's goldens and the oracle.

Interval outputs must be bit-exact: begin, end, row_offsets and rows.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from subsetix_b200 import synth
from tests.golden_io import get_set, load
from tests.gpu_util import assert_same, dev_set, host, iset, rand_set

pytestmark = pytest.mark.gpu

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")


def _ops():
    return {
        "union": sc.make_union,
        "intersection": sc.make_intersection,
        "difference": sc.make_difference,
        "symmetric_difference": sc.make_symmetric_difference,
        "complement": sc.make_complement,
    }


@pytest.fixture(scope="module")
def surfaces(cuda_device):
    b = sc.build_interval_set
    return {
        "A": b(row_offsets=[0, 2, 3], begin=[0, 6, 1], end=[4, 9, 5]),
        "B": b(row_offsets=[0, 1, 2], begin=[2, 0], end=[7, 4]),
        "C": b(row_offsets=[0, 1, 2], begin=[3, 2], end=[6, 3]),
        "D": b(row_offsets=[0, 1, 2], begin=[5, 5], end=[11, 8]),
        "E": b(row_offsets=[0, 1, 2], begin=[7, 6], end=[10, 9]),
    }


def _check(result, begin, end, offsets, rows=None):
    rows = list(range(len(offsets) - 1)) if rows is None else rows
    assert_same(result, (begin, end, offsets, rows))


# Golden vectors of the reference's own unit tests (subsetix_cupy/tests/test_expressions.py:154-309)

def test_nested_expression(surfaces):
    s = surfaces
    expr = sc.make_union(
        sc.make_difference(sc.make_intersection(sc.make_input(s["A"]), sc.make_input(s["B"])), sc.make_input(s["C"])),
        sc.make_intersection(sc.make_input(s["D"]), sc.make_input(s["E"])))
    _check(sc.evaluate(expr), [2, 6, 1, 3, 6], [3, 10, 2, 4, 8], [0, 2, 5])


def test_union_aligns_sparse_rows(surfaces):
    extra = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[1])
    _check(sc.evaluate(sc.make_union(sc.make_input(surfaces["A"]), sc.make_input(extra))),
           [0, 6, 1], [4, 9, 5], [0, 2, 3])


def test_difference_handles_empty_rhs(surfaces):
    empty = sc.build_interval_set(row_offsets=[0, 0, 0], begin=[], end=[])
    _check(sc.evaluate(sc.make_difference(sc.make_input(surfaces["A"]), sc.make_input(empty))),
           [0, 6, 1], [4, 9, 5], [0, 2, 3])


def test_union_sparse_row_ids(cuda_device):
    lhs = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[2], rows=[5])
    rhs = sc.build_interval_set(row_offsets=[0, 1], begin=[3], end=[4], rows=[7])
    _check(sc.evaluate(sc.make_union(sc.make_input(lhs), sc.make_input(rhs))), [0, 3], [2, 4], [0, 1, 2], [5, 7])


def test_symmetric_difference(surfaces):
    _check(sc.evaluate(sc.make_symmetric_difference(sc.make_input(surfaces["A"]), sc.make_input(surfaces["B"]))),
           [0, 4, 7, 0, 4], [2, 6, 9, 1, 5], [0, 3, 5])


def test_complement(surfaces):
    universe = sc.build_interval_set(row_offsets=[0, 1, 2], begin=[0, 0], end=[12, 6])
    _check(sc.evaluate(sc.make_complement(sc.make_input(universe), sc.make_input(surfaces["A"]))),
           [4, 9, 0, 5], [6, 12, 1, 6], [0, 2, 4])


def test_multishape_union(cuda_device):
    rect = sc.build_interval_set(row_offsets=[0, 2, 4, 6], begin=[0, 4, 1, 5, 2, 6], end=[2, 6, 3, 7, 4, 8])
    circ = sc.build_interval_set(row_offsets=[0, 1, 3, 4], begin=[1, 0, 4, 3], end=[5, 2, 6, 7])
    _check(sc.evaluate(sc.make_union(sc.make_input(rect), sc.make_input(circ))), [0, 0, 4, 2], [6, 3, 7, 8],
           [0, 1, 3, 4])
    ws = sc.CuPyWorkspace()
    _check(sc.evaluate(sc.make_union(sc.make_input(rect), sc.make_input(circ)), ws), [0, 0, 4, 2], [6, 3, 7, 8],
           [0, 1, 3, 4])


def test_backend_returns_device_arrays(surfaces):
    s = surfaces
    expr = sc.make_union(sc.make_intersection(sc.make_input(s["A"]), sc.make_input(s["B"])),
                         sc.make_difference(sc.make_input(s["D"]), sc.make_input(s["C"])))
    r = sc.evaluate(expr)
    assert isinstance(r.begin, torch.Tensor) and r.begin.is_cuda
    _check(r, [2, 6, 1, 5], [4, 11, 4, 8], [0, 2, 4])


def test_workspace_reuses_output_buffers(surfaces):
    ws = sc.CuPyWorkspace()
    expr = sc.make_union(sc.make_input(surfaces["A"]), sc.make_input(surfaces["B"]))
    r1 = sc.evaluate(expr, ws)
    p1 = r1.begin.data_ptr()
    del r1
    r2 = sc.evaluate(expr, ws)
    assert r2.begin.data_ptr() == p1


def test_interval_set_validation(cuda_device):
    with pytest.raises(TypeError):
        sc.IntervalSet(begin=torch.zeros(1, dtype=torch.int64, device="cuda"),
                       end=torch.zeros(1, dtype=torch.int32, device="cuda"),
                       row_offsets=torch.tensor([0, 1], dtype=torch.int32, device="cuda"), rows=[0])
    with pytest.raises(ValueError):
        sc.build_interval_set(row_offsets=[0, 2], begin=[0], end=[1])
    with pytest.raises(ValueError):
        sc.build_interval_set(row_offsets=[0, 1, 1], begin=[0], end=[1], rows=[3, 3])


# Fixtures produced by the reference itself

BIN = ["union", "intersection", "difference", "symmetric_difference", "complement"]


def _binop(name, a, b):
    return sc.evaluate(_ops()[name](sc.make_input(a), sc.make_input(b)))


def test_random_rows_256_setops(cuda_device):
    g = load("setops.npz")
    A, B = dev_set(get_set(g, "rows256/A")), dev_set(get_set(g, "rows256/B"))
    for op in BIN:
        assert_same(_binop(op, A, B), get_set(g, f"rows256/{op}"), op)


def test_fixture_binary_cases(cuda_device):
    g = load("setops.npz")
    for c in range(int(g["bin_count"])):
        A, B = dev_set(get_set(g, f"bin{c}/A")), dev_set(get_set(g, f"bin{c}/B"))
        for op in BIN:
            assert_same(_binop(op, A, B), get_set(g, f"bin{c}/{op}"), f"case {c} {op}")


EXPRS = {
    "e0": ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E"),
    "e1": ("union", ("intersection", ("difference", "D", "A"), "B"), ("symmetric_difference", "C", "E")),
    "e2": ("complement", ("union", "D", "E"), ("intersection", "A", "B")),
    "e3": ("intersection", ("union", "A", ("intersection", "B", "C")), ("difference", "E", "D")),
}


def _build(spec, leaves):
    if isinstance(spec, str):
        return sc.make_input(leaves[spec])
    return _ops()[spec[0]](_build(spec[1], leaves), _build(spec[2], leaves))


def test_fixture_expressions(cuda_device):
    g = load("setops.npz")
    for c in range(int(g["expr_count"])):
        leaves = {n: dev_set(get_set(g, f"expr{c}/{n}")) for n in "ABCDE"}
        for name, spec in EXPRS.items():
            assert_same(sc.evaluate(_build(spec, leaves)), get_set(g, f"expr{c}/{name}"), f"expr{c} {name}")
    leaves = {n: dev_set(get_set(g, f"shape512/{n}")) for n in "ABCDE"}
    assert_same(sc.evaluate(_build(EXPRS["e0"], leaves)), get_set(g, "shape512/e0"), "shape512")


def _random_canonical(rng, rows, width, mean_count, row_ids=None):
    begins, ends, off = [], [], [0]
    for _ in range(rows):
        k = int(rng.poisson(mean_count))
        x = int(rng.integers(-20, 20))
        for _ in range(k):
            x += int(rng.geometric(1 / 6.0))
            b = x
            x += int(rng.geometric(1 / 9.0))
            begins.append(b)
            ends.append(x)
        off.append(len(begins))
    rid = np.arange(rows, dtype=np.int32) if row_ids is None else row_ids
    return (np.asarray(begins, np.int32), np.asarray(ends, np.int32), np.asarray(off, np.int32), rid)


@pytest.mark.parametrize("mean_count", [0.5, 4.0, 40.0, 700.0])
def test_random_large_vs_oracle(cuda_device, mean_count):
    rng = np.random.default_rng(int(mean_count * 10))
    rows = max(4, int(40000 / max(mean_count, 1)))
    hs = [_random_canonical(rng, rows, 0, mean_count) for _ in range(5)]
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", hs)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", hs)}
    for name, spec in EXPRS.items():
        assert_same(sc.evaluate(_build(spec, leaves_d)), O.evaluate(spec, leaves_h), f"{name} m={mean_count}")
    for op in BIN:
        assert_same(_binop(op, leaves_d["A"], leaves_d["B"]), O.BINARY[op](leaves_h["A"], leaves_h["B"]), op)


def test_sparse_unaligned_rows_vs_oracle(cuda_device):
    rng = np.random.default_rng(7)
    hs = []
    for i in range(5):
        rid = np.sort(rng.choice(np.arange(-3000, 9000), size=3000, replace=False)).astype(np.int32)
        hs.append(_random_canonical(rng, rid.size, 0, 3.0, row_ids=rid))
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", hs)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", hs)}
    for name, spec in EXPRS.items():
        assert_same(sc.evaluate(_build(spec, leaves_d)), O.evaluate(spec, leaves_h), name)


def test_long_rows_take_exact_path(cuda_device):
    # one row far longer than a fused tile: the exact path must produce the same result
    rng = np.random.default_rng(11)
    hs = [_random_canonical(rng, 3, 0, 20000.0) for _ in range(2)]
    A, B = dev_set(hs[0]), dev_set(hs[1])
    for op in BIN:
        assert_same(_binop(op, A, B), O.BINARY[op](iset(hs[0]), iset(hs[1])), op)


def test_shapes_4096_expression(cuda_device):
    ops = synth.shape_operands(4096)
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", ops)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", ops)}
    assert_same(sc.evaluate(_build(EXPRS["e0"], leaves_d)), O.evaluate(EXPRS["e0"], leaves_h), "shapes4096")


def test_wide_coordinate_span_vs_oracle(cuda_device):
    # tiles whose coordinates span more than 2^24 take the 64-bit key path
    rng = np.random.default_rng(12)
    hs = []
    for _ in range(5):
        b, e, off, rid = _random_canonical(rng, 700, 0, 5.0)
        hs.append(((b.astype(np.int64) * 40000).astype(np.int32), (e.astype(np.int64) * 40000).astype(np.int32),
                   off, rid))
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", hs)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", hs)}
    for name, spec in EXPRS.items():
        assert_same(sc.evaluate(_build(spec, leaves_d)), O.evaluate(spec, leaves_h), name)


@pytest.mark.parametrize("tuning", [{"kernel": 1}, {"kernel": 1, "blocks_per_sm": 6}, {"kernel": 2},
                                    {"kernel": 3, "staging_cap": 256}, {"kernel": 3, "staging_cap": 12000},
                                    {"kernel": 4, "staging_cap": 256}, {"kernel": 4, "warps": 1},
                                    {"kernel": 4, "warps": 8}, {"kernel": 4, "staging_cap": 20000, "warps": 3},
                                    {"kernel": 4, "tile_rows": 16}, {"kernel": 5}, {"kernel": 5, "tile_rows": 32},
                                    {"kernel": 5, "tile_rows": 1, "warps": 1}, {"kernel": 5, "staging_cap": 64},
                                    {"kernel": 6}, {"kernel": 6, "tile_rows": 3, "warps": 1},
                                    {"kernel": 6, "staging_cap": 64}, {"kernel": 6, "tile_rows": 32},
                                    {"kernel": 7}, {"kernel": 7, "staging_cap": 64, "warps": 2}])
def test_tuning_never_changes_results(cuda_device, tuning):
    from subsetix_b200 import _core

    ops = synth.shape_operands(1024)
    leaves_h = {n: iset(h) for n, h in zip("ABCDE", ops)}
    leaves_d = {n: dev_set(h) for n, h in zip("ABCDE", ops)}
    saved = dict(_core.TUNING)
    try:
        _core.TUNING.clear()
        _core.TUNING.update(tuning)
        got = sc.evaluate(_build(EXPRS["e0"], leaves_d))
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)
    assert_same(got, O.evaluate(EXPRS["e0"], leaves_h), str(tuning))


def test_tile_boundaries_max(cuda_device):
    from subsetix_b200 import _core

    rng = np.random.default_rng(21)
    rows = 1003
    leaves = []
    host = []
    for _ in range(3):
        off = np.concatenate([[0], np.cumsum(rng.integers(0, 40, rows))]).astype(np.int32)
        n = int(off[-1])
        beg = rng.integers(-5000, 5000, n).astype(np.int32)
        end = (beg + rng.integers(1, 50, n)).astype(np.int32)
        host.append((off, beg, end))
        leaves.append((torch.as_tensor(beg, device="cuda"), torch.as_tensor(end, device="cuda"),
                       torch.as_tensor(off, device="cuda"), 0))
    for a, b in ((8, 32), (1, 7), (16, 1000), (5, 2000)):
        got = _core.max_tile_boundaries(leaves, rows, torch.device("cuda", 0), tile_rows=(a, b))
        stats = _core.tile_stats(leaves, rows, torch.device("cuda", 0), a, b)
        assert stats[:2] == tuple(got)
        want = []
        for tr in (a, b):
            edges = np.minimum(np.arange(0, rows + tr, tr), rows)
            want.append(2 * int(max(sum(o[edges[1:]] - o[edges[:-1]] for o, _, _ in host).max(), 0)))
        assert got == want, (a, b)
        span = 0
        for t0 in range(0, rows, a):
            lo, hi = None, None
            for off, beg, end in host:
                for r in range(t0, min(rows, t0 + a)):
                    if off[r + 1] > off[r]:
                        x0 = min(beg[off[r]], end[off[r]])
                        x1 = max(end[off[r + 1] - 1], beg[off[r + 1] - 1])
                        lo = x0 if lo is None else min(lo, x0)
                        hi = x1 if hi is None else max(hi, x1)
            if lo is not None:
                span = max(span, int(hi) - int(lo))
        assert stats[2] == span, (a, b)


MANY = {
    6: ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")),
        ("difference", "E", "F")),
    7: ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")),
        ("union", ("difference", "E", "F"), "G")),
    8: ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")),
        ("union", ("difference", "E", "F"), ("intersection", "G", "H"))),
}


@pytest.mark.parametrize("k", [6, 7, 8])
@pytest.mark.parametrize("tuning", [{}, {"kernel": 3}, {"kernel": 4}, {"kernel": 5}, {"kernel": 6}])
def test_many_leaf_expressions(cuda_device, k, tuning):
    # six to eight leaves: the truth table spans several words
    from subsetix_b200 import _core

    rng = np.random.default_rng(100 + k)
    names = "ABCDEFGH"[:k]
    hs = [_random_canonical(rng, 1500, 0, 6.0) for _ in names]
    leaves_h = {n: iset(h) for n, h in zip(names, hs)}
    leaves_d = {n: dev_set(h) for n, h in zip(names, hs)}
    saved = dict(_core.TUNING)
    try:
        _core.TUNING.clear()
        _core.TUNING.update(tuning)
        got = sc.evaluate(_build(MANY[k], leaves_d))
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)
    assert_same(got, O.evaluate(MANY[k], leaves_h), f"k={k} {tuning}")


@pytest.mark.parametrize("kernel", [6, 7])
def test_lookback_wait_gives_up_and_reports_timeout(cuda_device, kernel):
    """A tile that never publishes its look-back status: the tiles after it give up after a few polls,
    the sweep finishes and reports SX_FLAG_TIMEOUT, the public call raises, and the next regular call
    is exact (nothing hangs, the context stays usable)."""
    from subsetix_b200 import _core, _lib

    rows = 20000
    A = rand_set(rows, 4.0, seed=31, row0=0)
    B = rand_set(rows, 4.0, seed=32, row0=0)
    la, lb = dev_set(A), dev_set(B)
    specs = [(la.begin, la.end, la.row_offsets, 0), (lb.begin, lb.end, lb.row_offsets, 0)]
    tr = 8 if kernel == 6 else 16
    cap = _core.max_tile_boundaries(specs, rows, cuda_device, tile_rows=tr)
    tuning = {"kernel": kernel, "tile_rows": tr, "warps": 2, "staging_cap": cap, "wait_limit": 256, "withhold_tile": 5}
    table = [0b1110] + [0] * 7  # A | B over the state bits (A = 1, B = 2)
    _, _, _, result = _core.bool_eval_async(specs, rows, table, _lib.MODE_TABLE, cuda_device, tuning=tuning)
    total, flags = (int(x) for x in result.cpu())
    assert flags & _lib.FLAG_TIMEOUT
    saved = dict(_core.TUNING)
    _core.TUNING.clear()
    _core.TUNING.update(tuning)
    try:
        with pytest.raises(_lib.SubsetixError):
            sc.evaluate(sc.make_union(sc.make_input(la), sc.make_input(lb)))
    finally:
        _core.TUNING.clear()
        _core.TUNING.update(saved)
    got = sc.evaluate(sc.make_union(sc.make_input(la), sc.make_input(lb)))
    assert_same(got, O.union(iset(A), iset(B)))


def test_headline_expression_at_full_size_against_oracle(cuda_device):
    """((A|B)-(C&D))^E on the 4096^2 shapes stacked 128 times (37.9 M input intervals, the benchmark's batch)
    through the public evaluate(), equal to the oracle bit for bit."""
    import bench

    leaves = bench.workload(128)
    O, oleaves = bench._oracle_leaves(leaves)
    want = O.evaluate(bench.SPEC, oleaves)
    A, B, C, D, F = [sc.make_input(dev_set(h)) for h in leaves]
    got = sc.evaluate(sc.make_symmetric_difference(sc.make_difference(sc.make_union(A, B), sc.make_intersection(C, D)),
                                                   F))
    assert int(got.begin.shape[0]) > 20_000_000
    assert_same(got, tuple(want[:4]), "headline expression")
