"""The product's kernels against the reference's own kernels on the same GPU.

The reference compiles its CUDA-C kernel strings with NVRTC at run time and
NVRTC contracts multiplies into adds by default (``--fmad=true``).  Which
operations it fuses decides the last bit of every float32 result, so the
float32 parity target is the reference kernels run on this GPU:
``oracle/build_ref_nvrtc.py`` compiles them unchanged with the reference's
options, ``oracle/refgpu.py`` launches them with the reference's grid shapes.

Every comparison here is bit for bit: intervals, upwind values, gradient
magnitudes, threshold runs, prolonged and restricted fields.
"""

import re

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import refgpu
from tests.golden_io import load
from tests.gpu_util import assert_same, dev_set, host, rand_set

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="reference cubins not built (oracle/build_ref_nvrtc.py)")]

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")
rg = pytest.importorskip("subsetix_b200.subsetix_amr2.regrid")


@pytest.fixture(scope="module")
def ref(cuda_device):
    return refgpu.RefKernels(cuda_device)


def _t(x):
    return torch.as_tensor(x).cuda()


def _bits_equal(a, b, what):
    a = np.ascontiguousarray(torch.as_tensor(a).cpu().numpy())
    b = np.ascontiguousarray(torch.as_tensor(b).cpu().numpy())
    assert a.shape == b.shape and a.dtype == b.dtype, what
    as_int = np.int32 if a.dtype == np.float32 else np.int64
    diff = a.view(as_int) != b.view(as_int)
    n = int(diff.sum())
    assert n == 0, f"{what}: {n} of {a.size} values differ (first at {int(np.flatnonzero(diff)[0])})"


def _field(h, values):
    s = dev_set(h)
    f = sc.create_interval_field(s, fill_value=0.0, dtype=np.float32)
    f.values.copy_(torch.as_tensor(values, dtype=torch.float32, device="cuda"))
    return s, f


def _random_geometry(W, H, mean_k, seed):
    g = np.random.default_rng(seed)
    bs, es, offs = [], [], [0]
    for _ in range(H):
        k = min(int(g.poisson(mean_k)), W // 4)
        pts = np.sort(g.choice(W + 1, size=2 * k, replace=False))
        bs += list(pts[0::2])
        es += list(pts[1::2])
        offs.append(len(bs))
    return (np.array(bs, np.int32), np.array(es, np.int32), np.array(offs, np.int32), np.arange(H, dtype=np.int32))


def _gauss(n, sigma=0.05):
    xs = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(xs, xs)
    return np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / (2 * sigma ** 2)).astype(np.float32)


_VELOCITIES = [(1.0, 0.5, 0.5 / (1.5 * 2048), 1 / 2048, 1 / 2048),  # the fine level of the 1024^2 AMR run
               (1.0, 0.5, 0.5 / (1.5 * 2048), 1 / 1024, 1 / 1024),  # and its coarse level
               (0.7, -0.3, 0.37, 0.9, 1.1), (-1.3, 0.9, 0.05, 0.3, 0.7), (0.3, 0.123, 0.77, 1.0, 1.0),
               (1.7, -2.1, 0.013, 0.1, 0.1)]


@pytest.mark.parametrize("geom", ["sparse", "dense_rows", "gauss1024"])
def test_upwind_f32_bit_exact_vs_reference_kernel(ref, geom):
    rng = np.random.default_rng(3)
    if geom == "gauss1024":
        W = H = 1024
        h = (np.zeros(H, np.int32), np.full(H, W, np.int32), np.arange(H + 1, dtype=np.int32),
             np.arange(H, dtype=np.int32))
        vals = _gauss(W).reshape(-1)
    else:
        W, H = 512, 384
        h = _random_geometry(W, H, 3 if geom == "sparse" else 40, 11 if geom == "sparse" else 12)
        vals = rng.uniform(-1, 1, int((h[1] - h[0]).sum())).astype(np.float32)
    s, f = _field(h, vals)
    for a, b, dt, dx, dy in _VELOCITIES:
        want = ref.upwind_f32(s.begin, s.end, s.row_offsets, s.rows, f.interval_cell_offsets, f.values, width=W,
                              height=H, a=a, b=b, dt=dt, dx=dx, dy=dy)
        got = sc.step_upwind_interval(f, width=W, height=H, a=a, b=b, dt=dt, dx=dx, dy=dy)
        _bits_equal(got, want, f"upwind {geom} a={a} b={b} dt={dt} dx={dx}")


def test_upwind_fixture_inputs_vs_reference_kernel(ref):
    data = load("stencil_regrid.npz")
    keys = sorted({k.split("/")[0] for k in data if re.fullmatch(r"u\d+/params", k)})
    assert keys
    for key in keys:
        W, H, a, b, dt, dx, dy = data[f"{key}/params"].tolist()
        W, H = int(W), int(H)
        h = tuple(data[f"{key}/S/{part}"] for part in ("begin", "end", "row_offsets", "rows"))
        s, f = _field(h, data[f"{key}/values"])
        want = ref.upwind_f32(s.begin, s.end, s.row_offsets, s.rows, f.interval_cell_offsets, f.values, width=W,
                              height=H, a=a, b=b, dt=dt, dx=dx, dy=dy)
        got = sc.step_upwind_interval(f, width=W, height=H, a=a, b=b, dt=dt, dx=dx, dy=dy)
        _bits_equal(got, want, f"upwind fixture {key}")


@pytest.mark.parametrize("case", ["random", "gauss1024", "gauss_steep"])
def test_gradient_and_tags_bit_exact_vs_reference_kernels(ref, case):
    rng = np.random.default_rng(5)
    if case == "random":
        W, H = 512, 384
        v = rng.uniform(-1, 1, W * H).astype(np.float32)
        thresholds = [0.05, 0.3, 0.7]
    else:
        W = H = 1024
        v = _gauss(W, 0.05 if case == "gauss1024" else 0.01).reshape(-1)
        thresholds = [0.05, 0.05 / 1024, 0.003, 0.011]
    full = sc.full_interval_set(W, H)
    f = sc.create_interval_field(full, fill_value=0.0, dtype=np.float32)
    f.values.copy_(torch.as_tensor(v, device="cuda"))
    want = ref.gradient_flat(f.values, W, H)
    got = rg.gradient_magnitude_interval_field(f, width=W, height=H).values
    _bits_equal(got, want, f"gradient {case}")
    for thr in thresholds:
        t = max(thr, 1e-8)
        want_set = ref.threshold_intervals(want, W, H, t)
        gf = sc.create_interval_field(full, fill_value=0.0, dtype=np.float32)
        gf.values.copy_(want)
        assert_same(rg.intervals_above_threshold_interval_field(gf, width=W, height=H, threshold=t),
                    tuple(x.cpu().numpy() for x in want_set), f"threshold {case} {thr}")
        assert_same(rg.gradient_tag_threshold_interval_field(f, width=W, height=H, threshold=thr),
                    tuple(x.cpu().numpy() for x in want_set), f"gradient tag {case} {thr}")


@pytest.mark.parametrize("ratio", [2, 3, 4])
def test_prolong_restrict_f32_bit_exact_vs_reference_kernels(ref, ratio):
    rng = np.random.default_rng(20 + ratio)
    coarse_h = rand_set(60, 3.0, seed=40 + ratio, max_col=200, row0=0, min_per_row=1)
    coarse = O.ISet(*coarse_h)
    cvals = rng.uniform(-2, 2, int((coarse.end - coarse.begin).sum())).astype(np.float32)
    s, f = _field(coarse_h, cvals)
    # prolongation: the reference kernel fills the fine field on prolong_set(coarse)
    fine_set = O.prolong_set(coarse, ratio)
    fidx = O.coarse_to_fine_indices(coarse, fine_set, ratio)
    fine_off = O.cell_offsets(fine_set)
    want = torch.zeros(int(fine_off[-1]), dtype=torch.float32, device="cuda")
    ref.prolong_f32(_t(O.cell_offsets(coarse)), _t(fine_off), _t(fidx), ratio, f.values, want)
    got = sc.prolong_field(f, ratio)
    assert_same(got.interval_set, fine_set, "prolong set")
    _bits_equal(got.values, want, f"prolong x{ratio}")
    # restriction of a random fine field on that fine set, every reducer
    fvals = rng.uniform(-2, 2, int(fine_off[-1])).astype(np.float32)
    fs, ff = _field(fine_set, fvals)
    cset = O.restrict_set(fine_set, ratio)
    cidx = O.coarse_to_fine_indices(cset, fine_set, ratio)
    coff = O.cell_offsets(cset)
    for code, reducer in enumerate(("mean", "sum", "min", "max")):
        want = torch.zeros(int(coff[-1]), dtype=torch.float32, device="cuda")
        ref.restrict_f32(_t(coff), _t(fine_off), _t(cidx), ratio, code, ff.values, want)
        got = sc.restrict_field(ff, ratio, reducer=reducer)
        _bits_equal(got.values, want, f"restrict x{ratio} {reducer}")


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_binary_ops_match_reference_kernels(ref, seed):
    A = rand_set(300, 5.0, seed=100 + seed, row0=0)
    B = rand_set(300, 5.0, seed=200 + seed, row0=0)
    la, lb = dev_set(A), dev_set(B)
    for mode, make in (("union", sc.make_union), ("intersection", sc.make_intersection),
                       ("difference", sc.make_difference)):
        want = ref.apply_binary((la.begin, la.end, la.row_offsets, la.rows),
                                (lb.begin, lb.end, lb.row_offsets, lb.rows), mode)
        got = sc.evaluate(make(sc.make_input(la), sc.make_input(lb)))
        assert_same(got, tuple(x.cpu().numpy() for x in want), mode)


def test_shapes_expression_matches_reference_kernels(ref):
    from subsetix_b200 import synth

    hosts = synth.shape_operands(1024)
    sets = [dev_set(h) for h in hosts]
    leaves = {n: (s.begin, s.end, s.row_offsets, s.rows) for n, s in zip("ABCDE", sets)}
    spec = ("symmetric_difference", ("difference", ("union", "A", "B"), ("intersection", "C", "D")), "E")
    want = ref.evaluate(spec, leaves)
    A, B, C, D, E = [sc.make_input(s) for s in sets]
    got = sc.evaluate(sc.make_symmetric_difference(sc.make_difference(sc.make_union(A, B),
                                                                      sc.make_intersection(C, D)), E))
    assert_same(got, tuple(x.cpu().numpy() for x in want), "shapes expression")
