"""Morphology, multilevel sets and interval fields on the GPU.

Interval outputs are compared bit for bit (begin, end, row_offsets, rows)
with fixtures generated by the reference itself, and with the oracle on
larger seeded inputs.  Float32 field values must match the reference's bit
for bit; float64 values must match the FP64 oracle bit for bit (both follow
the same operation order without contraction).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.golden_io import error, get_set, has, load
from tests.gpu_util import assert_same, dev_set, host, iset, rand_set

pytestmark = pytest.mark.gpu

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")

MORPH = "morph.npz"
ML = "multilevel.npz"
STENCIL = "stencil_regrid.npz"


def _cases(data, prefix):
    return sorted({k.split("/")[0] for k in data if k.startswith(prefix) and k.split("/")[0][len(prefix):].isdigit()},
                  key=lambda s: int(s[len(prefix):]))


# ---------------------------------------------------------------- morphology

def test_morphology_fixtures(cuda_device):
    data = load(MORPH)
    checked = 0
    for case in _cases(data, "m"):
        S = dev_set(get_set(data, f"{case}/S"))
        for hx, hy in [(0, 0), (2, 0), (0, 1), (1, 1), (3, 2), (1, 4)]:
            assert_same(sc.dilate_interval_set(S, halo_x=hx, halo_y=hy), get_set(data, f"{case}/dilate_{hx}_{hy}"),
                        f"{case} dilate {hx},{hy}")
            checked += 1
        for w, h in [(8, 6), (16, 12), (1, 3)]:
            assert_same(sc.clip_interval_set(S, width=w, height=h), get_set(data, f"{case}/clip_{w}_{h}"),
                        f"{case} clip {w},{h}")
            assert_same(sc.erode_interval_set(S, halo_x=1, halo_y=1, width=w, height=h),
                        get_set(data, f"{case}/erode_{w}_{h}"), f"{case} erode {w},{h}")
            assert_same(sc.ghost_zones(S, halo_x=1, halo_y=1, width=w, height=h),
                        get_set(data, f"{case}/ghost_{w}_{h}"), f"{case} ghost {w},{h}")
            checked += 3
    assert checked >= 60 * 15


def test_morphology_random_rows_256(cuda_device):
    data = load(MORPH)
    A = dev_set(get_set(data, "rows256/A"))
    for hx, hy in [(1, 1), (2, 2), (4, 4), (3, 0)]:
        assert_same(sc.dilate_interval_set(A, halo_x=hx, halo_y=hy), get_set(data, f"rows256/dilate_{hx}_{hy}"))
        assert_same(sc.erode_interval_set(A, halo_x=hx, halo_y=hy, width=256, height=256),
                    get_set(data, f"rows256/erode_{hx}_{hy}"))


@pytest.mark.parametrize("hx,hy", [(1, 1), (2, 4), (0, 6), (3, 9), (5, 0)])
def test_dilate_random_against_oracle(cuda_device, hx, hy):
    h = rand_set(2048, 40.0, seed=hx * 10 + hy, row_stride=3)
    got = sc.dilate_interval_set(dev_set(h), halo_x=hx, halo_y=hy)
    exp = O.dilate(iset(h), hx, hy)
    assert_same(got, exp)


def test_clip_erode_random_against_oracle(cuda_device):
    h = rand_set(1024, 12.0, seed=5, row_stride=1, row0=-50)
    S = dev_set(h)
    W, H = 4000, 900
    assert_same(sc.clip_interval_set(S, width=W, height=H), O.clip(iset(h), W, H))
    assert_same(sc.erode_interval_set(S, 2, 1, width=W, height=H), O.erode(iset(h), 2, 1, width=W, height=H))
    assert_same(sc.ghost_zones(S, 1, 2, width=W, height=H), O.ghost_zones(iset(h), 1, 2, width=W, height=H))


def test_morphology_errors(cuda_device):
    S = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[3])
    with pytest.raises(ValueError):
        sc.dilate_interval_set(S, halo_x=-1)
    with pytest.raises(ValueError):
        sc.clip_interval_set(S, width=0, height=3)
    with pytest.raises(ValueError):
        sc.clip_interval_set(S, width=3, height=-1)
    with pytest.raises(TypeError):
        sc.translate_interval_set(S, dx=1.5)
    with pytest.raises(ValueError):
        sc.interior_for_direction(S, 0, 0)


def _compact(s):
    """Occupied rows with merged intervals (the reference's compaction)."""
    return O.build_from_rows(O.interval_rows(s), s.begin, s.end)


def _translate(s, dx, dy):
    return O.ISet(s.begin + dx, s.end + dx, s.row_offsets.copy(), s.rows + dy)


def test_translate_and_boundaries(cuda_device):
    h = rand_set(256, 6.0, seed=9, row_stride=1)
    S = dev_set(h)
    s = iset(h)
    t = sc.translate_interval_set(S, dx=3, dy=-2)
    assert_same(t, _translate(s, 3, -2))
    interior = _compact(O.intersection(s, _translate(s, -1, 0)))
    assert_same(sc.interior_for_direction(S, 1, 0), interior)
    assert_same(sc.boundary_for_direction(S, 1, 0), _compact(O.difference(s, interior)))
    inner = s
    for dx, dy in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        inner = O.intersection(inner, _translate(s, -dx, -dy))
    assert_same(sc.boundary_layer(S), _compact(O.difference(s, _compact(inner))))


# ---------------------------------------------------------------- multilevel sets

def test_prolong_restrict_set_fixtures(cuda_device):
    data = load(ML)
    for case in _cases(data, "p"):
        S = dev_set(get_set(data, f"{case}/S"))
        for r in (1, 2, 3, 4):
            assert_same(sc.prolong_set(S, r), get_set(data, f"{case}/prolong_{r}"), f"{case} prolong {r}")
            assert_same(sc.restrict_set(S, r), get_set(data, f"{case}/restrict_{r}"), f"{case} restrict {r}")
    S = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[3])
    assert sc.prolong_set(S, 1) is S


@pytest.mark.parametrize("r", [2, 3, 4, 8, 12])
def test_prolong_restrict_random_against_oracle(cuda_device, r):
    h = rand_set(3000, 20.0, seed=r, row_stride=2)
    S = dev_set(h)
    assert_same(sc.prolong_set(S, r), O.prolong_set(iset(h), r))
    assert_same(sc.restrict_set(S, r), O.restrict_set(iset(h), r))
    # restrict(prolong(S)) is S with touching intervals merged
    assert_same(sc.restrict_set(sc.prolong_set(S, r), r), O.restrict_set(O.prolong_set(iset(h), r), r))


# ---------------------------------------------------------------- fields

def _field(h, values, dtype=torch.float32):
    S = dev_set(h)
    f = sc.create_interval_field(S, fill_value=0.0, dtype=np.float32 if dtype == torch.float32 else np.float64)
    f.values.copy_(torch.as_tensor(np.asarray(values), device="cuda").to(dtype))
    return f


def _vals(x):
    return torch.as_tensor(x).cpu().numpy()


def test_field_fixtures(cuda_device):
    data = load(ML)
    n_fine = n_err = 0
    for case in _cases(data, "f"):
        h = get_set(data, f"{case}/S")
        f = _field(h, data[f"{case}/values"])
        for r in (2, 3):
            err = error(data, f"{case}/fine_{r}")
            if err is not None:
                with pytest.raises(ValueError):
                    sc.prolong_field(f, r)
                n_err += 1
                continue
            fine = sc.prolong_field(f, r)
            assert_same(fine.interval_set, get_set(data, f"{case}/fine_{r}"))
            np.testing.assert_array_equal(_vals(fine.values), data[f"{case}/fine_{r}/values"])
            noisy = sc.IntervalField(interval_set=fine.interval_set,
                                     values=torch.as_tensor(data[f"{case}/noisy_{r}"], device="cuda"),
                                     interval_cell_offsets=fine.interval_cell_offsets)
            for red in ("mean", "sum", "min", "max"):
                key = f"{case}/restrict_{r}_{red}"
                if error(data, key) is not None:
                    with pytest.raises(ValueError):
                        sc.restrict_field(noisy, r, reducer=red)
                    continue
                out = sc.restrict_field(noisy, r, reducer=red)
                assert_same(out.interval_set, get_set(data, key))
                assert out.values.dtype == torch.float32
                np.testing.assert_array_equal(_vals(out.values), data[f"{key}/values"], err_msg=key)
            n_fine += 1
    assert n_fine >= 20 and n_err >= 1


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_field_random_against_oracle(cuda_device, dtype):
    rng = np.random.default_rng(3)
    h = rand_set(1500, 10.0, seed=11, row_stride=1, min_per_row=1)
    npd = np.float32 if dtype == torch.float32 else np.float64
    s = iset(h)
    cf = O.create_field(s, 0.0, npd)
    cf.values[...] = rng.standard_normal(cf.values.size).astype(npd)
    f = _field(h, cf.values, dtype)
    for r in (2, 4):
        fine = sc.prolong_field(f, r, dtype=npd)
        exp = O.prolong_field(cf, r, dtype=npd)
        assert_same(fine.interval_set, exp.iset)
        np.testing.assert_array_equal(_vals(fine.values), exp.values)
        noisy_vals = rng.standard_normal(exp.values.size).astype(npd)
        noisy = sc.IntervalField(interval_set=fine.interval_set, values=torch.as_tensor(noisy_vals, device="cuda"),
                                 interval_cell_offsets=fine.interval_cell_offsets)
        for red in ("mean", "sum", "min", "max"):
            got = sc.restrict_field(noisy, r, reducer=red, dtype=npd)
            want = O.restrict_field(O.Field(exp.iset, noisy_vals, exp.offsets), r, red, dtype=npd)
            assert_same(got.interval_set, want.iset)
            np.testing.assert_array_equal(_vals(got.values), want.values, err_msg=red)


def test_restrict_field_misaligned_raises(cuda_device):
    h = rand_set(64, 3.0, seed=2, row_stride=1, min_per_row=1)
    f = _field(h, np.ones(int(np.sum(h[1] - h[0])), np.float32))
    with pytest.raises(ValueError):
        sc.restrict_field(f, 2)
    with pytest.raises(NameError):
        sc.restrict_field(f, 1)


def test_cell_access(cuda_device):
    S = sc.build_interval_set(row_offsets=[0, 2, 3], begin=[0, 6, 1], end=[4, 9, 5])
    f = sc.create_interval_field(S, fill_value=1.5, dtype=np.float32)
    assert f.cell_count == 11
    assert sc.set_cell(f, 0, 7, 4.0)
    assert not sc.set_cell(f, 0, 5, 4.0)
    assert float(sc.get_cell(f, 0, 7)) == 4.0
    assert sc.get_cell(f, 1, 0) is None
    with pytest.raises(IndexError):
        sc.get_cell(f, 5, 0)
    rows = torch.tensor([0, 0, 1, 1, 2, -1], dtype=torch.int32, device="cuda")
    cols = torch.tensor([3, 4, 4, 5, 0, 0], dtype=torch.int32, device="cuda")
    idx = sc.locate_interval_cells(f, rows, cols)
    assert idx.cpu().tolist() == [0, -1, 2, -1, -1, -1]


# ---------------------------------------------------------------- upwind

def test_upwind_fixtures(cuda_device):
    data = load(STENCIL)
    cases = _cases(data, "u")
    assert len(cases) == 15
    for case in cases:
        h = get_set(data, f"{case}/S")
        f = _field(h, data[f"{case}/values"])
        width, height, a, b, dt, dx, dy = data[f"{case}/params"].tolist()
        out = sc.step_upwind_interval(f, width=int(width), height=int(height), a=a, b=b, dt=dt, dx=dx, dy=dy)
        np.testing.assert_array_equal(_vals(out), data[f"{case}/out"], err_msg=case)
        buf = torch.empty_like(f.values)
        res = sc.step_upwind_interval(f, width=int(width), height=int(height), a=a, b=b, dt=dt, dx=dx, dy=dy, out=buf)
        assert res is buf
        np.testing.assert_array_equal(_vals(buf), data[f"{case}/out"])


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_upwind_random_against_oracle(cuda_device, dtype):
    npd = np.float32 if dtype == torch.float32 else np.float64
    rng = np.random.default_rng(7)
    W = H = 1024
    for seed, touching in ((1, False), (2, True)):
        h = rand_set(H, 30.0, seed=seed, row_stride=1, max_col=W, touching=touching, row0=0)
        s = iset(h)
        cf = O.create_field(s, 0.0, npd)
        cf.values[...] = rng.uniform(0, 1, cf.values.size).astype(npd)
        f = _field(h, cf.values, dtype)
        for a, b in ((1.0, 0.5), (-0.3, -0.8)):
            got = sc.step_upwind_interval(f, width=W, height=H, a=a, b=b, dt=0.2 / W, dx=1.0 / W, dy=1.0 / H)
            exp = O.upwind(cf, width=W, height=H, a=a, b=b, dt=0.2 / W, dx=1.0 / W, dy=1.0 / H, dtype=npd)
            np.testing.assert_array_equal(_vals(got), exp)


def test_upwind_rows_out_of_range(cuda_device):
    S = sc.build_interval_set(row_offsets=[0, 1, 2], begin=[0, 0], end=[2, 2], rows=[0, 5])
    f = sc.create_interval_field(S, fill_value=1.0, dtype=np.float32)
    with pytest.raises(ValueError):
        sc.step_upwind_interval(f, width=4, height=4, a=1.0, b=1.0, dt=0.1, dx=1.0, dy=1.0)
    with pytest.raises(ValueError):
        sc.step_upwind_interval(f, width=0, height=4, a=1.0, b=1.0, dt=0.1, dx=1.0, dy=1.0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_upwind_chunked_equals_generic(cuda_device, dtype):
    from subsetix_b200 import _core

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(13)
    cases = [rand_set(700, 25.0, seed=31, row_stride=1, touching=True, row0=0),   # ragged, touching, beyond width
             rand_set(300, 1.0, seed=32, row_stride=2, row0=1),                   # sparse rows, gaps between rows
             (np.zeros(64, np.int32), np.full(64, 5000, np.int32), np.arange(65, dtype=np.int32),
              np.arange(64, dtype=np.int32))]                                     # long single intervals
    shifted = rand_set(400, 12.0, seed=33, row_stride=1, touching=True, row0=0)
    cases.append((shifted[0] - 150, shifted[1] - 150, shifted[2], shifted[3]))    # columns on both sides of 0
    for h in cases:
        S = dev_set(h)
        H = int(h[3].max()) + 2
        W = 300
        b, e, off, rows = (torch.as_tensor(a, device=dev) for a in h)
        coff, cells = _core.cell_offsets(b, e, dev)
        lookup, bad = _core.row_lookup(rows, H, dev)
        assert not bad
        chunk_off, chunks = _core.upwind_plan(rows, off, b, e, coff, lookup, H, dev)
        table = _core.upwind_table(b, e, coff, chunk_off, chunks, cells, dev)
        v = torch.as_tensor(rng.standard_normal(cells), device=dev).to(dtype)
        for a_, b_ in ((0.6, 0.3), (-0.4, -0.9), (0.6, -0.3), (-0.4, 0.9), (0.0, -0.0)):  # every upwind side
            ref = torch.empty_like(v)
            _core.upwind(rows, off, b, e, coff, cells, lookup, v, ref, W, H, a_, b_, 1e-3, 1e-2, 1e-2, False, dev)
            for tab in (None, table):  # neighbour rows searched, then read from the plan's table
                got = torch.full_like(v, float("nan"))
                _core.upwind_chunked(off, b, e, coff, chunk_off, chunks, lookup, v, got, W, H, a_, b_, 1e-3, 1e-2,
                                     1e-2, dev, table=tab)
                assert torch.equal(got, ref), tab is None


def test_upwind_padded_cell_offsets(cuda_device):
    """Values laid out with gaps between intervals take the generic kernel and agree."""
    dev = torch.device("cuda", 0)
    h = rand_set(200, 9.0, seed=41, row_stride=1, touching=True, row0=0)
    S = dev_set(h)
    b, e = h[0].astype(np.int64), h[1].astype(np.int64)
    lens = e - b
    packed = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    padded = np.concatenate([[0], np.cumsum(lens + 3)]).astype(np.int32)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(int(packed[-1])).astype(np.float32)
    vp = np.zeros(int(padded[-1]), np.float32)
    for i in range(lens.size):
        vp[padded[i]:padded[i] + lens[i]] = v[packed[i]:packed[i + 1]]
    kw = dict(width=180, height=202, a=0.5, b=-0.7, dt=1e-3, dx=1e-2, dy=1e-2)
    f = sc.IntervalField(interval_set=S, values=torch.as_tensor(v, device=dev),
                         interval_cell_offsets=torch.as_tensor(packed, device=dev))
    fp = sc.IntervalField(interval_set=S, values=torch.as_tensor(vp, device=dev),
                          interval_cell_offsets=torch.as_tensor(padded, device=dev))
    ref = sc.step_upwind_interval(f, **kw).cpu().numpy()
    got = sc.step_upwind_interval(fp, **kw).cpu().numpy()
    for i in range(lens.size):
        assert np.array_equal(got[padded[i]:padded[i] + lens[i]], ref[packed[i]:packed[i + 1]])


def test_neighbour_table_with_gapped_offsets(cuda_device):
    """The table is exact wherever its byte offsets fit; gaps too wide for a byte are reported, not stored."""
    from subsetix_b200 import _core, _lib

    dev = torch.device("cuda", 0)
    h = rand_set(120, 6.0, seed=42, row_stride=1, touching=True, row0=0)
    b, e, off, rows = (torch.as_tensor(a, device=dev) for a in h)
    lens = (e - b).long()
    H, W = int(h[3].max()) + 2, 200
    lookup, bad = _core.row_lookup(rows, H, dev)
    assert not bad
    rng = np.random.default_rng(6)
    for gap, fits in ((2, True), (400, False)):
        coff = torch.zeros(lens.numel() + 1, dtype=torch.int32, device=dev)
        coff[1:] = torch.cumsum(lens + gap, 0).to(torch.int32)
        cells = int(coff[-1])
        chunk_off, chunks = _core.upwind_plan(rows, off, b, e, coff, lookup, H, dev)
        v = torch.as_tensor(rng.standard_normal(cells).astype(np.float32), device=dev)
        if not fits:
            with pytest.raises(_lib.SubsetixError, match="prefix sum"):
                _core.upwind_table(b, e, coff, chunk_off, chunks, cells, dev)
            continue
        table = _core.upwind_table(b, e, coff, chunk_off, chunks, cells, dev)
        ref = torch.zeros_like(v)
        got = torch.zeros_like(v)
        _core.upwind_chunked(off, b, e, coff, chunk_off, chunks, lookup, v, ref, W, H, 0.5, 0.5, 1e-3, 1e-2, 1e-2, dev)
        _core.upwind_chunked(off, b, e, coff, chunk_off, chunks, lookup, v, got, W, H, 0.5, 0.5, 1e-3, 1e-2, 1e-2, dev,
                             table=table)
        assert torch.equal(got, ref)


# ------------------------------------------------ percentile tagging and level helpers (reference fixtures)

def test_percentile_tagging_fixture(cuda_device):
    from subsetix_b200.subsetix_amr2 import regrid as rg

    data = load("levels.npz")
    for c in range(int(data["tag_count"])):
        grid = data[f"t{c}/data"]
        h, w = grid.shape
        f = sc.create_interval_field(sc.full_interval_set(w, h), fill_value=0.0, dtype=np.float32)
        f.values.copy_(torch.as_tensor(grid.ravel(), device="cuda"))
        for j, frac in enumerate(data[f"t{c}/fracs"].tolist()):
            assert_same(rg.gradient_tag_set(f, width=w, height=h, frac_high=frac), get_set(data, f"t{c}/tag_{j}"),
                        f"t{c} frac {frac}")


def test_level_helpers_fixture(cuda_device):
    from subsetix_b200.subsetix_cupy import multilevel as ml_mod

    data = load("levels.npz")
    for c in range(int(data["hier_count"])):
        ml = ml_mod.MultiLevel2D.create(3, base_ratio=2)
        ml.set_level(0, dev_set(get_set(data, f"h{c}/base")))
        assert_same(ml_mod.prolong_level_sets(ml, 0), get_set(data, f"h{c}/l1"))
        assert_same(ml_mod.prolong_level_sets(ml, 1), get_set(data, f"h{c}/l2"))
        assert_same(ml_mod.covered_by_fine(ml, 0), get_set(data, f"h{c}/covered0"))
        assert_same(ml_mod.coarse_only(ml.get_level(0), ml, 0), get_set(data, f"h{c}/coarse_only0"))
        assert_same(ml_mod.restrict_level_sets(ml, 1), get_set(data, f"h{c}/restricted1"))
        mf = ml_mod.MultiLevelField2D.create_from_geometry(ml, fill_value=0.0, dtype=np.float32)
        mf.get_level_field(0).values.copy_(torch.as_tensor(data[f"h{c}/f0"], device="cuda"))
        if error(data, f"h{c}/fields"):
            with pytest.raises(ValueError):
                ml_mod.prolong_level_field(ml, mf, 0)
                ml_mod.prolong_level_field(ml, mf, 1)
            continue
        np.testing.assert_array_equal(ml_mod.prolong_level_field(ml, mf, 0).values.cpu().numpy(), data[f"h{c}/pf1"])
        np.testing.assert_array_equal(ml_mod.prolong_level_field(ml, mf, 1).values.cpu().numpy(), data[f"h{c}/pf2"])
        mf.get_level_field(2).values.copy_(torch.as_tensor(data[f"h{c}/f2"], device="cuda"))
        for red in ("mean", "max"):
            got = ml_mod.restrict_level_field(ml, mf, 1, reducer=red).values.cpu().numpy()
            np.testing.assert_array_equal(got, data[f"h{c}/rf1_{red}"])
    with pytest.raises(IndexError):
        ml_mod.prolong_level_sets(ml_mod.MultiLevel2D.create(2), 1)
    with pytest.raises(ValueError):
        ml_mod.MultiLevel2D(ratios=[1, 3, 4], levels=[None] * 3).validate()
