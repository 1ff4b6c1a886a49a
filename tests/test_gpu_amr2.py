"""Two-level AMR on the GPU: regrid, subset transfers, synchronisation and the drivers.

Fixtures come from the reference itself (``tests/golden/make_golden.py``).
Interval outputs must match bit for bit; float32 field values too (the
kernels follow the reference's operation order without contraction).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.golden_io import get_set, load
from tests.gpu_util import assert_same, dev_set, iset, rand_set

pytestmark = pytest.mark.gpu

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")
amr = pytest.importorskip("subsetix_b200.subsetix_amr2")

from subsetix_b200.subsetix_amr2 import fields as F  # noqa: E402
from subsetix_b200.subsetix_amr2 import regrid as RG  # noqa: E402


def _vals(x):
    return torch.as_tensor(x).cpu().numpy()


def _grid_field(data):
    h, w = data.shape
    f = sc.create_interval_field(sc.full_interval_set(w, h), fill_value=0.0, dtype=np.float32)
    f.values.copy_(torch.as_tensor(data.reshape(-1), device="cuda"))
    return f


def test_regrid_fixtures(cuda_device):
    data = load("stencil_regrid.npz")
    n = int(data["regrid_count"])
    assert n == 9
    for g in range(n):
        key = f"g{g}"
        width, height, thr = data[f"{key}/params"].tolist()
        width, height = int(width), int(height)
        f = _grid_field(data[f"{key}/data"])
        grad = RG.gradient_magnitude_interval_field(f, width=width, height=height)
        np.testing.assert_array_equal(_vals(grad.values), data[f"{key}/grad"])
        tags = RG.gradient_tag_threshold_interval_field(f, width=width, height=height, threshold=thr)
        assert_same(tags, get_set(data, f"{key}/tags"), key)
        assert_same(amr.gradient_tag_threshold_set(f, width=width, height=height, threshold=thr),
                    get_set(data, f"{key}/tset"), key)
        for pad, mode in [(1, "von_neumann"), (1, "moore"), (2, "von_neumann"), (0, "moore")]:
            got = amr.enforce_two_level_grading_set(tags, padding=pad, mode=mode, width=width, height=height)
            assert_same(got, get_set(data, f"{key}/grade_{pad}_{mode}"), f"{key} grade {pad} {mode}")


def test_threshold_rle_large_against_oracle(cuda_device):
    rng = np.random.default_rng(4)
    for w, h in ((4096, 512), (1000, 333), (31, 7), (1, 5)):
        d = rng.uniform(0, 1, size=(h, w)).astype(np.float32)
        d = np.where(rng.uniform(size=(h, w)) < 0.5, 0.0, d).astype(np.float32)
        f = _grid_field(d)
        for thr in (0.05, 0.7):
            got = RG.intervals_above_threshold_interval_field(f, width=w, height=h, threshold=thr)
            assert_same(got, O.threshold_intervals(d.reshape(-1), w, h, thr))
            got = RG.gradient_tag_threshold_interval_field(f, width=w, height=h, threshold=thr)
            assert_same(got, O.gradient_tag_threshold(d.reshape(-1), w, h, thr))


def test_regrid_errors(cuda_device):
    f = _grid_field(np.zeros((4, 4), np.float32))
    with pytest.raises(ValueError):
        RG.gradient_magnitude_interval_field(f, width=5, height=4)
    with pytest.raises(ValueError):
        amr.enforce_two_level_grading_set(sc.full_interval_set(4, 4), padding=1, mode="diag", width=4, height=4)
    s = sc.full_interval_set(4, 4)
    assert amr.enforce_two_level_grading_set(s, padding=0, width=4, height=4) is s


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.int8, np.int32, np.int64, np.bool_])
def test_subset_gather_scatter_against_oracle(cuda_device, dtype):
    rng = np.random.default_rng(5)
    sup_h = rand_set(400, 6.0, seed=21, row_stride=1, row0=0)
    sup = O.ISet(*sup_h)
    sub = O.intersection(sup, O.ISet(*rand_set(300, 8.0, seed=22, row_stride=1, row0=50)))
    sub = O.ISet(sub.begin, sub.end, sub.row_offsets, sub.rows)
    vals = (rng.integers(-100, 100, size=int(O.cell_offsets(sup)[-1])) if dtype != np.bool_
            else rng.integers(0, 2, size=int(O.cell_offsets(sup)[-1]))).astype(dtype)
    sf = O.Field(sup, vals.copy(), O.cell_offsets(sup))
    exp = O.gather_subset(sf, sub)
    S = dev_set(sup_h)
    field = sc.create_interval_field(S, fill_value=0, dtype=dtype)
    field.values.copy_(torch.as_tensor(vals, device="cuda"))
    got = F.gather_interval_subset(field, dev_set((sub.begin, sub.end, sub.row_offsets, sub.rows)))
    np.testing.assert_array_equal(_vals(got.values), exp.values)
    # scatter a modified subset back
    newv = (exp.values * 2 + 1).astype(dtype) if dtype != np.bool_ else ~exp.values
    O.scatter_subset(sf, O.Field(exp.iset, newv, exp.offsets))
    got.values.copy_(torch.as_tensor(newv, device="cuda"))
    F.scatter_interval_subset(field, got)
    np.testing.assert_array_equal(_vals(field.values), sf.values)


def test_subset_missing_row_raises(cuda_device):
    sup = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[4], rows=[3])
    sub = sc.build_interval_set(row_offsets=[0, 1], begin=[0], end=[2], rows=[5])
    f = sc.create_interval_field(sup, fill_value=1.0, dtype=np.float32)
    with pytest.raises(ValueError):
        F.gather_interval_subset(f, sub)


def test_value_intervals_against_oracle(cuda_device):
    rng = np.random.default_rng(6)
    h = rand_set(500, 7.0, seed=23, row_stride=1, row0=0)
    s = O.ISet(*h)
    vals = rng.integers(-1, 2, size=int(O.cell_offsets(s)[-1])).astype(np.int8)
    field = sc.create_interval_field(dev_set(h), fill_value=0, dtype=np.int8)
    field.values.copy_(torch.as_tensor(vals, device="cuda"))
    for target in (1, 0, -1, 5):
        got = F._interval_field_value_intervals(field, target)
        assert_same(got, O.value_intervals(O.Field(s, vals, O.cell_offsets(s)), target))


def test_synchronize_against_oracle(cuda_device):
    rng = np.random.default_rng(8)
    W = H = 96
    r = 2
    tags = O.threshold_intervals(rng.uniform(0, 1, W * H).astype(np.float32), W, H, 0.8)
    refine = O.grading(tags, 1, "von_neumann", width=W, height=H)
    for dtype in (np.float32, np.float64):
        acts = O.Actions(W, H, r)
        acts.set_from(refine)
        cvals = rng.standard_normal(W * H).astype(dtype)
        fvals = rng.standard_normal(W * H * r * r).astype(dtype)
        cdom, fdom = O.full(W, H), O.full(W * r, H * r)
        cf = O.Field(cdom, cvals.copy(), O.cell_offsets(cdom))
        ff = O.Field(fdom, fvals.copy(), O.cell_offsets(fdom))
        O.synchronize(cf, ff, acts, r, dtype)
        actions = F.ActionField.full_grid(H, W, r)
        actions.set_from_interval_set(dev_set(refine))
        c = sc.create_interval_field(sc.full_interval_set(W, H), fill_value=0.0, dtype=dtype)
        c.values.copy_(torch.as_tensor(cvals, device="cuda"))
        f = sc.create_interval_field(sc.full_interval_set(W * r, H * r), fill_value=0.0, dtype=dtype)
        f.values.copy_(torch.as_tensor(fvals, device="cuda"))
        c2, f2 = amr.synchronize_interval_fields(c, f, actions, ratio=r, copy=True)
        np.testing.assert_array_equal(_vals(c2.values), cf.values)
        np.testing.assert_array_equal(_vals(f2.values), ff.values)
        np.testing.assert_array_equal(_vals(c.values), cvals)  # copy=True leaves inputs alone
        assert_same(actions.refine_set(), refine)
        assert_same(actions.fine_set(), O.prolong_set(refine, r))
        assert_same(actions.coarse_only_set(), acts.coarse_only())


def _gauss(res):
    xs = (np.arange(res) + 0.5) / res
    gx, gy = np.meshgrid(xs, xs)
    return np.exp(-((gx - 0.5) ** 2 + (gy - 0.5) ** 2) / (2 * 0.1 ** 2)).astype(np.float32)


@pytest.mark.parametrize("tag", ["sq32", "sq24", "gauss32"])
def test_amr2_simulation_fixtures(cuda_device, tag):
    data = load("amr.npz")
    res, steps, every, vx, vy, dt = data[f"{tag}/params"].tolist()
    res, steps, every = int(res), int(steps), int(every)
    config = amr.SimulationConfig(coarse_resolution=res, velocity=(vx, vy), cfl=0.5, refine_threshold=0.05, grading=1)
    sim = amr.AMR2Simulation(config)
    assert sim.dt == dt
    if tag.startswith("sq"):
        sim.initialize_square(squares=[amr.SquareSpec(center=(0.35, 0.4), half_width=(0.15, 0.1))])
    else:
        f = _grid_field(_gauss(res))
        sim.set_initial_field(f)
    st = sim.state
    np.testing.assert_array_equal(_vals(st.coarse_field.values), data[f"{tag}/coarse0"])
    np.testing.assert_array_equal(_vals(st.fine_field.values), data[f"{tag}/fine0"])
    assert_same(st.actions.refine_set(), get_set(data, f"{tag}/refine0"))
    seen = []
    state, stats = sim.run(steps=steps, regrid_every=every, listeners=[lambda s, t: seen.append(t.step)])
    assert seen == list(range(steps + 1)) and stats.step == steps
    np.testing.assert_array_equal(_vals(state.coarse_field.values), data[f"{tag}/coarse"])
    np.testing.assert_array_equal(_vals(state.fine_field.values), data[f"{tag}/fine"])
    assert_same(state.actions.refine_set(), get_set(data, f"{tag}/refine"))
    assert_same(state.geometry.coarse_only, get_set(data, f"{tag}/coarse_only"))
    assert_same(state.geometry.fine, get_set(data, f"{tag}/fine_set"))


def test_amr2_fp64_against_oracle(cuda_device):
    res, steps, every = 32, 6, 3
    u0 = _gauss(res).astype(np.float64)
    ref = O.AMR2(res, (1.0, 0.5), cfl=0.5, threshold=0.05, grading_pad=1, dtype=np.float64)
    ref.init(u0)
    ref.run(steps, every)
    sim = amr.AMR2Simulation(amr.SimulationConfig(coarse_resolution=res, velocity=(1.0, 0.5), cfl=0.5))
    f = sc.create_interval_field(sc.full_interval_set(res, res), fill_value=0.0, dtype=np.float64)
    f.values.copy_(torch.as_tensor(u0.reshape(-1), device="cuda"))
    sim.set_initial_field(f)
    state, _ = sim.run(steps=steps, regrid_every=every)
    assert state.coarse_field.values.dtype == torch.float64
    np.testing.assert_array_equal(_vals(state.coarse_field.values), ref.coarse.values)
    np.testing.assert_array_equal(_vals(state.fine_field.values), ref.fine.values)


def test_runner_fixture(cuda_device):
    data = load("amr.npz")

    def init_fn(f):
        f.coarse_field.values.fill_(1.0)
        f.fine_field.values.fill_(1.0)

    field = amr.run_two_level_simulation(amr.SimulationArgs(velocity=(0.1, 0.0), cfl=0.5, t0=0.0, tf=0.01,
                                                            min_level=2, max_level=3, refine_threshold=0.05,
                                                            grading=1), init_fn)
    np.testing.assert_array_equal(_vals(field.coarse_field.values), data["runner/coarse"])
    np.testing.assert_array_equal(_vals(field.fine_field.values), data["runner/fine"])


def test_mass_integral_matches_compensated_sum(cuda_device):
    from subsetix_b200 import _core

    rng = np.random.default_rng(9)
    for dtype in (np.float32, np.float64):
        v = (rng.standard_normal(3_000_001) * 1e3).astype(dtype)
        got = _core.mass_integral(torch.as_tensor(v, device="cuda"), 0.25, torch.device("cuda", 0))
        exp = O.mass_kahan(v, 0.25)
        assert abs(float(got.item()) - exp) <= 1e-13 * abs(exp) + 1e-300


def test_vtk_export(cuda_device, tmp_path):
    sim = amr.AMR2Simulation(amr.SimulationConfig(coarse_resolution=16, velocity=(1.0, 0.5), cfl=0.5))
    sim.initialize_square()
    exporter = amr.TwoLevelVTKExporter(str(tmp_path), every=1)
    sim.run(steps=1, exporters=[exporter])
    files = sorted(p.name for p in tmp_path.iterdir())
    assert files == ["amr2_mesh_step0000.vtu", "amr2_mesh_step0001.vtu"]
    raw = (tmp_path / files[0]).read_bytes()
    assert b"UnstructuredGrid" in raw and b'Name="ghost_mask"' in raw and b'Name="u"' in raw
    mesh = _read_vtu(tmp_path / files[0])
    state = sim.state
    # every coarse-only cell, ghost band included, appears once on level 0 with its value
    n0 = int((mesh["level"] == 0).sum())
    co = state.geometry.coarse_only
    assert n0 == int((co.end - co.begin).sum())
    assert mesh["points"].shape == (4 * mesh["u"].size, 3)


def _read_vtu(path):
    """The appended arrays of a raw-appended .vtu, by name (the layout the reference writes)."""
    import re

    raw = path.read_bytes()
    head, _, data = raw.partition(b"<AppendedData encoding=\"raw\">")
    data = data[data.index(b"_") + 1:]
    out = {}
    for m in re.finditer(rb'<DataArray type="(\w+)"(?: Name="(\w+)")?[^>]*offset="(\d+)"', head):
        typ, name, off = m.group(1).decode(), (m.group(2) or b"points").decode(), int(m.group(3))
        n = int(np.frombuffer(data[off:off + 8], "<u8")[0])
        dt = {"Int32": "<i4", "Float32": "<f4", "UInt8": "u1"}[typ]
        arr = np.frombuffer(data[off + 8:off + 8 + n], dt)
        out[name] = arr.reshape(-1, 3) if name == "points" else arr
    return out


def test_vtk_quads_device_equal_host(cuda_device, tmp_path):
    """Device quad assembly of an interval field equals the host assembly of the same cells as a mask."""
    from subsetix_b200.subsetix_cupy import export_vtk as vtk

    rng = np.random.default_rng(8)
    grid = rng.uniform(-1, 1, (24, 40)).astype(np.float32)
    f = _grid_field(grid)
    a = vtk.interval_field_quads(f, 1, 0.125, 0.25, 0.5, -1.0, 0)
    b = vtk.mask_quads(np.ones_like(grid, dtype=bool), grid, 1, 0.125, 0.25, 0.5, -1.0)
    np.testing.assert_array_equal(a.points, b.points)
    np.testing.assert_array_equal(a.values, b.values)
    vtk.write_unstructured_quads_vtu(str(tmp_path / "m.vtu"), [(f, 1, 0.125, 0.25, 0.5, -1.0, 1)])
    mesh = _read_vtu(tmp_path / "m.vtu")
    np.testing.assert_array_equal(mesh["u"], grid.ravel())
    assert set(mesh["ghost_mask"].tolist()) == {1} and set(mesh["types"].tolist()) == {9}


def test_amr2_simulation_128_physical_threshold(cuda_device):
    """The two-level AMR loop at 128^2 with the physical threshold 0.05 dx (12 % of the cells refined), 40 steps,
    regrid every 10: the drop-in AMR2Simulation and the fused engine against the reference's own run."""
    from subsetix_b200.subsetix_amr2.fused import FusedTwoLevelAMR

    data = load("amr_large.npz")
    res, steps, every, va, vb, dt, thr = data["g128/params"].tolist()
    res, steps, every = int(res), int(steps), int(every)
    u0 = data["g128/u0"]
    sim = amr.AMR2Simulation(amr.SimulationConfig(coarse_resolution=res, velocity=(va, vb), cfl=0.5,
                                                  refine_threshold=thr, grading=1))
    assert sim.dt == dt
    sim.set_initial_field(_grid_field(u0))
    assert_same(sim.state.actions.refine_set(), get_set(data, "g128/refine0"))
    state, _ = sim.run(steps=steps, regrid_every=every)
    np.testing.assert_array_equal(_vals(state.coarse_field.values), data["g128/coarse"])
    np.testing.assert_array_equal(_vals(state.fine_field.values), data["g128/fine"])
    assert_same(state.actions.refine_set(), get_set(data, "g128/refine"))
    assert_same(state.geometry.coarse_only, get_set(data, "g128/coarse_only"))
    eng = FusedTwoLevelAMR(torch.as_tensor(u0, device="cuda"), velocity=(va, vb), cfl=0.5, refine_threshold=thr)
    eng.run(steps, regrid_every=every)
    np.testing.assert_array_equal(_vals(eng.coarse_values).reshape(-1), data["g128/coarse"])
    np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), data["g128/fine"])
