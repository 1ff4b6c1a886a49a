"""The fused full-grid AMR engine against AMR2Simulation, the reference's fixtures and the FP64 oracle."""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.golden_io import get_set, load
from tests.gpu_util import assert_same, host

pytestmark = pytest.mark.gpu

amr = pytest.importorskip("subsetix_b200.subsetix_amr2")
from subsetix_b200.subsetix_amr2.fused import FusedTwoLevelAMR  # noqa: E402


def _vals(x):
    return torch.as_tensor(x).cpu().numpy()


def _gauss(res, sigma=0.1, cx=0.5, cy=0.5):
    xs = (np.arange(res) + 0.5) / res
    gx, gy = np.meshgrid(xs, xs)
    return np.exp(-((gx - cx) ** 2 + (gy - cy) ** 2) / (2 * sigma ** 2))


def _square(res):
    sim = amr.AMR2Simulation(amr.SimulationConfig(coarse_resolution=res, velocity=(1.0, 0.5), cfl=0.5))
    sim.initialize_square(squares=[amr.SquareSpec(center=(0.35, 0.4), half_width=(0.15, 0.1))])
    return sim.state.coarse_field.values.reshape(res, res).clone()


@pytest.mark.parametrize("tag", ["sq32", "sq24", "gauss32"])
@pytest.mark.parametrize("graph,fused", [(False, False), (False, True), (True, True), (True, False)])
def test_fused_matches_reference_fixtures(cuda_device, tag, graph, fused):
    data = load("amr.npz")
    res, steps, every, vx, vy, dt = data[f"{tag}/params"].tolist()
    res, steps, every = int(res), int(steps), int(every)
    u0 = _square(res) if tag.startswith("sq") else torch.as_tensor(_gauss(res).astype(np.float32), device="cuda")
    eng = FusedTwoLevelAMR(u0, velocity=(vx, vy), cfl=0.5, refine_threshold=0.05, grading=1, fused=fused)
    assert eng.dt == dt
    np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), data[f"{tag}/fine0"])
    assert_same(eng.refine_set(), get_set(data, f"{tag}/refine0"))
    eng.run(steps, regrid_every=every, graph=graph)
    np.testing.assert_array_equal(_vals(eng.coarse_values).reshape(-1), data[f"{tag}/coarse"])
    np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), data[f"{tag}/fine"])
    assert_same(eng.refine_set(), get_set(data, f"{tag}/refine"))


@pytest.mark.parametrize("mode,pad", [("von_neumann", 2), ("moore", 1), ("moore", 0)])
def test_fused_matches_amr2simulation(cuda_device, mode, pad):
    res, steps, every = 40, 9, 2
    u0 = torch.as_tensor(_gauss(res, 0.08, 0.4, 0.55).astype(np.float32), device="cuda")
    cfg = amr.SimulationConfig(coarse_resolution=res, velocity=(-0.7, 0.4), cfl=0.5, refine_threshold=0.03,
                               grading=pad, grading_mode=mode)
    sim = amr.AMR2Simulation(cfg)
    from subsetix_b200.subsetix_cupy import create_interval_field, full_interval_set

    f = create_interval_field(full_interval_set(res, res), fill_value=0.0, dtype=np.float32)
    f.values.copy_(u0.reshape(-1))
    sim.set_initial_field(f)
    state, _ = sim.run(steps=steps, regrid_every=every)
    eng = FusedTwoLevelAMR(u0, velocity=(-0.7, 0.4), cfl=0.5, refine_threshold=0.03, grading=pad, grading_mode=mode)
    eng.run(steps, regrid_every=every, graph=True)
    np.testing.assert_array_equal(_vals(eng.coarse_values).reshape(-1), _vals(state.coarse_field.values))
    np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), _vals(state.fine_field.values))
    assert_same(eng.refine_set(), host(state.actions.refine_set()))


def test_fused_fp64_matches_oracle(cuda_device):
    res, steps, every = 48, 12, 4
    u0 = _gauss(res, 0.07)
    ref = O.AMR2(res, (1.0, 0.5), cfl=0.5, threshold=0.05, grading_pad=1, dtype=np.float64)
    ref.init(u0)
    ref.run(steps, every)
    for fused in (True, False):
        eng = FusedTwoLevelAMR(torch.as_tensor(u0, device="cuda"), velocity=(1.0, 0.5), cfl=0.5, dtype=torch.float64,
                               fused=fused)
        eng.run(steps, regrid_every=every, graph=True)
        np.testing.assert_array_equal(_vals(eng.coarse_values).reshape(-1), ref.coarse.values)
        np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), ref.fine.values)


def test_fused_batch_equals_single_runs(cuda_device):
    res = 32
    inits = [_gauss(res, s, cx, 0.5).astype(np.float32) for s, cx in ((0.06, 0.3), (0.1, 0.5), (0.08, 0.7))]
    batch = torch.as_tensor(np.stack(inits), device="cuda")
    eng = FusedTwoLevelAMR(batch, velocity=(1.0, 0.5), cfl=0.5)
    eng.run(7, regrid_every=3)
    for i, u0 in enumerate(inits):
        one = FusedTwoLevelAMR(torch.as_tensor(u0, device="cuda"), velocity=(1.0, 0.5), cfl=0.5)
        one.run(7, regrid_every=3, graph=False)
        np.testing.assert_array_equal(_vals(eng.coarse_values[i]), _vals(one.coarse_values[0]))
        np.testing.assert_array_equal(_vals(eng.fine_values[i]), _vals(one.fine_values[0]))


def test_fused_fp32_error_and_mass(cuda_device):
    res, steps, every = 128, 40, 10
    u0 = _gauss(res, 0.05)
    e64 = FusedTwoLevelAMR(torch.as_tensor(u0, device="cuda"), velocity=(1.0, 0.5), cfl=0.5, dtype=torch.float64)
    e32 = FusedTwoLevelAMR(torch.as_tensor(u0.astype(np.float32), device="cuda"), velocity=(1.0, 0.5), cfl=0.5)
    m0 = float(e64.mass()[0])
    e64.run(steps, every)
    e32.run(steps, every)
    a = _vals(e32.fine_values).astype(np.float64)
    b = _vals(e64.fine_values)
    rel_l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel_l2 <= 1e-5, rel_l2
    m64, m32 = float(e64.mass()[0]), float(e32.mass()[0])
    assert abs(m32 - m64) <= 1e-5 * abs(m64)
    assert abs(m64 - m0) <= 1e-2 * abs(m0)  # zero-exterior upwind loses mass only at the boundary
    assert abs(float(e64.restriction_defect()[0])) <= 1e-12
    assert abs(float(e32.restriction_defect()[0])) <= 1e-5 * abs(m32)


def test_batched_uneven_sets_against_oracle(cuda_device):
    from subsetix_b200 import synth
    from subsetix_b200.batch import SetBatch, batched_binary, batched_upwind
    from tests.gpu_util import dev_set, iset

    sides, sets_a = synth.batched_uneven_sets(count=24, seed=3, side_hi=1024)
    _, sets_b = synth.batched_uneven_sets(count=24, seed=4, side_hi=1024)
    A = SetBatch.from_sets([dev_set(h) for h in sets_a], sides)
    B = SetBatch.from_sets([dev_set(h) for h in sets_b], sides)
    uni = batched_binary(A, B, "union").split()
    inter = batched_binary(A, B, "intersection").split()
    for i in range(len(sides)):
        assert_same(uni[i], O.union(iset(sets_a[i]), iset(sets_b[i])), f"union {i}")
        assert_same(inter[i], O.intersection(iset(sets_a[i]), iset(sets_b[i])), f"intersection {i}")
    # one FP32 upwind step of every set's field in one launch
    rng = np.random.default_rng(1)
    fields, values = [], []
    for h, side in zip(sets_a, sides):
        s = iset(h)
        f = O.create_field(s, 0.0, np.float32)
        f.values[...] = rng.uniform(0, 1, f.values.size).astype(np.float32)
        fields.append((f, side))
        values.append(f.values)
    vals = torch.as_tensor(np.concatenate(values), device="cuda")
    W = max(sides)
    got = _vals(batched_upwind(A, vals, width=W, a=1.0, b=-0.5, dt=1e-4, dx=1e-3, dy=1e-3))
    pos = 0
    for f, side in fields:
        exp = O.upwind(f, width=side, height=side, a=1.0, b=-0.5, dt=1e-4, dx=1e-3, dy=1e-3)
        np.testing.assert_array_equal(got[pos:pos + exp.size], exp)
        pos += exp.size


@pytest.mark.parametrize("velocity", [(0.9, -0.4), (-0.6, -0.8), (0.5, 0.7), (-0.8, 0.3)])  # every upwind side
@pytest.mark.parametrize("res", [32, 40])
def test_power_of_two_spacing_matches_division(cuda_device, res, velocity):
    # res 32 has power-of-two spacings (multiplication by the exact reciprocal),
    # res 40 does not (division); both must equal the FP64 oracle and AMR2Simulation
    u0 = _gauss(res, 0.08)
    ref = O.AMR2(res, velocity, cfl=0.5, threshold=0.05, grading_pad=1, dtype=np.float64)
    ref.init(u0)
    ref.run(6, 3)
    eng = FusedTwoLevelAMR(torch.as_tensor(u0, device="cuda"), velocity=velocity, cfl=0.5, dtype=torch.float64)
    eng.run(6, regrid_every=3)
    np.testing.assert_array_equal(_vals(eng.fine_values).reshape(-1), ref.fine.values)


@pytest.mark.parametrize("velocity", [(0.8, -0.6), (-0.5, -0.7)])
@pytest.mark.parametrize("res", [40, 70, 300])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_fused_step_any_width(cuda_device, res, dtype, velocity):
    # widths that leave partial warps and blocks: the one-kernel step equals the separate kernels
    u0 = torch.as_tensor(_gauss(res, 0.07), device="cuda")
    runs = []
    for fused in (True, False):
        eng = FusedTwoLevelAMR(u0, velocity=velocity, cfl=0.5, refine_threshold=0.05 / res, grading=1,
                               dtype=dtype, fused=fused)
        eng.run(9, regrid_every=4, graph=False)
        runs.append(eng)
    for lvl in ("coarse_values", "fine_values"):
        assert torch.equal(getattr(runs[0], lvl), getattr(runs[1], lvl)), lvl



def test_batched_upwind_per_set_spacing_and_graph_step(cuda_device):
    """Uneven batched sets, every set with dx = 1/side and its own CFL time step, against the oracle per set;
    the graph-captured BatchStep equals the direct calls."""
    from subsetix_b200 import synth
    from subsetix_b200.batch import BatchStep, SetBatch, batched_binary, batched_upwind
    from tests.gpu_util import dev_set, iset

    sides, sets_a = synth.batched_uneven_sets(count=20, seed=3, side_hi=700)
    _, sets_b = synth.batched_uneven_sets(count=20, seed=4, side_hi=700)
    A = SetBatch.from_sets([dev_set(h) for h in sets_a], sides)
    B = SetBatch.from_sets([dev_set(h) for h in sets_b], sides)
    rng = np.random.default_rng(11)
    fields, values = [], []
    for h in sets_a:
        f = O.create_field(iset(h), 0.0, np.float32)
        f.values[...] = rng.uniform(0, 1, f.values.size).astype(np.float32)
        fields.append(f)
        values.append(f.values)
    vals = torch.as_tensor(np.concatenate(values), device="cuda")
    dx = [1.0 / s for s in sides]
    dt = [0.5 / (1.0 / d + 0.5 / d) for d in dx]
    got = _vals(batched_upwind(A, vals, width=sides, a=1.0, b=0.5, dt=dt, dx=dx, dy=dx))
    pos = 0
    for f, side, h, t in zip(fields, sides, dx, dt):
        exp = O.upwind(f, width=side, height=side, a=1.0, b=0.5, dt=t, dx=h, dy=h)
        np.testing.assert_array_equal(got[pos:pos + exp.size], exp)
        pos += exp.size
    step = BatchStep(A, B, vals, width=sides, a=1.0, b=0.5, dt=dt, dx=dx, dy=dx)
    step()
    g = step.graph()
    step.out.zero_()
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_vals(step.out), got)
    for mine, ref in ((step.union(), batched_binary(A, B, "union")),
                      (step.intersection(), batched_binary(A, B, "intersection"))):
        for x, y in zip(mine.split(), ref.split()):
            assert_same(x, tuple(t.cpu().numpy() for t in (y.begin, y.end, y.row_offsets, y.rows)))


def test_batched_upwind_at_full_size_equals_per_set_calls(cuda_device):
    """The banded batch step on the benchmark's 256 uneven sets (238 M cells, dx = 1/side and a CFL time step per
    set) equals every set's own step_upwind_interval call bit for bit; that per-set path is the one checked against
    the oracle and the reference's kernels at smaller sizes."""
    from subsetix_b200 import synth
    from subsetix_b200.batch import SetBatch, batched_upwind
    from subsetix_b200.subsetix_cupy import create_interval_field, step_upwind_interval
    from subsetix_b200.subsetix_cupy.expressions import IntervalSet

    dev = torch.device("cuda", 0)
    sides, hosts = synth.batched_uneven_sets(count=256, seed=3)
    A = SetBatch.from_sets([IntervalSet._trusted(*(torch.as_tensor(x, device=dev) for x in h)) for h in hosts], sides)
    n = A.stencil_plan().cells
    assert n > 200_000_000
    vals = torch.rand(n, device=dev, generator=torch.Generator(device=dev).manual_seed(5))
    dx = [1.0 / s for s in sides]
    dt = [0.5 / (1.5 / h) for h in dx]
    got = batched_upwind(A, vals, width=sides, a=1.0, b=0.5, dt=dt, dx=dx, dy=dx)
    pos = 0
    for s, side, h, t in zip(A.split(), sides, dx, dt):
        f = create_interval_field(s, fill_value=0.0, dtype=np.float32)
        cells = int(f.values.numel())
        f.values.copy_(vals[pos:pos + cells])
        want = step_upwind_interval(f, width=side, height=side, a=1.0, b=0.5, dt=t, dx=h, dy=h)
        assert torch.equal(got[pos:pos + cells], want), side
        pos += cells
    assert pos == n


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_fused_step_at_full_size_equals_separate_kernels(cuda_device, dtype):
    """The benchmark's 1024^2 run with the physical threshold (part of the grid refined): the one-kernel step,
    which updates fine blocks only under refined cells, equals the separate upwind and synchronisation kernels."""
    res = 1024
    u0 = torch.as_tensor(_gauss(res, 0.05), device="cuda")
    runs = []
    for fused in (True, False):
        eng = FusedTwoLevelAMR(u0, velocity=(1.0, 0.5), cfl=0.5, refine_threshold=0.05 / res, grading=1, dtype=dtype,
                               fused=fused)
        eng.run(30, regrid_every=10)
        runs.append(eng)
    assert bool((runs[0].actions != 0).any())
    for lvl in ("coarse_values", "fine_values"):
        assert torch.equal(getattr(runs[0], lvl), getattr(runs[1], lvl)), lvl
