"""The adjoint upwind kernel and the differentiable multi-step advection.

Checks: the transpose identity <M v, w> = <v, M^T w> in FP64; the velocity
gradient against central differences; the gradient of a multi-level
advection loss against FP64 central finite differences on seeded
directions; checkpoint spacing does not change the gradient; FP32 against
FP64.
"""

import numpy as np
import pytest
import torch

from subsetix_b200 import synth
from tests.gpu_util import dev_set, rand_set

pytestmark = pytest.mark.gpu

adj = pytest.importorskip("subsetix_b200.adjoint")


def _level(h, width, height):
    return adj.Level(dev_set(h), width, height, 1.0 / width, 1.0 / height)


def _levels():
    """Nested three-level geometry: a full base grid, and disks at x2 and x4."""
    base = 64
    full = (np.zeros(base, np.int32), np.full(base, base, np.int32), np.arange(base + 1, dtype=np.int32),
            np.arange(base, dtype=np.int32))
    l1 = synth.disk_rows(2 * base, 0.3 * 2 * base)
    l2 = synth.disk_rows(4 * base, 0.15 * 4 * base)
    return [_level(full, base, base), _level(l1, 2 * base, 2 * base), _level(l2, 4 * base, 4 * base)]


@pytest.mark.parametrize("a,b", [(0.7, 0.4), (-0.5, 0.9), (0.3, -0.8), (-1.0, -0.2)])
@pytest.mark.parametrize("touching", [False, True])
def test_adjoint_transpose_identity(cuda_device, a, b, touching):
    h = rand_set(300, 8.0, seed=5, row_stride=1, max_col=280, touching=touching, row0=0)
    lvl = _level(h, 280, 300)
    rng = np.random.default_rng(0)
    n = lvl.cells
    v = torch.as_tensor(rng.standard_normal(n), device="cuda")
    w = torch.as_tensor(rng.standard_normal(n), device="cuda")
    dt = 1e-3
    mv = lvl.step(v, torch.empty_like(v), a, b, dt)
    g = torch.zeros(2, dtype=torch.float64, device="cuda")
    mtw = lvl.adjoint(w, v, a, b, dt, g)
    lhs = float(torch.dot(mv, w))
    rhs = float(torch.dot(v, mtw))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)
    # dL/da for L = <M(a) v, w>: M is affine in a for a fixed sign, so central differences are exact
    eps = 1e-3 * abs(a)
    lp = float(torch.dot(lvl.step(v, torch.empty_like(v), a + eps, b, dt), w))
    lm = float(torch.dot(lvl.step(v, torch.empty_like(v), a - eps, b, dt), w))
    assert abs(float(g[0]) - (lp - lm) / (2 * eps)) <= 1e-8 * max(abs(float(g[0])), 1.0)
    eps = 1e-3 * abs(b)
    lp = float(torch.dot(lvl.step(v, torch.empty_like(v), a, b + eps, dt), w))
    lm = float(torch.dot(lvl.step(v, torch.empty_like(v), a, b - eps, dt), w))
    assert abs(float(g[1]) - (lp - lm) / (2 * eps)) <= 1e-8 * max(abs(float(g[1])), 1.0)


def _gauss_on(lvl, cx, cy, sigma, dtype):
    s = lvl.interval_set
    b = s.begin.cpu().numpy()
    e = s.end.cpu().numpy()
    off = s.row_offsets.cpu().numpy()
    rows = s.rows.cpu().numpy()
    xs, ys = [], []
    for k, r in enumerate(rows):
        for i in range(off[k], off[k + 1]):
            x = np.arange(b[i], e[i])
            xs.append(x)
            ys.append(np.full(x.size, r))
    x = (np.concatenate(xs) + 0.5) / lvl.width
    y = (np.concatenate(ys) + 0.5) / lvl.height
    return torch.as_tensor(np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sigma ** 2)), dtype=dtype, device="cuda")


def _loss(levels, vel, u0, targets, dt, steps, every):
    uT = adj.advect(vel, levels, u0, dt=dt, steps=steps, checkpoint_every=every)
    return sum(0.5 * torch.sum((u - t) ** 2) for u, t in zip(uT, targets))


def test_advect_gradient_against_central_differences(cuda_device):
    levels = _levels()
    steps, every = 12, 5
    vel0 = torch.tensor([1.0, 0.5], dtype=torch.float64, device="cuda")
    dt = 0.5 / (1.0 / levels[-1].dx + 0.5 / levels[-1].dy)
    u0 = [_gauss_on(l, 0.5, 0.5, 0.1, torch.float64) for l in levels]
    targets = [_gauss_on(l, 0.53, 0.52, 0.1, torch.float64) for l in levels]
    vel = vel0.clone().requires_grad_(True)
    u0g = [u.clone().requires_grad_(True) for u in u0]
    loss = _loss(levels, vel, u0g, targets, dt, steps, every)
    loss.backward()
    rng = np.random.default_rng(42)
    eps = 1e-6
    worst = 0.0
    for _ in range(8):
        dv = torch.as_tensor(rng.standard_normal(2), device="cuda")
        du = [torch.as_tensor(rng.standard_normal(u.numel()), device="cuda") for u in u0]
        dirder = float(torch.dot(vel.grad, dv)) + sum(float(torch.dot(g.grad, d)) for g, d in zip(u0g, du))
        with torch.no_grad():
            lp = _loss(levels, vel0 + eps * dv, [u + eps * d for u, d in zip(u0, du)], targets, dt, steps, every)
            lm = _loss(levels, vel0 - eps * dv, [u - eps * d for u, d in zip(u0, du)], targets, dt, steps, every)
        fd = (float(lp) - float(lm)) / (2 * eps)
        worst = max(worst, abs(dirder - fd) / max(abs(fd), 1e-12))
    assert worst < 1e-6, worst


def test_checkpoint_spacing_and_fp32(cuda_device):
    levels = _levels()
    steps = 9
    dt = 0.5 / (1.0 / levels[-1].dx + 0.5 / levels[-1].dy)
    grads = {}
    for dtype in (torch.float64, torch.float32):
        for every in (1, 4, 9):
            vel = torch.tensor([0.8, -0.6], dtype=torch.float64, device="cuda", requires_grad=True)
            u0 = [_gauss_on(l, 0.45, 0.5, 0.12, dtype).requires_grad_(True) for l in levels]
            targets = [_gauss_on(l, 0.47, 0.49, 0.12, dtype) for l in levels]
            _loss(levels, vel, u0, targets, dt, steps, every).backward()
            grads[(dtype, every)] = (vel.grad.clone(), [u.grad.double().clone() for u in u0])
    for dtype in (torch.float64, torch.float32):
        ref_v, ref_u = grads[(dtype, 9)]
        for every in (1, 4):
            v, us = grads[(dtype, every)]
            assert torch.equal(v, ref_v)
            for a, b in zip(us, ref_u):
                assert torch.equal(a, b)
    v64, u64 = grads[(torch.float64, 9)]
    v32, u32 = grads[(torch.float32, 9)]
    assert float(torch.linalg.vector_norm(v32 - v64) / torch.linalg.vector_norm(v64)) < 1e-4
    for a, b in zip(u32, u64):
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) < 1e-5


@pytest.mark.parametrize("a,b", [(0.7, 0.4), (-0.5, -0.9), (0.7, -0.4), (-0.5, 0.9)])  # every upwind side
@pytest.mark.parametrize("table", [True, False])
def test_chunked_adjoint_equals_generic(cuda_device, a, b, table):
    from subsetix_b200 import _lib
    from subsetix_b200._runtime import ptr, stream_handle

    h = rand_set(400, 12.0, seed=8, row_stride=1, max_col=350, touching=True, row0=0)
    lvl = _level(h, 330, 400)      # some cells lie beyond the width
    assert lvl.chunk_off is not None and lvl.table is not None
    if not table:
        lvl.table = None           # neighbour rows searched instead of read from the plan's table
    rng = np.random.default_rng(3)
    w = torch.as_tensor(rng.standard_normal(lvl.cells), device="cuda")
    u = torch.as_tensor(rng.standard_normal(lvl.cells), device="cuda")
    g_chunk = torch.zeros(2, dtype=torch.float64, device="cuda")
    got = lvl.adjoint(w, u, a, b, 1e-3, g_chunk)
    lib = _lib.load()
    ref = torch.empty_like(w)
    g_ref = torch.empty(2, dtype=torch.float64, device="cuda")
    _lib.check(lib.sx_upwind_adjoint(_lib.SX_F64, ptr(lvl.rows), ptr(lvl.off), int(lvl.rows.numel()), ptr(lvl.begin),
                                     ptr(lvl.end), ptr(lvl.cell_off), int(lvl.begin.numel()), lvl.cells,
                                     ptr(lvl.lookup), ptr(w), ptr(u), ptr(ref), lvl.width, lvl.height, a, b, 1e-3,
                                     lvl.dx, lvl.dy, 0, ptr(g_ref), ptr(lvl.scratch), int(lvl.scratch.numel()),
                                     stream_handle(torch.device("cuda", 0))), "sx_upwind_adjoint")
    assert torch.equal(got, ref)
    assert torch.allclose(g_chunk, g_ref, rtol=1e-12, atol=0)


# ---------------------------------------------------------------------------------------------------------------
# Composite multi-level model: ghost filling from the coarser level, restriction onto it
# ---------------------------------------------------------------------------------------------------------------

def _hierarchy(base=24, radii=(0.3, 0.15)):
    hosts = synth.nested_disk_levels(base, list(radii))
    return adj.Hierarchy([dev_set(h) for h in hosts], base, base), hosts


def _cells_of(h):
    b, e, off, rows = h
    ys, xs = [], []
    for k, y in enumerate(rows):
        for i in range(off[k], off[k + 1]):
            x = np.arange(b[i], e[i])
            xs.append(x)
            ys.append(np.full(x.size, y))
    return np.concatenate(ys), np.concatenate(xs)


class _TorchComposite:
    """FP64 restatement of the composite step with torch operations (the reference gradient).

    Built from the host sets alone: each finer level is extended by its
    cross-shaped ghost ring inside the grid, ghost cells take their parent's
    value, every level takes an upwind step with zero outside its extended
    set, and covered coarse cells take the mean of their children.
    """

    def __init__(self, hosts, base, ratio=2):
        self.r = ratio
        self.levels = []
        for k, h in enumerate(hosts):
            n = base * ratio ** k
            ys, xs = _cells_of(h)
            inner = set(zip(ys.tolist(), xs.tolist()))
            cells = set(inner)
            if k:
                for y, x in inner:
                    for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
                        if 0 <= y + dy < n and 0 <= x + dx < n:
                            cells.add((y + dy, x + dx))
            order = sorted(cells)
            index = {c: i for i, c in enumerate(order)}
            nb = np.full((len(order), 4), -1, np.int64)
            for i, (y, x) in enumerate(order):
                for j, (dy, dx) in enumerate(((0, -1), (0, 1), (-1, 0), (1, 0))):
                    nb[i, j] = index.get((y + dy, x + dx), -1)
            inner_idx = np.array([index[(y, x)] for y, x in zip(ys.tolist(), xs.tolist())], np.int64)
            lvl = dict(n=n, order=order, index=index, nb=torch.as_tensor(nb, device="cuda"),
                       inner=torch.as_tensor(inner_idx, device="cuda"), inner_set=inner)
            if k:
                prev = self.levels[-1]
                ghosts = [c for c in order if c not in inner]
                lvl["gpos"] = torch.as_tensor([index[c] for c in ghosts], device="cuda")
                lvl["gpar"] = torch.as_tensor([prev["index"][(y // ratio, x // ratio)] for y, x in ghosts],
                                              device="cuda")
                cov = sorted({(y // ratio, x // ratio) for y, x in inner})
                lvl["cov"] = torch.as_tensor([prev["index"][c] for c in cov], device="cuda")
                lvl["child"] = torch.as_tensor([[index[(Y * ratio + dy, X * ratio + dx)] for dy in range(ratio)
                                                 for dx in range(ratio)] for Y, X in cov], device="cuda")
            self.levels.append(lvl)

    def _upwind(self, u, lvl, a, b, dt):
        dx = 1.0 / lvl["n"]
        nb = lvl["nb"]
        z = torch.zeros(1, dtype=u.dtype, device=u.device)
        ext = torch.cat([u, z])
        left, right, down, up = (ext[torch.where(nb[:, j] >= 0, nb[:, j], u.numel())] for j in range(4))
        dudx = (u - left) / dx if float(a) >= 0 else (right - u) / dx
        dudy = (u - down) / dx if float(b) >= 0 else (up - u) / dx
        return u - dt * (a * dudx + b * dudy)

    def step(self, us, a, b, dt):
        us = list(us)
        for k in range(1, len(us)):
            lvl = self.levels[k]
            us[k] = us[k].index_put((lvl["gpos"],), us[k - 1][lvl["gpar"]])
        us = [self._upwind(u, lvl, a, b, dt) for u, lvl in zip(us, self.levels)]
        for k in range(len(us) - 1, 0, -1):
            lvl = self.levels[k]
            us[k - 1] = us[k - 1].index_put((lvl["cov"],), us[k][lvl["child"]].sum(dim=1) / (self.r * self.r))
        return us

    def run(self, u0, vel, dt, steps):
        us = []
        for u, lvl in zip(u0, self.levels):
            x = torch.zeros(len(lvl["order"]), dtype=u.dtype, device=u.device)
            us.append(x.index_put((lvl["inner"],), u))
        for _ in range(steps):
            us = self.step(us, vel[0], vel[1], dt)
        return [u[lvl["inner"]] for u, lvl in zip(us, self.levels)]


def _gauss_cells(h, n, cx, cy, sigma):
    ys, xs = _cells_of(h)
    x, y = (xs + 0.5) / n, (ys + 0.5) / n
    return np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sigma ** 2))


def test_composite_step_matches_torch_restatement(cuda_device):
    H, hosts = _hierarchy()
    ref = _TorchComposite(hosts, 24)
    rng = np.random.default_rng(2)
    u0 = [torch.as_tensor(rng.standard_normal(n), device="cuda") for n in H.inner_cells]
    dt = 0.5 / (1.5 * 96)
    got = adj.advect_composite(torch.tensor([1.0, 0.5], dtype=torch.float64, device="cuda"), H, u0, dt=dt, steps=7)
    want = ref.run(u0, (1.0, 0.5), dt, 7)
    for g, w in zip(got, want):
        assert float((g - w).abs().max()) <= 1e-12 * max(float(w.abs().max()), 1.0)


def test_composite_transpose_identity(cuda_device):
    H, _ = _hierarchy()
    rng = np.random.default_rng(4)
    for a, b in ((0.7, 0.4), (-0.6, 0.9), (0.5, -1.1)):
        v = [torch.as_tensor(rng.standard_normal(n), device="cuda") for n in H.inner_cells]
        w = [torch.as_tensor(rng.standard_normal(n), device="cuda") for n in H.inner_cells]
        new, inputs = H.step(H.extend(v), a, b, 1e-3)
        mv = H.interior(new)
        g = torch.zeros(2, dtype=torch.float64, device="cuda")
        mtw = H.interior(H.step_adjoint(H.extend(w), inputs, a, b, 1e-3, g))
        lhs = sum(float(torch.dot(x, y)) for x, y in zip(mv, w))
        rhs = sum(float(torch.dot(x, y)) for x, y in zip(v, mtw))
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


def test_composite_gradient_matches_torch_autograd(cuda_device):
    """The hand-written adjoint against torch autograd through the FP64 restatement (the reference gradient)."""
    H, hosts = _hierarchy()
    ref = _TorchComposite(hosts, 24)
    rng = np.random.default_rng(6)
    steps, dt = 12, 0.5 / (1.5 * 96)
    u0 = [torch.as_tensor(_gauss_cells(h, 24 * 2 ** k, 0.5, 0.5, 0.12), device="cuda") for k, h in enumerate(hosts)]
    tg = [torch.as_tensor(rng.standard_normal(n) * 0.1, device="cuda") for n in H.inner_cells]

    def loss(out):
        return sum(0.5 * torch.sum((u - t) ** 2) for u, t in zip(out, tg))

    vel = torch.tensor([1.0, 0.5], dtype=torch.float64, device="cuda", requires_grad=True)
    ua = [u.clone().requires_grad_(True) for u in u0]
    loss(adj.advect_composite(vel, H, ua, dt=dt, steps=steps, checkpoint_every=5)).backward()
    vr = torch.tensor([1.0, 0.5], dtype=torch.float64, device="cuda", requires_grad=True)
    ur = [u.clone().requires_grad_(True) for u in u0]
    loss(ref.run(ur, vr, dt, steps)).backward()
    assert float((vel.grad - vr.grad).abs().max()) <= 1e-9 * float(vr.grad.abs().max())
    for a, b in zip(ua, ur):
        assert float((a.grad - b.grad).abs().max()) <= 1e-10 * max(float(b.grad.abs().max()), 1e-30)


def test_composite_gradient_against_central_differences(cuda_device):
    """FP32 adjoint of the composite model against FP64 central differences on 32 seeded directions."""
    H, hosts = _hierarchy(32)
    steps, every = 10, 4
    dt = 0.5 / (1.5 * 128)
    target = [torch.as_tensor(_gauss_cells(h, 32 * 2 ** k, 0.55, 0.525, 0.1), device="cuda")
              for k, h in enumerate(hosts)]
    u0 = [torch.as_tensor(_gauss_cells(h, 32 * 2 ** k, 0.5, 0.5, 0.1), device="cuda") for k, h in enumerate(hosts)]

    def loss(vel, us, dtype):
        out = adj.advect_composite(vel, H, [u.to(dtype) for u in us], dt=dt, steps=steps, checkpoint_every=every)
        return sum(0.5 * torch.sum((u.double() - t) ** 2) for u, t in zip(out, target))

    vel0 = torch.tensor([1.0, 0.5], dtype=torch.float64, device="cuda")
    vel = vel0.clone().requires_grad_(True)
    u32 = [u.float().requires_grad_(True) for u in u0]
    loss(vel, u32, torch.float32).backward()
    rng = np.random.default_rng(5)
    eps = 1e-6
    errs = []
    for _ in range(32):
        dv = torch.as_tensor(rng.standard_normal(2), device="cuda")
        du = [torch.as_tensor(rng.standard_normal(u.numel()), device="cuda") for u in u0]
        dirder = float(torch.dot(vel.grad, dv)) + sum(float(torch.dot(g.grad.double(), d)) for g, d in zip(u32, du))
        with torch.no_grad():
            lp = loss(vel0 + eps * dv, [u + eps * d for u, d in zip(u0, du)], torch.float64)
            lm = loss(vel0 - eps * dv, [u - eps * d for u, d in zip(u0, du)], torch.float64)
        fd = (float(lp) - float(lm)) / (2 * eps)
        errs.append(abs(dirder - fd) / max(abs(fd), 1e-12))
    assert max(errs) < 1e-4, max(errs)


def test_composite_graph_replays_equal_eager_launches(cuda_device):
    """Segments replayed as CUDA graphs give the same fields and gradients as the launches issued one by one."""
    H, hosts = _hierarchy()
    rng = np.random.default_rng(12)
    dt = 0.5 / (1.5 * 96)
    tg = [torch.as_tensor(rng.standard_normal(n), device="cuda", dtype=torch.float32) for n in H.inner_cells]
    results = []
    for graphs in (False, True, True):  # the second graph run replays the cached graphs
        vel = torch.tensor([0.8, -0.4], dtype=torch.float64, device="cuda", requires_grad=True)
        u0 = [torch.as_tensor(_gauss_cells(h, 24 * 2 ** k, 0.45, 0.5, 0.1), device="cuda",
                              dtype=torch.float32).requires_grad_(True) for k, h in enumerate(hosts)]
        out = adj.advect_composite(vel, H, u0, dt=dt, steps=13, checkpoint_every=5, graphs=graphs)
        sum(torch.sum((u - t) ** 2) for u, t in zip(out, tg)).backward()
        results.append(([o.detach().clone() for o in out], vel.grad.clone(), [u.grad.clone() for u in u0]))
    for other in results[1:]:
        for x, y in zip(results[0][0], other[0]):
            assert torch.equal(x, y)
        assert torch.equal(results[0][1], other[1])
        for x, y in zip(results[0][2], other[2]):
            assert torch.equal(x, y)


def test_composite_transpose_identity_at_full_size(cuda_device):
    """<A v, w> = <v, A^T w> in FP64 on the benchmark's three levels (2048^2 base, disks at x2 and x4, 13.7 M cells);
    the two sums are compared relative to the sum of the absolute products, the scale of their rounding."""
    base = 2048
    hosts = synth.nested_disk_levels(base, [0.3, 0.15])
    H = adj.Hierarchy([dev_set(h) for h in hosts], base, base)
    assert sum(H.inner_cells) > 10_000_000
    g0 = torch.Generator(device="cuda").manual_seed(9)
    v = [torch.randn(n, device="cuda", dtype=torch.float64, generator=g0) for n in H.inner_cells]
    w = [torch.randn(n, device="cuda", dtype=torch.float64, generator=g0) for n in H.inner_cells]
    a, b, dt = 0.8, -0.45, 0.5 / (1.5 * base * 4)
    new, inputs = H.step(H.extend(v), a, b, dt)
    mv = H.interior(new)
    g = torch.zeros(2, dtype=torch.float64, device="cuda")
    mtw = H.interior(H.step_adjoint(H.extend(w), inputs, a, b, dt, g))
    lhs = sum(float(torch.dot(x, y)) for x, y in zip(mv, w))
    rhs = sum(float(torch.dot(x, y)) for x, y in zip(v, mtw))
    scale = sum(float(torch.sum(torch.abs(x * y))) for x, y in zip(mv, w))
    assert abs(lhs - rhs) <= 1e-11 * scale, (lhs, rhs, scale)
