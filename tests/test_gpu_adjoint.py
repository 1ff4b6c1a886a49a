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


@pytest.mark.parametrize("a,b", [(0.7, 0.4), (-0.5, -0.9)])
def test_chunked_adjoint_equals_generic(cuda_device, a, b):
    from subsetix_b200 import _lib
    from subsetix_b200._runtime import ptr, stream_handle

    h = rand_set(400, 12.0, seed=8, row_stride=1, max_col=350, touching=True, row0=0)
    lvl = _level(h, 330, 400)      # some cells lie beyond the width
    assert lvl.chunk_off is not None
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
