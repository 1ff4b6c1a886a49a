"""Differentiable multi-step upwind advection on fixed interval geometry.

``advect`` runs ``steps`` first-order upwind steps on one or more interval
fields (levels) that share a velocity ``(a, b)`` and a time step, and is a
``torch.autograd.Function``: the backward pass applies the hand-written
adjoint kernel ``sx_upwind_adjoint`` step by step, which returns the
gradient with respect to the step's input and the gradient with respect to
the velocity (time step held fixed).  Forward states are kept only every
``checkpoint_every`` steps; the backward pass recomputes each segment from
its checkpoint, so memory holds ``steps / checkpoint_every + checkpoint_every``
states per level instead of ``steps``.

There is no counterpart in the reference, which has no derivatives.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import torch

from . import _core, _lib
from ._runtime import ptr, stream_handle
from .subsetix_cupy.expressions import IntervalSet, _t

_ROWS_UNSAFE = _lib.ROWS_UNSORTED_BEGIN | _lib.ROWS_OVERLAP | _lib.ROWS_EMPTY


@dataclass
class Level:
    """One level's geometry: an interval set in ``[0, width) x [0, height)`` and its cell spacing."""

    interval_set: IntervalSet
    width: int
    height: int
    dx: float
    dy: float

    def __post_init__(self):
        s = self.interval_set
        device = _t(s.row_offsets).device
        self.rows = _t(s.rows)
        self.off = _t(s.row_offsets)
        self.begin = _t(s.begin)
        self.end = _t(s.end)
        self.cell_off, self.cells = _core.cell_offsets(self.begin, self.end, device)
        self.lookup, bad = _core.row_lookup(self.rows, self.height, device)
        if bad:
            raise ValueError("interval_set rows exceed provided height")
        self.direct = not (_core.check_rows(self.begin, self.end, self.off, device) & _ROWS_UNSAFE)
        self.chunk_off, self.chunks = (_core.upwind_plan(self.rows, self.off, self.begin, self.end, self.cell_off,
                                                         self.lookup, self.height, device) if self.direct else (None, 0))
        self.device = device
        lib = _lib.load()
        nbytes = max(int(lib.sx_upwind_adjoint_scratch_bytes(self.cells)),
                     int(lib.sx_upwind_adjoint_chunked_scratch_bytes(self.chunks)))
        self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=device)

    def step(self, u: torch.Tensor, out: torch.Tensor, a: float, b: float, dt: float) -> torch.Tensor:
        if self.chunk_off is not None:
            _core.upwind_chunked(self.off, self.begin, self.end, self.cell_off, self.chunk_off, self.chunks,
                                 self.lookup, u, out, self.width, self.height, a, b, dt, self.dx, self.dy, self.device)
        else:
            _core.upwind(self.rows, self.off, self.begin, self.end, self.cell_off, self.cells, self.lookup, u, out,
                         self.width, self.height, a, b, dt, self.dx, self.dy, self.direct, self.device)
        return out

    def adjoint(self, w: torch.Tensor, u: torch.Tensor, a: float, b: float, dt: float, grad_ab: torch.Tensor
                ) -> torch.Tensor:
        """dL/du for one step, and dL/d(a, b) added into ``grad_ab`` (float64 device pair)."""
        lib = _lib.load()
        ubar = torch.empty_like(w)
        g = torch.empty(2, dtype=torch.float64, device=self.device)
        code = _lib.SX_F64 if w.dtype == torch.float64 else _lib.SX_F32
        if self.chunk_off is not None:
            _lib.check(lib.sx_upwind_adjoint_chunked(code, ptr(self.off), ptr(self.begin), ptr(self.end),
                                                     ptr(self.cell_off), ptr(self.chunk_off), self.chunks,
                                                     ptr(self.lookup), ptr(w), ptr(u), ptr(ubar), self.width,
                                                     self.height, a, b, dt, self.dx, self.dy, ptr(g),
                                                     ptr(self.scratch), int(self.scratch.numel()),
                                                     stream_handle(self.device)), "sx_upwind_adjoint_chunked")
            grad_ab += g
            return ubar
        _lib.check(lib.sx_upwind_adjoint(code, ptr(self.rows), ptr(self.off), int(self.rows.numel()), ptr(self.begin),
                                         ptr(self.end), ptr(self.cell_off), int(self.begin.numel()), self.cells,
                                         ptr(self.lookup), ptr(w), ptr(u), ptr(ubar), self.width, self.height, a, b,
                                         dt, self.dx, self.dy, 1 if self.direct else 0, ptr(g), ptr(self.scratch),
                                         int(self.scratch.numel()), stream_handle(self.device)), "sx_upwind_adjoint")
        grad_ab += g
        return ubar


def _run(levels: Sequence[Level], states: List[torch.Tensor], a: float, b: float, dt: float, n: int,
         keep: bool) -> List[List[torch.Tensor]]:
    """Advance every level ``n`` steps; with ``keep`` return all intermediate inputs per level."""
    trail: List[List[torch.Tensor]] = [[] for _ in levels]
    cur = list(states)
    for _ in range(n):
        for k, lvl in enumerate(levels):
            if keep:
                trail[k].append(cur[k])
            cur[k] = lvl.step(cur[k], torch.empty_like(cur[k]), a, b, dt)
    for k in range(len(levels)):
        trail[k].append(cur[k])
    return trail


class _Advect(torch.autograd.Function):
    @staticmethod
    def forward(ctx, velocity: torch.Tensor, levels, dt: float, steps: int, every: int, *u0):
        a, b = (float(v) for v in velocity.detach().cpu().tolist())
        checkpoints = [list(u.detach() for u in u0)]
        cur = [u.detach().contiguous() for u in u0]
        done = 0
        while done < steps:
            n = min(every, steps - done)
            trail = _run(levels, cur, a, b, dt, n, keep=False)
            cur = [t[-1] for t in trail]
            done += n
            if done < steps:
                checkpoints.append(list(cur))
        ctx.levels, ctx.dt, ctx.steps, ctx.every, ctx.ab = levels, dt, steps, every, (a, b)
        ctx.checkpoints = checkpoints
        ctx.vel_dtype = velocity.dtype
        ctx.vel_device = velocity.device
        return tuple(cur)

    @staticmethod
    def backward(ctx, *grad_out):
        levels, dt, steps, every = ctx.levels, ctx.dt, ctx.steps, ctx.every
        a, b = ctx.ab
        w = [g.contiguous() if g is not None else torch.zeros_like(c) for g, c in zip(grad_out, ctx.checkpoints[0])]
        grad_ab = torch.zeros(2, dtype=torch.float64, device=levels[0].device)
        seg_starts = list(range(0, steps, every))
        for si in reversed(range(len(seg_starts))):
            n = min(every, steps - seg_starts[si])
            trail = _run(levels, ctx.checkpoints[si], a, b, dt, n, keep=True)  # recompute the segment
            for j in reversed(range(n)):
                for k, lvl in enumerate(levels):
                    w[k] = lvl.adjoint(w[k], trail[k][j], a, b, dt, grad_ab)
        ctx.checkpoints = None
        grad_v = grad_ab.to(device=ctx.vel_device, dtype=ctx.vel_dtype)
        return (grad_v, None, None, None, None, *w)


def advect(velocity: torch.Tensor, levels: Sequence[Level], u0: Sequence[torch.Tensor], *, dt: float, steps: int,
           checkpoint_every: int = 10) -> Tuple[torch.Tensor, ...]:
    """``steps`` upwind steps of every level; differentiable in ``velocity`` (2 values) and ``u0``."""
    if len(levels) != len(u0):
        raise ValueError("one initial field per level")
    if steps < 0 or checkpoint_every < 1:
        raise ValueError("steps must be >= 0 and checkpoint_every >= 1")
    return _Advect.apply(velocity, tuple(levels), float(dt), int(steps), int(checkpoint_every), *u0)


__all__ = ["Level", "advect"]
