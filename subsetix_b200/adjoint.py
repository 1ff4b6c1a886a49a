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

``advect_composite`` couples nested levels the way a composite AMR step does
(:class:`Hierarchy`): before each step the ghost ring of every finer level
takes its coarse parents' values (injection), every level is advanced on its
cells plus that ring, and after the step the coarse cells under a finer level
take the mean of their children (restriction, finest level first).  Each
coupling is a gather or a block mean over index tables built once for the
fixed geometry (``sx_index_copy``, ``sx_index_block_mean``); the backward
pass applies their transposes (``sx_index_segment_add``,
``sx_index_block_mean_adj``) around the adjoint upwind kernel, in reverse
order.

There is no counterpart in the reference, which has no derivatives.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

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
        self.table = (_core.upwind_table(self.begin, self.end, self.cell_off, self.chunk_off, self.chunks, self.cells,
                                         device) if self.direct else None)
        self.device = device
        lib = _lib.load()
        nbytes = max(int(lib.sx_upwind_adjoint_scratch_bytes(self.cells)),
                     int(lib.sx_upwind_adjoint_chunked_scratch_bytes(self.chunks)))
        self.scratch = torch.empty(nbytes, dtype=torch.uint8, device=device)

    def step(self, u: torch.Tensor, out: torch.Tensor, a: float, b: float, dt: float) -> torch.Tensor:
        if self.chunk_off is not None:
            _core.upwind_chunked(self.off, self.begin, self.end, self.cell_off, self.chunk_off, self.chunks,
                                 self.lookup, u, out, self.width, self.height, a, b, dt, self.dx, self.dy, self.device,
                                 table=self.table)
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
                                                     ptr(self.lookup), ptr(self.table), ptr(w), ptr(u), ptr(ubar),
                                                     self.width,
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


# ---------------------------------------------------------------------------------------------------------------
# Nested levels coupled by ghost filling and restriction
# ---------------------------------------------------------------------------------------------------------------

def _cells(s: IntervalSet, cell_off: torch.Tensor):
    """(rows, cols) of every cell of ``s`` in value order, as int32 device tensors."""
    b, e, off, rows = _t(s.begin), _t(s.end), _t(s.row_offsets), _t(s.rows)
    n = int(b.numel())
    total = int(cell_off[-1].item()) if n else 0
    dev = off.device
    if total == 0:
        z = torch.zeros(0, dtype=torch.int32, device=dev)
        return z, z.clone()
    iv = torch.repeat_interleave(torch.arange(n, device=dev), (e - b).to(torch.int64))
    x = b[iv] + (torch.arange(total, device=dev, dtype=torch.int32) - cell_off[:-1][iv])
    irow = torch.repeat_interleave(rows, (off[1:] - off[:-1]).to(torch.int64))
    return irow[iv].to(torch.int32), x.to(torch.int32)


def _positions(s: IntervalSet, cell_off: torch.Tensor, rows: torch.Tensor, cols: torch.Tensor) -> torch.Tensor:
    """Value index of each cell (rows, cols) in a field on ``s``; -1 where the cell is not in ``s``."""
    from .subsetix_cupy.interval_field import IntervalField, locate_interval_cells

    if rows.numel() == 0:
        return rows.clone()
    f = IntervalField(interval_set=s, values=torch.empty(0, device=rows.device), interval_cell_offsets=cell_off)
    iv = torch.as_tensor(locate_interval_cells(f, rows, cols)).to(torch.int64)
    found = iv >= 0
    ivc = iv.clamp_min(0)
    pos = cell_off[ivc].to(torch.int64) + (cols.to(torch.int64) - _t(s.begin)[ivc].to(torch.int64))
    return torch.where(found, pos, torch.full_like(pos, -1)).to(torch.int32)


class Hierarchy:
    """Nested interval sets on grids refined by ``ratio`` per level, coupled as a composite AMR step.

    ``sets[k]`` lies in the ``(width * ratio**k) x (height * ratio**k)`` grid
    of level ``k``.  Every finer level needs its ghost ring (the cells next
    to it, left/right/below/above, inside the grid) to have parents in the
    coarser level's set, and every coarse cell under it to have all its
    ``ratio x ratio`` children in it; building a level from the prolongation
    of a coarse set that keeps a one-cell margin satisfies both.  Fields
    given to and returned by :func:`advect_composite` hold the cells of
    ``sets[k]`` in their usual order.
    """

    def __init__(self, sets: Sequence[IntervalSet], width: int, height: int, *, ratio: int = 2,
                 extent: Tuple[float, float] = (1.0, 1.0)):
        from .subsetix_cupy import (clip_interval_set, dilate_interval_set, evaluate, make_input, make_union,
                                    restrict_set)

        if not sets:
            raise ValueError("a hierarchy needs at least one level")
        self.ratio = r = int(ratio)
        if r < 2:
            raise ValueError("levels must be refined by a ratio of at least 2")
        self.levels: List[Level] = []
        self.inner: List[torch.Tensor] = []
        self.inner_cells: List[int] = []
        self.ghost: List[Optional[tuple]] = []
        self.cover: List[Optional[tuple]] = []
        self._segments: dict = {}
        for k, s in enumerate(sets):
            W, H = int(width) * r ** k, int(height) * r ** k
            if k == 0:
                ext = s
            else:
                cross = evaluate(make_union(make_input(dilate_interval_set(s, 1, 0)),
                                            make_input(dilate_interval_set(s, 0, 1))))
                ext = clip_interval_set(cross, width=W, height=H)
            lvl = Level(ext, W, H, extent[0] / W, extent[1] / H)
            self.levels.append(lvl)
            s_off, _ = _core.cell_offsets(_t(s.begin), _t(s.end), lvl.device)
            ys, xs = _cells(s, s_off)
            inner = _positions(ext, lvl.cell_off, ys, xs)
            if bool((inner < 0).any()):
                raise ValueError(f"level {k}: the set is not inside its grid")
            self.inner.append(inner)
            self.inner_cells.append(int(inner.numel()))
            if k == 0:
                self.ghost.append(None)
                self.cover.append(None)
                continue
            prev, prev_set = self.levels[k - 1], sets[k - 1]
            # ghost ring: cells of the extended set outside the set, with their parents on level k-1
            is_inner = torch.zeros(lvl.cells, dtype=torch.bool, device=lvl.device)
            is_inner[inner.to(torch.int64)] = True
            ey, ex = _cells(ext, lvl.cell_off)
            gpos = torch.nonzero(~is_inner).reshape(-1).to(torch.int32)
            py, px = torch.div(ey[gpos.to(torch.int64)], r, rounding_mode="floor"), \
                torch.div(ex[gpos.to(torch.int64)], r, rounding_mode="floor")
            ppos = _positions(prev.interval_set, prev.cell_off, py.to(torch.int32), px.to(torch.int32))
            p_set_off, _ = _core.cell_offsets(_t(prev_set.begin), _t(prev_set.end), lvl.device)
            if bool((ppos < 0).any()) or bool((_positions(prev_set, p_set_off, py.to(torch.int32),
                                                          px.to(torch.int32)) < 0).any()):
                raise ValueError(f"level {k}: its ghost ring is not covered by level {k - 1}")
            order = torch.argsort(ppos.to(torch.int64), stable=True)
            sp = ppos[order]
            uniq, counts = torch.unique_consecutive(sp, return_counts=True)
            seg_off = torch.zeros(uniq.numel() + 1, dtype=torch.int32, device=lvl.device)
            seg_off[1:] = torch.cumsum(counts, 0).to(torch.int32)
            self.ghost.append((gpos.contiguous(), ppos.contiguous(), seg_off, gpos[order].contiguous(),
                               uniq.to(torch.int32).contiguous()))
            # restriction: coarse cells under level k and their r x r children (sub-row outer, column inner)
            covered = restrict_set(s, r)
            c_off, _ = _core.cell_offsets(_t(covered.begin), _t(covered.end), lvl.device)
            cy, cx = _cells(covered, c_off)
            cpos = _positions(prev.interval_set, prev.cell_off, cy, cx)
            dy = torch.arange(r, device=lvl.device).repeat_interleave(r)
            dx = torch.arange(r, device=lvl.device).repeat(r)
            chy = (cy.to(torch.int64)[:, None] * r + dy[None, :]).reshape(-1).to(torch.int32)
            chx = (cx.to(torch.int64)[:, None] * r + dx[None, :]).reshape(-1).to(torch.int32)
            child = _positions(s, s_off, chy, chx)
            if bool((cpos < 0).any()) or bool((child < 0).any()):
                raise ValueError(f"level {k}: a coarse cell under it does not have all its children in it")
            child = inner[child.to(torch.int64)]
            self.cover.append((cpos.contiguous(), child.contiguous()))

    # -- the coupled step and its transpose ------------------------------------------------------------------------
    def _fill_ghosts(self, u: List[torch.Tensor]) -> None:
        lib = _lib.load()
        for k in range(1, len(self.levels)):
            gpos, ppos = self.ghost[k][0], self.ghost[k][1]
            _lib.check(lib.sx_index_copy(_code(u[k]), int(gpos.numel()), ptr(gpos), ptr(ppos), ptr(u[k - 1]),
                                         ptr(u[k]), stream_handle(u[k].device)), "sx_index_copy")

    def _restrict(self, u: List[torch.Tensor]) -> None:
        lib = _lib.load()
        r2 = self.ratio * self.ratio
        for k in range(len(self.levels) - 1, 0, -1):
            cpos, child = self.cover[k]
            _lib.check(lib.sx_index_block_mean(_code(u[k]), int(cpos.numel()), r2, 1.0 / r2, ptr(cpos), ptr(child),
                                               ptr(u[k]), ptr(u[k - 1]), stream_handle(u[k].device)),
                       "sx_index_block_mean")

    def step(self, u: List[torch.Tensor], a: float, b: float, dt: float) -> Tuple[List[torch.Tensor], List[torch.Tensor]]:
        """One coupled step of the extended-level fields ``u``; returns (new fields, upwind inputs)."""
        self._fill_ghosts(u)
        new = [lvl.step(x, torch.empty_like(x), a, b, dt) for lvl, x in zip(self.levels, u)]
        self._restrict(new)
        return new, u

    def step_adjoint(self, w: List[torch.Tensor], inputs: List[torch.Tensor], a: float, b: float, dt: float,
                     grad_ab: torch.Tensor) -> List[torch.Tensor]:
        """Transpose of :meth:`step` applied to ``w`` (modified); ``inputs`` are that step's upwind inputs."""
        lib = _lib.load()
        r2 = self.ratio * self.ratio
        for k in range(1, len(self.levels)):
            cpos, child = self.cover[k]
            _lib.check(lib.sx_index_block_mean_adj(_code(w[k]), int(cpos.numel()), r2, 1.0 / r2, ptr(cpos),
                                                   ptr(child), ptr(w[k - 1]), ptr(w[k]), stream_handle(w[k].device)),
                       "sx_index_block_mean_adj")
        w = [lvl.adjoint(x, u, a, b, dt, grad_ab) for lvl, x, u in zip(self.levels, w, inputs)]
        for k in range(len(self.levels) - 1, 0, -1):
            _, _, seg_off, src, dst = self.ghost[k]
            _lib.check(lib.sx_index_segment_add(_code(w[k]), int(dst.numel()), ptr(seg_off), ptr(src), ptr(dst),
                                                ptr(w[k]), ptr(w[k - 1]), 1, stream_handle(w[k].device)),
                       "sx_index_segment_add")
        return w

    # -- fields on the sets <-> fields on the extended sets ----------------------------------------------------------
    def extend(self, fields: Sequence[torch.Tensor]) -> List[torch.Tensor]:
        out = []
        lib = _lib.load()
        for lvl, inner, f in zip(self.levels, self.inner, fields):
            x = torch.zeros(lvl.cells, dtype=f.dtype, device=lvl.device)
            f = f.contiguous()
            _lib.check(lib.sx_index_copy(_code(x), int(inner.numel()), ptr(inner), None, ptr(f), ptr(x),
                                         stream_handle(lvl.device)), "sx_index_copy")
            out.append(x)
        return out

    def interior(self, fields: Sequence[torch.Tensor]) -> List[torch.Tensor]:
        out = []
        lib = _lib.load()
        for inner, x in zip(self.inner, fields):
            y = torch.empty(int(inner.numel()), dtype=x.dtype, device=x.device)
            _lib.check(lib.sx_index_copy(_code(x), int(inner.numel()), None, ptr(inner), ptr(x), ptr(y),
                                         stream_handle(x.device)), "sx_index_copy")
            out.append(y)
        return out


def _code(t: torch.Tensor) -> int:
    return _lib.SX_F64 if t.dtype == torch.float64 else _lib.SX_F32


def _run_composite(h: Hierarchy, states: List[torch.Tensor], a: float, b: float, dt: float, n: int, keep: bool):
    """``n`` coupled steps; with ``keep`` also the upwind inputs of every step."""
    inputs = []
    cur = list(states)
    for _ in range(n):
        cur, used = h.step(cur, a, b, dt)
        if keep:
            inputs.append(used)
    return cur, inputs


class _Segment:
    """``n`` coupled steps and their transposes as two CUDA graphs on fixed buffers.

    The forward graph runs the steps from ``inp`` and keeps every step's
    upwind inputs (``inputs``, the recomputation a backward pass needs); the
    backward graph applies the steps' transposes, last step first, from
    ``w_in`` to ``w_out`` and adds each step's velocity gradient onto
    ``grad`` (which the caller loads with the running sum).
    Velocity and time step are baked into the graphs.  Every launch of a
    segment becomes one graph replay instead of about seven launches per step
    issued from Python.
    """

    def __init__(self, h: "Hierarchy", n: int, a: float, b: float, dt: float, dtype: torch.dtype):
        dev = h.levels[0].device
        self.inp = [torch.zeros(lvl.cells, dtype=dtype, device=dev) for lvl in h.levels]
        self.w_in = [torch.zeros(lvl.cells, dtype=dtype, device=dev) for lvl in h.levels]
        self.grad = torch.zeros(2, dtype=torch.float64, device=dev)
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        self.fwd = torch.cuda.CUDAGraph()
        self.bwd = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            with torch.cuda.graph(self.fwd, stream=side):
                cur, self.inputs = _run_composite(h, list(self.inp), a, b, dt, n, keep=True)
                self.out = cur
            with torch.cuda.graph(self.bwd, stream=side):
                w = list(self.w_in)
                for j in reversed(range(n)):
                    w = h.step_adjoint(w, self.inputs[j], a, b, dt, self.grad)
                self.w_out = w
        torch.cuda.current_stream(dev).wait_stream(side)

    def forward(self, states: Sequence[torch.Tensor]) -> List[torch.Tensor]:
        for dst, src in zip(self.inp, states):
            dst.copy_(src)
        self.fwd.replay()
        return self.out

    def backward(self, w: Sequence[torch.Tensor]) -> List[torch.Tensor]:
        for dst, src in zip(self.w_in, w):
            dst.copy_(src)
        self.bwd.replay()
        return self.w_out


def _segment(h: "Hierarchy", n: int, a: float, b: float, dt: float, dtype: torch.dtype) -> _Segment:
    """Cached segment graphs of ``h`` (the two most recent parameter sets are kept)."""
    key = (n, a, b, dt, dtype)
    cache = h._segments
    seg = cache.pop(key, None)
    if seg is None:
        while len(cache) >= 2:
            cache.pop(next(iter(cache)))
        seg = _Segment(h, n, a, b, dt, dtype)
    cache[key] = seg
    return seg


class _AdvectComposite(torch.autograd.Function):
    @staticmethod
    def forward(ctx, velocity: torch.Tensor, h: Hierarchy, dt: float, steps: int, every: int, graphs: bool, *u0):
        a, b = (float(v) for v in velocity.detach().cpu().tolist())
        cur = h.extend([u.detach() for u in u0])
        checkpoints = [[x.clone() for x in cur]]
        done = 0
        while done < steps:
            n = min(every, steps - done)
            if graphs:
                cur = _segment(h, n, a, b, dt, cur[0].dtype).forward(cur)
            else:
                cur, _ = _run_composite(h, cur, a, b, dt, n, keep=False)
            done += n
            if done < steps:
                checkpoints.append([x.clone() for x in cur])
        ctx.h, ctx.dt, ctx.steps, ctx.every, ctx.ab, ctx.graphs = h, dt, steps, every, (a, b), graphs
        ctx.checkpoints = checkpoints
        ctx.vel = (velocity.dtype, velocity.device)
        return tuple(h.interior(cur))

    @staticmethod
    def backward(ctx, *grad_out):
        h, dt, steps, every = ctx.h, ctx.dt, ctx.steps, ctx.every
        a, b = ctx.ab
        zeros = [torch.zeros(n, dtype=c.dtype, device=c.device) for n, c in zip(h.inner_cells, ctx.checkpoints[0])]
        w = h.extend([g if g is not None else z for g, z in zip(grad_out, zeros)])
        grad_ab = torch.zeros(2, dtype=torch.float64, device=h.levels[0].device)
        starts = list(range(0, steps, every))
        for si in reversed(range(len(starts))):
            n = min(every, steps - starts[si])
            if ctx.graphs:
                # the graph adds every step's velocity gradient onto the running sum, in the eager order
                seg = _segment(h, n, a, b, dt, w[0].dtype)
                seg.grad.copy_(grad_ab)
                seg.forward(ctx.checkpoints[si])
                w = [x.clone() for x in seg.backward(w)]
                grad_ab.copy_(seg.grad)
            else:
                _, inputs = _run_composite(h, [x.clone() for x in ctx.checkpoints[si]], a, b, dt, n, keep=True)
                for j in reversed(range(n)):
                    w = h.step_adjoint(w, inputs[j], a, b, dt, grad_ab)
        ctx.checkpoints = None
        grads = h.interior(w)
        return (grad_ab.to(device=ctx.vel[1], dtype=ctx.vel[0]), None, None, None, None, None, *grads)


def advect_composite(velocity: torch.Tensor, hierarchy: Hierarchy, u0: Sequence[torch.Tensor], *, dt: float,
                     steps: int, checkpoint_every: int = 10, graphs: bool = True) -> Tuple[torch.Tensor, ...]:
    """``steps`` coupled steps of a :class:`Hierarchy`; differentiable in ``velocity`` (2 values) and ``u0``.

    ``u0[k]`` holds the cells of level ``k``'s set; so does each returned field.
    With ``graphs`` every checkpoint segment runs as a CUDA-graph replay (the
    graphs for a velocity and time step are captured on first use and kept for
    the two most recent ones); without, the same launches are issued one by
    one.  Results are the same either way.
    """
    if len(u0) != len(hierarchy.levels):
        raise ValueError("one initial field per level")
    for k, (u, n) in enumerate(zip(u0, hierarchy.inner_cells)):
        if int(u.numel()) != n:
            raise ValueError(f"level {k}: expected {n} values, got {int(u.numel())}")
    if steps < 0 or checkpoint_every < 1:
        raise ValueError("steps must be >= 0 and checkpoint_every >= 1")
    return _AdvectComposite.apply(velocity, hierarchy, float(dt), int(steps), int(checkpoint_every), bool(graphs),
                                  *u0)


__all__ = ["Level", "advect", "Hierarchy", "advect_composite"]
