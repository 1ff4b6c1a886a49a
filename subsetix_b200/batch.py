"""Many independent interval sets evaluated together, one launch per operation.

A batch lays its sets on disjoint row bands of one combined set: set ``i``
occupies rows ``base_i + row``, and consecutive bands are separated by at
least one empty row.  Row-wise operations (set algebra, morphology along
x) never mix rows, so one launch over the combined set evaluates the
operation for every set at once.  The upwind step reads rows ``y - 1`` and
``y + 1``, which are empty between bands, so the zero-exterior update of each
set is unchanged as long as every set lies inside its own domain
``[0, width_i) x [0, height_i)``; each band carries its own spacing and time
step (``sx_upwind_chunked_bands``), so set ``i`` gets exactly the values of
its own ``step_upwind_interval`` call with ``dx = dy = 1 / side_i``.

:class:`BatchStep` runs the union and intersection of two batches and one
upwind step of the first batch's field as three launches on fixed buffers
with no host synchronisation, so the whole step can be captured in one CUDA
graph and replayed; the three launches stay separate kernels because the two
sweeps write data-dependent output sizes through a look-back over their own
tiles, while the stencil walks a fixed chunk plan of different geometry.

This is the batching the reference lacks: there every set is one Python
call with its own launches and host synchronisations.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _core, _lib
from ._runtime import ptr, stream_handle
from .subsetix_cupy.expressions import IntervalSet, _t, apply_binary, truth_table, _remap
from .subsetix_cupy.interval_field import IntervalField
from .subsetix_cupy.interval_stencil import step_upwind_interval

I32 = torch.int32
_ROWS_UNSAFE = _lib.ROWS_UNSORTED_BEGIN | _lib.ROWS_OVERLAP | _lib.ROWS_EMPTY


@dataclass
class _StencilPlan:
    """Per-batch data of the banded stencil, built once: cell offsets, row lookup, chunk plan, row bands."""

    cell_off: torch.Tensor
    cells: int
    lookup: torch.Tensor
    height: int
    chunk_off: Optional[torch.Tensor]
    chunks: int
    row_band: torch.Tensor
    table: Optional[torch.Tensor] = None


@dataclass
class SetBatch:
    """Sets on disjoint row bands of ``combined``.

    ``bases[i]`` is the first row of band ``i`` and ``heights[i]`` its
    height (the set's rows lie in ``[0, heights[i])``).
    """

    combined: IntervalSet
    bases: List[int]
    heights: List[int]
    _plan: Optional[_StencilPlan] = field(default=None, repr=False, compare=False)
    _tables: dict = field(default_factory=dict, repr=False, compare=False)

    @classmethod
    def layout(cls, heights: Sequence[int], gap: int = 1) -> List[int]:
        bases, b = [], 0
        for h in heights:
            bases.append(b)
            b += int(h) + int(gap)
        return bases

    @classmethod
    def from_sets(cls, sets: Sequence[IntervalSet], heights: Sequence[int], gap: int = 1) -> "SetBatch":
        """Concatenate ``sets`` (rows of set ``i`` in ``[0, heights[i])``) onto bands."""
        if len(sets) != len(heights):
            raise ValueError("one height per set")
        if gap < 1:
            raise ValueError("bands must be separated by at least one empty row")
        bases = cls.layout(heights, gap)
        device = _t(sets[0].row_offsets).device
        begins = [_t(s.begin) for s in sets]
        ends = [_t(s.end) for s in sets]
        rows = [_t(s.rows) + b for s, b in zip(sets, bases)]
        counts = [_t(s.row_offsets)[1:] - _t(s.row_offsets)[:-1] for s in sets]
        cnt = torch.cat(counts) if counts else torch.zeros(0, dtype=I32, device=device)
        off = torch.zeros(int(cnt.numel()) + 1, dtype=I32, device=device)
        if cnt.numel():
            torch.cumsum(cnt, 0, out=off[1:])
        comb = IntervalSet._trusted(torch.cat(begins), torch.cat(ends), off, torch.cat(rows))
        return cls(comb, bases, [int(h) for h in heights])

    @property
    def total_rows(self) -> int:
        return self.bases[-1] + self.heights[-1] + 1 if self.bases else 1

    def split(self) -> List[IntervalSet]:
        """The per-set results, rows moved back to ``[0, height_i)`` (one host synchronisation)."""
        s = self.combined
        rows, off = _t(s.rows), _t(s.row_offsets)
        b, e = _t(s.begin), _t(s.end)
        edges = torch.tensor(self.bases + [self.bases[-1] + self.heights[-1]], dtype=I32, device=rows.device)
        cut = torch.searchsorted(rows, edges)
        at = torch.cat([cut.to(I32), off[cut.long()]]).cpu().tolist()
        n = len(self.bases)
        rcut, icut = at[: n + 1], at[n + 1:]
        out = []
        for i, base in enumerate(self.bases):
            r0, r1, lo, hi = rcut[i], rcut[i + 1], icut[i], icut[i + 1]
            out.append(IntervalSet._trusted(b[lo:hi], e[lo:hi], off[r0:r1 + 1] - lo, rows[r0:r1] - base))
        return out

    # -- the stencil's fixed data ---------------------------------------------------------------------------------
    def stencil_plan(self) -> _StencilPlan:
        """Cell offsets, row lookup, chunk plan and row bands of the combined set (built on first use)."""
        if self._plan is None:
            s = self.combined
            dev = _t(s.row_offsets).device
            b, e, off, rows = _t(s.begin), _t(s.end), _t(s.row_offsets), _t(s.rows)
            cell_off, cells = _core.cell_offsets(b, e, dev)
            H = self.total_rows
            lookup, bad = _core.row_lookup(rows, H, dev)
            if bad:
                raise ValueError("batch rows outside the band layout")
            direct = not (_core.check_rows(b, e, off, dev) & _ROWS_UNSAFE)
            chunk_off, chunks = (_core.upwind_plan(rows, off, b, e, cell_off, lookup, H, dev) if direct else (None, 0))
            table = _core.upwind_table(b, e, cell_off, chunk_off, chunks, cells, dev) if direct else None
            band = torch.full((H,), -1, dtype=I32, device=dev)
            for i, (base, h) in enumerate(zip(self.bases, self.heights)):
                band[base:base + h] = i
            self._plan = _StencilPlan(cell_off, cells, lookup, H, chunk_off, chunks, band, table)
        return self._plan

    def band_table(self, dtype: torch.dtype, spacing: Sequence[Tuple[float, float, float]]) -> torch.Tensor:
        """Device table of per-band (dx, dy, dt) in the kernel's form for ``dtype`` (cached per spacing)."""
        key = (dtype, tuple(tuple(float(x) for x in t) for t in spacing))
        got = self._tables.get(key)
        if got is None:
            if len(spacing) != len(self.bases):
                raise ValueError(f"{len(spacing)} spacings for {len(self.bases)} sets")
            code = _lib.SX_F64 if dtype == torch.float64 else _lib.SX_F32
            trip = np.ascontiguousarray(np.asarray(spacing, dtype=np.float64).reshape(-1))
            host = np.empty(4 * len(spacing), dtype=np.float64 if code == _lib.SX_F64 else np.float32)
            _lib.check(_lib.load().sx_upwind_band_table(code, trip.ctypes.data, len(spacing), host.ctypes.data),
                       "sx_upwind_band_table")
            got = torch.as_tensor(host).to(_t(self.combined.row_offsets).device)
            self._tables[key] = got
        return got


def batched_binary(lhs: SetBatch, rhs: SetBatch, mode: str) -> SetBatch:
    """``mode`` ("union", "intersection", "difference", "symmetric_difference") of every pair, one launch."""
    if lhs.bases != rhs.bases:
        raise ValueError("batches must share their band layout")
    return SetBatch(apply_binary(lhs.combined, rhs.combined, mode), list(lhs.bases), list(lhs.heights))


def _per_set(x, n: int, what: str) -> List[float]:
    if np.ndim(x) == 0:
        return [float(x)] * n
    vals = [float(v) for v in x]
    if len(vals) != n:
        raise ValueError(f"{what}: {len(vals)} values for {n} sets")
    return vals


def batched_upwind(batch: SetBatch, values: torch.Tensor, *, width, a: float, b: float, dt, dx, dy,
                   out: torch.Tensor | None = None) -> torch.Tensor:
    """One upwind step of every set's field (values stored set after set, row by row), one launch.

    ``dt``, ``dx``, ``dy`` and ``width`` are one number for every set or one
    value per set; set ``i`` must lie in ``[0, width_i) x [0, height_i)``.
    The steps of the sets do not interact (empty rows separate the bands),
    and each set's values equal its own ``step_upwind_interval`` call.
    """
    n = len(batch.bases)
    dts, dxs, dys = _per_set(dt, n, "dt"), _per_set(dx, n, "dx"), _per_set(dy, n, "dy")
    w = int(max(_per_set(width, n, "width")))
    vals = _t(values)
    plan = batch.stencil_plan()
    if int(vals.numel()) != plan.cells:
        raise ValueError(f"the batch has {plan.cells} cells, got {int(vals.numel())} values")
    res = torch.empty_like(vals) if out is None else _t(out)
    if plan.chunk_off is None:
        if len(set(zip(dts, dxs, dys))) != 1:
            raise ValueError("per-set spacing needs sorted, disjoint, non-empty intervals in every row")
        field = IntervalField(interval_set=batch.combined, values=vals, interval_cell_offsets=plan.cell_off)
        return step_upwind_interval(field, width=w, height=plan.height, a=a, b=b, dt=dts[0], dx=dxs[0], dy=dys[0],
                                    out=res)
    table = batch.band_table(vals.dtype, list(zip(dxs, dys, dts)))
    _upwind_bands(batch, plan, table, vals, res, w, a, b)
    return res


def _upwind_bands(batch: SetBatch, plan: _StencilPlan, table: torch.Tensor, vals: torch.Tensor, out: torch.Tensor,
                  width: int, a: float, b: float) -> None:
    s = batch.combined
    lib = _lib.load()
    code = _lib.SX_F64 if vals.dtype == torch.float64 else _lib.SX_F32
    _lib.check(lib.sx_upwind_chunked_bands(code, ptr(_t(s.row_offsets)), ptr(_t(s.begin)), ptr(_t(s.end)),
                                           ptr(plan.cell_off), ptr(plan.chunk_off), int(plan.chunks),
                                           ptr(plan.lookup), ptr(plan.table), ptr(vals), ptr(out), int(width),
                                           int(plan.height),
                                           float(a), float(b), ptr(plan.row_band), ptr(table), len(batch.bases),
                                           stream_handle(vals.device)), "sx_upwind_chunked_bands")


class BatchStep:
    """Union and intersection of two batches and one upwind step of the first's field, with no host sync.

    Everything a step needs is allocated here: output capacity for both set
    operations, their result pairs and scratch, the stencil's plan and band
    table, and the new values.  :meth:`__call__` enqueues the three launches;
    :meth:`graph` captures them once as a CUDA graph.  Set-operation results
    are read with :meth:`union` / :meth:`intersection` (one synchronisation).
    """

    def __init__(self, A: SetBatch, B: SetBatch, values: torch.Tensor, *, width, a: float, b: float, dt, dx, dy):
        if A.bases != B.bases or A.heights != B.heights:
            raise ValueError("batches must share their band layout")
        ra, rb = _t(A.combined.rows), _t(B.combined.rows)
        if ra.numel() != rb.numel() or not bool(torch.equal(ra, rb)):
            raise ValueError("BatchStep needs batches with identical row lists")
        self.A, self.B = A, B
        self.device = ra.device
        self.rows = int(ra.numel())
        n = len(A.bases)
        self.a, self.b = float(a), float(b)
        self.width = int(max(_per_set(width, n, "width")))
        self.values = _t(values)
        self.plan = A.stencil_plan()
        if self.plan.chunk_off is None:
            raise ValueError("BatchStep needs sorted, disjoint, non-empty intervals in every row")
        self.table = A.band_table(self.values.dtype, list(zip(_per_set(dx, n, "dx"), _per_set(dy, n, "dy"),
                                                               _per_set(dt, n, "dt"))))
        self.out = torch.empty_like(self.values)
        sa, sb = A.combined, B.combined
        self.leaves = [(_t(sa.begin), _t(sa.end), _t(sa.row_offsets), 0), (_t(sb.begin), _t(sb.end),
                                                                          _t(sb.row_offsets), 0)]
        cap = max(1, sum(int(x[0].numel()) for x in self.leaves))
        lib = _lib.load()
        self.scratch = torch.zeros(int(lib.sx_bool_workspace_bytes(self.rows)), dtype=torch.uint8, device=self.device)
        self.ops = {}
        for mode in ("union", "intersection"):
            node = _remap((mode, ("leaf", 0), ("leaf", 1)), {0: 0, 1: 1})
            tuning = _core.auto_tuning(self.leaves, self.rows, self.device)
            self.ops[mode] = dict(table=truth_table(node, 2), tuning=tuning,
                                  begin=torch.empty(cap, dtype=I32, device=self.device),
                                  end=torch.empty(cap, dtype=I32, device=self.device),
                                  offsets=torch.empty(self.rows + 1, dtype=I32, device=self.device),
                                  result=torch.zeros(2, dtype=I32, device=self.device))

    def __call__(self) -> None:
        for op in self.ops.values():
            _core.bool_eval_async(self.leaves, self.rows, op["table"], _lib.MODE_TABLE, self.device,
                                  out=(op["begin"], op["end"]), result=op["result"], offsets=op["offsets"],
                                  tuning=op["tuning"], scratch=self.scratch)
        _upwind_bands(self.A, self.plan, self.table, self.values, self.out, self.width, self.a, self.b)

    def graph(self) -> torch.cuda.CUDAGraph:
        """The three launches captured once (run :meth:`__call__` once before, to load every kernel)."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self()
        torch.cuda.current_stream(self.device).wait_stream(s)
        return g

    def _result(self, mode: str) -> SetBatch:
        op = self.ops[mode]
        total, flags = (int(x) for x in op["result"].cpu())
        if flags:
            raise _lib.SubsetixError(f"batched {mode}: the sweep reported flags {flags}")
        rows = _t(self.A.combined.rows)
        s = IntervalSet._trusted(op["begin"][:total], op["end"][:total], op["offsets"], rows)
        return SetBatch(s, list(self.A.bases), list(self.A.heights))

    def union(self) -> SetBatch:
        return self._result("union")

    def intersection(self) -> SetBatch:
        return self._result("intersection")


__all__ = ["SetBatch", "BatchStep", "batched_binary", "batched_upwind"]
