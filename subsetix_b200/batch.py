"""Many independent interval sets evaluated together, one launch per operation.

A batch lays its sets on disjoint row bands of one combined set: set ``i``
occupies rows ``base_i + row``, and consecutive bands are separated by at
least one empty row.  Row-wise operations (set algebra, morphology along
x) never mix rows, so one launch over the combined set evaluates the
operation for every set at once.  The upwind step reads rows ``y - 1`` and
``y + 1``, which are empty between bands, so the zero-exterior update of each
set is unchanged as long as every set lies inside its own domain
``[0, width_i) x [0, height_i)``.

This is the batching the reference lacks: there every set is one Python
call with its own launches and host synchronisations.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np
import torch

from . import _core, _lib
from .subsetix_cupy.expressions import IntervalSet, _t, apply_binary
from .subsetix_cupy.interval_field import IntervalField, create_interval_field
from .subsetix_cupy.interval_stencil import step_upwind_interval

I32 = torch.int32


@dataclass
class SetBatch:
    """Sets on disjoint row bands of ``combined``.

    ``bases[i]`` is the first row of band ``i`` and ``heights[i]`` its
    height (the set's rows lie in ``[0, heights[i])``).
    """

    combined: IntervalSet
    bases: List[int]
    heights: List[int]

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


def batched_binary(lhs: SetBatch, rhs: SetBatch, mode: str) -> SetBatch:
    """``mode`` ("union", "intersection", "difference", "symmetric_difference") of every pair, one launch."""
    if lhs.bases != rhs.bases:
        raise ValueError("batches must share their band layout")
    return SetBatch(apply_binary(lhs.combined, rhs.combined, mode), list(lhs.bases), list(lhs.heights))


def batched_upwind(batch: SetBatch, values: torch.Tensor, *, width: int, a: float, b: float, dt: float, dx: float,
                   dy: float, out: torch.Tensor | None = None) -> torch.Tensor:
    """One upwind step of every set's field (values stored set after set, row by row), one launch.

    Every set must lie in ``[0, width) x [0, height_i)``; the steps of the
    sets do not interact (empty rows separate the bands).
    """
    total_rows = batch.bases[-1] + batch.heights[-1] + 1
    field = IntervalField(interval_set=batch.combined, values=values,
                          interval_cell_offsets=_core.cell_offsets(_t(batch.combined.begin), _t(batch.combined.end),
                                                                   values.device)[0])
    return step_upwind_interval(field, width=width, height=total_rows, a=a, b=b, dt=dt, dx=dx, dy=dy, out=out)


__all__ = ["SetBatch", "batched_binary", "batched_upwind"]
