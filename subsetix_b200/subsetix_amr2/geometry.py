"""Two-level AMR geometry (drop-in for ``subsetix_amr2.geometry``).

Follows ``subsetix_amr2/geometry.py`` of the reference: the refine set,
its prolongation (fine set) and the coarse-only remainder, all computed on
the device with this package's set kernels.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import TYPE_CHECKING, Optional

from ..subsetix_cupy import (
    CuPyWorkspace,
    IntervalSet,
    clip_interval_set,
    dilate_interval_set,
    evaluate,
    make_difference,
    make_input,
    make_union,
    prolong_set,
)

if TYPE_CHECKING:
    from .fields import ActionField


def _clone_interval_set(interval_set: IntervalSet) -> IntervalSet:
    return interval_set.copy()


@dataclass
class TwoLevelGeometry:
    """Coarse domain, refine region, fine region and coarse-only region (``geometry.py:34-124``)."""

    ratio: int
    width: int
    height: int
    coarse: IntervalSet
    refine: IntervalSet
    fine: IntervalSet
    coarse_only: IntervalSet
    workspace: CuPyWorkspace

    @classmethod
    def from_action_field(cls, actions: "ActionField", *, workspace: Optional[CuPyWorkspace] = None
                          ) -> "TwoLevelGeometry":
        if actions.height <= 0 or actions.width <= 0:
            raise ValueError("action field must have positive dimensions")
        workspace = workspace or CuPyWorkspace()
        coarse = actions.coarse_interval_set()
        refine = actions.refine_set()
        fine = actions.fine_set()
        coarse_only = evaluate(make_difference(make_input(coarse), make_input(refine)), workspace=workspace)
        return cls(ratio=int(actions.ratio), width=actions.width, height=actions.height, coarse=coarse, refine=refine,
                   fine=fine, coarse_only=coarse_only, workspace=workspace)

    def with_action_field(self, actions: "ActionField") -> "TwoLevelGeometry":
        return TwoLevelGeometry.from_action_field(actions, workspace=self.workspace)

    def dilate_refine(self, halo: int = 1, *, mode: str = "von_neumann") -> "TwoLevelGeometry":
        """Grow the refine region by ``halo`` cells and rebuild the geometry (``geometry.py:83-124``)."""
        halo = int(halo)
        if halo <= 0:
            return self
        if mode not in {"von_neumann", "moore"}:
            raise ValueError("mode must be 'von_neumann' or 'moore'")
        if mode == "moore":
            dilated = dilate_interval_set(self.refine, halo_x=halo, halo_y=halo)
        else:
            horiz = dilate_interval_set(self.refine, halo_x=halo, halo_y=0)
            vert = dilate_interval_set(self.refine, halo_x=0, halo_y=halo)
            dilated = evaluate(make_union(make_input(horiz), make_input(vert)), workspace=self.workspace)
        dilated = clip_interval_set(dilated, width=self.width, height=self.height)
        refine_dense = clip_interval_set(self.refine, width=self.width, height=self.height)
        merged = evaluate(make_union(make_input(dilated), make_input(refine_dense)), workspace=self.workspace)
        clipped = clip_interval_set(merged, width=self.width, height=self.height)
        fine = prolong_set(clipped, self.ratio)
        coarse_only = evaluate(make_difference(make_input(self.coarse), make_input(clipped)), workspace=self.workspace)
        return TwoLevelGeometry(ratio=self.ratio, width=self.width, height=self.height, coarse=self.coarse,
                                refine=clipped, fine=fine, coarse_only=_clone_interval_set(coarse_only),
                                workspace=self.workspace)


__all__ = ["TwoLevelGeometry"]
