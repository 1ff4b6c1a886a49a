"""Two-level AMR geometry (drop-in for ``subsetix_amr2.geometry``).

A :class:`TwoLevelGeometry` names four interval sets of a two-level layout on
a regular ``width x height`` coarse grid (``subsetix_amr2/geometry.py:31-43``):
the coarse domain, the refine region, the refine region prolonged to the fine
grid, and the coarse cells outside the refine region.

Here all four come from one :class:`~.fields.ActionField`, which keeps its
int8 action bytes on the device and derives each set from them once
(value runs of the REFINE bytes, their prolongation, and the runs of every
other byte).  A geometry is therefore a cheap view of an action field, and
rebuilding it after a regrid costs one pass over the action bytes.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import TYPE_CHECKING, Optional

from ..subsetix_cupy import CuPyWorkspace, IntervalSet, evaluate, make_difference, make_input, prolong_set

if TYPE_CHECKING:
    from .fields import ActionField

_MODES = ("von_neumann", "moore")


@dataclass
class TwoLevelGeometry:
    """Coarse domain, refine region, fine region and coarse-only region of a two-level layout.

    ``workspace`` is kept for callers that evaluate expressions against the
    geometry's sets; the sets themselves never live in it.
    """

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
        """Geometry of an action field (``geometry.py:45-70``): every set is the field's cached one."""
        if min(int(actions.width), int(actions.height)) <= 0:
            raise ValueError("an action field with an empty grid has no geometry")
        return cls(ratio=int(actions.ratio), width=int(actions.width), height=int(actions.height),
                   coarse=actions.coarse_interval_set(), refine=actions.refine_set(), fine=actions.fine_set(),
                   coarse_only=actions.coarse_only_set(),
                   workspace=workspace if workspace is not None else CuPyWorkspace())

    def with_action_field(self, actions: "ActionField") -> "TwoLevelGeometry":
        """Geometry of ``actions`` that keeps this geometry's workspace (``geometry.py:72-81``)."""
        return type(self).from_action_field(actions, workspace=self.workspace)

    def dilate_refine(self, halo: int = 1, *, mode: str = "von_neumann") -> "TwoLevelGeometry":
        """Geometry whose refine region is grown by ``halo`` cells inside the domain (``geometry.py:83-124``).

        Growing the refine region this way is the 2:1 grading step: a box
        (``moore``) or a cross (``von_neumann``) dilation, united with the
        region and clipped to the grid.  The grading routine computes exactly
        that set, so it is reused here; the fine and coarse-only regions
        follow from the grown set.  ``halo <= 0`` returns this geometry.
        """
        from .regrid import enforce_two_level_grading_set

        halo = int(halo)
        if halo <= 0:
            return self
        if mode not in _MODES:
            raise ValueError(f"unknown dilation mode {mode!r}; expected one of {_MODES}")
        grown = enforce_two_level_grading_set(self.refine, padding=halo, mode=mode, width=self.width,
                                              height=self.height)
        rest = evaluate(make_difference(make_input(self.coarse), make_input(grown)))
        return TwoLevelGeometry(ratio=self.ratio, width=self.width, height=self.height, coarse=self.coarse,
                                refine=grown, fine=prolong_set(grown, self.ratio), coarse_only=rest.copy(),
                                workspace=self.workspace)


__all__ = ["TwoLevelGeometry"]
