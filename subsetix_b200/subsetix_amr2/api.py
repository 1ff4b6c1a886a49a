"""Samurai-style wrappers (drop-in for ``subsetix_amr2.api``).

``Box``, ``TwoLevelMesh``, ``ScalarField``, ``make_scalar_field`` and
``MRAdaptor`` follow ``subsetix_amr2/api.py`` of the reference.  They are
thin host objects over this package's device sets and fields.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from ..subsetix_cupy.expressions import IntervalSet
from ..subsetix_cupy.interval_field import IntervalField, create_interval_field
from ..subsetix_cupy.morphology import full_interval_set
from ..subsetix_cupy.multilevel import prolong_field
from .fields import ActionField, synchronize_interval_fields
from .geometry import TwoLevelGeometry
from .regrid import enforce_two_level_grading_set, gradient_tag_threshold_interval_field


@dataclass(frozen=True)
class Box:
    """Axis-aligned bounding box."""

    min_corner: tuple
    max_corner: tuple


class TwoLevelMesh:
    """Two-level mesh over a square coarse grid (``api.py:33-137``)."""

    def __init__(self, box: Box, min_level: int, max_level: int, *, ratio: int = 2,
                 coarse_resolution: Optional[int] = None):
        if min_level != 0 or max_level != 1:
            raise ValueError("current implementation supports two levels (0/1) only")
        self.box = box
        self.min_level = min_level
        self.max_level = max_level
        self.ratio = int(ratio)
        self.geometry: Optional[TwoLevelGeometry] = None
        self._base_resolution: Optional[int] = None
        self._coarse_interval: Optional[IntervalSet] = None
        self.actions: Optional[ActionField] = None
        if coarse_resolution is not None:
            self._base_resolution = int(coarse_resolution)
            if self._base_resolution <= 0:
                raise ValueError("coarse_resolution must be positive")
            self.initialise()

    def initialise(self, refine: IntervalSet | None = None) -> None:
        if self._base_resolution is None:
            raise RuntimeError("TwoLevelMesh.initialise requires coarse_resolution at construction time")
        rows = width = self._base_resolution
        coarse = self._coarse_interval
        if coarse is None or coarse.row_count != rows:
            coarse = full_interval_set(width, rows)
            self._coarse_interval = coarse
        actions = ActionField.from_interval_set(coarse, width=width, height=rows, ratio=self.ratio)
        if refine is not None:
            if not isinstance(refine, IntervalSet):
                raise TypeError("TwoLevelMesh.initialise expects an IntervalSet")
            if int(refine.row_offsets.shape[0]) - 1 != rows:
                raise ValueError("refine IntervalSet height mismatch with mesh resolution")
            actions.set_from_interval_set(refine)
        self.geometry = TwoLevelGeometry.from_action_field(actions)
        self._coarse_interval = actions.coarse_interval_set()
        self.actions = actions

    def regrid(self, refine: IntervalSet) -> TwoLevelGeometry:
        if not isinstance(refine, IntervalSet):
            raise TypeError("TwoLevelMesh.regrid expects an IntervalSet")
        rows = int(refine.row_offsets.shape[0]) - 1
        if self.geometry is None:
            if rows <= 0:
                raise ValueError("refine IntervalSet must describe at least one row")
            width = self._base_resolution or rows
            coarse = self._coarse_interval
            if coarse is None or coarse.row_count != rows:
                coarse = full_interval_set(width, rows)
                self._coarse_interval = coarse
            actions = ActionField.from_interval_set(coarse, width=width, height=rows, ratio=self.ratio)
            actions.set_from_interval_set(refine)
            self.geometry = TwoLevelGeometry.from_action_field(actions)
            self._base_resolution = width
        else:
            if rows != self.geometry.height:
                raise ValueError("refine IntervalSet height mismatch with existing geometry")
            actions = ActionField.from_interval_set(self.geometry.coarse, width=self.geometry.width, height=rows,
                                                    ratio=self.ratio)
            actions.set_from_interval_set(refine)
            self.geometry = self.geometry.with_action_field(actions)
        self._coarse_interval = self.geometry.coarse
        self.actions = actions
        return self.geometry

    def cell_length(self, level: int) -> float:
        if self.geometry is None:
            raise RuntimeError("mesh geometry not initialised")
        dx0 = (self.box.max_corner[0] - self.box.min_corner[0]) / float(self.geometry.width)
        return dx0 if level == self.min_level else dx0 / self.ratio


class ScalarField:
    """Coarse and fine full-grid fields bound to a mesh (``api.py:140-190``)."""

    def __init__(self, name: str, mesh: TwoLevelMesh, *, dtype=np.float32):
        self.name = name
        self.mesh = mesh
        self.dtype = np.dtype(dtype)
        if mesh.geometry is None:
            raise RuntimeError("mesh.initialise() must run before creating fields")
        self.resize()

    def interval_field(self, level: int) -> IntervalField:
        return self.coarse_field if level == self.mesh.min_level else self.fine_field

    def set_interval_fields(self, *, coarse: IntervalField | None = None, fine: IntervalField | None = None) -> None:
        if coarse is not None:
            if not isinstance(coarse, IntervalField):
                raise TypeError("coarse must be an IntervalField")
            self.coarse_field = coarse
        if fine is not None:
            if not isinstance(fine, IntervalField):
                raise TypeError("fine must be an IntervalField")
            self.fine_field = fine

    def resize(self) -> None:
        g = self.mesh.geometry
        if g is None:
            raise RuntimeError("mesh geometry not initialised")
        r = self.mesh.ratio
        self.coarse_field = create_interval_field(full_interval_set(g.width, g.height), fill_value=0.0,
                                                  dtype=self.dtype)
        self.fine_field = create_interval_field(full_interval_set(g.width * r, g.height * r), fill_value=0.0,
                                                dtype=self.dtype)

    def swap(self, other: "ScalarField") -> None:
        self.coarse_field, other.coarse_field = other.coarse_field, self.coarse_field
        self.fine_field, other.fine_field = other.fine_field, self.fine_field


def make_scalar_field(name: str, mesh: TwoLevelMesh, *, dtype=np.float32) -> ScalarField:
    return ScalarField(name, mesh, dtype=dtype)


class MRAdaptor:
    """Gradient tagging, grading, regrid, then prolongation and synchronisation (``api.py:197-237``)."""

    def __init__(self, field: ScalarField, *, refine_threshold: float, grading: int, mode: str = "von_neumann"):
        self.field = field
        self.mesh = field.mesh
        self.refine_threshold = float(refine_threshold)
        self.grading = int(grading)
        self.mode = mode

    def __call__(self) -> None:
        g = self.mesh.geometry
        if g is None:
            raise RuntimeError("mesh geometry not initialised")
        tags = gradient_tag_threshold_interval_field(self.field.coarse_field, width=g.width, height=g.height,
                                                     threshold=self.refine_threshold)
        graded = enforce_two_level_grading_set(tags, padding=self.grading, mode=self.mode, width=g.width,
                                               height=g.height)
        self.mesh.regrid(graded)
        dtype = np.float64 if self.field.dtype == np.float64 else np.float32
        self.field.fine_field = prolong_field(self.field.coarse_field, self.mesh.ratio, dtype=dtype)
        if self.mesh.actions is None:
            raise RuntimeError("mesh actions not initialised")
        synchronize_interval_fields(self.field.coarse_field, self.field.fine_field, self.mesh.actions,
                                    ratio=self.mesh.ratio, reducer="mean", fill_fine_outside=True, copy=False)


__all__ = ["Box", "TwoLevelMesh", "ScalarField", "make_scalar_field", "MRAdaptor"]
