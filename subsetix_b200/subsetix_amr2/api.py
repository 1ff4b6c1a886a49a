"""Samurai-style two-level wrappers (drop-in for ``subsetix_amr2.api``).

Public names, arguments and exception types follow the reference's
``subsetix_amr2/api.py``: a :class:`TwoLevelMesh` over a :class:`Box` with
levels 0 and 1, :class:`ScalarField` objects holding one whole-grid
interval field per level, and :class:`MRAdaptor`, which re-tags the refine
region from the coarse gradient, re-injects the fine level and synchronises.

Design here: the mesh's state is its :class:`~.fields.ActionField` (one int8
byte per coarse cell on the device); its :class:`~.geometry.TwoLevelGeometry`
is derived from those bytes when first read after a regrid.  The adaptor runs
on whole-grid fields with three dense kernels (gradient tag plus grading into
action bytes, injection, synchronisation) and no host synchronisation;
fields replaced by other geometry take the interval kernels instead.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

from .._runtime import like
from ..subsetix_cupy.expressions import IntervalSet, _t
from ..subsetix_cupy.interval_field import IntervalField, create_interval_field, torch_dtype
from ..subsetix_cupy.morphology import full_interval_set
from ..subsetix_cupy.multilevel import prolong_field
from . import _dense
from .fields import ActionField, synchronize_interval_fields
from .geometry import TwoLevelGeometry
from .regrid import enforce_two_level_grading_set, gradient_tag_threshold_interval_field


@dataclass(frozen=True)
class Box:
    """Axis-aligned physical domain ``[min_corner, max_corner]``."""

    min_corner: tuple
    max_corner: tuple


def _require_set(x, where: str) -> IntervalSet:
    if not isinstance(x, IntervalSet):
        raise TypeError(f"{where} takes an IntervalSet, not {type(x).__name__}")
    return x


class TwoLevelMesh:
    """Square two-level mesh (levels 0 and 1) whose refine region is held as action bytes."""

    def __init__(self, box: Box, min_level: int, max_level: int, *, ratio: int = 2,
                 coarse_resolution: Optional[int] = None):
        if (int(min_level), int(max_level)) != (0, 1):
            raise ValueError(f"TwoLevelMesh has levels 0 and 1 only, got {min_level}..{max_level}")
        self.box = box
        self.min_level = int(min_level)
        self.max_level = int(max_level)
        self.ratio = int(ratio)
        self.actions: Optional[ActionField] = None
        self._geometry: Optional[TwoLevelGeometry] = None
        self._n: Optional[int] = None
        if coarse_resolution is not None:
            if int(coarse_resolution) <= 0:
                raise ValueError(f"coarse_resolution must be at least 1, got {coarse_resolution}")
            self._n = int(coarse_resolution)
            self.initialise()

    # -- geometry, derived from the action bytes on demand ------------------------------------------------------------
    @property
    def geometry(self) -> Optional[TwoLevelGeometry]:
        if self._geometry is None and self.actions is not None:
            self._geometry = TwoLevelGeometry.from_action_field(self.actions)
        return self._geometry

    @geometry.setter
    def geometry(self, value: Optional[TwoLevelGeometry]) -> None:
        self._geometry = value

    def _adopt(self, actions: ActionField) -> None:
        """Make ``actions`` the mesh's refine state; the geometry follows on first read."""
        self.actions = actions
        self._geometry = None
        self._n = int(actions.height)

    def _mark(self, n: int, refine: Optional[IntervalSet]) -> TwoLevelGeometry:
        actions = ActionField.full_grid(n, n, self.ratio)
        if refine is not None:
            actions.set_from_interval_set(refine)
        self._adopt(actions)
        return self.geometry

    # -- public -------------------------------------------------------------------------------------------------------
    def initialise(self, refine: IntervalSet | None = None) -> None:
        """Reset the mesh to its coarse resolution, with ``refine`` (if given) marked for refinement."""
        if self._n is None:
            raise RuntimeError("TwoLevelMesh.initialise() needs the coarse_resolution given at construction")
        if refine is not None and _require_set(refine, "TwoLevelMesh.initialise").row_count != self._n:
            raise ValueError(f"the refine set has {refine.row_count} rows, the mesh {self._n}")
        self._mark(self._n, refine)

    def regrid(self, refine: IntervalSet) -> TwoLevelGeometry:
        """Mark ``refine`` for refinement (a mesh without geometry takes its size from it)."""
        rows = _require_set(refine, "TwoLevelMesh.regrid").row_count
        if self.actions is None:
            if rows <= 0:
                raise ValueError("the refine set of a new mesh must have at least one row")
            n = self._n or rows
        else:
            n = int(self.actions.height)
            if rows != n:
                raise ValueError(f"the refine set has {rows} rows, the mesh {n}")
        return self._mark(n, refine)

    def cell_length(self, level: int) -> float:
        """Cell width of ``level`` in box units."""
        if self.actions is None:
            raise RuntimeError("the mesh has no geometry yet")
        dx0 = (self.box.max_corner[0] - self.box.min_corner[0]) / float(self.actions.width)
        return dx0 if level == self.min_level else dx0 / self.ratio


def _whole_grid_field(width: int, height: int, dtype) -> IntervalField:
    return create_interval_field(full_interval_set(width, height), fill_value=0.0, dtype=dtype)


class ScalarField:
    """One whole-grid interval field per level of a :class:`TwoLevelMesh`, zero-filled."""

    def __init__(self, name: str, mesh: TwoLevelMesh, *, dtype=np.float32):
        self.name = name
        self.mesh = mesh
        self.dtype = np.dtype(dtype)
        if mesh.actions is None:
            raise RuntimeError("initialise the mesh before creating fields on it")
        self.coarse_field, self.fine_field = self._fresh()

    def _fresh(self):
        n, r = int(self.mesh.actions.height), int(self.mesh.ratio)
        return _whole_grid_field(n, n, self.dtype), _whole_grid_field(n * r, n * r, self.dtype)

    def interval_field(self, level: int) -> IntervalField:
        return self.coarse_field if level == self.mesh.min_level else self.fine_field

    def set_interval_fields(self, *, coarse: IntervalField | None = None, fine: IntervalField | None = None) -> None:
        for name, f in (("coarse", coarse), ("fine", fine)):
            if f is not None and not isinstance(f, IntervalField):
                raise TypeError(f"{name} must be an IntervalField, not {type(f).__name__}")
        if coarse is not None:
            self.coarse_field = coarse
        if fine is not None:
            self.fine_field = fine

    def resize(self) -> None:
        """Fresh zero fields on the mesh's current levels."""
        if self.mesh.actions is None:
            raise RuntimeError("the mesh has no geometry yet")
        self.coarse_field, self.fine_field = self._fresh()

    def swap(self, other: "ScalarField") -> None:
        self.coarse_field, other.coarse_field = other.coarse_field, self.coarse_field
        self.fine_field, other.fine_field = other.fine_field, self.fine_field


def make_scalar_field(name: str, mesh: TwoLevelMesh, *, dtype=np.float32) -> ScalarField:
    return ScalarField(name, mesh, dtype=dtype)


class MRAdaptor:
    """Refine where the coarse gradient reaches the threshold, graded; then re-inject and synchronise the fine level.

    The step is the reference's ``MRAdaptor.__call__`` (``api.py:199-237``):
    tag, grade, regrid the mesh, replace the fine field by the injection of
    the coarse field, synchronise in place.
    """

    def __init__(self, field: ScalarField, *, refine_threshold: float, grading: int, mode: str = "von_neumann"):
        self.field = field
        self.mesh = field.mesh
        self.refine_threshold = float(refine_threshold)
        self.grading = int(grading)
        self.mode = mode

    def __call__(self) -> None:
        mesh, f = self.mesh, self.field
        if mesh.actions is None:
            raise RuntimeError("the mesh has no geometry yet")
        n, r = int(mesh.actions.height), int(mesh.ratio)
        coarse = _dense.grid_values(f.coarse_field, n, n)
        if coarse is not None and self.mode in ("von_neumann", "moore"):
            self._whole_grid(coarse, n, r)
        else:
            self._intervals(n, r)

    def _whole_grid(self, coarse: torch.Tensor, n: int, r: int) -> None:
        mesh, f = self.mesh, self.field
        actions = ActionField.full_grid(n, n, r)
        _dense.regrid(coarse, _t(actions.field.values).view(n, n), threshold=self.refine_threshold, epsilon=1e-8,
                      padding=self.grading, mode=self.mode)
        actions._refine_set_cache = None
        mesh._adopt(actions)
        fine_set = full_interval_set(n * r, n * r)
        fine = torch.empty((n * r, n * r), dtype=coarse.dtype, device=coarse.device)
        _dense.sync(coarse, fine, None, r)
        _dense.sync(coarse, fine, _t(actions.field.values).view(n, n), r)
        offsets = torch.arange(0, n * n * r * r + 1, n * r, dtype=torch.int32, device=coarse.device)
        f.fine_field = IntervalField(interval_set=fine_set, values=like(f.coarse_field.values, fine.view(-1)),
                                     interval_cell_offsets=like(fine_set.begin, offsets))

    def _intervals(self, n: int, r: int) -> None:
        mesh, f = self.mesh, self.field
        tags = gradient_tag_threshold_interval_field(f.coarse_field, width=n, height=n,
                                                     threshold=self.refine_threshold)
        mesh.regrid(enforce_two_level_grading_set(tags, padding=self.grading, mode=self.mode, width=n, height=n))
        dtype = np.float64 if _t(f.coarse_field.values).dtype == torch.float64 else np.float32
        f.fine_field = prolong_field(f.coarse_field, r, dtype=dtype)
        synchronize_interval_fields(f.coarse_field, f.fine_field, mesh.actions, ratio=r, reducer="mean",
                                    fill_fine_outside=True, copy=False)


__all__ = ["Box", "TwoLevelMesh", "ScalarField", "make_scalar_field", "MRAdaptor"]
