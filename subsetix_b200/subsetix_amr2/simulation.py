"""Two-level AMR advection driver (drop-in for ``subsetix_amr2.simulation``).

The time loop, its order of operations and the public classes follow
``subsetix_amr2/simulation.py`` of the reference:

    for each step: synchronize; regrid every k steps; upwind on both levels;
    synchronize.

Every kernel underneath is this package's own.  Float32 fields follow the
reference.  A float64 initial field runs the whole loop in float64 (both
levels, restriction and prolongation), which the reference does not support.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Dict, Iterable, Sequence

import numpy as np
import torch

from ..subsetix_cupy.expressions import IntervalSet, _t
from ..subsetix_cupy.interval_field import IntervalField, create_interval_field, torch_dtype
from ..subsetix_cupy.interval_stencil import step_upwind_interval_field
from ..subsetix_cupy.morphology import full_interval_set
from ..subsetix_cupy.multilevel import prolong_field
from .export import save_two_level_vtk
from .fields import Action, ActionField, synchronize_interval_fields
from .geometry import TwoLevelGeometry
from .regrid import enforce_two_level_grading_set, gradient_tag_threshold_interval_field


@dataclass(frozen=True)
class SquareSpec:
    """Square patch ``[cx-hx, cx+hx] x [cy-hy, cy+hy]`` in unit coordinates with a value (``simulation.py:33-52``)."""

    center: tuple
    half_width: tuple
    value: float = 1.0


def build_square_interval_field(width: int, height: int, squares: Sequence[SquareSpec], *, dtype=np.float32
                                ) -> IntervalField:
    """Full-grid field with axis-aligned squares painted in (``simulation.py:55-97``).

    Cell ``i`` of an axis sits at ``i / (n - 1)``; a square covers the cells
    from ``ceil(lower)`` to ``floor(upper)`` on each axis.
    """
    if width <= 0 or height <= 0:
        raise ValueError("width and height must be positive")
    specs = list(squares)
    if not specs:
        raise ValueError("at least one SquareSpec is required")
    field = create_interval_field(full_interval_set(width, height), fill_value=0.0, dtype=dtype)
    grid = _t(field.values).view(height, width)
    xs = width - 1 if width > 1 else 1
    ys = height - 1 if height > 1 else 1
    for spec in specs:
        cx, cy = spec.center
        hx, hy = spec.half_width
        x0 = max(0, min(width - 1, math.ceil((cx - hx) * xs)))
        x1 = max(0, min(width - 1, math.floor((cx + hx) * xs)))
        y0 = max(0, min(height - 1, math.ceil((cy - hy) * ys)))
        y1 = max(0, min(height - 1, math.floor((cy + hy) * ys)))
        if x0 > x1 or y0 > y1:
            continue
        value = float(spec.value)
        if value == 0.0:
            continue
        grid[y0:y1 + 1, x0:x1 + 1] = value
    return field


@dataclass(frozen=True)
class SimulationConfig:
    coarse_resolution: int
    velocity: tuple
    cfl: float = 0.9
    refine_threshold: float = 0.05
    grading: int = 1
    grading_mode: str = "von_neumann"
    ratio: int = 2


@dataclass
class AMRState:
    coarse_field: IntervalField
    fine_field: IntervalField
    actions: ActionField
    geometry: TwoLevelGeometry

    @property
    def coarse(self):
        return self.coarse_field.values.reshape(self.geometry.height, self.geometry.width)

    @property
    def fine(self):
        r = self.geometry.ratio
        return self.fine_field.values.reshape(self.geometry.height * r, self.geometry.width * r)


@dataclass(frozen=True)
class SimulationStats:
    step: int
    time: float
    dt: float
    dx_coarse: float
    dy_coarse: float
    ratio: int


Callback = Callable[[AMRState, SimulationStats], None]


class AMR2Simulation:
    """Two-level advection with gradient-based regridding (``simulation.py:142-354``)."""

    def __init__(self, config: SimulationConfig):
        self.config = config
        self._validate_config()
        self.width = int(config.coarse_resolution)
        self.height = self.width
        self.dx_coarse = 1.0 / self.width
        self.dy_coarse = 1.0 / self.height
        self.dx_fine = self.dx_coarse / config.ratio
        self.dy_fine = self.dy_coarse / config.ratio
        denom = abs(config.velocity[0]) / self.dx_fine + abs(config.velocity[1]) / self.dy_fine
        self.dt = config.cfl / denom if denom > 0 else 0.0
        self.state = None
        self.current_step = 0
        self.current_time = 0.0

    # ---------------------------------------------------------------- public
    def initialize_square(self, *, squares: Sequence[SquareSpec] | None = None, amplitude: float = 1.0,
                          dtype=np.float32) -> None:
        specs = list(squares) if squares is not None else _DEFAULT_SQUARES
        coarse = build_square_interval_field(self.width, self.height, specs, dtype=dtype)
        if amplitude != 1.0:
            v = _t(coarse.values)
            v.mul_(float(np.dtype(dtype).type(float(amplitude))))
        self.set_initial_field(coarse)

    def set_initial_field(self, coarse_field: IntervalField) -> None:
        if not isinstance(coarse_field, IntervalField):
            raise TypeError("coarse_field must be an IntervalField")
        h, w = self.height, self.width
        s = coarse_field.interval_set
        if s.row_count != h:
            raise ValueError("coarse_field height mismatch with simulation domain")
        rows = _t(s.rows)
        if rows.numel() != h or not torch.equal(rows, torch.arange(h, dtype=rows.dtype, device=rows.device)):
            raise ValueError("coarse_field rows must match the simulation row ids [0, height)")
        off = _t(s.row_offsets)
        if not bool(((off[1:] - off[:-1]) == 1).all()):
            raise ValueError("coarse_field must contain exactly one interval per row")
        if not bool((_t(s.begin) == 0).all()) or not bool((_t(s.end) == w).all()):
            raise ValueError("coarse_field must cover the full width on every row")
        if int(coarse_field.values.shape[0]) != w * h:
            raise ValueError("coarse_field must hold width * height cells")
        refine = self._refine_from_gradient(coarse_field)
        actions = ActionField.full_grid(h, w, self.config.ratio, default=Action.KEEP)
        actions.set_from_interval_set(refine)
        geometry = self._build_geometry(actions)
        fine_field = prolong_field(coarse_field, self.config.ratio, dtype=self._dtype(coarse_field))
        self.state = AMRState(coarse_field=coarse_field, fine_field=fine_field, actions=actions, geometry=geometry)
        self.current_step = 0
        self.current_time = 0.0

    def run(self, *, steps: int, regrid_every: int = 1, exporters: Iterable[Callback] | None = None,
            listeners: Iterable[Callback] | None = None):
        state = self._require_state()
        exporters_list = list(exporters or [])
        listeners_list = list(listeners or [])
        stats = self._build_stats(step=self.current_step)
        self._dispatch(exporters_list, state, stats)
        self._dispatch(listeners_list, state, stats)
        period = max(1, int(regrid_every))
        for _ in range(int(steps)):
            self._synchronize()
            if self.current_step % period == 0:
                self._update_geometry()
            self._advance()
            self._synchronize()
            self.current_step += 1
            self.current_time += self.dt
            state = self._require_state()
            stats = self._build_stats(step=self.current_step)
            self._dispatch(exporters_list, state, stats)
            self._dispatch(listeners_list, state, stats)
        return state, stats

    # ------------------------------------------------------------- internals
    @staticmethod
    def _dtype(field: IntervalField):
        return np.float64 if _t(field.values).dtype == torch.float64 else np.float32

    def _validate_config(self) -> None:
        if self.config.coarse_resolution <= 0:
            raise ValueError("coarse_resolution must be positive")
        if self.config.ratio < 1:
            raise ValueError("ratio must be >= 1")
        if self.config.grading_mode not in {"von_neumann", "moore"}:
            raise ValueError("grading_mode must be 'von_neumann' or 'moore'")
        if self.config.refine_threshold <= 0.0:
            raise ValueError("refine_threshold must be > 0")

    def _require_state(self) -> AMRState:
        if self.state is None:
            raise RuntimeError("simulation not initialised")
        return self.state

    @staticmethod
    def _dispatch(callbacks, state, stats) -> None:
        for cb in callbacks:
            cb(state, stats)

    def _refine_from_gradient(self, field: IntervalField) -> IntervalSet:
        tagged = gradient_tag_threshold_interval_field(field, width=self.width, height=self.height,
                                                       threshold=self.config.refine_threshold)
        return enforce_two_level_grading_set(tagged, padding=self.config.grading, mode=self.config.grading_mode,
                                             width=self.width, height=self.height)

    def _build_geometry(self, actions: ActionField, workspace=None) -> TwoLevelGeometry:
        return TwoLevelGeometry.from_action_field(actions, workspace=workspace)

    def _synchronize(self) -> None:
        state = self._require_state()
        synchronize_interval_fields(state.coarse_field, state.fine_field, state.actions, ratio=self.config.ratio,
                                    reducer="mean", fill_fine_outside=True, copy=False)

    def _update_geometry(self) -> None:
        state = self._require_state()
        refine = self._refine_from_gradient(state.coarse_field)
        state.actions.set_from_interval_set(refine)
        workspace = state.geometry.workspace if state.geometry is not None else None
        state.geometry = self._build_geometry(state.actions, workspace=workspace)

    def _advance(self) -> None:
        state = self._require_state()
        a, b = self.config.velocity
        g = state.geometry
        r = g.ratio
        state.coarse_field = step_upwind_interval_field(state.coarse_field, width=g.width, height=g.height, a=a, b=b,
                                                        dt=self.dt, dx=self.dx_coarse, dy=self.dy_coarse)
        state.fine_field = step_upwind_interval_field(state.fine_field, width=g.width * r, height=g.height * r, a=a,
                                                      b=b, dt=self.dt, dx=self.dx_fine, dy=self.dy_fine)

    def _build_stats(self, *, step: int) -> SimulationStats:
        return SimulationStats(step=step, time=self.current_time, dt=self.dt, dx_coarse=self.dx_coarse,
                               dy_coarse=self.dy_coarse, ratio=self.config.ratio)


class TwoLevelVTKExporter:
    """Callback that writes the state to VTK every ``every`` steps (``simulation.py:357-404``)."""

    def __init__(self, directory: str, *, prefix: str = "amr2", every: int = 1, ghost_halo: int = 0):
        self.directory = directory
        self.prefix = prefix
        self.every = max(1, int(every))
        self.ghost_halo = max(0, int(ghost_halo))

    def __call__(self, state: AMRState, stats: SimulationStats) -> Dict[str, str] | None:
        if stats.step % self.every != 0:
            return None
        return save_two_level_vtk(self.directory, self.prefix, stats.step, coarse_field=state.coarse_field,
                                  fine_field=state.fine_field, refine_set=state.actions.refine_set(),
                                  coarse_only_set=state.geometry.coarse_only, fine_set=state.geometry.fine,
                                  dx_coarse=stats.dx_coarse, dy_coarse=stats.dy_coarse, ratio=stats.ratio,
                                  time_value=stats.time, ghost_halo=self.ghost_halo, width=state.geometry.width,
                                  height=state.geometry.height)


_DEFAULT_SQUARES = [SquareSpec(center=(0.30, 0.30), half_width=(0.10, 0.10))]

__all__ = [
    "AMR2Simulation",
    "AMRState",
    "SimulationConfig",
    "SimulationStats",
    "SquareSpec",
    "TwoLevelVTKExporter",
    "build_square_interval_field",
]
