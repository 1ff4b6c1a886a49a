"""Two-level AMR advection driver (drop-in for ``subsetix_amr2.simulation``).

Public classes, arguments and the order of a step follow the reference's
``AMR2Simulation`` (``subsetix_amr2/simulation.py:150-354``): a step is

    synchronize; regrid when the step index is a multiple of k;
    upwind on both levels; synchronize.

The reference accepts only a coarse field that covers the whole grid and
keeps the fine level as a whole grid too.  Every interval set of its loop is
therefore a rectangle or a mask on one, and this driver runs the loop on the
fused full-grid engine :class:`~.fused.FusedTwoLevelAMR`: one kernel per step
for upwind and synchronisation, one for gradient tagging plus grading, and
every whole regrid period replayed as one CUDA graph with no host
synchronisation.  The values are bit-identical to running the reference's
interval pipeline step by step.

The :class:`AMRState` handed to callbacks and returned by :meth:`run` is a
live view of the engine: its fields' ``values`` are the engine's current
buffers (writes to them feed the next step) and its action field reads the
engine's action bytes.  A view is valid until the next step; the interval
sets of the geometry are built from the action bytes only when asked for.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Dict, Iterable, List, Optional, Sequence

import numpy as np
import torch

from .._runtime import like
from ..subsetix_cupy.expressions import _t
from ..subsetix_cupy.interval_field import IntervalField, create_interval_field, torch_dtype
from ..subsetix_cupy.morphology import full_interval_set
from .export import save_two_level_vtk
from .fields import ActionField
from .fused import FusedTwoLevelAMR
from .geometry import TwoLevelGeometry

_GRADING_MODES = ("von_neumann", "moore")


@dataclass(frozen=True)
class SquareSpec:
    """Square ``[cx-hx, cx+hx] x [cy-hy, cy+hy]`` in unit coordinates holding ``value`` (``simulation.py:33-52``)."""

    center: tuple
    half_width: tuple
    value: float = 1.0


def _cell_span(lo: float, hi: float, n: int):
    """Cells ``i`` of an ``n``-cell axis whose position ``i / (n - 1)`` lies in ``[lo, hi]``, clamped to the axis."""
    scale = n - 1 if n > 1 else 1
    first = min(max(math.ceil(lo * scale), 0), n - 1)
    last = min(max(math.floor(hi * scale), 0), n - 1)
    return first, last


def build_square_interval_field(width: int, height: int, squares: Sequence[SquareSpec], *, dtype=np.float32
                                ) -> IntervalField:
    """Whole-grid field, zero except inside the squares (``simulation.py:55-97``); later squares overwrite earlier."""
    if width <= 0 or height <= 0:
        raise ValueError(f"grid must be non-empty, got {width} x {height}")
    specs = list(squares)
    if not specs:
        raise ValueError("build_square_interval_field needs at least one SquareSpec")
    field = create_interval_field(full_interval_set(width, height), fill_value=0.0, dtype=dtype)
    grid = _t(field.values).view(height, width)
    for spec in specs:
        x0, x1 = _cell_span(spec.center[0] - spec.half_width[0], spec.center[0] + spec.half_width[0], width)
        y0, y1 = _cell_span(spec.center[1] - spec.half_width[1], spec.center[1] + spec.half_width[1], height)
        if x0 <= x1 and y0 <= y1 and float(spec.value) != 0.0:
            grid[y0:y1 + 1, x0:x1 + 1] = float(spec.value)
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


class AMRState:
    """Coarse and fine fields, action field and geometry of a two-level run (``simulation.py:110-131``).

    ``geometry`` is derived from ``actions`` on first access unless given.
    """

    def __init__(self, coarse_field: IntervalField, fine_field: IntervalField, actions: ActionField,
                 geometry: Optional[TwoLevelGeometry] = None):
        self.coarse_field = coarse_field
        self.fine_field = fine_field
        self.actions = actions
        self._geometry = geometry

    @property
    def geometry(self) -> TwoLevelGeometry:
        if self._geometry is None:
            self._geometry = TwoLevelGeometry.from_action_field(self.actions)
        return self._geometry

    @geometry.setter
    def geometry(self, value: TwoLevelGeometry) -> None:
        self._geometry = value

    @property
    def coarse(self):
        return self.coarse_field.values.reshape(int(self.actions.height), int(self.actions.width))

    @property
    def fine(self):
        r = int(self.actions.ratio)
        return self.fine_field.values.reshape(int(self.actions.height) * r, int(self.actions.width) * r)

    def __repr__(self) -> str:
        return (f"AMRState(coarse={int(self.actions.height)}x{int(self.actions.width)}, "
                f"ratio={int(self.actions.ratio)}, dtype={_t(self.coarse_field.values).dtype})")


@dataclass(frozen=True)
class SimulationStats:
    step: int
    time: float
    dt: float
    dx_coarse: float
    dy_coarse: float
    ratio: int


Callback = Callable[[AMRState, SimulationStats], None]


def _check_config(cfg: SimulationConfig) -> None:
    if cfg.coarse_resolution <= 0:
        raise ValueError(f"coarse_resolution must be at least 1, got {cfg.coarse_resolution}")
    if cfg.ratio < 1:
        raise ValueError(f"refinement ratio must be at least 1, got {cfg.ratio}")
    if cfg.grading_mode not in _GRADING_MODES:
        raise ValueError(f"unknown grading_mode {cfg.grading_mode!r}; expected one of {_GRADING_MODES}")
    if not cfg.refine_threshold > 0.0:
        raise ValueError(f"refine_threshold must be positive, got {cfg.refine_threshold}")


def _whole_grid_values(field: IntervalField, width: int, height: int) -> torch.Tensor:
    """The values of ``field`` as a ``[height, width]`` tensor, after checking that it covers the whole grid."""
    if not isinstance(field, IntervalField):
        raise TypeError(f"expected an IntervalField, got {type(field).__name__}")
    s = field.interval_set
    if s.row_count != height:
        raise ValueError(f"the field has {s.row_count} rows, the grid {height}")
    rows = _t(s.rows)
    if not torch.equal(rows, torch.arange(height, dtype=rows.dtype, device=rows.device)):
        raise ValueError("the field's rows must be 0 .. height-1")
    off = _t(s.row_offsets)
    if not bool((off[1:] - off[:-1] == 1).all()):
        raise ValueError("the field must hold one interval per row")
    if not (bool((_t(s.begin) == 0).all()) and bool((_t(s.end) == width).all())):
        raise ValueError(f"every row of the field must be the interval [0, {width})")
    vals = _t(field.values)
    if int(vals.shape[0]) != width * height:
        raise ValueError(f"the field holds {int(vals.shape[0])} values, the grid {width * height} cells")
    return vals.view(height, width)


class AMR2Simulation:
    """Two-level advection with gradient-based regridding on the fused full-grid engine."""

    def __init__(self, config: SimulationConfig):
        _check_config(config)
        self.config = config
        self.width = self.height = int(config.coarse_resolution)
        self.dx_coarse = 1.0 / self.width
        self.dy_coarse = 1.0 / self.height
        self.dx_fine = self.dx_coarse / config.ratio
        self.dy_fine = self.dy_coarse / config.ratio
        rate = abs(config.velocity[0]) / self.dx_fine + abs(config.velocity[1]) / self.dy_fine
        self.dt = config.cfl / rate if rate > 0 else 0.0
        self.current_step = 0
        self.current_time = 0.0
        self._engine: Optional[FusedTwoLevelAMR] = None
        self._kind = None
        self._views = None
        self._cached = None

    # ------------------------------------------------------------------ setup
    def initialize_square(self, *, squares: Sequence[SquareSpec] | None = None, amplitude: float = 1.0,
                          dtype=np.float32) -> None:
        """Start from squares (the one default square when ``squares`` is None) scaled by ``amplitude``."""
        field = build_square_interval_field(self.width, self.height,
                                            list(squares) if squares is not None else _DEFAULT_SQUARES, dtype=dtype)
        if amplitude != 1.0:
            _t(field.values).mul_(float(np.dtype(dtype).type(float(amplitude))))
        self.set_initial_field(field)

    def set_initial_field(self, coarse_field: IntervalField) -> None:
        """Start from a whole-grid coarse field: refine from its gradient, fine level by injection."""
        values = _whole_grid_values(coarse_field, self.width, self.height)
        dtype = values.dtype if values.dtype in (torch.float32, torch.float64) else torch.float32
        cfg = self.config
        self._engine = FusedTwoLevelAMR(values, velocity=cfg.velocity, cfl=cfg.cfl,
                                        refine_threshold=cfg.refine_threshold, grading=cfg.grading,
                                        grading_mode=cfg.grading_mode, ratio=cfg.ratio, dtype=dtype)
        self._kind = coarse_field.values
        self._views = None
        self._cached = None
        self.current_step = 0
        self.current_time = 0.0

    @property
    def engine(self) -> FusedTwoLevelAMR:
        """The device engine (mass integrals, restriction defect, batched state)."""
        if self._engine is None:
            raise RuntimeError("call initialize_square() or set_initial_field() before running")
        return self._engine

    # ------------------------------------------------------------------ state
    def _domains(self):
        """Interval fields over the engine's buffers are rebuilt cheaply; their sets are made once."""
        if self._views is None:
            W, H, r = self.width, self.height, int(self.config.ratio)
            dev = self.engine.device
            coarse_set, fine_set = full_interval_set(W, H), full_interval_set(W * r, H * r)
            coarse_off = torch.arange(0, W * H + 1, W, dtype=torch.int32, device=dev)
            fine_off = torch.arange(0, W * H * r * r + 1, W * r, dtype=torch.int32, device=dev)
            self._views = (coarse_set, coarse_off, fine_set, fine_off)
        return self._views

    @property
    def state(self) -> Optional[AMRState]:
        """Live view of the current step (None before initialisation)."""
        if self._engine is None:
            return None
        eng = self._engine
        key = (eng.step_count, eng.cur)
        if self._cached is not None and self._cached[0] == key:
            return self._cached[1]
        coarse_set, coarse_off, fine_set, fine_off = self._domains()
        kind = self._kind
        coarse = IntervalField(interval_set=coarse_set, values=like(kind, eng.coarse_values[0].view(-1)),
                               interval_cell_offsets=like(coarse_set.begin, coarse_off))
        fine = IntervalField(interval_set=fine_set, values=like(kind, eng.fine_values[0].view(-1)),
                             interval_cell_offsets=like(fine_set.begin, fine_off))
        action_bytes = IntervalField(interval_set=coarse_set, values=like(kind, eng.actions[0].view(-1)),
                                     interval_cell_offsets=like(coarse_set.begin, coarse_off))
        actions = ActionField(field=action_bytes, ratio=int(self.config.ratio), width=self.width, height=self.height)
        view = AMRState(coarse_field=coarse, fine_field=fine, actions=actions)
        self._cached = (key, view)
        return view

    def _stats(self) -> SimulationStats:
        return SimulationStats(step=self.current_step, time=self.current_time, dt=self.dt, dx_coarse=self.dx_coarse,
                               dy_coarse=self.dy_coarse, ratio=self.config.ratio)

    def _notify(self, groups: List[List[Callback]]) -> tuple:
        state, stats = self.state, self._stats()
        for group in groups:
            for cb in group:
                cb(state, stats)
        return state, stats

    # ------------------------------------------------------------------ loop
    def run(self, *, steps: int, regrid_every: int = 1, exporters: Iterable[Callback] | None = None,
            listeners: Iterable[Callback] | None = None):
        """Advance ``steps`` steps; exporters then listeners are called before the first step and after each.

        Without callbacks the steps run as whole-period graph replays with no
        host synchronisation until the end; with callbacks each step is one
        replay followed by the callbacks.
        """
        eng = self.engine
        groups = [list(exporters or []), list(listeners or [])]
        period = max(1, int(regrid_every))
        state, stats = self._notify(groups)
        steps = int(steps)
        if steps <= 0:
            return state, stats
        if not any(groups):
            eng.run(steps, period)
            for _ in range(steps):
                self.current_step += 1
                self.current_time += self.dt
            return self.state, self._stats()
        for _ in range(steps):
            eng.run(1, period)
            self.current_step += 1
            self.current_time += self.dt
            state, stats = self._notify(groups)
        return state, stats


class TwoLevelVTKExporter:
    """Callback writing the state as VTK every ``every`` steps (``simulation.py:357-404``)."""

    def __init__(self, directory: str, *, prefix: str = "amr2", every: int = 1, ghost_halo: int = 0):
        self.directory = directory
        self.prefix = prefix
        self.every = max(1, int(every))
        self.ghost_halo = max(0, int(ghost_halo))

    def __call__(self, state: AMRState, stats: SimulationStats) -> Dict[str, str] | None:
        if stats.step % self.every:
            return None
        geo = state.geometry
        return save_two_level_vtk(self.directory, self.prefix, stats.step, coarse_field=state.coarse_field,
                                  fine_field=state.fine_field, refine_set=geo.refine,
                                  coarse_only_set=geo.coarse_only, fine_set=geo.fine, dx_coarse=stats.dx_coarse,
                                  dy_coarse=stats.dy_coarse, ratio=stats.ratio, time_value=stats.time,
                                  ghost_halo=self.ghost_halo, width=geo.width, height=geo.height)


# The square the reference's demo starts from (simulation.py:407-409).
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
