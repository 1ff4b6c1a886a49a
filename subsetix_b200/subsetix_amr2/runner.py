"""Samurai-style two-level advection run (drop-in for ``subsetix_amr2.runner``).

The public dataclasses, ``parse_simulation_args`` (its flags and defaults are
the command-line contract) and the helpers keep the reference's names and
arguments (``subsetix_amr2/runner.py``).  A run follows the reference's time
loop (``runner.py:172-249``):

    adapt (tag, grade, regrid, re-inject the fine level, synchronise);
    synchronise again; upwind both levels with dt = min(cfl step, tf - t);
    swap the new levels in; write a snapshot when due.

On the whole-grid fields that :class:`~.api.ScalarField` creates, a step is
six dense launches with no host synchronisation (``_dense``); snapshots build
interval sets from the action bytes only when written.
"""

from __future__ import annotations

import argparse
import math
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Sequence

from ..subsetix_cupy.interval_stencil import step_upwind_interval_field
from . import _dense
from .api import Box, MRAdaptor, ScalarField, TwoLevelMesh, make_scalar_field
from .export import save_two_level_vtk
from .fields import synchronize_interval_fields


@dataclass(frozen=True)
class OutputOptions:
    directory: Path
    prefix: str = "amr2"
    every: int = 10
    ghost_halo: int = 1

    def __post_init__(self) -> None:
        if self.every <= 0:
            raise ValueError(f"snapshots need a positive interval, got every={self.every}")


@dataclass(frozen=True)
class SimulationArgs:
    """Domain, velocity, time span, levels and refinement settings of one run."""

    min_corner: tuple = (0.0, 0.0)
    max_corner: tuple = (1.0, 1.0)
    velocity: tuple = (1.0, 1.0)
    cfl: float = 0.5
    t0: float = 0.0
    tf: float = 0.1
    min_level: int = 4
    max_level: int = 5
    refine_threshold: float = 0.05
    grading: int = 1
    grading_mode: str = "von_neumann"
    output: OutputOptions | None = None


# flag, destination, argparse keywords: the command line of runner.py:52-80.
_FLAGS = (
    ("--min-corner", "min_corner", dict(type=float, nargs=2, default=(0.0, 0.0), help="lower box corner x y")),
    ("--max-corner", "max_corner", dict(type=float, nargs=2, default=(1.0, 1.0), help="upper box corner x y")),
    ("--velocity", "velocity", dict(type=float, nargs=2, default=(1.0, 1.0), help="advection velocity a b")),
    ("--cfl", "cfl", dict(type=float, default=0.5, help="CFL number on the fine level")),
    ("--Ti", "t0", dict(type=float, default=0.0, help="start time")),
    ("--Tf", "tf", dict(type=float, default=0.1, help="end time")),
    ("--min-level", "min_level", dict(type=int, default=4, help="coarse level (2**level cells per side)")),
    ("--max-level", "max_level", dict(type=int, default=5, help="fine level (min-level + 1)")),
    ("--refine-threshold", "refine_threshold", dict(type=float, default=0.05, help="gradient tag threshold")),
    ("--grading", "grading", dict(type=int, default=1, help="grading padding in coarse cells")),
    ("--grading-mode", "grading_mode", dict(type=str, choices=["von_neumann", "moore"], default="von_neumann",
                                            help="grading stencil")),
    ("--vtk-dir", "vtk_dir", dict(type=Path, default=None, help="write VTK snapshots into this folder")),
    ("--vtk-prefix", "vtk_prefix", dict(type=str, default="amr2", help="snapshot file prefix")),
    ("--vtk-every", "vtk_every", dict(type=int, default=10, help="steps between snapshots")),
    ("--ghost-halo", "ghost_halo", dict(type=int, default=1, help="ghost layer width in snapshots")),
)
_PAIRS = ("min_corner", "max_corner", "velocity")
_SCALARS = {"cfl": float, "t0": float, "tf": float, "min_level": int, "max_level": int,
            "refine_threshold": float, "grading": int, "grading_mode": str}


def parse_simulation_args(argv: Sequence[str] | None = None) -> SimulationArgs:
    """Command-line arguments of a run (the reference's flags and defaults)."""
    parser = argparse.ArgumentParser(description="two-level interval-set AMR advection")
    for flag, dest, kw in _FLAGS:
        parser.add_argument(flag, dest=dest, **kw)
    ns = vars(parser.parse_args(argv))
    values = {k: tuple(float(x) for x in ns[k]) for k in _PAIRS}
    values.update({k: cast(ns[k]) for k, cast in _SCALARS.items()})
    if ns["vtk_dir"] is not None:
        values["output"] = OutputOptions(directory=Path(ns["vtk_dir"]), prefix=str(ns["vtk_prefix"]),
                                         every=int(ns["vtk_every"]), ghost_halo=int(ns["ghost_halo"]))
    args = SimulationArgs(**values)
    _validate_args(args)
    return args


def _validate_args(args: SimulationArgs) -> None:
    if args.max_level - args.min_level != 1:
        raise ValueError(f"a two-level run needs max_level = min_level + 1, got {args.min_level}, {args.max_level}")
    if args.tf < args.t0:
        raise ValueError(f"end time {args.tf} precedes start time {args.t0}")
    if not args.refine_threshold > 0.0:
        raise ValueError(f"refine_threshold must be positive, got {args.refine_threshold}")


def build_mesh(args: SimulationArgs, ratio: int = 2) -> TwoLevelMesh:
    """Mesh of ``2**min_level`` coarse cells per side over the run's box."""
    return TwoLevelMesh(Box(args.min_corner, args.max_corner), 0, 1, ratio=ratio,
                        coarse_resolution=2 ** int(args.min_level))


def _mesh_parts(field: ScalarField):
    mesh = field.mesh
    if mesh.actions is None:
        raise RuntimeError("the mesh has no geometry yet")
    return mesh, int(mesh.actions.height), int(mesh.ratio)


def update_ghost(field: ScalarField) -> None:
    """Synchronise the two levels of ``field`` in place (restrict into refined cells, inject elsewhere)."""
    mesh, n, r = _mesh_parts(field)
    coarse = _dense.grid_values(field.coarse_field, n, n)
    fine = _dense.grid_values(field.fine_field, n * r, n * r)
    if coarse is not None and fine is not None and coarse.dtype == fine.dtype:
        from ..subsetix_cupy.expressions import _t

        _dense.sync(coarse, fine, _t(mesh.actions.field.values).view(n, n), r)
        return
    synchronize_interval_fields(field.coarse_field, field.fine_field, mesh.actions, ratio=r, reducer="mean",
                                fill_fine_outside=True, copy=False)


def save_snapshot(output: OutputOptions, mesh: TwoLevelMesh, field: ScalarField, step: int, *,
                  time_value: float) -> None:
    """Write both levels and the geometry of ``mesh`` as VTK files."""
    geo = mesh.geometry
    if geo is None:
        raise RuntimeError("the mesh has no geometry yet")
    (x0, y0), (x1, y1) = mesh.box.min_corner, mesh.box.max_corner
    save_two_level_vtk(os.fspath(output.directory), output.prefix, step, coarse_field=field.coarse_field,
                       fine_field=field.fine_field, refine_set=geo.refine, coarse_only_set=geo.coarse_only,
                       fine_set=geo.fine, dx_coarse=(x1 - x0) / geo.width, dy_coarse=(y1 - y0) / geo.height,
                       ratio=mesh.ratio, time_value=time_value, ghost_halo=output.ghost_halo, width=geo.width,
                       height=geo.height)


def _cfl_step(args: SimulationArgs, dx: float, dy: float) -> float:
    a, b = args.velocity
    rate = abs(a) / dx + abs(b) / dy
    dt = args.cfl / rate if rate > 0 else max(args.tf - args.t0, 0.0)
    if dt <= 0.0:
        raise ValueError(f"the time step is not positive (dt = {dt})")
    return dt


def _advance(field: ScalarField, nxt: ScalarField, n: int, r: int, args: SimulationArgs, dt: float,
             spacing) -> None:
    """Upwind both levels of ``field`` into ``nxt`` (whole grids in place, other geometry through intervals)."""
    (dx0, dy0), (dx1, dy1) = spacing
    a, b = args.velocity
    levels = ((field.coarse_field, nxt.coarse_field, n, dx0, dy0), (field.fine_field, nxt.fine_field, n * r, dx1, dy1))
    dense = [(_dense.grid_values(src, m, m), _dense.grid_values(dst, m, m)) for src, dst, m, _, _ in levels]
    if all(s is not None and d is not None and s.dtype == d.dtype for s, d in dense):
        for (s, d), (_, _, _, dx, dy) in zip(dense, levels):
            _dense.upwind(s, d, a=a, b=b, dt=dt, dx=dx, dy=dy)
        return
    new = [step_upwind_interval_field(src, width=m, height=m, a=a, b=b, dt=dt, dx=dx, dy=dy)
           for src, _, m, dx, dy in levels]
    nxt.set_interval_fields(coarse=new[0], fine=new[1])


def run_two_level_simulation(args: SimulationArgs, init_fn: Callable[[ScalarField], None]) -> ScalarField:
    """Advect ``u`` (initialised by ``init_fn``) from ``t0`` to ``tf``; returns the final field."""
    mesh = build_mesh(args)
    field = make_scalar_field("u", mesh)
    init_fn(field)
    update_ghost(field)
    adapt = MRAdaptor(field, refine_threshold=args.refine_threshold, grading=args.grading, mode=args.grading_mode)
    adapt()
    n, r = int(mesh.actions.height), int(mesh.ratio)
    dx0 = (args.max_corner[0] - args.min_corner[0]) / n
    dy0 = (args.max_corner[1] - args.min_corner[1]) / n
    spacing = ((dx0, dy0), (dx0 / r, dy0 / r))
    dt = _cfl_step(args, *spacing[1])
    if args.output is not None:
        args.output.directory.mkdir(parents=True, exist_ok=True)
        save_snapshot(args.output, mesh, field, 0, time_value=args.t0)
    nxt = make_scalar_field("unp1", mesh)
    t, step = args.t0, 0
    while t < args.tf:
        adapt()
        h = min(dt, args.tf - t)
        update_ghost(field)
        _advance(field, nxt, n, r, args, h, spacing)
        field.swap(nxt)
        t = min(args.tf, t + h)
        step += 1
        if args.output is not None and (step % args.output.every == 0 or math.isclose(t, args.tf)):
            save_snapshot(args.output, mesh, field, step, time_value=t)
    return field


__all__ = [
    "OutputOptions",
    "SimulationArgs",
    "parse_simulation_args",
    "build_mesh",
    "update_ghost",
    "save_snapshot",
    "run_two_level_simulation",
]
