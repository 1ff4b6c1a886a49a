"""Samurai-style two-level advection driver (drop-in for ``subsetix_amr2.runner``).

Follows ``subsetix_amr2/runner.py`` of the reference: adapt, synchronise,
upwind both levels, swap, until ``tf``.
"""

from __future__ import annotations

import argparse
import math
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Callable, Sequence

from ..subsetix_cupy.interval_stencil import step_upwind_interval_field
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
            raise ValueError("OutputOptions.every must be > 0")


@dataclass(frozen=True)
class SimulationArgs:
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


def parse_simulation_args(argv: Sequence[str] | None = None) -> SimulationArgs:
    p = argparse.ArgumentParser(description="Samurai-style two-level AMR driver (subsetix)")
    p.add_argument("--min-corner", type=float, nargs=2, default=(0.0, 0.0))
    p.add_argument("--max-corner", type=float, nargs=2, default=(1.0, 1.0))
    p.add_argument("--velocity", type=float, nargs=2, default=(1.0, 1.0))
    p.add_argument("--cfl", type=float, default=0.5)
    p.add_argument("--Ti", dest="t0", type=float, default=0.0, help="Initial time")
    p.add_argument("--Tf", dest="tf", type=float, default=0.1, help="Final time")
    p.add_argument("--min-level", type=int, default=4)
    p.add_argument("--max-level", type=int, default=5)
    p.add_argument("--refine-threshold", type=float, default=0.05)
    p.add_argument("--grading", type=int, default=1)
    p.add_argument("--grading-mode", type=str, choices=["von_neumann", "moore"], default="von_neumann")
    p.add_argument("--vtk-dir", type=Path, default=None, help="Directory for VTK outputs")
    p.add_argument("--vtk-prefix", type=str, default="amr2")
    p.add_argument("--vtk-every", type=int, default=10)
    p.add_argument("--ghost-halo", type=int, default=1)
    ns = p.parse_args(argv)
    output = None
    if ns.vtk_dir is not None:
        output = OutputOptions(directory=Path(ns.vtk_dir), prefix=str(ns.vtk_prefix), every=int(ns.vtk_every),
                               ghost_halo=int(ns.ghost_halo))
    args = SimulationArgs(min_corner=tuple(float(v) for v in ns.min_corner),
                          max_corner=tuple(float(v) for v in ns.max_corner),
                          velocity=tuple(float(v) for v in ns.velocity), cfl=float(ns.cfl), t0=float(ns.t0),
                          tf=float(ns.tf), min_level=int(ns.min_level), max_level=int(ns.max_level),
                          refine_threshold=float(ns.refine_threshold), grading=int(ns.grading),
                          grading_mode=ns.grading_mode, output=output)
    _validate_args(args)
    return args


def _validate_args(args: SimulationArgs) -> None:
    if args.max_level != args.min_level + 1:
        raise ValueError("two-level driver expects max_level = min_level + 1")
    if args.tf < args.t0:
        raise ValueError("tf must be >= t0")
    if args.refine_threshold <= 0.0:
        raise ValueError("refine_threshold must be > 0")


def build_mesh(args: SimulationArgs, ratio: int = 2) -> TwoLevelMesh:
    return TwoLevelMesh(Box(args.min_corner, args.max_corner), 0, 1, ratio=ratio,
                        coarse_resolution=1 << args.min_level)


def update_ghost(field: ScalarField) -> None:
    if field.mesh.geometry is None:
        raise RuntimeError("mesh geometry not initialised")
    if field.mesh.actions is None:
        raise RuntimeError("mesh actions not initialised")
    synchronize_interval_fields(field.coarse_field, field.fine_field, field.mesh.actions, ratio=field.mesh.ratio,
                                reducer="mean", fill_fine_outside=True, copy=False)


def save_snapshot(output: OutputOptions, mesh: TwoLevelMesh, field: ScalarField, step: int, *,
                  time_value: float) -> None:
    g = mesh.geometry
    if g is None:
        raise RuntimeError("mesh geometry not initialised")
    save_two_level_vtk(os.fspath(output.directory), output.prefix, step, coarse_field=field.coarse_field,
                       fine_field=field.fine_field, refine_set=g.refine, coarse_only_set=g.coarse_only,
                       fine_set=g.fine, dx_coarse=(mesh.box.max_corner[0] - mesh.box.min_corner[0]) / g.width,
                       dy_coarse=(mesh.box.max_corner[1] - mesh.box.min_corner[1]) / g.height, ratio=mesh.ratio,
                       time_value=time_value, ghost_halo=output.ghost_halo, width=g.width, height=g.height)


def run_two_level_simulation(args: SimulationArgs, init_fn: Callable[[ScalarField], None]) -> ScalarField:
    """Run from ``t0`` to ``tf`` and return the final field (``runner.py:172-249``)."""
    mesh = build_mesh(args)
    field = make_scalar_field("u", mesh)
    init_fn(field)
    update_ghost(field)
    adaptor = MRAdaptor(field, refine_threshold=args.refine_threshold, grading=args.grading,
                        mode=args.grading_mode)
    adaptor()
    g = mesh.geometry
    assert g is not None
    a, b = args.velocity
    dx0 = (args.max_corner[0] - args.min_corner[0]) / g.width
    dy0 = (args.max_corner[1] - args.min_corner[1]) / g.height
    dx1, dy1 = dx0 / mesh.ratio, dy0 / mesh.ratio
    denom = abs(a) / dx1 + abs(b) / dy1
    dt = args.cfl / denom if denom > 0 else max(args.tf - args.t0, 0.0)
    if dt <= 0.0:
        raise ValueError("invalid CFL configuration (dt <= 0)")
    if args.output is not None:
        args.output.directory.mkdir(parents=True, exist_ok=True)
        save_snapshot(args.output, mesh, field, 0, time_value=args.t0)
    unp1 = make_scalar_field("unp1", mesh)
    t = args.t0
    step = 0
    while t < args.tf:
        adaptor()
        dt_step = min(dt, args.tf - t)
        update_ghost(field)
        unp1.resize()
        g = mesh.geometry
        if g is None:
            raise RuntimeError("mesh geometry not initialised")
        r = mesh.ratio
        coarse_next = step_upwind_interval_field(field.coarse_field, width=g.width, height=g.height, a=a, b=b,
                                                 dt=dt_step, dx=dx0, dy=dy0)
        fine_next = step_upwind_interval_field(field.fine_field, width=g.width * r, height=g.height * r, a=a, b=b,
                                               dt=dt_step, dx=dx1, dy=dy1)
        unp1.set_interval_fields(coarse=coarse_next, fine=fine_next)
        field.swap(unp1)
        t = min(args.tf, t + dt_step)
        step += 1
        if args.output is not None and (step % args.output.every == 0 or math.isclose(t, args.tf)):
            save_snapshot(args.output, mesh, field, step, time_value=t)
    return field


__all__ = ["OutputOptions", "SimulationArgs", "parse_simulation_args", "build_mesh", "update_ghost",
           "save_snapshot", "run_two_level_simulation"]
