"""Drop-in for the reference's ``subsetix_amr2`` package (two-level AMR on interval sets).

Names and semantics follow ``subsetix_amr2/__init__.py`` of the reference;
the device work runs on this package's sm_100a kernels.
"""

from .geometry import TwoLevelGeometry
from .regrid import gradient_tag_threshold_set, gradient_tag_set, enforce_two_level_grading_set
from .fields import synchronize_interval_fields
from .export import save_two_level_vtk
from .api import Box, MRAdaptor, TwoLevelMesh, make_scalar_field
from .runner import (
    OutputOptions,
    SimulationArgs,
    build_mesh,
    parse_simulation_args,
    run_two_level_simulation,
    save_snapshot,
    update_ghost,
)
from .simulation import (
    AMR2Simulation,
    AMRState,
    SimulationConfig,
    SimulationStats,
    SquareSpec,
    TwoLevelVTKExporter,
    build_square_interval_field,
)

__all__ = [
    "TwoLevelGeometry",
    "gradient_tag_set",
    "gradient_tag_threshold_set",
    "enforce_two_level_grading_set",
    "synchronize_interval_fields",
    "save_two_level_vtk",
    "Box",
    "TwoLevelMesh",
    "make_scalar_field",
    "MRAdaptor",
    "OutputOptions",
    "SimulationArgs",
    "parse_simulation_args",
    "build_mesh",
    "run_two_level_simulation",
    "save_snapshot",
    "update_ghost",
    "AMR2Simulation",
    "AMRState",
    "SimulationConfig",
    "SimulationStats",
    "SquareSpec",
    "TwoLevelVTKExporter",
    "build_square_interval_field",
]
