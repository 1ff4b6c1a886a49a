"""Drop-in for the reference's ``subsetix_cupy`` package (interval sets on the GPU).

Names and semantics follow ``subsetix_cupy/__init__.py`` of the reference.
The kernels behind them are this package's own sm_100a CUDA code, reached
through the C ABI in ``include/subsetix_b200.h``.
"""

from .expressions import (
    Expr,
    IntervalSet,
    CuPyWorkspace,
    build_interval_set,
    evaluate,
    make_difference,
    make_complement,
    make_input,
    make_intersection,
    make_symmetric_difference,
    make_union,
)
from .interval_field import IntervalField, create_interval_field, get_cell, set_cell, locate_interval_cells
from .multilevel import (
    MultiLevel2D,
    MultiLevelField2D,
    covered_by_fine,
    coarse_only,
    prolong_field,
    prolong_level_field,
    prolong_level_sets,
    prolong_set,
    restrict_field,
    restrict_level_field,
    restrict_level_sets,
    restrict_set,
)
from .morphology import (
    translate_interval_set,
    interior_for_direction,
    boundary_for_direction,
    boundary_layer,
    dilate_interval_set,
    erode_interval_set,
    full_interval_set,
    ghost_zones,
    clip_interval_set,
)
from .interval_stencil import step_upwind_interval, step_upwind_interval_field

__all__ = [
    "Expr",
    "IntervalSet",
    "CuPyWorkspace",
    "build_interval_set",
    "evaluate",
    "make_difference",
    "make_complement",
    "make_input",
    "make_intersection",
    "make_symmetric_difference",
    "make_union",
    "IntervalField",
    "create_interval_field",
    "get_cell",
    "set_cell",
    "locate_interval_cells",
    "MultiLevel2D",
    "MultiLevelField2D",
    "prolong_set",
    "restrict_set",
    "prolong_field",
    "restrict_field",
    "prolong_level_sets",
    "restrict_level_sets",
    "prolong_level_field",
    "restrict_level_field",
    "covered_by_fine",
    "coarse_only",
    "translate_interval_set",
    "interior_for_direction",
    "boundary_for_direction",
    "boundary_layer",
    "dilate_interval_set",
    "erode_interval_set",
    "ghost_zones",
    "full_interval_set",
    "clip_interval_set",
    "step_upwind_interval",
    "step_upwind_interval_field",
]
