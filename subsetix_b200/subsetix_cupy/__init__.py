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
]
