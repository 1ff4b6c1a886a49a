"""ctypes bindings to ``libsubsetix_b200.so`` (declared in include/subsetix_b200.h).

The library must exist in-tree.  ``python -m subsetix_b200.build`` or
``__graft_entry__.build()`` produces it.  There is no fallback
implementation: if the library is missing or cannot load, every operation
raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsubsetix_b200.so")

SX_OK = 0
SX_ERR_INVALID = 1
SX_ERR_CUDA = 2
SX_ERR_CAPACITY = 3
SX_ERR_WORKSPACE = 4

MODE_TABLE = 0
MODE_UNION = 1

FLAG_CONTRACT = 1
FLAG_LONG_TILE = 2
FLAG_CAPACITY = 4
FLAG_TIMEOUT = 8

c_i32p = ctypes.POINTER(ctypes.c_int32)
c_vp = ctypes.c_void_p


class SxLeaf(ctypes.Structure):
    _fields_ = [("begin", c_vp), ("end", c_vp), ("row_offsets", c_vp), ("row_ends", c_vp), ("widen", ctypes.c_int32),
                ("scale", ctypes.c_int32)]


class SxTuning(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32), ("staging_cap", ctypes.c_int32),
                ("warps", ctypes.c_int32), ("tile_rows", ctypes.c_int32), ("wait_limit", ctypes.c_int32),
                ("withhold_tile", ctypes.c_int32)]


class SxRowList(ctypes.Structure):
    _fields_ = [("rows", c_vp), ("row_offsets", c_vp), ("count", ctypes.c_int32), ("shift", ctypes.c_int32),
                ("skip_empty", ctypes.c_int32), ("div", ctypes.c_int32), ("phase", ctypes.c_int32)]


# name -> (restype, argtypes)
_SIGNATURES = {
    "sx_abi_version": (ctypes.c_int, []),
    "sx_last_error": (ctypes.c_char_p, []),
    "sx_bool_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32]),
    "sx_bool_eval": (ctypes.c_int, [ctypes.POINTER(SxLeaf), ctypes.c_int, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, c_vp, c_vp, c_vp, ctypes.c_int64,
                                    c_vp, c_vp, ctypes.c_size_t, ctypes.POINTER(SxTuning), c_vp]),
    "sx_bool_eval_static": (ctypes.c_int, [ctypes.POINTER(SxLeaf), ctypes.c_int, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, c_vp, c_vp, c_vp,
                                           ctypes.c_int64, c_vp, c_vp]),
    "sx_exact_setop": (ctypes.c_int, [ctypes.c_int, ctypes.c_int32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                      c_vp, c_vp, c_vp]),
    "sx_merge_rows": (ctypes.c_int, [ctypes.c_int32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "sx_scan_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int64]),
    "sx_scan_i32": (ctypes.c_int, [c_vp, ctypes.c_int64, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_align_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32]),
    "sx_align_rows": (ctypes.c_int, [ctypes.POINTER(SxRowList), ctypes.c_int, ctypes.c_int32, ctypes.c_int32, c_vp,
                                     ctypes.c_int32, ctypes.POINTER(c_vp), ctypes.POINTER(c_vp), c_vp, c_vp,
                                     ctypes.c_size_t, c_vp]),
    "sx_tile_boundaries_max": (ctypes.c_int, [ctypes.POINTER(SxLeaf), ctypes.c_int, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_int32, c_vp, c_vp]),
    "sx_check_rows": (ctypes.c_int, [c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int64, c_vp, c_vp]),
    "sx_cell_offsets": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int64, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_prolong_set_workspace_bytes": (ctypes.c_size_t, [ctypes.c_int32]),
    "sx_prolong_set": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, c_vp,
                                      c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_prolong_field": (ctypes.c_int, [ctypes.c_int, c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp,
                                        ctypes.c_int32, c_vp, c_vp, c_vp]),
    "sx_prolong_field_f32": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp, ctypes.c_int32,
                                            c_vp, c_vp, c_vp]),
    "sx_prolong_field_f64": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp, ctypes.c_int32,
                                            c_vp, c_vp, c_vp]),
    "sx_coarse_fine_check": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp,
                                            ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int32, c_vp,
                                            c_vp]),
    "sx_restrict_field": (ctypes.c_int, [ctypes.c_int, c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp,
                                         ctypes.c_int32, ctypes.c_int, c_vp, c_vp, c_vp]),
    "sx_restrict_field_f32": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp, ctypes.c_int32,
                                             ctypes.c_int, c_vp, c_vp, c_vp]),
    "sx_restrict_field_f64": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, ctypes.c_int64, c_vp, c_vp, ctypes.c_int32,
                                             ctypes.c_int, c_vp, c_vp, c_vp]),
    "sx_subset_rows": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int32, ctypes.c_int64, c_vp, ctypes.c_int32, c_vp, c_vp,
                                      c_vp]),
    "sx_subset_copy": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                      ctypes.c_int32, c_vp, c_vp, ctypes.c_int, c_vp]),
    "sx_row_lookup": (ctypes.c_int, [c_vp, ctypes.c_int32, ctypes.c_int32, c_vp, c_vp, c_vp]),
    "sx_upwind": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64,
                                 ctypes.c_int64, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 c_vp]),
    "sx_upwind_plan": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int64, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_upwind_plan_fill": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp,
                                           ctypes.c_int64, c_vp, ctypes.c_int32, c_vp, c_vp]),
    "sx_upwind_plan_table": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp, c_vp]),
    "sx_upwind_chunked": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp, c_vp,
                                         c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, c_vp]),
    "sx_upwind_f32": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64,
                                     c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, c_vp]),
    "sx_upwind_f64": (ctypes.c_int, [c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64, ctypes.c_int64,
                                     c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     c_vp]),
    "sx_upwind_adjoint_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int64]),
    "sx_upwind_adjoint": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int64,
                                         ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_upwind_adjoint_chunked_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int64]),
    "sx_upwind_adjoint_chunked": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp,
                                                 c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 c_vp, c_vp, ctypes.c_size_t, c_vp]),
    "sx_threshold_rle": (ctypes.c_int, [c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_int, c_vp,
                                        c_vp, c_vp, c_vp, c_vp]),
    "sx_gradient_magnitude": (ctypes.c_int, [c_vp, ctypes.c_int32, ctypes.c_int32, c_vp, c_vp]),
    "sx_gradient_threshold_rle": (ctypes.c_int, [c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, c_vp, c_vp,
                                                 c_vp, c_vp, c_vp]),
    "sx_locate_cells": (ctypes.c_int, [c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, ctypes.c_int64, c_vp,
                                       c_vp]),
    "sx_value_runs": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                     c_vp]),
    "sx_gather_i32": (ctypes.c_int, [c_vp, ctypes.c_int32, c_vp, c_vp, c_vp]),
    "sx_upwind_band_table": (ctypes.c_int, [ctypes.c_int, c_vp, ctypes.c_int32, c_vp]),
    "sx_upwind_chunked_bands": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int64, c_vp, c_vp,
                                               c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                               ctypes.c_double, c_vp, c_vp, ctypes.c_int32, c_vp]),
    "sx_cell_quads": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, ctypes.c_int32, c_vp, c_vp, c_vp, ctypes.c_int32, c_vp,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, c_vp, c_vp, c_vp]),
    "sx_index_copy": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "sx_index_block_mean": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int32, ctypes.c_double, c_vp, c_vp,
                                           c_vp, c_vp, c_vp]),
    "sx_index_block_mean_adj": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int32, ctypes.c_double, c_vp,
                                               c_vp, c_vp, c_vp, c_vp]),
    "sx_index_segment_add": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int,
                                            c_vp]),
    "sx_upwind_full": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, c_vp]),
    "sx_amr_sync_full": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, c_vp]),
    "sx_amr_step_full": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, c_vp]),
    "sx_amr_regrid_full": (ctypes.c_int, [ctypes.c_int, c_vp, c_vp, c_vp, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_float, ctypes.c_int32, ctypes.c_int, c_vp]),
    "sx_mass_integral": (ctypes.c_int, [ctypes.c_int, c_vp, ctypes.c_int64, ctypes.c_double, c_vp, ctypes.c_int, c_vp,
                                        c_vp]),
    "sx_mass_integral_f64": (ctypes.c_int, [c_vp, ctypes.c_int64, ctypes.c_double, c_vp, ctypes.c_int, c_vp, c_vp]),
}

SX_F32 = 0
SX_F64 = 1

ROWS_UNSORTED_BEGIN = 1
ROWS_OVERLAP = 2
ROWS_EMPTY = 4
ROWS_TOUCH = 8
ROWS_UNSORTED_END = 16

_lock = threading.Lock()
_lib = None


class SubsetixError(RuntimeError):
    """A C-ABI call failed (CUDA error, capacity or workspace problem)."""


def load():
    """Load the shared library and bind every declared symbol."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m subsetix_b200.build` (no CPU fallback exists)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (restype, argtypes) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def exported_symbols():
    return list(_SIGNATURES)


def last_error() -> str:
    msg = load().sx_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc == SX_OK:
        return
    msg = last_error()
    if rc == SX_ERR_INVALID:
        raise ValueError(f"{what}: {msg}")
    raise SubsetixError(f"{what} failed ({rc}): {msg}")
