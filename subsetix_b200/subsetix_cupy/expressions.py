"""Interval sets and lazy set-algebra expressions (drop-in for ``subsetix_cupy.expressions``).

Public names, argument meanings and exceptions follow the reference module
(``subsetix_cupy/expressions.py``).  The compute path is new.

* A whole expression tree is compiled into one truth table over its distinct
  leaves, up to 8 of them.  The tree is evaluated by one fused kernel launch
  (``sx_bool_eval``) instead of one count/scan/write round trip per binary
  node.  Trees with more leaves are split at the root.
* Inputs outside the fused path's contract (touching, overlapping, empty or
  unsorted intervals in a row) are detected on the device.  The same tree is
  then re-evaluated node by node with the exact reference-order kernels, so
  the result is the reference's for every input.
* Arrays are torch tensors.  CuPy arrays are accepted without copying, and
  CuPy inputs give CuPy outputs.  No CPU path exists: without a CUDA device
  every operation raises.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _core, _lib
from .._runtime import current_device, is_cupy, like, to_tensor

try:  # the reference exposes the CuPy module it runs on; None when CuPy is absent
    import cupy as _REAL_CUPY  # type: ignore
except Exception:  # pragma: no cover
    _REAL_CUPY = None

I32 = torch.int32


def _require_cupy():
    """Array module for results: CuPy when installed, torch otherwise."""
    return _REAL_CUPY if _REAL_CUPY is not None else torch


def _t(x) -> torch.Tensor:
    return to_tensor(x)


def _i32(x, device=None) -> torch.Tensor:
    if isinstance(x, (list, tuple)) or (isinstance(x, np.ndarray)):
        arr = np.asarray(x, dtype=np.int32).reshape(-1) if len(np.shape(x)) else np.asarray(x, dtype=np.int32)
        return torch.as_tensor(arr, device=device or current_device())
    return to_tensor(x, dtype=I32, device=device)


def _dtype_ok(x) -> bool:
    if isinstance(x, torch.Tensor):
        return x.dtype == torch.int32
    if is_cupy(x):
        return x.dtype == np.int32
    return np.asarray(x).dtype == np.int32


@dataclass(frozen=True)
class IntervalSet:
    """Half-open ``[begin, end)`` intervals in compressed-row layout.

    The invariants are the reference's (``expressions.py:144-227``):
    ``row_offsets`` has ``row_count + 1`` entries and starts at 0, and its
    last entry is the interval count.  ``rows`` is one-dimensional, strictly
    increasing, and ``row_count`` long.
    """

    begin: Any
    end: Any
    row_offsets: Any
    rows: Any

    def __post_init__(self) -> None:
        for name in ("begin", "end", "row_offsets"):
            if not _dtype_ok(getattr(self, name)):
                raise TypeError(f"{name} must use int32 precision")
        b, e, off = self.begin, self.end, self.row_offsets
        if tuple(b.shape) != tuple(e.shape):
            raise ValueError("begin and end must share the same shape")
        if len(off.shape) != 1:
            raise ValueError("row_offsets must be one-dimensional")
        if self.rows is None:
            raise ValueError("rows must be provided")
        rows = self.rows
        if not (isinstance(rows, torch.Tensor) or is_cupy(rows)):
            rows = _i32(rows, device=_t(off).device if (isinstance(off, torch.Tensor) or is_cupy(off)) else None)
            rows = like(self.begin, rows)
        elif not _dtype_ok(rows):
            rows = like(rows, _t(rows).to(I32))
        if len(rows.shape) != 1:
            raise ValueError("rows must be one-dimensional")
        offt = _t(off)
        nint = int(np.prod(b.shape)) if len(b.shape) else 1
        R = int(offt.numel()) - 1
        if int(rows.shape[0]) != R:
            # checked after the first/last entries in the reference; both raise ValueError
            first = int(offt[0]) if offt.numel() else 0
            if first != 0:
                raise ValueError("row_offsets must start at zero")
            if int(offt[-1]) != nint:
                raise ValueError("row_offsets last entry must match interval count")
            raise ValueError("rows length must match row_offsets size - 1")
        # one synchronising read covers the three value checks
        rt = _t(rows)
        checks = torch.stack([
            offt[0] != 0,
            offt[-1] != nint,
            (rt[1:] <= rt[:-1]).any() if R > 1 else torch.zeros((), dtype=torch.bool, device=offt.device),
        ]).cpu()
        if bool(checks[0]):
            raise ValueError("row_offsets must start at zero")
        if bool(checks[1]):
            raise ValueError("row_offsets last entry must match interval count")
        if bool(checks[2]):
            raise ValueError("rows must be strictly increasing")
        object.__setattr__(self, "rows", rows)

    @classmethod
    def _trusted(cls, begin, end, row_offsets, rows, dense: Optional[int] = None) -> "IntervalSet":
        """Build without validation (outputs of this package's own kernels)."""
        obj = object.__new__(cls)
        object.__setattr__(obj, "begin", begin)
        object.__setattr__(obj, "end", end)
        object.__setattr__(obj, "row_offsets", row_offsets)
        object.__setattr__(obj, "rows", rows)
        if dense is not None:
            object.__setattr__(obj, "_dense_rows", int(dense))
        return obj

    @property
    def row_count(self) -> int:
        return int(self.row_offsets.shape[0] - 1)

    def rows_index(self):
        return self.rows

    def interval_rows(self):
        """Row id of every interval (``expressions.py:236-249``)."""
        off = _t(self.row_offsets)
        n = int(self.begin.shape[0]) if len(self.begin.shape) else 0
        if off.numel() <= 1 or n == 0:
            return like(self.begin, torch.zeros(0, dtype=I32, device=off.device))
        counts = (off[1:] - off[:-1]).to(torch.int64)
        return like(self.begin, torch.repeat_interleave(_t(self.rows), counts, output_size=n))

    def copy(self) -> "IntervalSet":
        c = lambda x: like(x, _t(x).clone())  # noqa: E731
        return IntervalSet._trusted(c(self.begin), c(self.end), c(self.row_offsets), c(self.rows),
                                    getattr(self, "_dense_rows", None))


def _dense_key(s: IntervalSet) -> Optional[int]:
    return getattr(s, "_dense_rows", None)


class CuPyWorkspace:
    """Reusable output storage for evaluations.

    Output buffers are pooled across iterations.  A result produced with a
    workspace may be recycled by the next top-level :func:`evaluate` call;
    copy it if it must outlive that call (``expressions.py:261-325``).
    Unlike the reference, intermediate nodes never share a buffer with
    their operands, so nested expressions and xor are also correct with a
    workspace.
    """

    def __init__(self, cp_module=None):
        self._cp = cp_module
        self._counts = None
        self._counts_capacity = 0
        self._offsets = None
        self._offsets_capacity = 0
        self._buffers: List[Tuple[torch.Tensor, torch.Tensor]] = []
        self._buffers_capacity: List[int] = []
        self._buffers_in_use: List[bool] = []
        self._depth = 0

    def _reset_iteration(self) -> None:
        for i in range(len(self._buffers_in_use)):
            self._buffers_in_use[i] = False

    def _enter(self) -> None:
        if self._depth == 0:
            self._reset_iteration()
        self._depth += 1

    def _exit(self) -> None:
        self._depth = max(self._depth - 1, 0)

    def ensure_counts(self, row_count: int):
        if self._counts is None or self._counts_capacity < row_count:
            self._counts = torch.empty(row_count, dtype=I32, device=current_device())
            self._counts_capacity = row_count
        return self._counts[:row_count]

    def ensure_offsets(self, row_count: int):
        need = row_count + 1
        if self._offsets is None or self._offsets_capacity < need:
            self._offsets = torch.empty(need, dtype=I32, device=current_device())
            self._offsets_capacity = need
        return self._offsets[:need]

    def acquire_output(self, total: int, device=None):
        for i, (used, cap) in enumerate(zip(self._buffers_in_use, self._buffers_capacity)):
            if not used and cap >= total:
                self._buffers_in_use[i] = True
                b, e = self._buffers[i]
                return b[:total], e[:total]
        dev = device or current_device()
        b = torch.empty(max(total, 1), dtype=I32, device=dev)
        e = torch.empty(max(total, 1), dtype=I32, device=dev)
        self._buffers.append((b, e))
        self._buffers_capacity.append(max(total, 1))
        self._buffers_in_use.append(True)
        return b[:total], e[:total]


# ---------------------------------------------------------------------------
# Expression nodes
# ---------------------------------------------------------------------------

class Expr:
    """Base expression node."""

    def evaluate(self, workspace: Optional[CuPyWorkspace] = None) -> IntervalSet:
        raise NotImplementedError


class _InputExpr(Expr):
    def __init__(self, interval_set: IntervalSet):
        self._set = interval_set

    def evaluate(self, workspace=None) -> IntervalSet:
        return self._set


class _CallableExpr(Expr):
    def __init__(self, func):
        self._func = func

    def evaluate(self, workspace=None) -> IntervalSet:
        return self._func(workspace)


_MODES = ("union", "intersection", "difference", "symmetric_difference")


class _BinaryExpr(Expr):
    def __init__(self, lhs: Expr, rhs: Expr, mode: str):
        if mode not in _MODES:
            raise ValueError(f"unsupported operation {mode!r}")
        self._lhs = lhs
        self._rhs = rhs
        self._mode = mode

    def evaluate(self, workspace=None) -> IntervalSet:
        return _evaluate_tree(self, workspace)


def make_input(interval_set: IntervalSet) -> Expr:
    """Wrap an :class:`IntervalSet` so it can take part in expressions."""
    return _InputExpr(interval_set)


def make_intersection(lhs: Expr, rhs: Expr) -> Expr:
    return _BinaryExpr(lhs, rhs, "intersection")


def make_union(lhs: Expr, rhs: Expr) -> Expr:
    return _BinaryExpr(lhs, rhs, "union")


def make_difference(lhs: Expr, rhs: Expr) -> Expr:
    return _BinaryExpr(lhs, rhs, "difference")


def make_symmetric_difference(lhs: Expr, rhs: Expr) -> Expr:
    """(lhs \\ rhs) | (rhs \\ lhs) (``expressions.py:380-388``)."""
    return _BinaryExpr(lhs, rhs, "symmetric_difference")


def make_complement(universe: Expr, subset: Expr) -> Expr:
    """universe \\ subset (``expressions.py:391-399``)."""
    return _BinaryExpr(universe, subset, "difference")


def evaluate(expr: Expr, workspace: Optional[CuPyWorkspace] = None) -> IntervalSet:
    """Evaluate ``expr`` and return a new :class:`IntervalSet`."""
    if workspace is not None:
        workspace._enter()
        try:
            return expr.evaluate(workspace)
        finally:
            workspace._exit()
    return expr.evaluate(None)


def build_interval_set(row_offsets: Sequence[int], begin: Sequence[int], end: Sequence[int], *,
                       rows: Optional[Sequence[int]] = None) -> IntervalSet:
    """Build an :class:`IntervalSet` from sequences; values are coerced to int32 (``expressions.py:413-443``)."""
    dev = None
    for x in (row_offsets, begin, end):
        if isinstance(x, torch.Tensor) and x.is_cuda:
            dev = x.device
    off = _i32(row_offsets, dev)
    b = _i32(begin, off.device)
    e = _i32(end, off.device)
    last = int(off[-1])
    if last != int(b.numel()):
        raise ValueError("row_offsets final entry must equal the interval count")
    kind = next((x for x in (row_offsets, begin, end) if is_cupy(x)), None)
    if rows is None:
        r = torch.arange(int(off.numel()) - 1, dtype=I32, device=off.device)
        s = IntervalSet(like(kind, b), like(kind, e), like(kind, off), like(kind, r))
        object.__setattr__(s, "_dense_rows", int(r.numel()))
        return s
    return IntervalSet(like(kind, b), like(kind, e), like(kind, off), like(kind, _i32(rows, off.device)))


# ---------------------------------------------------------------------------
# Evaluation
# ---------------------------------------------------------------------------

_FUSED_MAX_LEAVES = 8


def _collect(expr: Expr, leaves: List[IntervalSet], index: Dict[int, int], workspace) -> Any:
    """Return a compiled node: ('leaf', i) or (mode, lhs, rhs)."""
    if isinstance(expr, _BinaryExpr):
        return (expr._mode, _collect(expr._lhs, leaves, index, workspace), _collect(expr._rhs, leaves, index, workspace))
    s = expr.evaluate(workspace)
    if not isinstance(s, IntervalSet):
        raise TypeError("expression leaves must evaluate to IntervalSet")
    key = id(s)
    if key not in index:
        index[key] = len(leaves)
        leaves.append(s)
    return ("leaf", index[key])


def _count_leaves(node) -> int:
    return 1 if node[0] == "leaf" else _count_leaves(node[1]) + _count_leaves(node[2])


def _eval_bool(node, state: int) -> bool:
    op = node[0]
    if op == "leaf":
        return bool((state >> node[1]) & 1)
    a = _eval_bool(node[1], state)
    b = _eval_bool(node[2], state)
    if op == "union":
        return a or b
    if op == "intersection":
        return a and b
    if op == "difference":
        return a and not b
    return a != b


def truth_table(node, k: int) -> List[int]:
    words = [0] * 8
    for state in range(1 << k):
        if _eval_bool(node, state):
            words[state >> 5] |= 1 << (state & 31)
    return words


def _same_rows(sets: Sequence[IntervalSet]) -> bool:
    first = sets[0]
    keys = [_dense_key(s) for s in sets]
    if keys[0] is not None and all(k == keys[0] for k in keys):
        return True
    n0 = int(first.rows.shape[0])
    if any(int(s.rows.shape[0]) != n0 for s in sets):
        return False
    r0 = _t(first.rows)
    others = [_t(s.rows) for s in sets[1:] if _t(s.rows).data_ptr() != r0.data_ptr() or n0 == 0]
    if not others or n0 == 0:
        return True
    # one device comparison and one read-back for all the sets
    same = torch.stack([torch.eq(r0, o).all() for o in others])
    return bool(same.all())


def _row_bounds(sets: Sequence[IntervalSet]) -> Tuple[int, int]:
    ends = []
    for s in sets:
        r = _t(s.rows)
        if r.numel():
            ends.append(r[0:1])
            ends.append(r[-1:])
    if not ends:
        return 0, 0
    host = torch.cat(ends).cpu()
    return int(host.min()), int(host.max())


def _aligned(sets: Sequence[IntervalSet], device):
    """Common rows and per-set aligned offsets (``expressions.py:131-141``)."""
    if _same_rows(sets):
        return _t(sets[0].rows), [_t(s.row_offsets) for s in sets], _dense_key(sets[0])
    lo, hi = _row_bounds(sets)
    lists = [(_t(s.rows), _t(s.row_offsets), 0, False) for s in sets]
    rows_out, offs = _core.align_rows(lists, lo, hi, device, [True] * len(sets))
    return rows_out, offs, None


def _wrap(kind, b, e, off, rows, dense) -> IntervalSet:
    return IntervalSet._trusted(like(kind, b), like(kind, e), like(kind, off), like(kind, rows), dense)


def _fused(node, leaves: List[IntervalSet], workspace) -> Optional[IntervalSet]:
    """One fused launch; None when the exact path must run instead."""
    device = _t(leaves[0].row_offsets).device
    rows_out, offs, dense = _aligned(leaves, device)
    R = int(rows_out.numel())
    kind = leaves[0].begin
    if R == 0:
        z = torch.zeros(0, dtype=I32, device=device)
        return _wrap(kind, z, z.clone(), torch.zeros(1, dtype=I32, device=device), rows_out, dense)
    k = len(leaves)
    table = truth_table(node, k)
    cap = max(1, sum(int(s.begin.shape[0]) for s in leaves))
    out = workspace.acquire_output(cap, device) if workspace is not None else None
    specs = [(_t(s.begin), _t(s.end), off, 0) for s, off in zip(leaves, offs)]
    ob, oe, ooff, total, flags = _core.bool_eval(specs, R, table, _lib.MODE_TABLE, device, out=out)
    if flags & (_lib.FLAG_CONTRACT | _lib.FLAG_LONG_TILE):
        return None
    if flags & (_lib.FLAG_CAPACITY | _lib.FLAG_TIMEOUT):
        raise _lib.SubsetixError(f"fused set evaluation failed (flags={flags})")
    return _wrap(kind, ob[:total], oe[:total], ooff, rows_out, dense)


def _exact_binary(lhs: IntervalSet, rhs: IntervalSet, mode: str) -> IntervalSet:
    """One binary op in the reference's order (``expressions.py:446-528``)."""
    if mode == "symmetric_difference":
        return _exact_binary(_exact_binary(lhs, rhs, "difference"), _exact_binary(rhs, lhs, "difference"), "union")
    device = _t(lhs.row_offsets).device
    rows_out, offs, dense = _aligned([lhs, rhs], device)
    R = int(rows_out.numel())
    kind = lhs.begin
    if R == 0:
        z = torch.zeros(0, dtype=I32, device=device)
        return _wrap(kind, z, z.clone(), torch.zeros(1, dtype=I32, device=device), rows_out, dense)
    op = {"union": _core.OP_UNION, "intersection": _core.OP_INTERSECTION, "difference": _core.OP_DIFFERENCE}[mode]
    ob, oe, off = _core.exact_setop(op, (_t(lhs.begin), _t(lhs.end), offs[0]), (_t(rhs.begin), _t(rhs.end), offs[1]),
                                    R, device)
    return _wrap(kind, ob, oe, off, rows_out, dense)


def _exact_tree(node, leaves: List[IntervalSet]) -> IntervalSet:
    if node[0] == "leaf":
        return leaves[node[1]]
    return _exact_binary(_exact_tree(node[1], leaves), _exact_tree(node[2], leaves), node[0])


def _evaluate_compiled(node, leaves: List[IntervalSet], workspace) -> IntervalSet:
    if node[0] == "leaf":
        return leaves[node[1]]
    used = sorted(_leaf_ids(node))
    if len(used) > _FUSED_MAX_LEAVES:
        lhs = _evaluate_compiled(node[1], leaves, workspace)
        rhs = _evaluate_compiled(node[2], leaves, workspace)
        return _evaluate_compiled((node[0], ("leaf", 0), ("leaf", 1)), [lhs, rhs], workspace)
    remap = {old: new for new, old in enumerate(used)}
    local = _remap(node, remap)
    sub = [leaves[i] for i in used]
    result = _fused(local, sub, workspace)
    if result is None:
        result = _exact_tree(local, sub)
    return result


def _leaf_ids(node) -> set:
    if node[0] == "leaf":
        return {node[1]}
    return _leaf_ids(node[1]) | _leaf_ids(node[2])


def _remap(node, remap):
    if node[0] == "leaf":
        return ("leaf", remap[node[1]])
    return (node[0], _remap(node[1], remap), _remap(node[2], remap))


def _evaluate_tree(expr: Expr, workspace) -> IntervalSet:
    leaves: List[IntervalSet] = []
    node = _collect(expr, leaves, {}, workspace)
    for s in leaves:
        if not (isinstance(s.begin, torch.Tensor) or is_cupy(s.begin)):
            raise TypeError("Inputs must be device arrays; CPU fallback is disabled")
    return _evaluate_compiled(node, leaves, workspace)


def apply_binary(lhs: IntervalSet, rhs: IntervalSet, mode: str, workspace=None) -> IntervalSet:
    """Functional form of one binary operation (the reference's ``_apply_binary``)."""
    if lhs is rhs:
        return _evaluate_compiled((mode, ("leaf", 0), ("leaf", 0)), [lhs], workspace)
    return _evaluate_compiled((mode, ("leaf", 0), ("leaf", 1)), [lhs, rhs], workspace)


_apply_binary = apply_binary
_OPERATION_CODES = {"union": 0, "intersection": 1, "difference": 2}

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
