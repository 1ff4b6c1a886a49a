"""The reference's own kernels, NVRTC-compiled, launched on torch tensors.

TEST INFRASTRUCTURE ONLY: this module is a checker and a baseline, never part
of the product path.  It loads the cubins that ``oracle/build_ref_nvrtc.py``
built from the reference's kernel strings (unchanged source, CuPy's NVRTC
options) and launches them through the CUDA driver API on torch's current
stream, with the grid and block shapes the reference uses.  The host steps
around each launch (row lookups, prefix sums, output allocation, the
``.item()`` reads) are restated with torch, in the reference's order:

* upwind: ``subsetix_cupy/interval_stencil.py:126-219`` (grid = intervals,
  block 128);
* gradient magnitude: ``subsetix_amr2/regrid.py:233-274`` (block 256);
* threshold run-lengths: ``subsetix_amr2/regrid.py:277-333`` (one 32-lane
  block per row, count, cumsum, write);
* prolong / restrict field: ``subsetix_cupy/multilevel.py:385-407,452-479``
  (grid = coarse intervals, block 128);
* binary set operations: ``subsetix_cupy/expressions.py:446-528`` (K1 count,
  cumsum, one host read of the total, K2 write; block 128), with the row
  alignment of ``expressions.py:58-141`` for operands that share a row list;
* expression trees: ``expressions.py:328-410`` (one binary launch pair per
  node; xor as two differences and a union).

The result of every float kernel here is what the real reference computes on
this GPU, FMA contraction included.
"""

from __future__ import annotations

import ctypes
import json
import os
from typing import Dict, Tuple

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
CUBIN_DIR = os.path.join(HERE, "_ref", "nvrtc")

_CTYPES = {
    "int": ctypes.c_int32,
    "unsigned int": ctypes.c_uint32,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "long long": ctypes.c_int64,
    "bool": ctypes.c_bool,
    "signed char": ctypes.c_int8,
}


def available() -> bool:
    return os.path.exists(os.path.join(CUBIN_DIR, "manifest.json"))


class _Driver:
    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        cu = self.cu
        cu.cuInit.argtypes = [ctypes.c_uint]
        cu.cuCtxGetCurrent.argtypes = [ctypes.POINTER(ctypes.c_void_p)]
        cu.cuModuleLoadData.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        cu.cuModuleGetFunction.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_char_p]
        cu.cuLaunchKernel.argtypes = [ctypes.c_void_p] + [ctypes.c_uint] * 7 + [
            ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
        self.check(cu.cuInit(0), "cuInit")

    @staticmethod
    def check(rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what} failed with CUDA driver error {rc}")


class RefKernels:
    """Loaded reference cubins; ``launch`` runs one with the reference's arguments."""

    def __init__(self, device: torch.device | int | None = None):
        if not available():
            raise RuntimeError("reference cubins missing: run oracle/build_ref_nvrtc.py where the reference is mounted")
        with open(os.path.join(CUBIN_DIR, "manifest.json")) as fh:
            self.manifest = json.load(fh)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   (device if isinstance(device, int) else device.index or 0))
        torch.zeros(1, device=self.device)  # makes torch's primary context current on this thread
        self.drv = _Driver()
        ctx = ctypes.c_void_p()
        self.drv.check(self.drv.cu.cuCtxGetCurrent(ctypes.byref(ctx)), "cuCtxGetCurrent")
        if not ctx.value:
            raise RuntimeError("no current CUDA context after torch initialisation")
        self._funcs: Dict[str, Tuple[ctypes.c_void_p, list]] = {}
        self._images = []

    def _function(self, key: str):
        got = self._funcs.get(key)
        if got is not None:
            return got
        entry = self.manifest["kernels"][key]
        with open(os.path.join(CUBIN_DIR, f"{key}.cubin"), "rb") as fh:
            image = ctypes.create_string_buffer(fh.read())
        self._images.append(image)
        mod = ctypes.c_void_p()
        self.drv.check(self.drv.cu.cuModuleLoadData(ctypes.byref(mod), image), f"cuModuleLoadData({key})")
        fn = ctypes.c_void_p()
        self.drv.check(self.drv.cu.cuModuleGetFunction(ctypes.byref(fn), mod, entry["function"].encode()),
                       f"cuModuleGetFunction({key})")
        got = (fn, entry["params"])
        self._funcs[key] = got
        return got

    def launch(self, key: str, grid, block, *args) -> None:
        fn, params = self._function(key)
        if len(args) != len(params):
            raise TypeError(f"{key}: expected {len(params)} arguments, got {len(args)}")
        grid = tuple(int(g) for g in (grid if isinstance(grid, tuple) else (grid,))) + (1, 1)
        block = tuple(int(b) for b in (block if isinstance(block, tuple) else (block,))) + (1, 1)
        if grid[0] * grid[1] * grid[2] == 0:
            return
        holders = []
        for (ctype, is_ptr), value in zip(params, args):
            if is_ptr:
                if not isinstance(value, torch.Tensor) or value.device != self.device:
                    raise TypeError(f"{key}: pointer arguments must be tensors on {self.device}")
                if value.numel() and not value.is_contiguous():
                    raise ValueError(f"{key}: pointer argument is not contiguous")
                holders.append(ctypes.c_void_p(value.data_ptr() if value.numel() else 0))
            else:
                holders.append(_CTYPES[ctype](value))
        slots = (ctypes.c_void_p * len(holders))(*[ctypes.cast(ctypes.byref(h), ctypes.c_void_p) for h in holders])
        stream = torch.cuda.current_stream(self.device).cuda_stream
        self.drv.check(self.drv.cu.cuLaunchKernel(fn, grid[0], grid[1], grid[2], block[0], block[1], block[2], 0,
                                                  ctypes.c_void_p(stream), slots, None), f"cuLaunchKernel({key})")

    # -- field kernels --------------------------------------------------------------------------------------------

    def upwind_f32(self, begin, end, row_offsets, rows, cell_offsets, values, *, width, height, a, b, dt, dx, dy):
        """``step_upwind_interval`` (``interval_stencil.py:126-219``) on float32 values."""
        dev = self.device
        n = int(begin.numel())
        out = torch.empty_like(values, dtype=torch.float32)
        if n == 0:
            out.fill_(0.0)
            return out
        counts = (row_offsets[1:] - row_offsets[:-1]).to(torch.int64)
        row_ids = torch.repeat_interleave(rows.to(torch.int32), counts)
        lookup = torch.full((int(height),), -1, dtype=torch.int32, device=dev)
        lookup[rows.to(torch.int64)] = torch.arange(rows.numel(), dtype=torch.int32, device=dev)
        ords = lookup[row_ids.to(torch.int64)]
        if int(ords.min().item()) < 0:
            raise ValueError("interval_set rows exceed provided height")
        self.launch("interval_upwind", (n,), (128,), row_ids, begin, end, row_offsets, cell_offsets, ords, lookup,
                    values.to(torch.float32).contiguous(), out, n, int(width), int(height), float(a), float(b),
                    float(dt), float(dx), float(dy))
        return out

    def gradient_flat(self, values, width: int, height: int):
        """``gradient_magnitude_interval_field`` (``regrid.py:233-274``)."""
        data = values.to(torch.float32).contiguous()
        out = torch.empty(width * height, dtype=torch.float32, device=self.device)
        block = 256
        self.launch("subsetix_gradient_magnitude_flat", (max(1, (width * height + block - 1) // block),), (block,),
                    data, int(width), int(height), out)
        return out

    def threshold_intervals(self, values, width: int, height: int, threshold: float):
        """``intervals_above_threshold_interval_field`` (``regrid.py:277-333``): (begin, end, offsets, rows)."""
        dev = self.device
        data = values.to(torch.float32).contiguous()
        counts = torch.zeros(height, dtype=torch.int32, device=dev)
        self.launch("subsetix_count_threshold_intervals", (height,), (32,), data, int(height), int(width),
                    float(threshold), counts)
        offsets = torch.zeros(height + 1, dtype=torch.int32, device=dev)
        offsets[1:] = torch.cumsum(counts, 0, dtype=torch.int32)
        total = int(offsets[-1].item())
        begin = torch.empty(total, dtype=torch.int32, device=dev)
        end = torch.empty(total, dtype=torch.int32, device=dev)
        if total:
            self.launch("subsetix_write_threshold_intervals", (height,), (32,), data, int(height), int(width),
                        float(threshold), offsets, begin, end)
        return begin, end, offsets, torch.arange(height, dtype=torch.int32, device=dev)

    def prolong_f32(self, coarse_offsets, fine_offsets, fine_interval_indices, ratio, coarse_values, fine_values):
        n = int(coarse_offsets.numel()) - 1
        self.launch("prolong_field_f32", (n,), (128,), coarse_offsets, fine_offsets, fine_interval_indices,
                    int(ratio), n, coarse_values.to(torch.float32).contiguous(), fine_values)
        return fine_values

    def restrict_f32(self, coarse_offsets, fine_offsets, fine_interval_indices, ratio, reducer, fine_values,
                     coarse_values):
        n = int(coarse_offsets.numel()) - 1
        norm = float(torch.tensor(1.0 / (ratio * ratio) if reducer == 0 else 1.0, dtype=torch.float32))
        self.launch("restrict_field_f32", (n,), (128,), coarse_offsets, fine_offsets, fine_interval_indices,
                    int(ratio), n, int(reducer), norm, fine_values.to(torch.float32).contiguous(), coarse_values)
        return coarse_values

    # -- set algebra ----------------------------------------------------------------------------------------------

    _OPS = {"union": 0, "intersection": 1, "difference": 2}

    def apply_binary(self, lhs, rhs, mode: str):
        """``_apply_binary`` (``expressions.py:446-528``) for operands on one row list.

        ``lhs``/``rhs`` are ``(begin, end, row_offsets, rows)`` tuples.  The
        reference first checks whether the row lists are equal (one device
        reduction and host read, ``expressions.py:131-135``); only that case is
        restated, which is the case of every operand in the bench workload.
        """
        dev = self.device
        lb, le, lo, lr = lhs
        rb, re_, ro, rr = rhs
        if lr.numel() != rr.numel() or not bool(torch.equal(lr, rr)):
            raise NotImplementedError("row lists differ: alignment is not restated here")
        rows = int(lo.numel()) - 1
        if rows == 0:
            z = torch.zeros(0, dtype=torch.int32, device=dev)
            return z, z, torch.zeros(1, dtype=torch.int32, device=dev), lr
        counts = torch.empty(rows, dtype=torch.int32, device=dev)
        grid = ((rows + 127) // 128,)
        op = self._OPS[mode]
        self.launch("count_segments", grid, (128,), lb, le, lo, rb, re_, ro, rows, op, counts)
        offsets = torch.empty(rows + 1, dtype=torch.int32, device=dev)
        offsets[0] = 0
        torch.cumsum(counts, 0, dtype=torch.int32, out=offsets[1:])
        total = int(offsets[-1].item())
        if total == 0:
            z = torch.zeros(0, dtype=torch.int32, device=dev)
            return z, z, offsets, lr
        ob = torch.empty(total, dtype=torch.int32, device=dev)
        oe = torch.empty(total, dtype=torch.int32, device=dev)
        self.launch("write_segments", grid, (128,), lb, le, lo, rb, re_, ro, offsets, rows, op, ob, oe)
        return ob, oe, offsets, lr

    def evaluate(self, spec, leaves):
        """Evaluate a nested ``(op, lhs, rhs)`` tree over named leaves node by node, as ``Expr`` trees do."""
        if isinstance(spec, str):
            return leaves[spec]
        op, l_spec, r_spec = spec
        lhs = self.evaluate(l_spec, leaves)
        rhs = self.evaluate(r_spec, leaves)
        if op == "symmetric_difference":
            return self.apply_binary(self.apply_binary(lhs, rhs, "difference"),
                                     self.apply_binary(rhs, lhs, "difference"), "union")
        return self.apply_binary(lhs, rhs, op)
