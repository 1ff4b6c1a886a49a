"""CPU execution of CUDA-C RawKernel sources (oracle test infrastructure).

This module is part of the oracle, not of the product.  Only the tests and
the golden-fixture generator use it.  It lets the reference package run on a
machine without a GPU.  The reference builds its kernels from CUDA-C source
strings through ``cupy.RawKernel`` (for example ``subsetix_cupy/kernels.py:239-289``).
The NumPy-backed ``cupy`` stand-in in ``oracle/refshim/cupy`` hands those
strings to :class:`CpuRawKernel`.  That class compiles them as ordinary C++
with ``g++``, using a prelude that maps the CUDA keywords and thread indices
onto host code, and runs the launch grid as loops.

Two launch modes exist:

* Independent threads.  These kernels never talk to each other, so blocks
  and threads run one after another.
* Lock-step warps.  Kernels that call ``__ballot_sync`` (the regrid run-length
  encoders, ``subsetix_amr2/regrid.py:20-124``) run each lane as a real host
  thread.  The lanes of a warp meet at a barrier on every ballot, so every
  lane sees the same 32-bit vote mask a GPU warp would.

Floating point is compiled with hardware FMA and ``-ffp-contract=fast``.
The reference's GPU build (NVRTC, ``--fmad=true`` by default) fuses each
multiply into the add or subtract that consumes it, the first product of a
sum first; GCC's contraction makes the same choices on these kernels (the
upwind update becomes ``fma(-dt, fma(a, du_dx, b * du_dy), c)``, the
gradient norm ``sqrt(fma(gx, gx, gy * gy))``), so float results equal the
reference's GPU results.  In one place GCC's own grouping differs from
NVRTC's: inside the gradient kernel (``regrid.py:217``) it fuses the second
product of ``gx * gx + gy * gy``.  That expression is therefore pinned, in
the copy of the source handed to the host compiler, to the grouping NVRTC
emits (``_CONTRACTION_PINS``).  Both were checked against the reference's
kernels compiled with NVRTC and run on a B200, on every cell of the probe
inputs; the GPU tests keep checking the product against those kernels on
the fixture inputs.  Integer results are exact.

The sources are read at run time from the reference package that the caller
imported.  Nothing from the reference is stored in this repository.  Compiled
objects are cached under ``oracle/_ref/shim_cache``, which git ignores.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import re
import subprocess
import threading
from typing import Any, List, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_CACHE_DIR = os.path.join(os.path.dirname(_HERE), "_ref", "shim_cache")
_FLAGS = ("-std=c++20", "-O2", "-mfma", "-ffp-contract=fast", "-fPIC", "-shared", "-w")
# source text -> the same expression with NVRTC's fusion written out (host compile only)
_CONTRACTION_PINS = {"sqrtf(gx * gx + gy * gy)": "sqrtf(fmaf(gx, gx, gy * gy))"}
_LOCK = threading.Lock()

_PRELUDE = r"""
#include <math.h>
#include <stdint.h>
#include <barrier>
#include <thread>
#include <vector>
#include <functional>
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__ __restrict
struct sxshim_dim3 { unsigned int x, y, z; };
static thread_local sxshim_dim3 threadIdx, blockIdx;
static sxshim_dim3 blockDim, gridDim;
struct sxshim_warp {
    std::barrier<>* bar;
    unsigned int votes[32];
};
static thread_local sxshim_warp* sxshim_my_warp = nullptr;
static thread_local int sxshim_lane = 0;
static inline unsigned int __ballot_sync(unsigned int mask, int pred) {
    sxshim_warp* w = sxshim_my_warp;
    w->votes[sxshim_lane] = pred ? 1u : 0u;
    w->bar->arrive_and_wait();
    unsigned int out = 0u;
    for (int l = 0; l < 32; ++l) {
        if (w->votes[l]) out |= (1u << l);
    }
    w->bar->arrive_and_wait();
    return out & mask;
}
static inline int __popc(unsigned int x) { return __builtin_popcount(x); }
static inline int __ffs(int x) { return __builtin_ffs(x); }
"""

_LAUNCHER = r"""
extern "C" int sxshim_launch_@NAME@(unsigned int gx, unsigned int gy, unsigned int gz,
                                   unsigned int bx, unsigned int by, unsigned int bz,
                                   void** args, int lockstep)
{
    gridDim.x = gx; gridDim.y = gy; gridDim.z = gz;
    blockDim.x = bx; blockDim.y = by; blockDim.z = bz;
    auto body = [&]() { @NAME@(@ARGS@); };
    for (unsigned int z = 0; z < gz; ++z)
    for (unsigned int y = 0; y < gy; ++y)
    for (unsigned int x = 0; x < gx; ++x) {
        sxshim_dim3 blk = {x, y, z};
        if (!lockstep) {
            blockIdx = blk;
            for (unsigned int tz = 0; tz < bz; ++tz)
            for (unsigned int ty = 0; ty < by; ++ty)
            for (unsigned int tx = 0; tx < bx; ++tx) {
                threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
                body();
            }
        } else {
            unsigned int n = bx * by * bz;
            unsigned int nwarps = (n + 31u) / 32u;
            std::vector<sxshim_warp> warps(nwarps);
            std::vector<std::barrier<>*> bars;
            for (unsigned int w = 0; w < nwarps; ++w) {
                unsigned int lanes = (w + 1u) * 32u <= n ? 32u : n - w * 32u;
                warps[w].bar = new std::barrier<>((std::ptrdiff_t)lanes);
                for (int l = 0; l < 32; ++l) warps[w].votes[l] = 0u;
            }
            std::vector<std::thread> threads;
            for (unsigned int t = 0; t < n; ++t) {
                threads.emplace_back([&, t]() {
                    blockIdx = blk;
                    threadIdx.x = t % bx; threadIdx.y = (t / bx) % by; threadIdx.z = t / (bx * by);
                    sxshim_my_warp = &warps[t / 32u];
                    sxshim_lane = (int)(t % 32u);
                    body();
                    sxshim_my_warp->bar->arrive_and_drop();
                });
            }
            for (auto& th : threads) th.join();
            for (unsigned int w = 0; w < nwarps; ++w) delete warps[w].bar;
        }
    }
    return 0;
}
"""

_SCALAR_TYPES = {
    "int": ctypes.c_int32,
    "unsigned int": ctypes.c_uint32,
    "unsigned": ctypes.c_uint32,
    "float": ctypes.c_float,
    "double": ctypes.c_double,
    "long long": ctypes.c_int64,
    "bool": ctypes.c_bool,
    "signed char": ctypes.c_int8,
}


def _parse_params(source: str, name: str) -> List[Tuple[str, bool]]:
    match = re.search(r"\bvoid\s+" + re.escape(name) + r"\s*\(([^)]*)\)", source, re.S)
    if match is None:
        raise RuntimeError(f"kernel {name!r} not found in source")
    params: List[Tuple[str, bool]] = []
    for raw in match.group(1).split(","):
        text = " ".join(raw.replace("\n", " ").split())
        if not text:
            continue
        is_ptr = "*" in text
        ident = re.findall(r"[A-Za-z_][A-Za-z_0-9]*", text)[-1]
        ctype = text[: text.rfind(ident)].strip()
        ctype = ctype.replace("__restrict__", "").replace("const", "").strip()
        ctype = " ".join(ctype.split())
        params.append((ctype, is_ptr))
    return params


class CpuRawKernel:
    """Compile a CUDA-C kernel string as C++ and run its grid on the host."""

    def __init__(self, code: str, name: str, options: Sequence[str] = ()):
        self.code = code
        self.name = name
        self.options = tuple(options)
        self._fn = None
        self._params: List[Tuple[str, bool]] = []
        self._lockstep = "__ballot_sync" in code

    def _compile(self) -> None:
        params = _parse_params(self.code, self.name)
        arg_exprs = []
        for idx, (ctype, is_ptr) in enumerate(params):
            if is_ptr:
                base = ctype.replace("*", "").strip()
                arg_exprs.append(f"({base}*)(*(void**)args[{idx}])")
            else:
                arg_exprs.append(f"*({ctype}*)args[{idx}]")
        launcher = _LAUNCHER.replace("@NAME@", self.name).replace("@ARGS@", ", ".join(arg_exprs))
        code = self.code
        for text, pinned in _CONTRACTION_PINS.items():
            code = code.replace(text, pinned)
        full = _PRELUDE + "\n" + code + "\n" + launcher
        digest = hashlib.sha256((" ".join(_FLAGS) + full).encode()).hexdigest()[:20]
        os.makedirs(_CACHE_DIR, exist_ok=True)
        so_path = os.path.join(_CACHE_DIR, f"{self.name}_{digest}.so")
        with _LOCK:
            if not os.path.exists(so_path):
                tmp = so_path + f".{os.getpid()}.tmp"
                cmd = ["g++", *_FLAGS, "-x", "c++", "-", "-o", tmp, "-lpthread"]
                proc = subprocess.run(cmd, input=full.encode(), capture_output=True)
                if proc.returncode != 0:
                    raise RuntimeError(
                        f"g++ failed for kernel {self.name}:\n{proc.stderr.decode()[:4000]}"
                    )
                os.replace(tmp, so_path)
        lib = ctypes.CDLL(so_path)
        fn = getattr(lib, f"sxshim_launch_{self.name}")
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_uint] * 6 + [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
        self._fn = fn
        self._params = params
        self._lib = lib

    def __call__(self, grid, block, args, **_kwargs) -> None:
        if self._fn is None:
            self._compile()
        grid = tuple(int(g) for g in (grid if isinstance(grid, tuple) else (grid,)))
        block = tuple(int(b) for b in (block if isinstance(block, tuple) else (block,)))
        grid = grid + (1,) * (3 - len(grid))
        block = block + (1,) * (3 - len(block))
        if len(args) != len(self._params):
            raise TypeError(f"{self.name}: expected {len(self._params)} args, got {len(args)}")
        keep: List[Any] = []
        slots = (ctypes.c_void_p * len(args))()
        for idx, ((ctype, is_ptr), value) in enumerate(zip(self._params, args)):
            if is_ptr:
                arr = value
                if not isinstance(arr, np.ndarray):
                    raise TypeError(f"{self.name}: argument {idx} must be an array")
                if arr.size and not arr.flags.c_contiguous:
                    raise ValueError(f"{self.name}: argument {idx} is not contiguous")
                holder = ctypes.c_void_p(arr.__array_interface__["data"][0] if arr.size else 0)
                keep.append(holder)
                slots[idx] = ctypes.cast(ctypes.pointer(holder), ctypes.c_void_p)
            else:
                ct = _SCALAR_TYPES.get(ctype)
                if ct is None:
                    raise TypeError(f"{self.name}: unsupported scalar type {ctype!r}")
                holder = ct(value.item() if hasattr(value, "item") else value)
                keep.append(holder)
                slots[idx] = ctypes.cast(ctypes.pointer(holder), ctypes.c_void_p)
        total_blocks = grid[0] * grid[1] * grid[2]
        if total_blocks == 0:
            return
        rc = self._fn(grid[0], grid[1], grid[2], block[0], block[1], block[2], slots,
                      1 if self._lockstep else 0)
        if rc != 0:
            raise RuntimeError(f"{self.name}: launch failed ({rc})")
