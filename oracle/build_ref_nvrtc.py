"""Compile the reference's own CUDA-C kernel strings for the GPU with NVRTC.

TEST INFRASTRUCTURE ONLY.  The cubins this recipe writes are the checker for
the product's float arithmetic and the "reference kernels" leg of the bench;
the product never loads them.

The reference builds every kernel at run time through ``cupy.RawKernel``
with NVRTC and the options it passes there, ``("--std=c++11",)`` for almost
all of them (``subsetix_cupy/kernels.py:254-277``,
``subsetix_cupy/interval_stencil.py:116-123``, ``subsetix_amr2/regrid.py:20-178``,
``subsetix_amr2/fields.py:297``, ``subsetix_cupy/interval_field.py:243``).
NVRTC's defaults then apply, in particular ``--fmad=true``: a multiply that
feeds an add may be fused into one FMA.  A host build of the same source
cannot say which multiplies the GPU compiler fuses, so the float outputs of
the real reference are only known from these kernels run on the GPU.

How the sources are obtained: a child process puts the NumPy stand-in for
``cupy`` (``oracle/refshim``) and the reference checkout on ``sys.path``,
imports the reference modules and calls their kernel getters.  The stand-in's
``RawKernel`` records ``(code, name, options)`` without compiling anything.
The child compiles each source with NVRTC, adding only the target
architecture (``sm_100``, what CuPy passes for a compute capability 10.0
device), and writes one cubin per kernel plus ``manifest.json`` (kernel name
-> parameter types) into ``oracle/_ref/nvrtc/``.  No reference source is
written anywhere; ``oracle/_ref/`` is git-ignored and travels to the GPU
machine with the other built files.

Usage::

    python oracle/build_ref_nvrtc.py [--reference DIR] [--force]
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref", "nvrtc")
MANIFEST = os.path.join(OUT_DIR, "manifest.json")
ARCH = "--gpu-architecture=sm_100"

# (module, getter expression) pairs evaluated in the child; each yields one
# RawKernel or a tuple of them.  The subset-copy getter yields one kernel per
# value type under one function name; those cubins are keyed ``name@dtype``.
_SUBSET_TYPES = ("float32", "float64", "int8", "int32", "int64", "bool")
_GETTERS = [
    ("subsetix_cupy.kernels", "get_kernels(cp)"),
    ("subsetix_cupy.interval_stencil", "_get_interval_upwind_kernel()"),
    ("subsetix_cupy.interval_field", "_get_locate_kernel()"),
    ("subsetix_amr2.regrid", "(_COUNT_INTERVALS, _WRITE_INTERVALS, _GRADIENT_MAGNITUDE_KERNEL, "
                             "_get_gradient_flat_kernel())"),
    ("subsetix_amr2.fields", "tuple(_get_interval_subset_kernel(m, t) for m in ('gather', 'scatter') "
                             "for t in _SUBSET_TYPES)"),
]


def _child(reference: str, out_dir: str) -> None:
    sys.dont_write_bytecode = True
    sys.path.insert(0, reference)
    sys.path.insert(0, os.path.join(HERE, "refshim"))
    import importlib

    import cupy as cp  # the NumPy stand-in: RawKernel only records its arguments
    from cuda.bindings import nvrtc

    spec = importlib.util.spec_from_file_location("sx_cpu_rawkernel", os.path.join(HERE, "refshim", "cpu_rawkernel.py"))
    rk = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(rk)

    kernels = []
    for mod_name, expr in _GETTERS:
        mod = importlib.import_module(mod_name)
        got = eval(expr, {**vars(mod), "cp": cp, "_SUBSET_TYPES": _SUBSET_TYPES})
        got = [k for k in (got if isinstance(got, tuple) else (got,)) if k is not None]
        if mod_name == "subsetix_amr2.fields":
            keys = [f"{k.name}@{t}" for k, t in zip(got, _SUBSET_TYPES * 2)]
        else:
            keys = [k.name for k in got]
        kernels += list(zip(keys, got))

    def check(res, prog=None):
        err = res[0]
        if err != nvrtc.nvrtcResult.NVRTC_SUCCESS:
            log = ""
            if prog is not None:
                _, size = nvrtc.nvrtcGetProgramLogSize(prog)
                buf = b" " * size
                nvrtc.nvrtcGetProgramLog(prog, buf)
                log = buf.decode(errors="replace")
            raise RuntimeError(f"NVRTC failed: {err}\n{log}")
        return res[1:] if len(res) > 1 else None

    os.makedirs(out_dir, exist_ok=True)
    manifest = {"nvrtc_version": list(check(nvrtc.nvrtcVersion())), "arch": ARCH, "kernels": {}}
    for key, k in kernels:
        prog, = check(nvrtc.nvrtcCreateProgram(k.code.encode(), f"{k.name}.cu".encode(), 0, [], []))
        opts = [o.encode() for o in k.options] + [ARCH.encode()]
        check(nvrtc.nvrtcCompileProgram(prog, len(opts), opts), prog)
        size, = check(nvrtc.nvrtcGetCUBINSize(prog))
        cubin = b" " * size
        check(nvrtc.nvrtcGetCUBIN(prog, cubin))
        nvrtc.nvrtcDestroyProgram(prog)
        with open(os.path.join(out_dir, f"{key}.cubin"), "wb") as fh:
            fh.write(cubin)
        params = rk._parse_params(k.code, k.name)
        manifest["kernels"][key] = {"function": k.name, "params": [[t, bool(p)] for t, p in params],
                                    "options": list(k.options)}
    with open(os.path.join(out_dir, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)


def build(reference: str = "/root/reference", force: bool = False) -> str | None:
    """Build the cubins when the reference checkout is present; return the folder or None."""
    if not os.path.isdir(os.path.join(reference, "subsetix_cupy")):
        return None
    if not force and os.path.exists(MANIFEST):
        return OUT_DIR
    env = dict(os.environ)
    env.pop("PYTHONPATH", None)
    subprocess.run([sys.executable, os.path.abspath(__file__), "--child", "--reference", reference],
                   check=True, env=env, cwd=HERE)
    return OUT_DIR


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--child", action="store_true")
    args = ap.parse_args()
    if args.child:
        _child(args.reference, OUT_DIR)
    else:
        print(build(args.reference, force=args.force))
