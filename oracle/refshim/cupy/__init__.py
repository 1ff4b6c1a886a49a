"""NumPy-backed stand-in for the ``cupy`` module (oracle test infrastructure).

It is not part of the product.  The reference package imports ``cupy`` at
module level (``subsetix_cupy/expressions.py:19-24``,
``subsetix_amr2/fields.py:7``).  Placing this directory first on ``sys.path``
lets the reference's own Python code, and its kernel strings, run unchanged on
a machine without a GPU.  The tests and ``tests/golden/make_golden.py`` use it
to check the oracle against the reference.

How the mapping works:

* :class:`ndarray` is a ``numpy.ndarray`` subclass.  It adds ``.get()`` and
  ``.data.ptr``, and makes scalar indexing return a 0-d array, as CuPy does.
* Module attributes not defined here fall through to NumPy.  Array results
  are returned as :class:`ndarray`.
* ``RawKernel`` compiles the CUDA-C string for the host (``cpu_rawkernel``).
"""

from __future__ import annotations

import numpy as _np

import importlib.util as _ilu
import os as _os

_spec = _ilu.spec_from_file_location(
    "sx_refshim_cpu_rawkernel",
    _os.path.join(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))), "cpu_rawkernel.py"),
)
_cpu_rawkernel = _ilu.module_from_spec(_spec)
_spec.loader.exec_module(_cpu_rawkernel)

__version__ = "0.0.0-numpy-shim"


class _DataPtr:
    __slots__ = ("ptr",)

    def __init__(self, ptr: int):
        self.ptr = ptr


class ndarray(_np.ndarray):
    """NumPy array that answers the parts of the CuPy array API the reference uses."""

    def get(self, stream=None, order="C", out=None):  # noqa: D401 - CuPy signature
        return _np.array(self, copy=True)

    @property
    def data(self):  # type: ignore[override]
        return _DataPtr(int(self.__array_interface__["data"][0]))

    def __getitem__(self, key):
        # CuPy wraps out-of-range integer-array indices instead of raising;
        # the reference's alignment checks rely on that (multilevel.py:445-451).
        if isinstance(key, _np.ndarray) and key.dtype.kind in "iu" and self.ndim >= 1:
            n = self.shape[0]
            key = _np.asarray(key).view(_np.ndarray) % n if n > 0 else key
        out = super().__getitem__(key)
        if not isinstance(out, _np.ndarray):
            return _np.asarray(out).view(ndarray)
        return out

    def take(self, indices, axis=None, out=None, mode="wrap"):
        return _wrap(super().take(_np.asarray(indices), axis=axis, out=out, mode="wrap"))

    def astype(self, dtype, order="K", casting="unsafe", subok=True, copy=True):
        return _wrap(super().astype(dtype, order=order, casting=casting, subok=subok, copy=copy))

    def __array_wrap__(self, obj, context=None, return_scalar=False):
        result = super().__array_wrap__(obj, context, return_scalar)
        return result


def _wrap(value):
    if isinstance(value, ndarray):
        return value
    if isinstance(value, _np.ndarray):
        return value.view(ndarray)
    if isinstance(value, tuple):
        return tuple(_wrap(v) for v in value)
    if isinstance(value, list):
        return [_wrap(v) for v in value]
    return value


def _unwrap(value):
    if isinstance(value, ndarray):
        return value.view(_np.ndarray)
    if isinstance(value, (list, tuple)):
        return type(value)(_unwrap(v) for v in value)
    return value


def _make(fn):
    def wrapped(*args, **kwargs):
        out_arg = kwargs.get("out")
        result = fn(*args, **kwargs)
        if out_arg is not None and isinstance(out_arg, ndarray):
            return out_arg
        return _wrap(result)

    wrapped.__name__ = getattr(fn, "__name__", "wrapped")
    return wrapped


def asarray(a, dtype=None, order=None):
    if isinstance(a, ndarray) and (dtype is None or _np.dtype(dtype) == a.dtype):
        return a
    return _np.asarray(a, dtype=dtype, order=order).view(ndarray)


def array(obj, dtype=None, copy=True, order="K", subok=False, ndmin=0):
    out = _np.array(obj, dtype=dtype, copy=bool(copy) if copy is not None else None, order=order, ndmin=ndmin)
    return out.view(ndarray)


def asnumpy(a, stream=None, order="C", out=None):
    if isinstance(a, _np.ndarray):
        return _np.array(a.view(_np.ndarray), copy=True)
    return _np.asarray(a)


def empty(shape, dtype=float, order="C"):
    return _np.empty(shape, dtype=dtype, order=order).view(ndarray)


def RawKernel(code, name, options=(), backend="nvrtc", translate_cucomplex=False, **_kw):
    return _cpu_rawkernel.CpuRawKernel(code, name, options)


int8 = _np.int8
int32 = _np.int32
int64 = _np.int64
uint8 = _np.uint8
float32 = _np.float32
float64 = _np.float64
bool_ = _np.bool_
dtype = _np.dtype
newaxis = None


def __getattr__(name):
    attr = getattr(_np, name)
    if callable(attr) and not isinstance(attr, type):
        return _make(attr)
    return attr


from . import testing  # noqa: E402,F401
from . import cuda  # noqa: E402,F401
from . import random  # noqa: E402,F401
