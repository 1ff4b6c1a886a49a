"""Device plumbing for the Python layer: arrays, streams and workspaces.

* Arrays.  Internally every device array is a ``torch.Tensor``.  CuPy
  arrays, or any object that exports ``__cuda_array_interface__`` or
  DLPack, are wrapped without a copy.  Results are handed back in the
  caller's array kind (see :func:`like`).
* Streams.  Kernels are enqueued on the current torch stream of the
  tensors' device.
* Workspaces.  The C ABI needs caller-owned scratch for its scan state.
  One zero-filled buffer is kept per (device, stream) and grows on demand.
  The kernels leave it clean after every call.
"""

from __future__ import annotations

import threading
from typing import Any, Dict, Tuple

import numpy as np
import torch

from . import _lib

_state = threading.local()

try:  # CuPy is optional; torch works alone
    import cupy as _cupy  # type: ignore
except Exception:  # pragma: no cover - cupy absent in this image
    _cupy = None


def require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA device required; subsetix_b200 has no CPU fallback")


def current_device() -> torch.device:
    require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def is_cupy(x) -> bool:
    return _cupy is not None and isinstance(x, _cupy.ndarray)


def to_tensor(x, dtype=None, device=None) -> torch.Tensor:
    """Zero-copy view of a device array as a torch tensor (host data is copied to the device)."""
    if isinstance(x, torch.Tensor):
        t = x
    elif is_cupy(x):
        t = torch.from_dlpack(x)
    elif hasattr(x, "__cuda_array_interface__"):
        t = torch.as_tensor(x, device="cuda")
    elif hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
        t = torch.from_dlpack(x)
    else:
        t = torch.as_tensor(np.asarray(x))
    if device is None:
        device = t.device if t.is_cuda else current_device()
    if t.device != device:
        t = t.to(device)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t


def like(kind_source, t: torch.Tensor):
    """Return ``t`` in the array kind of ``kind_source`` (CuPy in -> CuPy out)."""
    if is_cupy(kind_source):
        return _cupy.from_dlpack(t)
    return t


def stream_handle(device: torch.device) -> int:
    return int(torch.cuda.current_stream(device).cuda_stream)


class _Workspace:
    __slots__ = ("buf",)

    def __init__(self):
        self.buf = None


def workspace(device: torch.device, nbytes: int) -> Tuple[int, int]:
    """Pointer and size of the scratch buffer for the current stream (grown to ``nbytes``)."""
    pools: Dict[Tuple[int, int], _Workspace] = getattr(_state, "pools", None)
    if pools is None:
        pools = {}
        _state.pools = pools
    key = (device.index, stream_handle(device))
    ws = pools.get(key)
    if ws is None:
        ws = _Workspace()
        pools[key] = ws
    need = max(int(nbytes), 4096)
    if ws.buf is None or ws.buf.numel() < need:
        size = max(need, 2 * (ws.buf.numel() if ws.buf is not None else 0))
        # The old buffer may still be in use by queued kernels; the caching
        # allocator keeps its memory alive until the stream passes this point.
        ws.buf = torch.zeros(size, dtype=torch.uint8, device=device)
    return ws.buf.data_ptr(), ws.buf.numel()


def reset_workspaces() -> None:
    """Drop every workspace (after a failed launch left a scan state dirty)."""
    _state.pools = {}


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr() if t.numel() else None


def read_pair(result: torch.Tensor) -> Tuple[int, int]:
    """Synchronising read of a device ``result`` pair (count, flags)."""
    host = result.cpu()
    return int(host[0]), int(host[1])
