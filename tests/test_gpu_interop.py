"""Zero-copy ingestion: objects that export only ``__cuda_array_interface__`` or only DLPack.

The drop-in takes CuPy arrays, torch tensors, or any device array exposing
one of the two protocols, without copying them: the data pointer of the
input reaches the kernels unchanged.  Results come back as torch tensors for
such inputs (CuPy inputs give CuPy outputs when CuPy is installed).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.gpu_util import assert_same, iset, rand_set

pytestmark = pytest.mark.gpu

sc = pytest.importorskip("subsetix_b200.subsetix_cupy")


class CAIOnly:
    """A device array that speaks only the CUDA array interface (as Numba or PyCUDA arrays do)."""

    def __init__(self, t: torch.Tensor):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__


class DLPackOnly:
    """A device array that speaks only DLPack (as JAX or TensorFlow arrays do)."""

    def __init__(self, t: torch.Tensor):
        self._t = t

    def __dlpack__(self, stream=None, **kwargs):
        return self._t.__dlpack__(stream=stream) if stream is not None else self._t.__dlpack__()

    def __dlpack_device__(self):
        return self._t.__dlpack_device__()


@pytest.mark.parametrize("wrap", [CAIOnly, DLPackOnly])
def test_foreign_device_arrays_are_used_in_place(cuda_device, wrap):
    from subsetix_b200._runtime import to_tensor

    A = rand_set(200, 4.0, seed=41, row0=0)
    B = rand_set(200, 4.0, seed=42, row0=0)
    dev = {k: [torch.as_tensor(a, device="cuda") for a in h] for k, h in (("A", A), ("B", B))}
    for t in dev["A"]:
        assert to_tensor(wrap(t)).data_ptr() == t.data_ptr()
    sets = {k: sc.build_interval_set(row_offsets=wrap(v[2]), begin=wrap(v[0]), end=wrap(v[1]), rows=wrap(v[3]))
            for k, v in dev.items()}
    assert torch.as_tensor(sets["A"].begin).data_ptr() == dev["A"][0].data_ptr()
    got = sc.evaluate(sc.make_union(sc.make_input(sets["A"]), sc.make_input(sets["B"])))
    assert isinstance(got.begin, torch.Tensor)
    assert_same(got, O.union(iset(A), iset(B)))
