"""Access to the committed golden fixtures (``tests/golden/*.npz``)."""

from __future__ import annotations

import functools
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@functools.lru_cache(maxsize=None)
def load(name: str):
    with np.load(os.path.join(GOLDEN, name), allow_pickle=False) as data:
        return {k: data[k] for k in data.files}


def has(data, key: str) -> bool:
    return f"{key}/begin" in data or key in data


def get_set(data, key: str):
    return (data[f"{key}/begin"], data[f"{key}/end"], data[f"{key}/row_offsets"], data[f"{key}/rows"])


def error(data, key: str):
    k = f"{key}/error"
    return str(data[k]) if k in data else None
