"""``cupy.random`` stand-in backed by NumPy's legacy generator (oracle test infrastructure)."""

import numpy as _np


def seed(value=None):
    _np.random.seed(value)


def random(size=None, dtype=float):
    return _np.random.random(size).astype(dtype).view(__import__("cupy").ndarray)
