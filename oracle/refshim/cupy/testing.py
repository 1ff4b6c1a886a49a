"""``cupy.testing`` stand-in: NumPy's assertions on host copies (oracle test infrastructure)."""

import numpy as _np


def _host(x):
    return _np.asarray(x.view(_np.ndarray) if isinstance(x, _np.ndarray) else x)


def assert_array_equal(x, y, err_msg="", verbose=True, strict=False):
    _np.testing.assert_array_equal(_host(x), _host(y), err_msg=err_msg, verbose=verbose, strict=strict)


def assert_allclose(actual, desired, rtol=1e-7, atol=0, err_msg="", verbose=True):
    _np.testing.assert_allclose(_host(actual), _host(desired), rtol=rtol, atol=atol, err_msg=err_msg, verbose=verbose)


def assert_array_almost_equal(x, y, decimal=6, err_msg="", verbose=True):
    _np.testing.assert_array_almost_equal(_host(x), _host(y), decimal=decimal, err_msg=err_msg, verbose=verbose)
