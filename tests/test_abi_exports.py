"""The C-ABI library loads and exports every function include/subsetix_b200.h declares (no GPU needed)."""

import ctypes
import os
import re

import pytest

from subsetix_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "subsetix_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sx_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert names, "no declarations parsed"
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binds_every_declared_symbol():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_abi_version_and_error_string_without_gpu():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    lib = _lib.load()
    assert lib.sx_abi_version() == 1
    # an invalid call fails on the host, before touching the device
    rc = lib.sx_bool_eval(None, 0, 1, None, 0, None, None, None, 0, None, None, 0, None, None)
    assert rc == _lib.SX_ERR_INVALID
    assert "k=0" in _lib.last_error()
