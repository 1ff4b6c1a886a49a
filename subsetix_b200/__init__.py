"""B200-native (sm_100a) interval-set AMR hot path.

The subpackages ``subsetix_b200.subsetix_cupy`` and
``subsetix_b200.subsetix_amr2`` mirror the reference packages of the same
names.  :func:`enable_dropin` registers them under their original top-level
names, so existing ``import subsetix_cupy`` code runs unchanged on this
implementation.
"""

from __future__ import annotations

import sys

__version__ = "0.1.0"


def enable_dropin() -> None:
    """Make ``import subsetix_cupy`` / ``import subsetix_amr2`` resolve to this package."""
    import importlib

    for name in ("subsetix_cupy", "subsetix_amr2"):
        try:
            mod = importlib.import_module(f"subsetix_b200.{name}")
        except ImportError:
            continue
        sys.modules.setdefault(name, mod)
        for sub, m in list(sys.modules.items()):
            prefix = f"subsetix_b200.{name}."
            if sub.startswith(prefix):
                sys.modules.setdefault(name + "." + sub[len(prefix):], m)


def library_path() -> str:
    from ._lib import LIB_PATH

    return LIB_PATH
