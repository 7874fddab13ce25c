"""Locate and load the native library (``lib/libdyphur_b200.so``).

The library is built in-tree by ``dyphur_b200.build`` (nvcc, sm_100a). There
is no fallback: a missing library is an ImportError-style failure.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libdyphur_b200.so")

_lock = threading.Lock()
_lib = None


class NativeLibraryMissing(ImportError):
    pass


def load_library() -> ctypes.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise NativeLibraryMissing(
                    f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'` "
                    "or `python -m dyphur_b200.build`")
            _lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        return _lib
