"""Loader for the in-tree CUDA library libgrace_b200.so.

The library is built by grace_b200/build.py (nvcc, sm_100a).  Loading fails
loudly when it is missing: there is no CPU fallback for the hot path.
"""
import ctypes
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrace_b200.so")
_lib = None


class LibraryMissing(RuntimeError):
    pass


def load():
    """Load and bind libgrace_b200.so (every symbol of include/grace_b200.h)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(
            f"{LIB_PATH} is missing; build it with `python -m grace_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in abi.PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, what):
    if rc != abi.OK:
        raise RuntimeError(f"{what} failed with status {rc}")
    return rc
