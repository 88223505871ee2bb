"""Loader for the in-tree CUDA library libgrace_b200.so.

The library is built by grace_b200/build.py (nvcc, sm_100a).  Loading fails
loudly when it is missing: there is no CPU fallback for the hot path.
"""
import ctypes
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgrace_b200.so")
# the same sources with every multiply and add rounded on its own
# (nvcc -fmad=false), for parity tests that need the oracle's rounding
EXACT_LIB_PATH = os.path.join(_HERE, "libgrace_b200_exact.so")
_libs = {}


class LibraryMissing(RuntimeError):
    pass


def load(variant="default"):
    """Load and bind libgrace_b200.so, or with variant="exact" its -fmad=false
    build (every symbol of include/grace_b200.h)."""
    if variant in _libs:
        return _libs[variant]
    path = {"default": LIB_PATH, "exact": EXACT_LIB_PATH}[variant]
    if not os.path.exists(path):
        raise LibraryMissing(
            f"{path} is missing; build it with `python -m grace_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in abi.PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[variant] = lib
    return lib


def check(rc, what):
    if rc != abi.OK:
        raise RuntimeError(f"{what} failed with status {rc}")
    return rc
