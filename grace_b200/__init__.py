"""B200-native replacement of GRACE's Cowling GRMHD stage (sm_100a, FP64).

The compute lives in libgrace_b200.so behind the C ABI of
include/grace_b200.h; this package is the host-side mirror of the reference's
interface (grace_b200.host) plus parameter helpers and synthetic workloads.
"""
from . import abi, params  # noqa: F401

__all__ = ["abi", "params", "host", "workloads"]
