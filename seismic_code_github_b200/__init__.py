"""B200-native finite-difference wave-propagation engine (sm_100a CUDA behind a C ABI).

The compute path is libseisfd.so (include/seisfd.h); `seisfd` is its ctypes binding and
`workloads` builds the seeded synthetic benchmark cases.
"""
from . import seisfd  # noqa: F401

__all__ = ["seisfd"]
