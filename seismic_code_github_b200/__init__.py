"""B200-native finite-difference wave-propagation engine (sm_100a CUDA behind a C ABI).

The compute path is libseisfd.so (include/seisfd.h); `seisfd` is its ctypes binding and
`workloads` builds the seeded synthetic benchmark cases.  Submodules are imported on first
use, so that `workloads` (plain numpy) can be imported without touching the binding.
"""
import importlib

__all__ = ["seisfd", "workloads", "sharding"]


def __getattr__(name):
    if name in __all__:
        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
