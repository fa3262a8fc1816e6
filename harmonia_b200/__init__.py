"""harmonia-b200: Harmonia's batched B+tree query path, B200-native.

The product is the CUDA library ``libharmonia.so`` behind the C ABI in
``include/harmonia.h``; this package holds its build script, a ctypes
binding (``native``), the host-side mirror of the reference's tree interface
(``BPlusTree``), the seeded workload generator (``datagen``) and the serving
loop binding (``serving``).
"""
from .native import HarmoniaError  # noqa: F401
from .tree import BPlusTree, launch_count, trim_memory, MAX_KEY, NOT_FOUND  # noqa: F401

__all__ = ["BPlusTree", "HarmoniaError", "launch_count", "trim_memory", "MAX_KEY", "NOT_FOUND"]
