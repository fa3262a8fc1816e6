"""Reference dataset files through the C ABI (hm_read_keys, hm_read_ranges,
hm_write_keys): one signed decimal key per line, ranges as two lines (start,
end), as the reference's data generator writes them
(open-harmonia/script/generate-data/generate.py) and its harness reads them
(open-harmonia/src/main.cpp:50-67, open-harmonia/src/range.cu:349-355)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .native import check, lib


def read_keys(path: str) -> np.ndarray:
    """All keys of a key file, in file order, as int64."""
    n = ctypes.c_size_t()
    p = os.fsencode(path)
    check(lib().hm_read_keys(p, None, 0, ctypes.byref(n)), "hm_read_keys")
    keys = np.empty(max(n.value, 1), np.int64)
    check(lib().hm_read_keys(p, keys.ctypes.data, len(keys), ctypes.byref(n)), "hm_read_keys")
    return keys[: n.value]


def read_ranges(path: str):
    """(start, end) int64 arrays of a range file."""
    n = ctypes.c_size_t()
    p = os.fsencode(path)
    check(lib().hm_read_ranges(p, None, None, 0, ctypes.byref(n)), "hm_read_ranges")
    start = np.empty(max(n.value, 1), np.int64)
    end = np.empty(max(n.value, 1), np.int64)
    check(lib().hm_read_ranges(p, start.ctypes.data, end.ctypes.data, len(start), ctypes.byref(n)),
          "hm_read_ranges")
    return start[: n.value], end[: n.value]


def write_keys(path: str, keys) -> None:
    """Writes keys one per line."""
    k = np.ascontiguousarray(np.asarray(keys, dtype=np.int64))
    check(lib().hm_write_keys(os.fsencode(path), k.ctypes.data if len(k) else None, len(k)), "hm_write_keys")
