"""ctypes binding of the C ABI in include/harmonia.h (libharmonia.so).

The library is built in-tree by harmonia_b200/build.py.  Loading fails loudly
when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libharmonia.so")

HM_OK = 0
ERRORS = {
    -1: "HM_EINVAL", -2: "HM_ENOMEM", -3: "HM_EDUPLICATE", -4: "HM_EMAXKEY", -5: "HM_ECUDA",
    -6: "HM_ECAPACITY", -7: "HM_ETIMEOUT", -8: "HM_ENODEVICE", -9: "HM_EBUSY",
    -10: "HM_ECANCELLED", -11: "HM_ETOOLARGE", -12: "HM_EIO",
}
HM_ECAPACITY = -6
HM_UPSERT_SUPPLIED = 0
HM_UPSERT_REF_KEY_MINUS_1 = 1

# Every symbol include/harmonia.h declares.
EXPORTS = (
    "hm_config_default", "hm_bulk_load", "hm_search", "hm_search_batches", "hm_range",
    "hm_range_between", "hm_set_wait_limit",    "hm_upsert_batch", "hm_export", "hm_tree_get_info", "hm_set_search_config",
    "hm_get_config", "hm_autotune", "hm_sync", "hm_free", "hm_strerror", "hm_launch_count",
    "hm_profile", "hm_profile_read", "hm_plan_create", "hm_plan_launch", "hm_plan_free",
    "hm_search_noalloc", "hm_server_config_default", "hm_server_start", "hm_server_submit",
    "hm_server_wait", "hm_server_get_stats", "hm_server_reset_stats", "hm_server_stop", "hm_server_free",
    "hm_last_cuda_error", "hm_read_keys", "hm_read_ranges", "hm_write_keys", "hm_snapshot_save",
    "hm_snapshot_load", "hm_delete_batch", "hm_search_baseline", "hm_trim_memory",
)
HM_NOALLOC_MAX_QUERIES = 1 << 20


class HarmoniaError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = ERRORS.get(code, str(code))
        msg = _lib.hm_strerror(code).decode() if _lib is not None else name
        if _lib is not None and code in (-2, -5, -8):
            buf = ctypes.create_string_buffer(256)
            if _lib.hm_last_cuda_error(buf, 256):
                msg += "; " + buf.value.decode()
        super().__init__(f"{what}: {name} ({msg})" if what else f"{name} ({msg})")


class Config(ctypes.Structure):
    _fields_ = [("fanout", ctypes.c_int), ("leaf_cap", ctypes.c_int), ("inner_fill", ctypes.c_int),
                ("leaf_fill", ctypes.c_int), ("group_width", ctypes.c_int),
                ("queries_per_group", ctypes.c_int), ("sort_bits", ctypes.c_int),
                ("smem_bytes", ctypes.c_int), ("cache_hints", ctypes.c_int), ("join", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class TreeInfo(ctypes.Structure):
    _fields_ = [("fanout", ctypes.c_int), ("leaf_cap", ctypes.c_int), ("height", ctypes.c_int),
                ("inner_row_words", ctypes.c_int), ("leaf_row_words", ctypes.c_int),
                ("leaf_index_words", ctypes.c_int), ("smem_levels", ctypes.c_int),
                ("n_keys", ctypes.c_int64), ("n_inner", ctypes.c_int64), ("n_leaf", ctypes.c_int64),
                ("lvl_start", ctypes.c_int64 * 33),
                ("inner", ctypes.c_void_p), ("prefix", ctypes.c_void_p),
                ("leaf_rows", ctypes.c_void_p),
                ("leaf_cnt", ctypes.c_void_p), ("leaf_base", ctypes.c_void_p),
                ("device_bytes", ctypes.c_size_t)]


class StageTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


class Batch(ctypes.Structure):
    _fields_ = [("q", ctypes.c_void_p), ("out", ctypes.c_void_p), ("n", ctypes.c_int64)]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libharmonia.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -c 'import __graft_entry__ as g; g.build()'` "
                           "or `python harmonia_b200/build.py` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    P, I, SZ = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    PT = ctypes.POINTER(ctypes.c_void_p)
    L.hm_config_default.argtypes = [ctypes.POINTER(Config)]
    L.hm_trim_memory.argtypes = [ctypes.POINTER(SZ)]
    L.hm_bulk_load.argtypes = [P, P, SZ, ctypes.POINTER(Config), PT]
    L.hm_search.argtypes = [P, P, SZ, P, P]
    L.hm_search_batches.argtypes = [P, ctypes.POINTER(Batch), I, P]
    L.hm_range.argtypes = [P, P, P, SZ, P, P, P, SZ, ctypes.POINTER(SZ), P]
    L.hm_range_between.argtypes = [P, P, P, SZ, P, P, P, SZ, ctypes.POINTER(SZ), P]
    L.hm_upsert_batch.argtypes = [P, P, P, SZ, I, P]
    L.hm_export.argtypes = [P, P, P, SZ, ctypes.POINTER(SZ)]
    L.hm_tree_get_info.argtypes = [P, ctypes.POINTER(TreeInfo)]
    L.hm_set_search_config.argtypes = [P, ctypes.POINTER(Config)]
    L.hm_get_config.argtypes = [P, ctypes.POINTER(Config)]
    L.hm_autotune.argtypes = [P, P, SZ, ctypes.POINTER(Config)]
    L.hm_sync.argtypes = [P, P]
    L.hm_set_wait_limit.argtypes = [P, ctypes.c_int64]
    L.hm_free.argtypes = [P]
    L.hm_strerror.argtypes = [I]
    L.hm_strerror.restype = ctypes.c_char_p
    L.hm_launch_count.argtypes = []
    L.hm_launch_count.restype = ctypes.c_uint64
    L.hm_last_cuda_error.argtypes = [ctypes.c_char_p, SZ]
    L.hm_profile.argtypes = [P, I]
    L.hm_plan_create.argtypes = [P, ctypes.POINTER(Batch), I, PT]
    L.hm_plan_launch.argtypes = [P, P]
    L.hm_plan_free.argtypes = [P]
    L.hm_search_noalloc.argtypes = [P, P, SZ, P, P]
    L.hm_profile_read.argtypes = [P, ctypes.POINTER(StageTime), I, ctypes.POINTER(I)]
    C = ctypes.c_char_p
    L.hm_read_keys.argtypes = [C, P, SZ, ctypes.POINTER(SZ)]
    L.hm_read_ranges.argtypes = [C, P, P, SZ, ctypes.POINTER(SZ)]
    L.hm_write_keys.argtypes = [C, P, SZ]
    L.hm_snapshot_save.argtypes = [P, C]
    L.hm_snapshot_load.argtypes = [C, ctypes.POINTER(Config), PT]
    L.hm_delete_batch.argtypes = [P, P, SZ, ctypes.POINTER(SZ), P]
    L.hm_search_baseline.argtypes = [P, I, P, SZ, P, P]
    _lib = L
    return L


def check(code: int, what: str = "") -> None:
    if code != HM_OK:
        raise HarmoniaError(code, what)


def default_config(**overrides) -> Config:
    """Library defaults with overrides; fills left unset follow the chosen
    fanout / leaf capacity (the library fills a zero fill with the capacity)."""
    c = Config()
    check(lib().hm_config_default(ctypes.byref(c)), "hm_config_default")
    c.inner_fill = 0
    c.leaf_fill = 0
    for k, v in overrides.items():
        if v is not None:
            setattr(c, k, int(v))
    return c
