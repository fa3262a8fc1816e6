"""Host-side mirror of the reference's tree interface over the C ABI.

The reference's operator surface is the C++ class BPlusTree
(open-harmonia/src/bpt.h:342-561: insert, search, range_search, sort,
insert_parallel_Newupdate_batch) plus one GPU experiment function per CLI
option (open-harmonia/src/ppi-bpt.h:4-98).  ``BPlusTree`` below keeps those
names and argument meanings for the batched forms:

* ``BPlusTree.bulk_load(keys, values)`` stands in for the insert loop +
  ``sort()`` + ``prepareGPU_*`` upload (open-harmonia/src/main.cpp:50-67,151-152);
* ``search(keys)`` returns the value or -1 per key (BPlusTree::search,
  open-harmonia/src/bpt.cpp:673-680);
* ``range_search(start, length)`` returns the first ``length`` records with
  key >= start (open-harmonia/src/cpu-range.cpp:129-183 with end = Max_Key);
* ``insert_parallel_Newupdate_batch(keys, values)`` applies one update batch
  with the reference's rule (existing key -> key-1,
  open-harmonia/src/bpt-ppi-update-batch.cpp:47); ``upsert`` takes the
  supplied value for existing keys.

Buffers may be numpy arrays (host) or CUDA torch tensors (device); results
come back in the same kind.  Errors raise HarmoniaError with the HM_E* code.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import native
from .native import HarmoniaError, check, lib  # noqa: F401

MAX_KEY = 2**63 - 1
NOT_FOUND = -1


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x) -> int:
    if _is_torch(x):
        return x.data_ptr()
    return x.ctypes.data


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)


def _as_i64(x):
    if _is_torch(x):
        import torch
        if x.dtype != torch.int64 or not x.is_contiguous():
            x = x.to(torch.int64).contiguous()
        return x
    return np.ascontiguousarray(x, dtype=np.int64)


def _as_i32(x):
    if _is_torch(x):
        import torch
        if x.dtype != torch.int32 or not x.is_contiguous():
            x = x.to(torch.int32).contiguous()
        return x
    return np.ascontiguousarray(x, dtype=np.int32)


def _empty_like(x, n: int, dtype="int64"):
    if _is_torch(x):
        import torch
        return torch.empty(n, dtype=getattr(torch, dtype), device=x.device)
    return np.empty(n, dtype=dtype)


class BPlusTree:
    """A device-resident batched B+tree (one hm_tree handle)."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)

    # ---- construction ----
    @classmethod
    def bulk_load(cls, keys, values, fanout: int = 64, leaf_cap: int = 16, inner_fill=None,
                  leaf_fill=None, group_width=None, queries_per_group=None, sort_bits=None,
                  smem_bytes=None) -> "BPlusTree":
        keys = _as_i64(keys)
        values = _as_i64(values)
        if len(keys) != len(values):
            raise ValueError("keys and values differ in length")
        cfg = native.default_config(fanout=fanout, leaf_cap=leaf_cap, inner_fill=inner_fill,
                                    leaf_fill=leaf_fill, group_width=group_width,
                                    queries_per_group=queries_per_group, sort_bits=sort_bits,
                                    smem_bytes=smem_bytes)
        h = ctypes.c_void_p()
        n = len(keys)
        check(lib().hm_bulk_load(_ptr(keys) if n else None, _ptr(values) if n else None, n,
                                 ctypes.byref(cfg), ctypes.byref(h)), "hm_bulk_load")
        return cls(h.value)

    @classmethod
    def from_reference_file(cls, path: str, **config) -> "BPlusTree":
        """Bulk-loads the keys of a reference insert file (one decimal key per
        line) with value = key, as the reference's main() inserts them
        (open-harmonia/src/main.cpp:56-66)."""
        from .files import read_keys

        keys = read_keys(path)
        return cls.bulk_load(keys, keys.copy(), **config)

    def save(self, path: str) -> None:
        """Writes a snapshot (sorted contents + configuration) to path."""
        check(lib().hm_snapshot_save(self._h, os.fsencode(path)), "hm_snapshot_save")

    @classmethod
    def load(cls, path: str, **config) -> "BPlusTree":
        """Bulk-loads a snapshot; keyword arguments override the saved
        configuration (fanout, leaf_cap, fills, search settings)."""
        h = ctypes.c_void_p()
        cfg = None
        if config:
            cfg = native.default_config(**config)
        check(lib().hm_snapshot_load(os.fsencode(path), ctypes.byref(cfg) if cfg is not None else None,
                                     ctypes.byref(h)), "hm_snapshot_load")
        return cls(h.value)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(lib().hm_free(self._h), "hm_free")
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # ---- queries ----
    def search(self, keys, out=None, stream=None):
        keys = _as_i64(keys)
        n = len(keys)
        if out is None:
            out = _empty_like(keys, n)
        if n:
            check(lib().hm_search(self._h, _ptr(keys), n, _ptr(out), _stream_ptr(stream)), "hm_search")
        return out

    def search_pointer_baseline(self, keys, out=None, stream=None):
        """The HB+-style pointer-chasing comparison kernel (device buffers);
        same results as search()."""
        n = len(keys)
        if out is None:
            out = _empty_like(keys, n)
        if n:
            check(lib().hm_search_baseline(self._h, 1, _ptr(keys), n, _ptr(out), _stream_ptr(stream)),
                  "hm_search_baseline")
        return out

    def search_batches(self, batches, stream=None) -> None:
        """batches: list of (queries, out) CUDA tensors, searched in one launch."""
        arr = (native.Batch * max(len(batches), 1))()
        for i, (q, o) in enumerate(batches):
            arr[i].q = _ptr(q)
            arr[i].out = _ptr(o)
            arr[i].n = len(q)
        check(lib().hm_search_batches(self._h, arr, len(batches), _stream_ptr(stream)), "hm_search_batches")

    def plan(self, batches) -> "Plan":
        """Captures a CUDA graph searching these (queries, out) CUDA tensor pairs."""
        return Plan(self, batches)

    def range_search(self, start, length, stream=None):
        """Returns (offsets[n+1], keys, values): query i owns [offsets[i], offsets[i+1])."""
        start = _as_i64(start)
        length = _as_i32(length)
        n = len(start)
        offsets = _empty_like(start, n + 1)
        cap = int(length.clip(min=0).sum()) if n else 0
        okeys = _empty_like(start, max(cap, 1))
        ovals = _empty_like(start, max(cap, 1))
        total = ctypes.c_size_t()
        check(lib().hm_range(self._h, _ptr(start) if n else None, _ptr(length) if n else None, n,
                             _ptr(offsets), _ptr(okeys), _ptr(ovals), cap, ctypes.byref(total),
                             _stream_ptr(stream)), "hm_range")
        m = total.value
        return offsets, okeys[:m], ovals[:m]

    def range_between(self, start, end, cap=None, stream=None):
        """Inclusive ranges, as the reference's BPlusTree::range_search:
        every record with start[i] <= key <= end[i].  Returns (offsets[n+1],
        keys, values).  cap bounds the record count (default: counted by a
        first call that returns HM_ECAPACITY with the total)."""
        start = _as_i64(start)
        end = _as_i64(end)
        if len(start) != len(end):
            raise ValueError("start and end differ in length")
        n = len(start)
        offsets = _empty_like(start, n + 1)
        total = ctypes.c_size_t()

        def call(c, ok, ov):
            return lib().hm_range_between(self._h, _ptr(start) if n else None, _ptr(end) if n else None, n,
                                          _ptr(offsets), _ptr(ok) if ok is not None else None,
                                          _ptr(ov) if ov is not None else None, c, ctypes.byref(total),
                                          _stream_ptr(stream))

        if cap is None:
            rc = call(0, None, None)
            if rc not in (0, native.HM_ECAPACITY):
                check(rc, "hm_range_between")
            cap = total.value
        okeys = _empty_like(start, max(cap, 1))
        ovals = _empty_like(start, max(cap, 1))
        check(call(cap, okeys, ovals), "hm_range_between")
        m = total.value
        return offsets, okeys[:m], ovals[:m]

    # ---- updates ----
    def delete(self, keys, stream=None) -> int:
        """One delete epoch: removes the stored keys among keys; returns how
        many were removed (the reference has no working delete)."""
        keys = _as_i64(keys)
        removed = ctypes.c_size_t()
        check(lib().hm_delete_batch(self._h, _ptr(keys) if len(keys) else None, len(keys),
                                    ctypes.byref(removed), _stream_ptr(stream)), "hm_delete_batch")
        return int(removed.value)

    def upsert(self, keys, values, ref_rule: bool = False, stream=None) -> None:
        keys = _as_i64(keys)
        values = _as_i64(values)
        if len(keys) != len(values):
            raise ValueError("keys and values differ in length")
        flags = native.HM_UPSERT_REF_KEY_MINUS_1 if ref_rule else native.HM_UPSERT_SUPPLIED
        if len(keys):
            check(lib().hm_upsert_batch(self._h, _ptr(keys), _ptr(values), len(keys), flags,
                                        _stream_ptr(stream)), "hm_upsert_batch")

    def insert_parallel_Newupdate_batch(self, keys, values) -> None:  # noqa: N802 (reference name)
        """The reference's update rule: existing keys take key-1, new keys their value."""
        self.upsert(keys, values, ref_rule=True)

    # ---- inspection ----
    def info(self) -> native.TreeInfo:
        i = native.TreeInfo()
        check(lib().hm_tree_get_info(self._h, ctypes.byref(i)), "hm_tree_get_info")
        return i

    @property
    def size(self) -> int:
        return int(self.info().n_keys)

    def export(self):
        n = self.size
        k = np.empty(max(n, 1), np.int64)
        v = np.empty(max(n, 1), np.int64)
        got = ctypes.c_size_t()
        check(lib().hm_export(self._h, k.ctypes.data, v.ctypes.data, n, ctypes.byref(got)), "hm_export")
        return k[: got.value], v[: got.value]

    def config(self) -> dict:
        c = native.Config()
        check(lib().hm_get_config(self._h, ctypes.byref(c)), "hm_get_config")
        return c.as_dict()

    def set_search_config(self, **kw) -> None:
        c = native.Config()
        check(lib().hm_get_config(self._h, ctypes.byref(c)), "hm_get_config")
        for k, v in kw.items():
            setattr(c, k, int(v))
        check(lib().hm_set_search_config(self._h, ctypes.byref(c)), "hm_set_search_config")

    def autotune(self, sample_keys) -> dict:
        best = native.Config()
        check(lib().hm_autotune(self._h, _ptr(sample_keys), len(sample_keys), ctypes.byref(best)), "hm_autotune")
        return best.as_dict()

    def profile(self, enable: bool = True) -> None:
        """Per-stage CUDA-event timing on the stages' own streams (off by default)."""
        check(lib().hm_profile(self._h, 1 if enable else 0), "hm_profile")

    def profile_read(self) -> dict:
        """{stage: (launches, total_ms)} since the last read; clears the record."""
        arr = (native.StageTime * 8)()
        n = ctypes.c_int()
        check(lib().hm_profile_read(self._h, arr, 8, ctypes.byref(n)), "hm_profile_read")
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(min(n.value, 8))}

    def set_wait_limit(self, polls: int) -> None:
        """Polls of the search kernel's bounded wait for its staged top levels
        (default 2^24); 0 makes every such wait give up (HM_ETIMEOUT)."""
        check(lib().hm_set_wait_limit(self._h, int(polls)), "hm_set_wait_limit")

    def sync(self, stream=None) -> None:
        check(lib().hm_sync(self._h, _stream_ptr(stream)), "hm_sync")

    def layout(self) -> dict:
        """Copies the device arrays to host numpy (tests compare them bit for bit)."""
        from cuda.bindings import runtime as rt

        i = self.info()

        def grab(ptr, count, itemsize, dtype):
            out = np.empty(count, dtype=dtype)
            if count:
                (err,) = rt.cudaMemcpy(out.ctypes.data, ptr, count * itemsize,
                                       rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
                if err != rt.cudaError_t.cudaSuccess:
                    raise RuntimeError(f"cudaMemcpy failed: {err}")
            return out

        self.sync()
        return {
            "height": i.height,
            "lvl_start": list(i.lvl_start[: i.height + 1]),
            "n_inner": i.n_inner,
            "n_leaf": i.n_leaf,
            "inner": grab(i.inner, i.n_inner * i.inner_row_words, 8, np.int64),
            "prefix": grab(i.prefix, i.n_inner, 4, np.int32),
            "leaf_rows": grab(i.leaf_rows, i.n_leaf * i.leaf_row_words, 8, np.int64),
            "leaf_cnt": grab(i.leaf_cnt, i.n_leaf, 4, np.int32),
            "leaf_base": grab(i.leaf_base, i.n_leaf, 8, np.int64),
        }


class Plan:
    """A batch set captured as a CUDA graph (hm_plan); launch() replays it."""

    def __init__(self, tree: BPlusTree, batches):
        self._tree = tree  # keeps the tree alive while the plan exists
        self._bufs = list(batches)
        arr = (native.Batch * max(len(batches), 1))()
        for i, (q, o) in enumerate(batches):
            arr[i].q = _ptr(q)
            arr[i].out = _ptr(o)
            arr[i].n = len(q)
        h = ctypes.c_void_p()
        check(lib().hm_plan_create(tree.handle, arr, len(batches), ctypes.byref(h)), "hm_plan_create")
        self._h = h

    def launch(self, stream=None) -> None:
        check(lib().hm_plan_launch(self._h, _stream_ptr(stream)), "hm_plan_launch")

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(lib().hm_plan_free(self._h), "hm_plan_free")
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count() -> int:
    """Kernel launches issued by libharmonia.so in this process."""
    return int(lib().hm_launch_count())


def trim_memory() -> int:
    """Frees the device blocks the library keeps for reuse (arenas,
    temporaries and scratch of freed trees); returns the bytes freed."""
    out = ctypes.c_size_t()
    check(lib().hm_trim_memory(ctypes.byref(out)), "hm_trim_memory")
    return int(out.value)
