"""Test infrastructure only: ctypes access to the two CPU oracles.

* ``PortTree`` wraps ``libhmoracle.so``, the plain-C restatement
  (oracle/hm_oracle.c) on the product's device layout.
* ``RefTree`` wraps ``_ref/libhmref.so``, the reference's own CPU B+tree
  (open-harmonia/src) compiled from its sources by ``make ref``.

Only tests, the smoke check and bench.py's reference/cpu_baseline arm import
this module.  The product path never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libhmoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhmref.so")
CFB_SO = os.path.join(HERE, "_ref", "libhmref_cfb.so")
GPU_SO = os.path.join(HERE, "_ref", "libhmref_gpu.so")
MAX_KEY = 2**63 - 1

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_L = ctypes.c_long


def build(ref: bool = False) -> None:
    """Compile the restatement (and the reference library when asked)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "port"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class _Params(ctypes.Structure):
    _fields_ = [("fanout", ctypes.c_int), ("leaf_cap", ctypes.c_int),
                ("inner_fill", ctypes.c_int), ("leaf_fill", ctypes.c_int)]


class _Tree(ctypes.Structure):
    _fields_ = [("p", _Params), ("height", ctypes.c_int), ("inner_row", ctypes.c_int),
                ("leaf_row", ctypes.c_int), ("leaf_index", ctypes.c_int),
                ("n_keys", _I64), ("n_inner", _I64), ("n_leaf", _I64),
                ("lvl_start", _I64 * 33),
                ("inner", _P), ("prefix", _P), ("leaf_rows", _P),
                ("leaf_cnt", _P), ("leaf_base", _P)]


_port = None


def _port_lib():
    global _port
    if _port is None:
        lib = ctypes.CDLL(PORT_SO)
        lib.hmo_build.argtypes = [_P, _P, _I64, ctypes.POINTER(_Params), ctypes.POINTER(_Tree)]
        lib.hmo_build.restype = ctypes.c_int
        lib.hmo_free.argtypes = [ctypes.POINTER(_Tree)]
        lib.hmo_search.argtypes = [ctypes.POINTER(_Tree), _P, _I64, _P]
        lib.hmo_range.argtypes = [ctypes.POINTER(_Tree), _P, _P, _I64, _P, _P, _P, _I64]
        lib.hmo_range.restype = _I64
        lib.hmo_range_between.argtypes = [ctypes.POINTER(_Tree), _P, _P, _I64, _P, _P, _P, _I64]
        lib.hmo_range_between.restype = _I64
        lib.hmo_export.argtypes = [ctypes.POINTER(_Tree), _P, _P, _I64]
        lib.hmo_export.restype = _I64
        lib.hmo_upsert.argtypes = [_P, _P, _I64, _P, _P, _I64, ctypes.c_int, _P, _P, _I64]
        lib.hmo_upsert.restype = _I64
        lib.hmo_splitmix64.argtypes = [ctypes.c_uint64]
        lib.hmo_splitmix64.restype = ctypes.c_uint64
        lib.hmo_shape.argtypes = [_I64, ctypes.POINTER(_Params), ctypes.POINTER(ctypes.c_int),
                                  _P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]
        lib.hmo_shape.restype = ctypes.c_int
        _port = lib
    return _port


def splitmix64(x: int) -> int:
    return int(_port_lib().hmo_splitmix64(ctypes.c_uint64(x)))


def params(fanout=64, leaf_cap=16, inner_fill=None, leaf_fill=None) -> _Params:
    return _Params(fanout, leaf_cap, inner_fill or fanout, leaf_fill or leaf_cap)


def shape(n: int, fanout=64, leaf_cap=16, inner_fill=None, leaf_fill=None):
    """(height, lvl_start list, n_inner, n_leaf) of a bulk-loaded tree."""
    p = params(fanout, leaf_cap, inner_fill, leaf_fill)
    h = ctypes.c_int()
    ls = np.zeros(33, np.int64)
    ni, nl = _I64(), _I64()
    rc = _port_lib().hmo_shape(n, ctypes.byref(p), ctypes.byref(h), _ptr(ls), ctypes.byref(ni), ctypes.byref(nl))
    if rc:
        raise ValueError("bad tree parameters")
    return h.value, ls[: h.value + 1].tolist(), ni.value, nl.value


class PortTree:
    """The C restatement built over sorted unique keys."""

    def __init__(self, sorted_keys, vals, fanout=64, leaf_cap=16, inner_fill=None, leaf_fill=None):
        self._k = np.ascontiguousarray(sorted_keys, dtype=np.int64)
        self._v = np.ascontiguousarray(vals, dtype=np.int64)
        self.p = params(fanout, leaf_cap, inner_fill, leaf_fill)
        self.t = _Tree()
        rc = _port_lib().hmo_build(_ptr(self._k), _ptr(self._v), len(self._k), ctypes.byref(self.p), ctypes.byref(self.t))
        if rc:
            raise ValueError(f"hmo_build failed: {rc}")

    def __del__(self):
        if getattr(self, "t", None) is not None and _port is not None:
            _port.hmo_free(ctypes.byref(self.t))
            self.t = None

    def _arr(self, ptr, count, ctype, dtype):
        if count == 0:
            return np.zeros(0, dtype)
        buf = (ctype * count).from_address(ptr)
        return np.ctypeslib.as_array(buf).view(dtype).copy()

    def layout(self) -> dict:
        t = self.t
        return {
            "height": t.height,
            "lvl_start": list(t.lvl_start[: t.height + 1]),
            "n_inner": t.n_inner,
            "n_leaf": t.n_leaf,
            "inner": self._arr(t.inner, t.n_inner * t.inner_row, ctypes.c_int64, np.int64),
            "prefix": self._arr(t.prefix, t.n_inner, ctypes.c_int32, np.int32),
            "leaf_rows": self._arr(t.leaf_rows, t.n_leaf * t.leaf_row, ctypes.c_int64, np.int64),
            "leaf_cnt": self._arr(t.leaf_cnt, t.n_leaf, ctypes.c_int32, np.int32),
            "leaf_base": self._arr(t.leaf_base, t.n_leaf, ctypes.c_int64, np.int64),
        }

    def search(self, q) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.int64)
        out = np.empty_like(q)
        _port_lib().hmo_search(ctypes.byref(self.t), _ptr(q), len(q), _ptr(out))
        return out

    def range(self, start, length):
        start = np.ascontiguousarray(start, dtype=np.int64)
        length = np.ascontiguousarray(length, dtype=np.int32)
        n = len(start)
        cap = int(np.clip(length, 0, None).sum())
        off = np.empty(n + 1, np.int64)
        ok = np.empty(max(cap, 1), np.int64)
        ov = np.empty(max(cap, 1), np.int64)
        tot = _port_lib().hmo_range(ctypes.byref(self.t), _ptr(start), _ptr(length), n, _ptr(off), _ptr(ok), _ptr(ov), cap)
        return off, ok[:tot], ov[:tot]

    def range_between(self, start, end):
        """Inclusive ranges: every record with start[i] <= key <= end[i]."""
        start = np.ascontiguousarray(start, dtype=np.int64)
        end = np.ascontiguousarray(end, dtype=np.int64)
        n = len(start)
        off = np.empty(n + 1, np.int64)
        cap = max(4 * n, 1 << 12)
        while True:
            ok = np.empty(cap, np.int64)
            ov = np.empty(cap, np.int64)
            tot = _port_lib().hmo_range_between(ctypes.byref(self.t), _ptr(start), _ptr(end), n, _ptr(off),
                                                _ptr(ok), _ptr(ov), cap)
            if tot >= 0:
                return off, ok[:tot], ov[:tot]
            cap *= 4

    def export(self):
        n = self.t.n_keys
        k = np.empty(max(n, 1), np.int64)
        v = np.empty(max(n, 1), np.int64)
        m = _port_lib().hmo_export(ctypes.byref(self.t), _ptr(k), _ptr(v), n)
        return k[:m], v[:m]


def upsert_set(skeys, svals, bkeys, bvals, ref_rule: bool = False):
    """Sorted contents after one upsert batch (last occurrence wins)."""
    skeys = np.ascontiguousarray(skeys, dtype=np.int64)
    svals = np.ascontiguousarray(svals, dtype=np.int64)
    bkeys = np.ascontiguousarray(bkeys, dtype=np.int64)
    bvals = np.ascontiguousarray(bvals, dtype=np.int64)
    cap = len(skeys) + len(bkeys)
    ok = np.empty(max(cap, 1), np.int64)
    ov = np.empty(max(cap, 1), np.int64)
    m = _port_lib().hmo_upsert(_ptr(skeys), _ptr(svals), len(skeys), _ptr(bkeys), _ptr(bvals), len(bkeys),
                               1 if ref_rule else 0, _ptr(ok), _ptr(ov), cap)
    if m < 0:
        raise ValueError(f"hmo_upsert failed: {m}")
    return ok[:m], ov[:m]


_ref = None


def delete_set(skeys, svals, dkeys):
    """Contents after removing dkeys (set semantics; the reference's remove
    is an empty stub, open-harmonia/src/bpt.cpp:771-773, so this is the
    specification, not a restatement)."""
    keep = ~np.isin(skeys, np.asarray(dkeys, np.int64))
    return skeys[keep], svals[keep]


def gpu_ref_available() -> bool:
    return os.path.exists(GPU_SO)


def _ref_lib(path: str = REF_SO):
    global _ref
    if _ref is None:
        _ref = {}
    if path not in _ref:
        lib = ctypes.CDLL(path)
        lib.hmref_build.argtypes = [_P, _P, _L]
        lib.hmref_build.restype = _P
        for f in ("hmref_height",):
            getattr(lib, f).argtypes = [_P]
            getattr(lib, f).restype = ctypes.c_int
        for f in ("hmref_inner_nodes", "hmref_big_leaves"):
            getattr(lib, f).argtypes = [_P]
            getattr(lib, f).restype = _L
        lib.hmref_search.argtypes = [_P, _P, _L, _P, ctypes.c_int]
        lib.hmref_search_prefetch.argtypes = [_P, _P, _L, _P, ctypes.c_int]
        lib.hmref_range.argtypes = [_P, _P, _P, _L, _P, _P, _P, _L]
        lib.hmref_range.restype = _L
        lib.hmref_range_between.argtypes = [_P, _P, _P, _L, _P, _P, _P, _L, ctypes.c_int]
        lib.hmref_range_timed.argtypes = [_P, _P, _P, _L, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        lib.hmref_range_timed.restype = _L
        lib.hmref_range_between.restype = _L
        lib.hmref_upsert.argtypes = [_P, _P, _P, _L, _L, _L]
        lib.hmref_upsert.restype = ctypes.c_int
        lib.hmref_export.argtypes = [_P, _P, _P, _L]
        lib.hmref_export.restype = _L
        if path == GPU_SO:
            lib.hmrefgpu_prepare.argtypes = [_P]
            lib.hmrefgpu_prepare.restype = _P
            lib.hmrefgpu_free.argtypes = [_P]
            lib.hmrefgpu_check.argtypes = [_P, _P, _L]
            lib.hmrefgpu_check.restype = _L
            lib.hmrefgpu_search.argtypes = [_P, _P, _L, _P, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                            ctypes.POINTER(ctypes.c_float)]
            lib.hmrefgpu_search.restype = ctypes.c_int
            lib.hmrefgpu_emulate.argtypes = [_P, _P, _L, _P]
        _ref[path] = lib
    return _ref[path]


class RefTree:
    """The reference's PPI tree, built by inserting keys in the given order.
    gpu=True loads the library that also holds the reference's GPU search
    (oracle/_ref/libhmref_gpu.so), for RefGpuSearch."""

    def __init__(self, keys, vals, gpu: bool = False):
        self._k = np.ascontiguousarray(keys, dtype=np.int64)
        self._v = np.ascontiguousarray(vals, dtype=np.int64)
        self.lib_path = GPU_SO if gpu else REF_SO
        self.h = _ref_lib(self.lib_path).hmref_build(_ptr(self._k), _ptr(self._v), len(self._k))
        if not self.h:
            raise ValueError("the reference needs more than 4 keys for a PPI tree")

    @property
    def height(self) -> int:
        return _ref_lib(self.lib_path).hmref_height(self.h)

    def search(self, q, threads: int = 0) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.int64)
        out = np.empty_like(q)
        _ref_lib(self.lib_path).hmref_search(self.h, _ptr(q), len(q), _ptr(out), threads)
        return out

    def search_prefetch(self, q, threads: int = 0) -> np.ndarray:
        """The reference's software-pipelined search (16 queries per group,
        AVX2 child search, prefetch of each next node); fresh trees only."""
        q = np.ascontiguousarray(q, dtype=np.int64)
        out = np.empty_like(q)
        _ref_lib(self.lib_path).hmref_search_prefetch(self.h, _ptr(q), len(q), _ptr(out), threads)
        return out

    def range(self, start, length):
        start = np.ascontiguousarray(start, dtype=np.int64)
        length = np.ascontiguousarray(length, dtype=np.int32)
        n = len(start)
        cap = int(np.clip(length, 0, None).sum())
        off = np.empty(n + 1, np.int64)
        ok = np.empty(max(cap, 1), np.int64)
        ov = np.empty(max(cap, 1), np.int64)
        tot = _ref_lib(self.lib_path).hmref_range(self.h, _ptr(start), _ptr(length), n, _ptr(off), _ptr(ok), _ptr(ov), cap)
        return off, ok[:tot], ov[:tot]

    def range_timed(self, start, length, threads: int = 0):
        """The range walk over all queries in parallel (OpenMP, as the
        reference's CPU range experiment runs it), without compaction:
        returns (records, checksum)."""
        start = np.ascontiguousarray(start, dtype=np.int64)
        length = np.ascontiguousarray(length, dtype=np.int32)
        cs = ctypes.c_longlong()
        tot = _ref_lib(self.lib_path).hmref_range_timed(self.h, _ptr(start), _ptr(length), len(start), threads, ctypes.byref(cs))
        return int(tot), int(cs.value)

    def range_between(self, start, end, walk: bool = False):
        """Inclusive ranges by BPlusTree::range_search: every record with
        start[i] <= key <= end[i] (offsets, keys, values, compacted).  After
        an update, or with walk=True, the same walk over the update-aware
        descent (ref_driver.cpp range_between_walk)."""
        start = np.ascontiguousarray(start, dtype=np.int64)
        end = np.ascontiguousarray(end, dtype=np.int64)
        n = len(start)
        off = np.empty(n + 1, np.int64)
        cap = max(4 * n, 1 << 12)
        while True:
            ok = np.empty(cap, np.int64)
            ov = np.empty(cap, np.int64)
            tot = _ref_lib(self.lib_path).hmref_range_between(self.h, _ptr(start), _ptr(end), n, _ptr(off), _ptr(ok),
                                                 _ptr(ov), cap, 1 if walk else 0)
            if tot >= 0:
                return off, ok[:tot], ov[:tot]
            cap *= 4

    def upsert(self, keys, vals, syn_batch: int = 0, rebuild_batch: int = 0) -> None:
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        vals = np.ascontiguousarray(vals, dtype=np.int64)
        _ref_lib(self.lib_path).hmref_upsert(self.h, _ptr(keys), _ptr(vals), len(keys), syn_batch, rebuild_batch)

    def export(self):
        cap = 1 << 12
        while True:
            k = np.empty(cap, np.int64)
            v = np.empty(cap, np.int64)
            m = _ref_lib(self.lib_path).hmref_export(self.h, _ptr(k), _ptr(v), cap)
            if m >= 0:
                return k[:m], v[:m]
            cap *= 4


_cfb = None


def cfb_available() -> bool:
    return os.path.exists(CFB_SO)


def _cfb_lib():
    global _cfb
    if _cfb is None:
        lib = ctypes.CDLL(CFB_SO)
        lib.hmcfb_order.restype = ctypes.c_int
        lib.hmcfb_build.argtypes = [_P, _P, _L]
        lib.hmcfb_build.restype = _P
        lib.hmcfb_search.argtypes = [_P, _P, _L, _P, ctypes.c_int]
        _cfb = lib
    return _cfb


class CfbTree:
    """The reference's pointer B+tree at order 128 (open-harmonia/regular_bpt),
    built by insert() in the given key order; search is its find()."""

    def __init__(self, keys, vals):
        self._k = np.ascontiguousarray(keys, dtype=np.int64)
        self._v = np.ascontiguousarray(vals, dtype=np.int64)
        self.h = _cfb_lib().hmcfb_build(_ptr(self._k), _ptr(self._v), len(self._k))

    @property
    def order(self) -> int:
        return _cfb_lib().hmcfb_order()

    def search(self, q, threads: int = 0) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.int64)
        out = np.empty_like(q)
        _cfb_lib().hmcfb_search(self.h, _ptr(q), len(q), _ptr(out), threads)
        return out


class RefGpuSearch:
    """The reference's own GPU point search (open-harmonia/src/full-multi-
    prefix-sort-8thread.cu: CUB SortPairs on bits [48, 64) and the 8-thread
    kernel) on a RefTree built with gpu=True, through oracle/ref_gpu_driver.cu."""

    def __init__(self, tree: RefTree):
        if tree.lib_path != GPU_SO:
            raise ValueError("build the RefTree with gpu=True")
        self.tree = tree
        self.lib = _ref_lib(GPU_SO)
        self.g = self.lib.hmrefgpu_prepare(tree.h)
        if not self.g:
            raise RuntimeError("hmrefgpu_prepare failed (no device, or out of memory)")

    def check(self, q) -> int:
        """Keys the kernel would search outside the tree's arrays (CPU only)."""
        q = np.ascontiguousarray(q, dtype=np.int64)
        return int(self.lib.hmrefgpu_check(self.tree.h, _ptr(q), len(q)))

    def search(self, q, reps: int = 3):
        """(values, mean device ms of sort + kernel, device ms with copies)."""
        q = np.ascontiguousarray(q, dtype=np.int64)
        out = np.full(len(q), -7, np.int64)
        md, mc = ctypes.c_float(), ctypes.c_float()
        rc = self.lib.hmrefgpu_search(self.g, _ptr(q), len(q), _ptr(out), reps, ctypes.byref(md), ctypes.byref(mc))
        if rc != 0:
            raise RuntimeError(f"hmrefgpu_search failed: {rc}")
        return out, float(md.value), float(mc.value)

    def close(self):
        if self.g:
            self.lib.hmrefgpu_free(self.g)
            self.g = None


def check_gpu_ref_batch(tree: RefTree, q) -> int:
    """The CPU check of the reference GPU kernel's index path alone."""
    q = np.ascontiguousarray(q, dtype=np.int64)
    return int(_ref_lib(GPU_SO).hmrefgpu_check(tree.h, _ptr(q), len(q)))


def emulate_gpu_ref(tree: RefTree, q) -> np.ndarray:
    """The reference GPU kernel's computation run on the CPU (for locating
    where its results depart from the CPU search); -7 marks refused keys."""
    q = np.ascontiguousarray(q, dtype=np.int64)
    out = np.empty_like(q)
    _ref_lib(GPU_SO).hmrefgpu_emulate(tree.h, _ptr(q), len(q), _ptr(out))
    return out

