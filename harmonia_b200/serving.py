"""Python binding of the serving loop (hm_server_* in include/harmonia.h).

A ``Server`` wraps one tree.  ``search``, ``range`` and ``upsert`` submit a
request with host (numpy) buffers and return a ``Ticket``; ``Ticket.wait()``
blocks until the dispatcher has answered it and returns the result.  The
ticket keeps the request's buffers alive until then, as the C API requires.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native
from .native import HarmoniaError, check, lib

HM_REQ_SEARCH, HM_REQ_RANGE, HM_REQ_UPSERT, HM_REQ_DELETE = 0, 1, 2, 3


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("keys", ctypes.c_void_p), ("lens", ctypes.c_void_p),
                ("vals", ctypes.c_void_p), ("n", ctypes.c_size_t), ("out", ctypes.c_void_p),
                ("offsets", ctypes.c_void_p), ("out_keys", ctypes.c_void_p), ("out_vals", ctypes.c_void_p),
                ("out_cap", ctypes.c_size_t), ("flags", ctypes.c_int)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device_budget_bytes", ctypes.c_size_t), ("max_queue", ctypes.c_int), ("streams", ctypes.c_int),
                ("max_launch_queries", ctypes.c_int64), ("device_wait_limit_ms", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("epochs", ctypes.c_uint64), ("queries", ctypes.c_uint64),
                ("pending", ctypes.c_uint64), ("p50_us", ctypes.c_double), ("p99_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("elapsed_s", ctypes.c_double),
                ("queue_p50_us", ctypes.c_double), ("queue_p99_us", ctypes.c_double),
                ("stage_p50_us", ctypes.c_double), ("stage_p99_us", ctypes.c_double),
                ("device_p50_us", ctypes.c_double), ("device_p99_us", ctypes.c_double),
                ("finish_p50_us", ctypes.c_double), ("finish_p99_us", ctypes.c_double),
                ("epoch_drain_mean_us", ctypes.c_double), ("epoch_apply_mean_us", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    L = lib()
    P = ctypes.c_void_p
    L.hm_server_config_default.argtypes = [ctypes.POINTER(ServerConfig)]
    L.hm_server_start.argtypes = [P, ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]
    L.hm_server_submit.argtypes = [P, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]
    L.hm_server_wait.argtypes = [P, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]
    L.hm_server_get_stats.argtypes = [P, ctypes.POINTER(ServerStats)]
    L.hm_server_reset_stats.argtypes = [P]
    L.hm_server_stop.argtypes = [P]
    L.hm_server_free.argtypes = [P]
    _bound = True
    return L


def _is_cuda_tensor(a) -> bool:
    return getattr(a, "is_cuda", False) is True and hasattr(a, "data_ptr")


class Ticket:
    def __init__(self, server: "Server", ticket: int, kind: int, keep: tuple, result):
        self.server = server
        self.ticket = ticket
        self.kind = kind
        self._keep = keep  # buffers the dispatcher reads/writes until done
        self._result = result
        self.status = None

    def wait(self, timeout_us: int = -1, check_status: bool = True):
        if self.status is not None:  # already collected
            if check_status and self.status != 0:
                raise HarmoniaError(self.status, "request")
            return self._result()
        st = ctypes.c_int()
        rc = _bind().hm_server_wait(self.server._h, self.ticket, timeout_us, ctypes.byref(st))
        if rc != 0:
            raise HarmoniaError(rc, "hm_server_wait")
        self.status = st.value
        if check_status and st.value != 0:
            raise HarmoniaError(st.value, "request")
        return self._result()


class Server:
    def __init__(self, tree, device_budget_bytes=None, max_queue=None, streams=None, max_launch_queries=None,
                 device_wait_limit_ms=None):
        L = _bind()
        cfg = ServerConfig()
        check(L.hm_server_config_default(ctypes.byref(cfg)), "hm_server_config_default")
        for k, v in (("device_budget_bytes", device_budget_bytes), ("max_queue", max_queue), ("streams", streams),
                     ("max_launch_queries", max_launch_queries), ("device_wait_limit_ms", device_wait_limit_ms)):
            if v is not None:
                setattr(cfg, k, int(v))
        h = ctypes.c_void_p()
        check(L.hm_server_start(tree.handle, ctypes.byref(cfg), ctypes.byref(h)), "hm_server_start")
        self._h = h
        self._tree = tree

    def _submit(self, req: Request) -> int:
        t = ctypes.c_uint64()
        rc = _bind().hm_server_submit(self._h, ctypes.byref(req), ctypes.byref(t))
        if rc != 0:
            raise HarmoniaError(rc, "hm_server_submit")
        return t.value

    def search(self, keys, out=None) -> Ticket:
        """Point search; out (optional) receives the values.  keys and out in
        page-locked memory (e.g. numpy views of torch tensors made with
        pin_memory=True) are copied by DMA without a staging copy; so are
        contiguous int64 torch CUDA tensors (device memory), which may be
        passed for either."""
        if _is_cuda_tensor(keys) or _is_cuda_tensor(out):
            return self._search_tensors(keys, out)
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        if out is None:
            out = np.empty(len(keys), np.int64)
        elif out.dtype != np.int64 or not out.flags.c_contiguous or len(out) != len(keys):
            raise ValueError("out must be a contiguous int64 array as long as keys")
        r = Request(kind=HM_REQ_SEARCH, keys=keys.ctypes.data, n=len(keys), out=out.ctypes.data)
        return Ticket(self, self._submit(r), HM_REQ_SEARCH, (keys, out), lambda: out)

    def _search_tensors(self, keys, out):
        import torch
        if not _is_cuda_tensor(keys):
            keys = np.ascontiguousarray(keys, dtype=np.int64)
        n = len(keys)
        if out is None:
            out = np.empty(n, np.int64)
        for a in (keys, out):
            if _is_cuda_tensor(a):
                if a.dtype != torch.int64 or not a.is_contiguous():
                    raise ValueError("CUDA tensors must be contiguous int64")
            elif a.dtype != np.int64 or not a.flags.c_contiguous:
                raise ValueError("host buffers must be contiguous int64 arrays")
        if len(out) != n:
            raise ValueError("out must be as long as keys")

        def ptr(a):
            return a.data_ptr() if _is_cuda_tensor(a) else a.ctypes.data

        r = Request(kind=HM_REQ_SEARCH, keys=ptr(keys), n=n, out=ptr(out))
        return Ticket(self, self._submit(r), HM_REQ_SEARCH, (keys, out), lambda: out)

    def range(self, start, length, cap=None) -> Ticket:
        start = np.ascontiguousarray(start, dtype=np.int64)
        length = np.ascontiguousarray(length, dtype=np.int32)
        n = len(start)
        cap = int(length.clip(min=0).sum()) if cap is None else int(cap)
        offsets = np.empty(n + 1, np.int64)
        ok = np.empty(max(cap, 1), np.int64)
        ov = np.empty(max(cap, 1), np.int64)
        r = Request(kind=HM_REQ_RANGE, keys=start.ctypes.data, lens=length.ctypes.data, n=n,
                    offsets=offsets.ctypes.data, out_keys=ok.ctypes.data, out_vals=ov.ctypes.data, out_cap=cap)
        return Ticket(self, self._submit(r), HM_REQ_RANGE, (start, length, offsets, ok, ov),
                      lambda: (offsets, ok[: offsets[-1]], ov[: offsets[-1]]))

    def upsert(self, keys, vals, ref_rule: bool = False) -> Ticket:
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        vals = np.ascontiguousarray(vals, dtype=np.int64)
        r = Request(kind=HM_REQ_UPSERT, keys=keys.ctypes.data, vals=vals.ctypes.data, n=len(keys),
                    flags=native.HM_UPSERT_REF_KEY_MINUS_1 if ref_rule else native.HM_UPSERT_SUPPLIED)
        return Ticket(self, self._submit(r), HM_REQ_UPSERT, (keys, vals), lambda: None)

    def delete(self, keys) -> Ticket:
        """Removes the stored keys among keys (an epoch barrier, like upsert)."""
        keys = np.ascontiguousarray(np.asarray(keys, dtype=np.int64))
        r = Request(kind=HM_REQ_DELETE, keys=keys.ctypes.data, n=len(keys))
        return Ticket(self, self._submit(r), HM_REQ_DELETE, (keys,), lambda: None)

    def stats(self) -> dict:
        s = ServerStats()
        check(_bind().hm_server_get_stats(self._h, ctypes.byref(s)), "hm_server_get_stats")
        return s.as_dict()

    def reset_stats(self) -> None:
        check(_bind().hm_server_reset_stats(self._h), "hm_server_reset_stats")

    def stop(self) -> None:
        """Cancels queued requests, finishes those in flight; tickets stay waitable."""
        if self._h is not None and self._h.value:
            check(_bind().hm_server_stop(self._h), "hm_server_stop")

    def close(self) -> None:
        if self._h is not None and self._h.value:
            check(_bind().hm_server_free(self._h), "hm_server_free")
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
