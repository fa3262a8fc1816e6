"""GPU tests of the serving loop: results in the mix equal results alone,
continuous batching from several submitter threads, and the host-side
failure paths (admission refusals, cancellation, timeouts, bad requests).
No test faults or hangs the GPU: every failure is made on the host."""
import threading
import time

import numpy as np
import pytest

from harmonia_b200 import BPlusTree, HarmoniaError, datagen as dg
from harmonia_b200.serving import Server
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def make_tree(n=1 << 18, seed=3, leaf_fill=12):
    keys = dg.gen_keys(n, seed)
    return keys, BPlusTree.bulk_load(keys, dg.values_for(keys), leaf_fill=leaf_fill)


def request_mix(keys, count, seed):
    """90% point (80% hits) / 5% range (1..128) / 5% upsert (half new, half existing)."""
    rng = np.random.default_rng(seed)
    live = np.sort(keys)
    out = []
    for i in range(count):
        u = rng.random()
        m = int(np.exp(rng.uniform(np.log(64), np.log(1 << 14))))
        if u < 0.90:
            out.append(("search", dg.gen_point_queries(live, m, 0.8, seed * 1000 + i)))
        elif u < 0.95:
            out.append(("range", dg.gen_ranges(max(1, m // 64), 1, 128, seed * 1000 + i)))
        else:
            bk, bv = dg.gen_upserts(live, max(2, m // 8), 0.5, seed * 1000 + i)
            out.append(("upsert", (bk, bv)))
            live = np.union1d(live, bk)
    return out


def expected_results(keys, reqs):
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    tree = po.PortTree(sk, sv)
    exp = []
    for kind, data in reqs:
        if kind == "search":
            exp.append(tree.search(data))
        elif kind == "range":
            exp.append(tree.range(*data))
        else:
            sk, sv = po.upsert_set(sk, sv, *data)
            tree = po.PortTree(sk, sv)
            exp.append(None)
    return exp, sk, sv


def check(kind, got, exp):
    if kind == "search":
        assert (got == exp).all()
    elif kind == "range":
        assert all((a == b).all() for a, b in zip(got, exp))


def test_mixed_stream_results_equal_results_alone():
    keys, tree = make_tree()
    reqs = request_mix(keys, 300, seed=5)
    exp, sk, sv = expected_results(keys, reqs)
    with tree, Server(tree, streams=3, max_launch_queries=1 << 16) as srv:
        tickets = []
        for kind, data in reqs:
            if kind == "search":
                tickets.append(srv.search(data))
            elif kind == "range":
                tickets.append(srv.range(*data))
            else:
                tickets.append(srv.upsert(*data))
        for (kind, _), tk, e in zip(reqs, tickets, exp):
            check(kind, tk.wait(), e)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["launches"] < len(reqs)  # reads were coalesced
        assert st["p99_us"] >= st["p50_us"] > 0
        xk, xv = tree.export()
        assert (xk == sk).all() and (xv == sv).all()
    # the same requests one at a time (each waited before the next) give the same answers
    keys2, tree2 = make_tree()
    with tree2, Server(tree2, streams=1) as srv:
        for (kind, data), e in zip(reqs[:120], exp[:120]):
            tk = srv.search(data) if kind == "search" else srv.range(*data) if kind == "range" else srv.upsert(*data)
            check(kind, tk.wait(), e)


def test_page_locked_buffers_mixed_with_pageable():
    """Point requests whose keys and/or out are page-locked go by DMA, the
    others through staging, coalesced into the same launches and around
    upsert epochs; every answer equals the oracle's."""
    keys, tree = make_tree(1 << 18, seed=21)
    reqs = request_mix(keys, 200, seed=23)
    exp, sk, sv = expected_results(keys, reqs)
    rng = np.random.default_rng(29)

    def pinned(a):
        b = torch.empty(len(a), dtype=torch.int64, pin_memory=True).numpy()
        b[:] = a
        return b

    kinds = []
    with tree, Server(tree, streams=3, max_launch_queries=1 << 15) as srv:
        tickets = []
        for kind, data in reqs:
            if kind == "search":
                mode = int(rng.integers(0, 4))  # bit 0: keys pinned, bit 1: out pinned
                kinds.append(mode)
                q = pinned(data) if mode & 1 else data
                out = torch.empty(len(data), dtype=torch.int64, pin_memory=True).numpy() if mode & 2 else None
                tickets.append(srv.search(q, out=out))
            elif kind == "range":
                tickets.append(srv.range(*data))
            else:
                tickets.append(srv.upsert(*data))
        for (kind, _), tk, e in zip(reqs, tickets, exp):
            check(kind, tk.wait(), e)
        assert srv.stats()["failed"] == 0
    assert set(kinds) == {0, 1, 2, 3}


def test_device_buffers():
    """Point requests whose keys and/or out are CUDA tensors (device memory)
    are copied by DMA (device to device), mixed with host requests."""
    keys, tree = make_tree(1 << 18, seed=31)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with tree, Server(tree, streams=2, max_launch_queries=1 << 15) as srv:
        qs = [dg.gen_point_queries(keys, 1000 + 111 * i, 0.7, seed=40 + i) for i in range(12)]
        tks, outs = [], []
        for i, q in enumerate(qs):
            mode = i % 4  # bit 0: keys on the device, bit 1: out on the device
            kq = torch.from_numpy(q).cuda() if mode & 1 else q
            out = torch.empty(len(q), dtype=torch.int64, device="cuda") if mode & 2 else None
            tks.append(srv.search(kq, out=out))
        for q, tk in zip(qs, tks):
            got = tk.wait()
            got = got.cpu().numpy() if hasattr(got, "cpu") else got
            assert (got == oracle.search(q)).all()


def test_concurrent_submitters_continuous_batching():
    keys, tree = make_tree(1 << 19, seed=9)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    errors = []
    with tree, Server(tree, streams=4, max_launch_queries=1 << 15) as srv:
        def worker(w):
            try:
                for i in range(40):
                    q = dg.gen_point_queries(keys, 1000 + 37 * i + w, 0.8, seed=w * 100 + i)
                    got = srv.search(q).wait()
                    if not (got == oracle.search(q)).all():
                        errors.append((w, i))
            except Exception as e:  # pragma: no cover - reported below
                errors.append(repr(e))
        ths = [threading.Thread(target=worker, args=(w,)) for w in range(6)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        st = srv.stats()
    assert not errors
    assert st["completed"] == 240


def test_admission_refusals_and_bad_requests():
    keys, tree = make_tree(1 << 14, seed=11)
    with tree, Server(tree, device_budget_bytes=1 << 16, max_queue=4) as srv:
        with pytest.raises(HarmoniaError) as e:  # one request larger than the whole budget
            srv.search(np.zeros(1 << 13, np.int64))
        assert e.value.code == -9
        from harmonia_b200.serving import Request, _bind
        import ctypes
        bad = Request(kind=7, n=1)
        t = ctypes.c_uint64()
        assert _bind().hm_server_submit(srv._h, ctypes.byref(bad), ctypes.byref(t)) == -1
        bad = Request(kind=0, n=5)  # null buffers
        assert _bind().hm_server_submit(srv._h, ctypes.byref(bad), ctypes.byref(t)) == -1
        ok = srv.search(keys[:100]).wait()
        assert (ok >= 0).all()
        assert srv.stats()["rejected"] >= 1


def test_stop_cancels_queued_and_wait_times_out():
    keys, tree = make_tree(1 << 20, seed=13)
    with tree, Server(tree, streams=1, max_launch_queries=1 << 20) as srv:
        qs = [dg.gen_point_queries(keys, 1 << 20, 0.5, seed=i) for i in range(12)]
        big = [srv.search(q) for q in qs]  # submitted back to back: most stay queued
        with pytest.raises(HarmoniaError) as e:  # still queued: a zero wait times out
            big[-1].wait(timeout_us=0)
        assert e.value.code == -7
        t_end = time.monotonic() + 10.0  # the first request has left the queue (launched)
        while srv.stats()["launches"] < 1 and time.monotonic() < t_end:
            time.sleep(0.001)
        srv.stop()  # queued requests are cancelled, in-flight ones finish
        statuses = []
        for tk in big:
            try:
                tk.wait(check_status=False)
            except HarmoniaError:
                pass
            statuses.append(tk.status)
        assert statuses[0] == 0
        assert -10 in statuses  # HM_ECANCELLED for the ones still queued
        with pytest.raises(HarmoniaError) as e:
            srv.search(keys[:10])
        assert e.value.code == -10


def test_c5_serving_replay_matches_reference():
    """The seeded serving stream on a 2^25-key tree (400 requests: point
    searches, ranges and upsert epochs, sizes 64..2^20) submitted back to back
    to a server with three launch slots: every read's result and the final
    contents against the reference replaying the same stream in submission
    order (golden.json c5_serving_replay)."""
    from tests.helpers import digest, load_golden
    g = load_golden()["c5_serving_replay"]
    keys = dg.gen_keys(g["n"], g["key_seed"])
    stream = dg.gen_serving_stream(keys, g["count"], g["seed"])
    assert "".join(r[0][0] for r in stream) == g["kinds"]
    tree = BPlusTree.bulk_load(torch.from_numpy(keys).cuda(), torch.from_numpy(dg.values_for(keys)).cuda(),
                               leaf_fill=12)
    with tree, Server(tree, streams=3, max_launch_queries=1 << 22, device_budget_bytes=2 << 30) as srv:
        tickets = []
        for req in stream:
            if req[0] == "search":
                tickets.append(srv.search(req[1]))
            elif req[0] == "range":
                tickets.append(srv.range(req[1], req[2]))
            else:
                tickets.append(srv.upsert(req[1], req[2]))
        reads = []
        for req, tk in zip(stream, tickets):
            r = tk.wait()
            if req[0] == "search":
                reads.append(digest(r))
            elif req[0] == "range":
                reads.append(digest(*r))
        bad = [i for i, (a, b) in enumerate(zip(reads, g["read_digests"])) if a != b]
        assert len(reads) == len(g["read_digests"]) and not bad, f"reads {bad[:8]} differ"
        st = srv.stats()
        assert st["failed"] == 0 and st["completed"] == g["count"]
        ek, ev = tree.export()
        assert len(ek) == g["n_after"] and digest(ek, ev) == g["export_digest"]
