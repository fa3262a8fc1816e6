"""Read-only calls on one tree that overlap on the device.

The C ABI lets read-only calls (hm_search, hm_range, hm_search_batches,
hm_export) on one tree run concurrently on different streams, from one host
thread or several.  Each call leases its own block of the tree's scratch pool;
a block is ordered after its previous use, and a block that is too small is
replaced by a larger one (the old one is freed with the tree), so no call
frees device memory while others run.  The bucket join's
boundary cache is filled once under the tree's lock, and later callers wait on
the fill's event.

These tests enqueue work on several streams without synchronising in between,
with sizes that make scratch blocks grow mid-sequence, and compare every result
with the oracle (exact: integer results)."""
import threading

import numpy as np
import pytest

from harmonia_b200 import BPlusTree, datagen as dg
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def tree_1m():
    keys = dg.gen_keys(1 << 20, seed=31)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    t = BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)))
    yield keys, sk, oracle, t
    t.close()


def test_searches_and_range_on_three_streams_overlap(tree_1m):
    keys, sk, oracle, t = tree_1m
    # pre-sort at every size, so every search needs scratch; descent, no join
    t.set_search_config(sort_bits=8, join=2)
    try:
        sizes_1 = [4096, 1 << 21]  # the second call grows stream 1's block
        size_2 = 3 << 20
        qs1 = [dg.gen_point_queries(keys, m, 0.6, seed=100 + i) for i, m in enumerate(sizes_1)]
        q2 = dg.gen_point_queries(keys, size_2, 0.6, seed=110)
        st, ln = dg.gen_ranges(1 << 16, 1, 64, seed=111)
        d1 = [cuda(q) for q in qs1]
        d2 = cuda(q2)
        o1 = [torch.full_like(d, -7) for d in d1]
        o2 = torch.full_like(d2, -7)
        dst, dln = cuda(st), cuda(ln.astype(np.int32))
        torch.cuda.synchronize()
        s1, s2, s3 = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        t.search(d1[0], o1[0], stream=s1)
        t.search(d2, o2, stream=s2)
        t.search(d1[1], o1[1], stream=s1)
        off, rk, rv = t.range_search(dst, dln, stream=s3)  # returns once its total is known
        o3 = torch.full_like(d1[0], -7)
        t.search(d1[0], o3, stream=s2)  # reuses stream 2's block after its first call
        torch.cuda.synchronize()
        for q, o in zip(qs1, o1):
            assert (o.cpu().numpy() == oracle.search(q)).all()
        assert (o2.cpu().numpy() == oracle.search(q2)).all()
        assert (o3.cpu().numpy() == oracle.search(qs1[0])).all()
        eoff, ek, ev = oracle.range(st, ln)
        assert (off.cpu().numpy() == eoff).all()
        assert (rk.cpu().numpy() == ek).all() and (rv.cpu().numpy() == ev).all()
    finally:
        t.set_search_config(sort_bits=-1, join=-1)


def test_join_calls_on_two_streams_share_the_boundary_cache():
    """A fresh tree's first two joins start on two streams at once: one fills
    the bucket-boundary cache, the other waits for the fill (or fills it
    first); both answers must be exact."""
    keys = dg.gen_keys(1 << 20, seed=41)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys))) as t:
        t.set_search_config(join=1)
        qa = dg.gen_point_queries(keys, 1 << 22, 0.9, seed=42)
        qb = dg.gen_zipf_queries(sk, 3 << 20, 0.99, seed=43)
        da, db = cuda(qa), cuda(qb)
        oa, ob = torch.empty_like(da), torch.empty_like(db)
        torch.cuda.synchronize()
        sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
        t.search(da, oa, stream=sa)
        t.search(db, ob, stream=sb)
        torch.cuda.synchronize()
        assert (oa.cpu().numpy() == oracle.search(qa)).all()
        assert (ob.cpu().numpy() == oracle.search(qb)).all()


def test_host_threads_on_own_and_shared_streams(tree_1m):
    """Four host threads issue searches and ranges at once: three on streams
    of their own, two of them sharing one stream.  Calls from two threads on
    one stream still get separate scratch blocks."""
    keys, sk, oracle, t = tree_1m
    t.set_search_config(sort_bits=8, join=2)
    shared = torch.cuda.Stream()
    streams = [torch.cuda.Stream(), torch.cuda.Stream(), shared, shared]
    work, errors = [], []
    for w in range(4):
        items = []
        for c in range(3):
            m = [1000, 1 << 18, 700001][(w + c) % 3]
            q = dg.gen_point_queries(keys, m, 0.5, seed=200 + 10 * w + c)
            st, ln = dg.gen_ranges(2048, 1, 32, seed=300 + 10 * w + c)
            items.append((q, cuda(q), st, ln))
        work.append(items)
    torch.cuda.synchronize()
    results = [[None] * 3 for _ in range(4)]

    def run(w):
        try:
            with torch.cuda.stream(streams[w]):
                for c, (q, dq, st, ln) in enumerate(work[w]):
                    out = torch.empty_like(dq)
                    t.search(dq, out, stream=streams[w])
                    rng = t.range_search(st, ln, stream=streams[w])  # host buffers: returns when done
                    streams[w].synchronize()
                    results[w][c] = (out.cpu().numpy(), rng)
        except Exception as e:  # reported on the main thread
            errors.append(e)

    try:
        th = [threading.Thread(target=run, args=(w,)) for w in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        assert not errors, errors
        for w in range(4):
            for c, (q, dq, st, ln) in enumerate(work[w]):
                got, (off, rk, rv) = results[w][c]
                assert (got == oracle.search(q)).all(), (w, c)
                eoff, ek, ev = oracle.range(st, ln)
                assert (off == eoff).all() and (rk == ek).all() and (rv == ev).all(), (w, c)
    finally:
        t.set_search_config(sort_bits=-1, join=-1)
