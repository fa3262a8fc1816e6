"""GPU tests of delete epochs (hm_delete_batch) and of reads after them.

The reference's BPlusTree::remove is an empty stub
(open-harmonia/src/bpt.cpp:771-773), so the specification is set semantics:
the contents after a delete are the contents before minus the deleted keys,
and point searches, range scans (first L records with key >= start) and
exports see exactly those contents.  The oracle is the C restatement
(oracle/hm_oracle.c) built on the expected contents."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, datagen as dg
from harmonia_b200.serving import Server
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def check_reads(t, ek, ev, seed):
    oracle = po.PortTree(ek, ev)
    xk, xv = t.export()
    assert (xk == ek).all() and (xv == ev).all()
    q = dg.gen_point_queries(ek if len(ek) else np.array([1], np.int64), 1 << 15, 0.5, seed)
    assert (t.search(q) == oracle.search(q)).all()
    assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all()
    start, length = dg.gen_ranges(4096, 1, 256, seed + 1)
    got = t.range_search(start, length)
    exp = oracle.range(start, length)
    assert all((a == b).all() for a, b in zip(got, exp))


@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_delete_in_place(fanout, leaf_cap):
    keys = dg.gen_keys(1 << 18, 31)
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    rng = np.random.default_rng(32)
    present = rng.choice(keys, 20000, replace=False)
    absent = dg.gen_point_queries(keys, 3000, 0.0, 33)
    batch = np.concatenate([present, absent, present[:500], np.array([2**63 - 1, -(2**63)], np.int64)])
    rng.shuffle(batch)
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=fanout, leaf_cap=leaf_cap,
                             leaf_fill=leaf_cap * 3 // 4) as t:
        gen0 = t.info().n_leaf
        removed = t.delete(cuda(batch))
        assert removed == len(present)
        ek, ev = po.delete_set(sk, sv, batch)
        assert t.size == len(ek) and t.info().n_leaf == gen0  # compacted in place
        check_reads(t, ek, ev, 34)
        # the bucket join on a large batch over the compacted leaves
        t.set_search_config(join=1)
        q = dg.gen_point_queries(sk, 1 << 20, 0.9, 35)
        assert (t.search(cuda(q)).cpu().numpy() == po.PortTree(ek, ev).search(q)).all()
        t.set_search_config(join=-1)
        # deleted keys can be stored again
        t.upsert(present[:1000], present[:1000] + 7)
        ek2, ev2 = po.upsert_set(ek, ev, present[:1000], present[:1000] + 7)
        check_reads(t, ek2, ev2, 36)
        assert t.delete(present[:1000]) == 1000  # and removed again
        check_reads(t, ek, ev, 37)


def test_emptied_leaves_rebuild_and_plans_follow():
    keys = dg.gen_keys(1 << 17, 41)
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        q = dg.gen_point_queries(sk, 1 << 16, 0.8, 42)
        dq, dout = cuda(q), torch.empty(len(q), dtype=torch.int64, device="cuda")
        with t.plan([(dq, dout)]) as plan:
            gone = sk[1000:9000]  # whole leaves: forces the rebuild
            assert t.delete(gone) == len(gone)
            ek, ev = po.delete_set(sk, sv, gone)
            check_reads(t, ek, ev, 43)
            plan.launch()
            torch.cuda.synchronize()
            assert (dout.cpu().numpy() == po.PortTree(ek, ev).search(q)).all()


def test_delete_everything_then_refill():
    keys = dg.gen_keys(5000, 44)
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        assert t.delete(keys) == len(keys)
        assert t.size == 0
        assert (t.search(keys) == -1).all()
        assert t.delete(keys) == 0
        t.upsert(keys[:100], dg.values_for(keys[:100]))
        sk = np.sort(keys[:100])
        check_reads(t, sk, dg.values_for(sk), 45)


def test_deletes_in_the_serving_stream():
    keys = dg.gen_keys(1 << 16, 51)
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    victims = sk[::7]
    with BPlusTree.bulk_load(keys, dg.values_for(keys), leaf_fill=12) as t, Server(t, streams=2) as srv:
        before = srv.search(victims)
        gone = srv.delete(victims)
        after = srv.search(victims)
        rest = srv.search(sk)
        assert (before.wait() == dg.values_for(victims)).all()  # submitted before the delete
        gone.wait()
        assert (after.wait() == -1).all()
        ek, ev = po.delete_set(sk, sv, victims)
        assert (rest.wait() == po.PortTree(ek, ev).search(sk)).all()
        xk, xv = t.export()
        assert (xk == ek).all() and (xv == ev).all()
