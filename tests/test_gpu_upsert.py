"""GPU parity tests of the epoch upsert (in-place merge and rebuild paths)."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, HarmoniaError, datagen as dg
from oracle import pyoracle as po
from tests.helpers import digest, load_golden, load_small

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLD = load_golden()


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("leaf_fill", [12, 16])
def test_c1_two_epochs_match_reference(leaf_fill):
    g0, g1, g2 = GOLD["c1_point"], GOLD["c1_upsert"], GOLD["c1_upsert2"]
    keys = dg.gen_keys(g0["n"], g0["key_seed"])
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=leaf_fill) as t:
        bk, bv = dg.gen_upserts(keys, g1["m"], g1["new_frac"], g1["seed"])
        t.upsert(cuda(bk), cuda(bv))
        ek, ev = t.export()
        assert len(ek) == g1["n_after"] and digest(ek, ev) == g1["export_digest"]
        assert digest(t.search(cuda(bk)).cpu().numpy()) == g1["search_digest"]
        bk2, bv2 = dg.gen_upserts(ek, g2["m"], g2["new_frac"], g2["seed"])
        t.upsert(bk2, bv2)  # host buffers
        ek2, ev2 = t.export()
        assert digest(ek2, ev2) == g2["export_digest"]
        assert digest(t.search(cuda(bk2)).cpu().numpy()) == g2["search_digest"]


def test_small_golden_reference_rule():
    s = load_small()
    keys = dg.gen_keys(int(s["n"]), int(s["key_seed"]))
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=128, leaf_cap=64, leaf_fill=40) as t:
        # the reference's rule ignores the supplied value of existing keys
        vals = np.where(np.isin(s["u_keys"], keys), 999, s["u_vals"])
        t.insert_parallel_Newupdate_batch(vals * 0 + s["u_keys"], vals)
        ek, ev = t.export()
        assert (ek == s["after_keys"]).all() and (ev == s["after_vals"]).all()


def test_duplicates_in_batch_last_wins():
    keys = np.arange(0, 2000, 2, dtype=np.int64)
    with BPlusTree.bulk_load(keys, keys * 10) as t:
        bk = np.array([4, 5, 4, 5, 7, 1999], np.int64)
        bv = np.array([1, 2, 3, 4, 5, 6], np.int64)
        t.upsert(bk, bv)
        ek, ev = po.upsert_set(keys, keys * 10, bk, bv)
        xk, xv = t.export()
        assert (xk == ek).all() and (xv == ev).all()
        assert t.search(cuda(np.array([4, 5, 7, 1999, 3], np.int64))).cpu().tolist() == [3, 4, 5, 6, -1]


@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_overflow_triggers_rebuild(fanout, leaf_cap):
    keys = dg.gen_keys(5000, seed=31)
    vals = dg.values_for(keys)
    with BPlusTree.bulk_load(keys, vals, fanout=fanout, leaf_cap=leaf_cap) as t:  # full leaves
        h0 = t.info().n_leaf
        bk, bv = dg.gen_upserts(keys, 6000, 0.9, seed=32)
        t.upsert(bk, bv)
        sk = np.sort(keys)
        ek, ev = po.upsert_set(sk, dg.values_for(sk), bk, bv)
        xk, xv = t.export()
        assert (xk == ek).all() and (xv == ev).all()
        assert t.info().n_leaf > h0
        q = np.concatenate([bk, dg.gen_point_queries(keys, 5000, 0.5, seed=33)])
        assert (t.search(cuda(q)).cpu().numpy() == po.PortTree(ek, ev).search(q)).all()
        st, ln = dg.gen_ranges(300, 1, 100, seed=34)
        got = t.range_search(st, ln)
        exp = po.PortTree(ek, ev).range(st, ln)
        assert all((a == b).all() for a, b in zip(got, exp))


def test_upsert_into_empty_tree_and_errors():
    with BPlusTree.bulk_load(np.zeros(0, np.int64), np.zeros(0, np.int64)) as t:
        bk = np.array([5, -3, 100], np.int64)
        t.upsert(bk, bk + 1)
        k, v = t.export()
        assert k.tolist() == [-3, 5, 100] and v.tolist() == [-2, 6, 101]
        with pytest.raises(HarmoniaError) as e:
            t.upsert(np.array([1, 2**63 - 1], np.int64), np.zeros(2, np.int64))
        assert e.value.code == -4
        assert t.export()[0].tolist() == [-3, 5, 100]


def test_oversized_batches_are_rejected_before_any_copy():
    """Upsert and delete batches hold at most 2^31 - 1 keys (the batch sort
    carries 32-bit input positions): a larger count gets HM_ETOOLARGE at the
    entry point, before a byte of the (here one-element) buffers is read, and
    the tree is unchanged."""
    import ctypes
    from harmonia_b200.native import lib
    with BPlusTree.bulk_load(np.array([1, 2, 3], np.int64), np.array([10, 20, 30], np.int64)) as t:
        one = torch.zeros(1, dtype=torch.int64, device="cuda")
        p = ctypes.c_void_p(one.data_ptr())
        assert lib().hm_upsert_batch(t._h, p, p, 1 << 31, 0, None) == -11
        removed = ctypes.c_size_t(7)
        assert lib().hm_delete_batch(t._h, p, 1 << 31, ctypes.byref(removed), None) == -11
        assert removed.value == 0
        k, v = t.export()
        assert k.tolist() == [1, 2, 3] and v.tolist() == [10, 20, 30]


def test_many_small_epochs_stay_exact():
    keys = dg.gen_keys(1 << 14, seed=41)
    sk, sv = np.sort(keys), dg.values_for(np.sort(keys))
    with BPlusTree.bulk_load(keys, dg.values_for(keys), leaf_fill=12) as t:
        for e in range(12):
            bk, bv = dg.gen_upserts(sk, 700, 0.5, seed=50 + e)
            t.upsert(cuda(bk), cuda(bv))
            sk, sv = po.upsert_set(sk, sv, bk, bv)
        xk, xv = t.export()
        assert (xk == sk).all() and (xv == sv).all()


def test_tiny_batches_on_a_large_tree():
    """In-place epochs of a few keys on a tree with far more leaves than keys
    in the batch (the rescan of leaf_base spans all leaves)."""
    keys = dg.gen_keys(1 << 21, seed=71)
    sk, sv = np.sort(keys), dg.values_for(np.sort(keys))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=12) as t:
        for e, m in enumerate((1, 3, 10, 64, 2)):
            bk, bv = dg.gen_upserts(sk, m, 0.5, seed=700 + e)
            t.upsert(bk, bv)
            sk, sv = po.upsert_set(sk, sv, bk, bv)
        xk, xv = t.export()
        assert (xk == sk).all() and (xv == sv).all()
        st, ln = dg.gen_ranges(2000, 1, 128, seed=77)
        got = t.range_search(st, ln)
        exp = po.PortTree(sk, sv).range(st, ln)
        assert all((a == b).all() for a, b in zip(got, exp))


def test_reused_device_blocks_stay_exact():
    """Trees built after others were freed (and after rebuilds) take their
    arenas, temporaries and scratch from the library's block cache; their
    contents and answers stay exact, and hm_trim_memory frees the cache."""
    from harmonia_b200 import trim_memory
    keys = dg.gen_keys(1 << 18, seed=131)
    sk, sv = np.sort(keys), dg.values_for(np.sort(keys))
    for rep in range(3):
        with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys))) as t:  # full leaves
            bk, bv = dg.gen_upserts(sk, 20000, 0.5, seed=140 + rep)  # overflows: a rebuild
            t.upsert(cuda(bk), cuda(bv))
            ek, ev = po.upsert_set(sk, sv, bk, bv)
            xk, xv = t.export()
            assert (xk == ek).all() and (xv == ev).all()
            q = dg.gen_point_queries(ek, 1 << 17, 0.7, seed=150 + rep)
            assert (t.search(cuda(q)).cpu().numpy() == po.PortTree(ek, ev).search(q)).all()
    assert trim_memory() > 0
    assert trim_memory() == 0


@pytest.mark.parametrize("fanout,leaf_cap,fill", [(64, 16, 12), (128, 64, 48)])
def test_small_epochs_one_kernel_path(fanout, leaf_cap, fill):
    """Epochs of at most 1024 keys go through the one-kernel path when every
    new key fits its leaf, and fall back to the general path (untouched tree
    first) when one does not: duplicates, both value rules, new smallest and
    largest keys (the join's bucket range moves), a full leaf, ranges and
    searches through the descent and the bucket join after every epoch."""
    keys = dg.gen_keys(1 << 18, seed=91)
    sk, sv = np.sort(keys), dg.values_for(np.sort(keys))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), fanout=fanout, leaf_cap=leaf_cap,
                             leaf_fill=fill) as t:
        lo, hi = int(sk[0]), int(sk[-1])
        crowd = np.arange(int(sk[100]) + 1, int(sk[100]) + 1 + 3 * leaf_cap, dtype=np.int64)  # overflows one leaf
        crowd = crowd[~np.isin(crowd, sk)][:leaf_cap]
        epochs = [
            (dg.gen_upserts(sk, 1000, 0.5, seed=92), 0),
            ((np.array([lo - 5, hi + 5, lo - 5, int(sk[7])], np.int64), np.array([1, 2, 3, 4], np.int64)), 0),
            (dg.gen_upserts(sk, 64, 0.3, seed=93), 1),
            ((crowd, crowd + 7), 0),
            (dg.gen_upserts(sk, 1024, 0.6, seed=94), 1),
        ]
        for (bk, bv), ref in epochs:
            if ref:
                t.insert_parallel_Newupdate_batch(bk, bv)
                bv = np.where(np.isin(bk, sk), bk - 1, bv)
                # the reference rule: an existing key's value becomes key - 1
                last = {}
                for k, v in zip(bk.tolist(), bv.tolist()):
                    last[k] = v
                bk = np.array(list(last.keys()), np.int64)
                bv = np.array(list(last.values()), np.int64)
            else:
                t.upsert(cuda(bk), cuda(bv))
            sk, sv = po.upsert_set(sk, sv, bk, bv)
            xk, xv = t.export()
            assert (xk == sk).all() and (xv == sv).all()
            oracle = po.PortTree(sk, sv)
            q = np.concatenate([bk, dg.gen_point_queries(sk, 1 << 18, 0.7, seed=95), [sk[0] - 1, sk[-1] + 1]])
            for join in (2, 1):
                t.set_search_config(join=join)
                assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all(), join
            t.set_search_config(join=-1)
            st, ln = dg.gen_ranges(500, 1, 100, seed=96)
            st[:3] = [sk[0], sk[-1], bk[0]]
            got = t.range_search(st, ln)
            assert all((a == b).all() for a, b in zip(got, oracle.range(st, ln)))
            room = np.int64(2**63 - 2) - st  # inclusive ranges rank their ends through leaf_base
            en = st + np.minimum(room, np.int64(1) << 44)
            got = t.range_between(st, en)
            assert all((a == b).all() for a, b in zip(got, oracle.range_between(st, en)))


@pytest.mark.parametrize("fanout,leaf_cap,fill", [(64, 16, 12), (128, 64, 48), (64, 64, 40)])
def test_overflowing_leaf_rebalances_its_subtree(fanout, leaf_cap, fill):
    # new keys packed into one leaf's key range overflow it while its subtree
    # (the last-level inner node's leaves) still has room: the subtree is
    # re-spread in place, the arena and the leaf count stay, plans need no
    # re-capture, and every read matches the oracle
    keys = dg.gen_keys(1 << 17, seed=61)
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=fanout, leaf_cap=leaf_cap, leaf_fill=fill) as t:
        info0 = t.info()
        q = dg.gen_point_queries(sk, 1 << 15, 0.8, seed=62)
        dq, dout = cuda(q), torch.empty(len(q), dtype=torch.int64, device="cuda")
        t.set_search_config(join=1)  # the join keeps its bucket boundaries per tree shape
        assert (t.search(dq).cpu().numpy() == po.PortTree(sk, sv).search(q)).all()
        t.set_search_config(join=-1)
        with t.plan([(dq, dout)]) as plan:
            ek, ev = sk, sv
            for epoch, at in enumerate((5000, 5000, 70000)):
                j = at + int(np.argmax(np.diff(ek[at:at + 40])))  # the widest gap near `at`
                lo, hi = int(ek[j]), int(ek[j + 1])
                room = leaf_cap - fill + 3
                new = np.unique(lo + 1 + (np.arange(room) * max(1, (hi - lo - 1) // (room + 1))))
                new = new[(new > lo) & (new < hi)]
                assert len(new) > leaf_cap - fill, "the gap must hold enough keys to overflow a leaf"
                upd = ek[j - 3: j]
                bk = np.concatenate([new, upd])
                bv = bk * 3 + epoch
                t.upsert(bk, bv)
                ek, ev = po.upsert_set(ek, ev, bk, bv)
                info = t.info()
                assert info.n_leaf == info0.n_leaf and info.leaf_rows == info0.leaf_rows  # no rebuild
                xk, xv = t.export()
                assert (xk == ek).all() and (xv == ev).all()
                oracle = po.PortTree(ek, ev)
                q2 = np.concatenate([bk, q])
                assert (t.search(cuda(q2)).cpu().numpy() == oracle.search(q2)).all()
                t.set_search_config(join=1)  # after the in-place rebalance
                assert (t.search(cuda(q2)).cpu().numpy() == oracle.search(q2)).all()
                t.set_search_config(join=-1)
                st, ln = dg.gen_ranges(2000, 1, 200, seed=63 + epoch)
                st[:50] = bk[:50] if len(bk) >= 50 else st[:50]
                got = t.range_search(st, ln)
                exp = oracle.range(st, ln)
                assert all((a == b).all() for a, b in zip(got, exp))
                plan.launch()
                torch.cuda.synchronize()
                assert (dout.cpu().numpy() == oracle.search(q)).all()
            # the join over rebalanced leaves (first keys must still order the leaves)
            t.set_search_config(join=1)
            big = dg.gen_point_queries(ek, 1 << 19, 0.9, seed=70)
            assert (t.search(cuda(big)).cpu().numpy() == po.PortTree(ek, ev).search(big)).all()
            t.set_search_config(join=-1)
