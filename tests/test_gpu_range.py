"""GPU parity tests of the range scan with prefix-sum compaction."""
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


@pytest.fixture(scope="module")
def c1():
    g = GOLD["c1_point"]
    keys = dg.gen_keys(g["n"], g["key_seed"])
    sk = np.sort(keys)
    t = BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)))
    yield keys, sk, t
    t.close()


def test_c1_range_digest_device_and_host(c1):
    keys, sk, t = c1
    g = GOLD["c1_range"]
    st, ln = dg.gen_ranges(g["m"], g["lo"], g["hi"], g["seed"])
    off, k, v = t.range_search(cuda(st), cuda(ln))
    assert digest(off.cpu().numpy(), k.cpu().numpy(), v.cpu().numpy()) == g["digest"]
    off, k, v = t.range_search(st, ln)
    assert digest(off, k, v) == g["digest"]


@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (64, 64), (128, 16), (128, 64)])
def test_small_golden(fanout, leaf_cap):
    s = load_small()
    keys = dg.gen_keys(int(s["n"]), int(s["key_seed"]))
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=fanout, leaf_cap=leaf_cap) as t:
        off, k, v = t.range_search(s["r_start"], s["r_len"])
        assert (off == s["r_off"]).all() and (k == s["r_keys"]).all() and (v == s["r_vals"]).all()


def test_edge_ranges(c1):
    keys, sk, t = c1
    st = np.array([sk[0], sk[-1], sk[-1] + 1, 2**63 - 1, -(2**63), sk[5] + 1, sk[100], sk[-2]], np.int64)
    ln = np.array([3, 5, 4, 9, 2, 0, -3, 1000], np.int32)
    exp = po.PortTree(sk, dg.values_for(sk)).range(st, ln)
    got = t.range_search(cuda(st), cuda(ln))
    for a, b in zip(got, exp):
        assert (a.cpu().numpy() == b).all()
    assert exp[0][-1] == 3 + 1 + 0 + 0 + 2 + 0 + 0 + 2


def test_capacity_error(c1):
    keys, sk, t = c1
    st = cuda(np.array([sk[0]], np.int64))
    ln = cuda(np.array([10], np.int32))
    import ctypes
    from harmonia_b200 import native
    off = torch.empty(2, dtype=torch.int64, device="cuda")
    ok = torch.empty(4, dtype=torch.int64, device="cuda")
    tot = ctypes.c_size_t()
    rc = native.lib().hm_range(t.handle, st.data_ptr(), ln.data_ptr(), 1, off.data_ptr(), ok.data_ptr(),
                               ok.data_ptr(), 4, ctypes.byref(tot), None)
    assert rc == -6 and tot.value == 10


def test_empty_tree_and_empty_batch():
    with BPlusTree.bulk_load(np.zeros(0, np.int64), np.zeros(0, np.int64)) as t:
        off, k, v = t.range_search(np.array([0, 5], np.int64), np.array([3, 3], np.int32))
        assert off.tolist() == [0, 0, 0] and len(k) == 0
        off, k, v = t.range_search(np.zeros(0, np.int64), np.zeros(0, np.int32))
        assert off.tolist() == [0]


@pytest.mark.parametrize("leaf_cap,fill", [(16, 1), (16, 3), (64, 5)])
def test_ranges_across_many_sparse_leaves(leaf_cap, fill):
    # a few keys per leaf: one range spans up to 256 leaves, so the copy walks
    # several 32-leaf windows of leaf_base, with ranges starting and ending
    # anywhere inside them and running past the last key
    keys = dg.gen_keys(20000, seed=31)
    sk = np.sort(keys)
    sv = dg.values_for(sk)
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_cap=leaf_cap, leaf_fill=fill) as t:
        st, ln = dg.gen_ranges(3000, 1, 256, seed=32)
        st[:40] = sk[np.arange(40) * 400]   # exact key starts
        st[40:48] = sk[-8:]                 # near the end: the copy stops at the last key
        ln[:48] = 256
        oracle = po.PortTree(sk, sv)
        got = t.range_search(cuda(st), cuda(ln))
        exp = oracle.range(st, ln)
        for a, b in zip(got, exp):
            assert (a.cpu().numpy() == b).all()
        # after deletes leave leaves of uneven size (none empty)
        gone = sk[5:20000:3]
        t.delete(gone)
        ek = np.setdiff1d(sk, gone)
        got = t.range_search(cuda(st), cuda(ln))
        exp = po.PortTree(ek, dg.values_for(ek)).range(st, ln)
        for a, b in zip(got, exp):
            assert (a.cpu().numpy() == b).all()


# ---- inclusive ranges [start, end] (hm_range_between) ----

def _eq(got, exp):
    for a, b in zip(got, exp):
        a = a.cpu().numpy() if hasattr(a, "cpu") else a
        assert len(a) == len(b) and (a == b).all()


def test_c1_range_between_digest_before_and_after_upsert():
    """The reference's BPlusTree::range_search outputs (golden digests) on the
    C1 tree, then again after the C1 upsert epoch."""
    g, gu, ga = GOLD["c1_range_between"], GOLD["c1_upsert"], GOLD["c1_range_between_after"]
    keys = dg.gen_keys(GOLD["c1_point"]["n"], GOLD["c1_point"]["key_seed"])
    st, en = dg.gen_range_pairs(g["m"], g["n_keys"], g["lo"], g["hi"], g["seed"])
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=12) as t:
        off, k, v = t.range_between(cuda(st), cuda(en))
        assert digest(off.cpu().numpy(), k.cpu().numpy(), v.cpu().numpy()) == g["digest"]
        off, k, v = t.range_between(st, en)  # host buffers
        assert digest(off, k, v) == g["digest"]
        bk, bv = dg.gen_upserts(keys, gu["m"], gu["new_frac"], gu["seed"])
        t.upsert(bk, bv)
        off, k, v = t.range_between(cuda(st), cuda(en))
        assert digest(off.cpu().numpy(), k.cpu().numpy(), v.cpu().numpy()) == ga["digest"]


@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (64, 64), (128, 16), (128, 64)])
def test_range_between_matches_oracle(fanout, leaf_cap):
    keys = dg.gen_keys(50000, seed=61)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), fanout=fanout, leaf_cap=leaf_cap) as t:
        st, en = dg.gen_range_pairs(5000, len(keys), 1, 300, seed=62)
        _eq(t.range_between(cuda(st), cuda(en)), oracle.range_between(st, en))


def test_range_between_edges(c1):
    keys, sk, t = c1
    mx = 2**63 - 1
    st = np.array([sk[0], sk[10], sk[-1], sk[-1] + 1, -(2**63), sk[5] + 1, sk[100], sk[-3], 0, sk[7], mx, sk[50]],
                  np.int64)
    en = np.array([sk[0], sk[10], mx, mx, sk[2], sk[6] - 1, sk[99], mx, -1, sk[7] - 1, mx, sk[50] + 1], np.int64)
    exp = po.PortTree(sk, dg.values_for(sk)).range_between(st, en)
    # one key, one key, last key to the end, past the end, from the lowest
    # int64, a gap between keys, end < start, the last three keys, end < 0,
    # end < start by one, Max_Key alone, a key and the gap after it
    assert np.diff(exp[0]).tolist() == [1, 1, 1, 0, 3, 0, 0, 3, 0, 0, 0, 1]
    _eq(t.range_between(cuda(st), cuda(en)), exp)
    _eq(t.range_between(st, en), exp)


def test_range_between_capacity_and_empty():
    import ctypes
    from harmonia_b200 import native
    keys = dg.gen_keys(4096, seed=63)
    sk = np.sort(keys)
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        st, en = cuda(np.array([sk[0]], np.int64)), cuda(np.array([sk[9]], np.int64))
        off = torch.empty(2, dtype=torch.int64, device="cuda")
        ok = torch.empty(4, dtype=torch.int64, device="cuda")
        tot = ctypes.c_size_t()
        rc = native.lib().hm_range_between(t.handle, st.data_ptr(), en.data_ptr(), 1, off.data_ptr(),
                                           ok.data_ptr(), ok.data_ptr(), 4, ctypes.byref(tot), None)
        assert rc == native.HM_ECAPACITY and tot.value == 10
        off, k, v = t.range_between(np.zeros(0, np.int64), np.zeros(0, np.int64))
        assert off.tolist() == [0] and len(k) == 0
    with BPlusTree.bulk_load(np.zeros(0, np.int64), np.zeros(0, np.int64)) as t:
        off, k, v = t.range_between(np.array([0, -5], np.int64), np.array([100, 2**62], np.int64))
        assert off.tolist() == [0, 0, 0]


def test_range_between_after_deletes_on_sparse_leaves():
    keys = dg.gen_keys(20000, seed=64)
    sk = np.sort(keys)
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=3) as t:
        st, en = dg.gen_range_pairs(3000, len(keys), 1, 400, seed=65)
        gone = sk[7:20000:3]
        t.delete(gone)
        ek = np.setdiff1d(sk, gone)
        _eq(t.range_between(cuda(st), cuda(en)), po.PortTree(ek, dg.values_for(ek)).range_between(st, en))
