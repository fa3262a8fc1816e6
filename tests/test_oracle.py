"""CPU tests of the oracle: the C restatement is pinned to the reference's own
CPU B+tree through the golden fixtures (and directly, where the reference
library is built in this checkout)."""
import numpy as np
import pytest

from harmonia_b200 import datagen as dg
from oracle import pyoracle as po
from tests.helpers import digest, load_golden, load_small

GOLD = load_golden()


def test_splitmix64_numpy_matches_c():
    xs = np.array([0, 1, 2, 12345, 2**63 - 1, 2**64 - 1], dtype=np.uint64)
    got = dg.splitmix64(xs)
    assert [int(g) for g in got] == [po.splitmix64(int(x)) for x in xs]


def test_generated_keys_distinct_and_sentinel_free():
    k = dg.gen_keys(1 << 18, seed=3)
    assert len(np.unique(k)) == len(k)
    assert (k >= 0).all() and (k != dg.MAX_KEY).all()
    assert (dg.values_for(k) >= 0).all()
    assert (dg.gen_keys(1000, seed=3) == k[:1000]).all()  # prefix-stable, seeded


def test_port_matches_small_golden():
    s = load_small()
    keys = dg.gen_keys(int(s["n"]), int(s["key_seed"]))
    sk = np.sort(keys)
    for fanout, leaf_cap in [(64, 16), (64, 64), (128, 16), (128, 64)]:
        t = po.PortTree(sk, dg.values_for(sk), fanout=fanout, leaf_cap=leaf_cap)
        assert (t.search(s["q"]) == s["res"]).all()
        off, k, v = t.range(s["r_start"], s["r_len"])
        assert (off == s["r_off"]).all() and (k == s["r_keys"]).all() and (v == s["r_vals"]).all()
    ek, ev = po.upsert_set(sk, dg.values_for(sk), s["u_keys"], s["u_vals"])
    assert (ek == s["after_keys"]).all() and (ev == s["after_vals"]).all()


@pytest.fixture(scope="module")
def c1():
    g = GOLD["c1_point"]
    keys = dg.gen_keys(g["n"], g["key_seed"])
    sk = np.sort(keys)
    return keys, sk, dg.values_for(sk)


def test_port_matches_c1_point_digest(c1):
    keys, sk, sv = c1
    g = GOLD["c1_point"]
    q = dg.gen_point_queries(keys, g["m"], g["hit"], g["q_seed"])
    out = po.PortTree(sk, sv).search(q)
    assert digest(out) == g["digest"]
    assert int((out >= 0).sum()) == g["hits"]


def test_port_matches_c1_zipf_and_range_digests(c1):
    keys, sk, sv = c1
    t = po.PortTree(sk, sv, fanout=128, leaf_cap=64)
    g = GOLD["c1_zipf"]
    q = dg.gen_zipf_queries(sk, g["m"], g["theta"], g["q_seed"])
    assert digest(t.search(q)) == g["digest"]
    g = GOLD["c1_range"]
    st, ln = dg.gen_ranges(g["m"], g["lo"], g["hi"], g["seed"])
    off, k, v = t.range(st, ln)
    assert digest(off, k, v) == g["digest"]


def test_port_matches_c1_upsert_digests(c1):
    keys, sk, sv = c1
    g1, g2 = GOLD["c1_upsert"], GOLD["c1_upsert2"]
    bk, bv = dg.gen_upserts(keys, g1["m"], g1["new_frac"], g1["seed"])
    ek, ev = po.upsert_set(sk, sv, bk, bv)
    assert len(ek) == g1["n_after"] and digest(ek, ev) == g1["export_digest"]
    assert digest(po.PortTree(ek, ev).search(bk)) == g1["search_digest"]
    bk2, bv2 = dg.gen_upserts(ek, g2["m"], g2["new_frac"], g2["seed"])
    ek2, ev2 = po.upsert_set(ek, ev, bk2, bv2)
    assert digest(ek2, ev2) == g2["export_digest"]
    assert digest(po.PortTree(ek2, ev2).search(bk2)) == g2["search_digest"]


def test_reference_rule_upsert_equals_supplied_key_minus_1(c1):
    keys, sk, sv = c1
    bk, bv = dg.gen_upserts(keys, 4096, 0.5, 21)
    a = po.upsert_set(sk, sv, bk, bv)
    b = po.upsert_set(sk, sv, bk, np.where(np.isin(bk, sk), 12345, bv), ref_rule=True)
    assert (a[0] == b[0]).all() and (a[1] == b[1]).all()


# One case of the direct upsert comparison, run in a child process: the
# reference ends its process (exit code 0) when an update would split the
# root (open-harmonia/src/bpt.cpp:336-339), which must fail the test rather
# than end the test run.
_UPSERT_CASE = """
import sys, numpy as np
sys.path.insert(0, sys.argv[4])
from harmonia_b200 import datagen as dg
from oracle import pyoracle as po
n, frac, seed = int(sys.argv[1]), float(sys.argv[2]), int(sys.argv[3])
keys = dg.gen_keys(n, seed)
cur_k = np.sort(keys)
cur_v = dg.values_for(cur_k)
ref = po.RefTree(keys, dg.values_for(keys))
for e in range(2):
    bk, bv = dg.gen_upserts(cur_k, max(1, n // 8), frac, seed * 10 + e)
    ref.upsert(bk, bv)
    cur_k, cur_v = po.upsert_set(cur_k, cur_v, bk, bv, ref_rule=True)
    rk, rv = ref.export()
    assert len(rk) == len(cur_k) and (rk == cur_k).all() and (rv == cur_v).all(), ("contents", e)
    q = dg.gen_point_queries(cur_k, 4096, 0.5, seed + e)
    assert (ref.search(q) == po.PortTree(cur_k, cur_v).search(q)).all(), ("search", e)
print("CASE-OK", len(cur_k))
"""


@pytest.mark.skipif(not po.ref_available(), reason="reference library not built in this checkout")
@pytest.mark.parametrize("frac", [0.0, 0.05, 0.5, 1.0])
@pytest.mark.parametrize("n", [5000, 1 << 16, 1 << 18])
def test_upsert_restatement_matches_reference_batched_update(n, frac):
    """The restatement of an upsert epoch (po.upsert_set under the reference's
    rule, the oracle of every GPU upsert test) against the reference's own
    BPlusTree::insert_parallel_Newupdate_batch
    (open-harmonia/src/bpt-ppi-update-batch.cpp:86-200): two epochs of n/8
    keys in a row, from no new keys to all new, the sorted contents equal
    after each, and searches through the reference's post-update descent
    equal the restatement's on the new contents."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _UPSERT_CASE, str(n), str(frac), "7", root],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "CASE-OK" in r.stdout, (r.returncode, r.stdout[-500:], r.stderr[-2000:])


def test_upsert_last_occurrence_wins():
    sk = np.array([10, 20, 30], np.int64)
    sv = np.array([1, 2, 3], np.int64)
    k, v = po.upsert_set(sk, sv, np.array([20, 5, 20, 5], np.int64), np.array([7, 8, 9, 10], np.int64))
    assert k.tolist() == [5, 10, 20, 30] and v.tolist() == [10, 1, 9, 3]


@pytest.mark.parametrize("n", [0, 1, 2, 15, 16, 17, 63, 64, 65, 1000, 4097])
@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_port_layout_invariants(n, fanout, leaf_cap):
    keys = np.sort(dg.gen_keys(n, seed=n + 1))
    vals = dg.values_for(keys)
    t = po.PortTree(keys, vals, fanout=fanout, leaf_cap=leaf_cap)
    L = t.layout()
    h, ls, ni, nl = po.shape(n, fanout, leaf_cap)
    assert (L["height"], L["lvl_start"], L["n_inner"], L["n_leaf"]) == (h, ls, ni, nl)
    row = fanout // 8 + fanout
    inner = L["inner"].reshape(ni, row)
    # prefix is the running sum of child counts (CFB: prefix[i+1] = prefix[i] + children_i)
    nchild = [int((inner[i, fanout // 8:] != po.MAX_KEY).sum()) + 1 for i in range(ni)]
    assert L["prefix"][0] == 1 or ni == 1 and L["prefix"][0] == ni
    for i in range(ni - 1):
        assert L["prefix"][i + 1] == L["prefix"][i] + nchild[i]
    assert L["prefix"][ni - 1] + nchild[ni - 1] == ni + nl
    # index words mirror every 8th key
    for i in range(ni):
        for j in range(fanout // 8):
            s = 8 * (j + 1)
            assert inner[i, j] == (inner[i, fanout // 8 + s] if s < fanout else po.MAX_KEY)
    assert int(L["leaf_cnt"].sum()) == n
    assert (np.concatenate([[0], np.cumsum(L["leaf_cnt"])[:-1]]) == L["leaf_base"]).all()
    ek, ev = t.export()
    assert (ek == keys).all() and (ev == vals).all()
    if n:
        q = np.concatenate([keys, keys + 1, [np.int64(-(2**63)), po.MAX_KEY]])
        exp = np.concatenate([vals, np.where(np.isin(keys + 1, keys), -1, -1), [-1, -1]])
        exp[n:2 * n] = np.where(np.isin(keys + 1, keys), np.interp(keys + 1, keys, vals).astype(np.int64), -1)
        assert (t.search(q)[:n] == vals).all()
        assert (t.search(q)[-2:] == -1).all()


@pytest.mark.skipif(not po.ref_available(), reason="reference library not built in this checkout")
@pytest.mark.parametrize("n", [5, 100, 5000, 1 << 16])
@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (64, 64), (128, 16), (128, 64)])
def test_port_matches_reference_directly(n, fanout, leaf_cap):
    keys = dg.gen_keys(n, seed=100 + n)
    vals = dg.values_for(keys)
    ref = po.RefTree(keys, vals)
    sk = np.sort(keys)
    t = po.PortTree(sk, dg.values_for(sk), fanout=fanout, leaf_cap=leaf_cap)
    q = dg.gen_point_queries(keys, 20000, 0.5, seed=n)
    q[:3] = [sk[0], sk[-1], -7]
    assert (ref.search(q) == t.search(q)).all()
    st, ln = dg.gen_ranges(500, 1, 300, seed=n)
    st[:2] = [sk[0], sk[-1]]
    a, b = ref.range(st, ln), t.range(st, ln)
    assert all((x == y).all() for x, y in zip(a, b))


@pytest.mark.skipif(not po.ref_available(), reason="reference library not built in this checkout")
@pytest.mark.parametrize("n", [5, 100, 5000, 1 << 16])
def test_reference_prefetch_search_equals_its_plain_search(n):
    """The reference's software-pipelined CPU search (timed as a second CPU
    figure) answers as its plain search does, including a ragged tail."""
    keys = dg.gen_keys(n, seed=300 + n)
    ref = po.RefTree(keys, dg.values_for(keys))
    q = dg.gen_point_queries(keys, 20003, 0.5, seed=n)
    q[:3] = [keys.min(), keys.max(), -7]
    assert (ref.search_prefetch(q) == ref.search(q)).all()
    assert (ref.search_prefetch(q, threads=3) == ref.search(q)).all()


def test_port_matches_c1_range_between_digests(c1):
    """Inclusive ranges (BPlusTree::range_search) before and after the first
    C1 upsert epoch, on two layouts of the restatement."""
    keys, sk, sv = c1
    g = GOLD["c1_range_between"]
    st, en = dg.gen_range_pairs(g["m"], g["n_keys"], g["lo"], g["hi"], g["seed"])
    for fanout, leaf_cap in [(64, 16), (128, 64)]:
        off, k, v = po.PortTree(sk, sv, fanout=fanout, leaf_cap=leaf_cap).range_between(st, en)
        assert digest(off, k, v) == g["digest"] and len(k) == g["records"]
    gu, ga = GOLD["c1_upsert"], GOLD["c1_range_between_after"]
    bk, bv = dg.gen_upserts(keys, gu["m"], gu["new_frac"], gu["seed"])
    ek, ev = po.upsert_set(sk, sv, bk, bv)
    off, k, v = po.PortTree(ek, ev).range_between(st, en)
    assert digest(off, k, v) == ga["digest"] and len(k) == ga["records"]


def test_port_range_between_edges():
    sk = np.arange(10, 1000, 10, dtype=np.int64)  # 10, 20, ..., 990
    t = po.PortTree(sk, sk * 3, leaf_cap=16)
    st = np.array([10, 15, 990, 995, -5, 500, 500, 0, 200], np.int64)
    en = np.array([10, 25, 990, 2000, 5, 499, 500, po.MAX_KEY, 100], np.int64)
    off, k, v = t.range_between(st, en)
    want = [[10], [20], [990], [], [], [], [500], list(range(10, 1000, 10)), []]
    assert np.diff(off).tolist() == [len(w) for w in want]
    assert k.tolist() == sum(want, []) and (v == k * 3).all()


@pytest.mark.skipif(not po.ref_available(), reason="reference library not built in this checkout")
@pytest.mark.parametrize("n", [5, 100, 5000, 1 << 16])
def test_range_between_port_and_reference_walk_match_reference(n):
    """The reference's own range_search, its walk over the update-aware
    descent (used after updates), and the restatement agree; after an upsert
    epoch the walk and the restatement on the upserted contents agree."""
    keys = dg.gen_keys(n, seed=300 + n)
    vals = dg.values_for(keys)
    ref = po.RefTree(keys, vals)
    sk = np.sort(keys)
    st, en = dg.gen_range_pairs(3000, n, 1, 40, seed=n)
    st[:4] = [sk[0], sk[-1], sk[n // 2], sk[0] - 1]
    en[:4] = [sk[0], sk[-1] + 1, sk[n // 2] - 1, sk[min(3, n - 1)]]
    a = ref.range_between(st, en)
    b = ref.range_between(st, en, walk=True)
    c = po.PortTree(sk, dg.values_for(sk)).range_between(st, en)
    assert all((x == y).all() for x, y in zip(a, b))
    assert all((x == y).all() for x, y in zip(a, c))
    bk, bv = dg.gen_upserts(keys, max(2, n // 4), 0.5, seed=n + 1)
    ref.upsert(bk, bv)
    ek, ev = po.upsert_set(sk, dg.values_for(sk), bk, bv)
    a = ref.range_between(st, en)
    c = po.PortTree(ek, ev).range_between(st, en)
    assert all((x == y).all() for x, y in zip(a, c))


@pytest.mark.skipif(not po.cfb_available(), reason="fanout-128 reference library not built in this checkout")
@pytest.mark.parametrize("n", [5, 1000, 1 << 16])
def test_fanout128_reference_matches_port(n):
    """The reference's pointer B+tree at order 128 (regular_bpt, find()) and
    the fanout-128 restatement give the same point results."""
    keys = dg.gen_keys(n, seed=500 + n)
    vals = dg.values_for(keys)
    cfb = po.CfbTree(keys, vals)
    assert cfb.order == 128
    sk = np.sort(keys)
    q = dg.gen_point_queries(keys, 20000, 0.5, seed=n)
    q[:3] = [sk[0], sk[-1], -7]
    assert (cfb.search(q) == po.PortTree(sk, dg.values_for(sk), fanout=128).search(q)).all()


@pytest.mark.skipif(not po.gpu_ref_available(), reason="reference GPU library not built in this checkout")
def test_reference_gpu_library_cpu_side():
    """The library holding the reference's GPU search also holds its CPU tree
    (same answers as the plain reference library), and the CPU check of the
    GPU kernel's index path accepts the seeded workloads (uniform and Zipf)."""
    keys = dg.gen_keys(1 << 16, seed=77)
    vals = dg.values_for(keys)
    t = po.RefTree(keys, vals, gpu=True)
    q = dg.gen_point_queries(keys, 1 << 16, 0.5, seed=78)
    assert (t.search(q) == po.RefTree(keys, vals).search(q)).all()
    assert po.check_gpu_ref_batch(t, q) == 0
    assert po.check_gpu_ref_batch(t, dg.gen_zipf_queries(np.sort(keys), 1 << 16, 0.99, seed=79)) == 0
    assert po.check_gpu_ref_batch(t, np.array([po.MAX_KEY], np.int64)) == 1  # never sent to the kernel
