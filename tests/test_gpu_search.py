"""GPU parity tests of the bulk loader and the point search, through the C ABI.

Bit-exact against the oracle: the C restatement (layout and results) and the
reference CPU tree's golden digests."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, HarmoniaError, datagen as dg, native
from oracle import pyoracle as po
from tests.helpers import digest, load_golden, load_small

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLD = load_golden()
CONFIGS = [(64, 16), (64, 64), (128, 16), (128, 64)]


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.fixture(scope="module")
def c1():
    g = GOLD["c1_point"]
    keys = dg.gen_keys(g["n"], g["key_seed"])
    vals = dg.values_for(keys)
    sk = np.sort(keys)
    t = BPlusTree.bulk_load(cuda(keys), cuda(vals))
    yield keys, sk, t
    t.close()


@pytest.mark.parametrize("n", [0, 1, 2, 15, 16, 17, 64, 1000, 4097, 1 << 16])
@pytest.mark.parametrize("fanout,leaf_cap", CONFIGS)
def test_bulk_load_layout_bit_exact(n, fanout, leaf_cap):
    keys = dg.gen_keys(n, seed=n + 5)
    vals = dg.values_for(keys)
    sk = np.sort(keys)
    exp = po.PortTree(sk, dg.values_for(sk), fanout=fanout, leaf_cap=leaf_cap).layout()
    with BPlusTree.bulk_load(keys, vals, fanout=fanout, leaf_cap=leaf_cap) as t:
        got = t.layout()
    for k in ("height", "lvl_start", "n_inner", "n_leaf"):
        assert got[k] == exp[k], k
    for k in ("inner", "prefix", "leaf_rows", "leaf_cnt", "leaf_base"):
        assert (got[k] == exp[k]).all(), k


@pytest.mark.parametrize("inner_fill,leaf_fill", [(2, 1), (3, 5), (33, 12), (64, 16)])
def test_bulk_load_partial_fill_layout(inner_fill, leaf_fill):
    keys = dg.gen_keys(20000, seed=9)
    sk = np.sort(keys)
    exp = po.PortTree(sk, dg.values_for(sk), 64, 16, inner_fill, leaf_fill).layout()
    with BPlusTree.bulk_load(keys, dg.values_for(keys), 64, 16, inner_fill, leaf_fill) as t:
        got = t.layout()
    for k in ("inner", "prefix", "leaf_rows", "leaf_cnt", "leaf_base"):
        assert (got[k] == exp[k]).all(), k


def test_c1_point_digest(c1):
    keys, sk, t = c1
    g = GOLD["c1_point"]
    q = dg.gen_point_queries(keys, g["m"], g["hit"], g["q_seed"])
    out = t.search(cuda(q)).cpu().numpy()
    assert digest(out) == g["digest"]


def test_c1_zipf_digest(c1):
    keys, sk, t = c1
    g = GOLD["c1_zipf"]
    q = dg.gen_zipf_queries(sk, g["m"], g["theta"], g["q_seed"])
    assert digest(t.search(cuda(q)).cpu().numpy()) == g["digest"]


@pytest.mark.parametrize("w", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("qpg", [1, 2, 4])
def test_every_group_width_and_depth(c1, w, qpg):
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, 300001, 0.7, seed=w * 10 + qpg)
    exp = po.PortTree(sk, dg.values_for(sk)).search(q)
    t.set_search_config(group_width=w, queries_per_group=qpg, sort_bits=0, join=2)
    try:
        assert (t.search(cuda(q)).cpu().numpy() == exp).all()
    finally:
        t.set_search_config(group_width=4, queries_per_group=1, sort_bits=-1, join=-1)


@pytest.mark.parametrize("bits", [1, 4, 8, 9, 12, 16])
def test_presort_bits(c1, bits):
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, 1 << 19, 0.9, seed=bits)
    exp = po.PortTree(sk, dg.values_for(sk)).search(q)
    t.set_search_config(sort_bits=bits, join=2)
    try:
        assert (t.search(cuda(q)).cpu().numpy() == exp).all()
    finally:
        t.set_search_config(sort_bits=-1, join=-1)


@pytest.mark.parametrize("fanout,leaf_cap", CONFIGS)
def test_configs_against_small_golden(fanout, leaf_cap):
    s = load_small()
    keys = dg.gen_keys(int(s["n"]), int(s["key_seed"]))
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=fanout, leaf_cap=leaf_cap) as t:
        assert (t.search(cuda(s["q"])).cpu().numpy() == s["res"]).all()
        assert (t.search(s["q"]) == s["res"]).all()  # host buffers


def test_host_pageable_and_pinned_buffers(c1):
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, (1 << 22) * 2 + 12345, 0.5, seed=77)  # more chunks than the ring holds
    exp = po.PortTree(sk, dg.values_for(sk)).search(q)
    assert (t.search(q) == exp).all()
    qp = torch.from_numpy(q).pin_memory()
    op = torch.empty_like(qp).pin_memory()
    t.search(qp, op)
    assert (op.numpy() == exp).all()


def test_edge_queries(c1):
    keys, sk, t = c1
    q = np.array([sk[0], sk[-1], sk[0] - 1, sk[-1] + 1, -(2**63), 2**63 - 1, -1, 0], dtype=np.int64)
    exp = po.PortTree(sk, dg.values_for(sk)).search(q)
    assert exp[-3] == -1 and exp[2] == -1
    for n in (1, 3, len(q)):
        assert (t.search(cuda(q[:n])).cpu().numpy() == exp[:n]).all()
    assert len(t.search(cuda(q[:0]))) == 0


def test_negative_and_extreme_keys():
    keys = np.array([-(2**63), -5, -1, 0, 7, 2**63 - 2], dtype=np.int64)
    vals = np.arange(6, dtype=np.int64) * 3
    with BPlusTree.bulk_load(keys[::-1].copy(), vals[::-1].copy()) as t:
        q = np.concatenate([keys, [-4, 1, 2**63 - 1, 8]])
        got = t.search(cuda(q)).cpu().numpy()
        assert got.tolist() == vals.tolist() + [-1, -1, -1, -1]


def test_empty_and_single_key_trees():
    with BPlusTree.bulk_load(np.zeros(0, np.int64), np.zeros(0, np.int64)) as t:
        assert (t.search(cuda(np.array([0, 5, -5], np.int64))).cpu().numpy() == -1).all()
        assert t.size == 0
    with BPlusTree.bulk_load(np.array([42], np.int64), np.array([7], np.int64)) as t:
        assert t.search(cuda(np.array([42, 41, 43], np.int64))).cpu().tolist() == [7, -1, -1]


def test_bulk_load_errors():
    with pytest.raises(HarmoniaError) as e:
        BPlusTree.bulk_load(np.array([3, 1, 3], np.int64), np.zeros(3, np.int64))
    assert e.value.code == -3
    with pytest.raises(HarmoniaError) as e:
        BPlusTree.bulk_load(np.array([1, 2**63 - 1], np.int64), np.zeros(2, np.int64))
    assert e.value.code == -4
    with pytest.raises(HarmoniaError) as e:
        BPlusTree.bulk_load(np.array([1], np.int64), np.zeros(1, np.int64), fanout=96)
    assert e.value.code == -1


def test_search_batches_uneven(c1):
    keys, sk, t = c1
    oracle = po.PortTree(sk, dg.values_for(sk))
    sizes = [1, 2, 255, 256, 257, 1000, 4096, 70001, 3, 0, 12345]
    qs = [dg.gen_point_queries(keys, m, 0.5, seed=300 + i) for i, m in enumerate(sizes)]
    dq = [cuda(q) for q in qs]
    outs = [torch.full((len(q),), -77, dtype=torch.int64, device="cuda") for q in qs]
    t.search_batches(list(zip(dq, outs)))
    for q, o in zip(qs, outs):
        assert (o.cpu().numpy() == oracle.search(q)).all()


def test_autotune_keeps_results_exact(c1):
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, 1 << 18, 0.9, seed=5)
    best = t.autotune(cuda(q))
    assert best["group_width"] in (2, 4, 8, 16, 32)
    assert best["join"] in (-1, 2)  # the join is left to the automatic choice or switched off
    exp = po.PortTree(sk, dg.values_for(sk)).search(q)
    assert (t.search(cuda(q)).cpu().numpy() == exp).all()
    t.set_search_config(group_width=4, queries_per_group=1, sort_bits=-1, join=-1)


def test_launches_come_from_the_library(c1):
    keys, sk, t = c1
    before = native.lib().hm_launch_count()
    t.search(cuda(keys[:1000]))
    torch.cuda.synchronize()
    assert native.lib().hm_launch_count() > before


def test_search_batches_large_presorted_union(c1):
    """Large sets take the gather / joint pre-sort / scatter-back path."""
    keys, sk, t = c1
    oracle = po.PortTree(sk, dg.values_for(sk))
    sizes = [1 << 20, 1000, 1 << 19, 5, 777777]
    qs = [dg.gen_point_queries(keys, m, 0.6, seed=400 + i) for i, m in enumerate(sizes)]
    outs = [torch.full((len(q),), -77, dtype=torch.int64, device="cuda") for q in qs]
    for bits in (16, 8, 0):
        t.set_search_config(sort_bits=bits)
        for o in outs:
            o.fill_(-77)
        t.search_batches(list(zip([cuda(q) for q in qs], outs)))
        for q, o in zip(qs, outs):
            assert (o.cpu().numpy() == oracle.search(q)).all(), bits
    t.set_search_config(sort_bits=-1)


def test_search_batches_bucket_join_placed(c1):
    """A batch set through the bucket join with results placed in first-pass
    order (total under 2^25 queries): the first pass reads every batch in
    place, the join writes first-pass positions, the one inverse pass writes
    each batch's output; the same through a captured plan."""
    keys, sk, t = c1
    oracle = po.PortTree(sk, dg.values_for(sk))
    sizes = [1 << 20, 1000, 1 << 19, 5, 777777, 8192, 8193]
    qs = [cuda(dg.gen_point_queries(keys, m, 0.6, seed=500 + i)) for i, m in enumerate(sizes)]
    outs = [torch.full((len(q),), -77, dtype=torch.int64, device="cuda") for q in qs]
    t.set_search_config(join=1)
    try:
        t.search_batches(list(zip(qs, outs)))
        for q, o in zip(qs, outs):
            assert (o.cpu().numpy() == oracle.search(q.cpu().numpy())).all()
        plan = t.plan(list(zip(qs, outs)))
        for rep in range(2):
            for o in outs:
                o.fill_(-77)
            plan.launch()
            torch.cuda.synchronize()
            for q, o in zip(qs, outs):
                assert (o.cpu().numpy() == oracle.search(q.cpu().numpy())).all(), rep
        plan.close()
    finally:
        t.set_search_config(join=-1)


def test_plan_replay_matches_and_follows_rebuild():
    keys = dg.gen_keys(1 << 18, seed=61)
    vals = dg.values_for(keys)
    sk = np.sort(keys)
    with BPlusTree.bulk_load(cuda(keys), cuda(vals)) as t:
        sizes = [3 << 20, 4096, 1, 100000]
        qs = [cuda(dg.gen_point_queries(keys, m, 0.5, seed=70 + i)) for i, m in enumerate(sizes)]
        outs = [torch.empty_like(q) for q in qs]
        plan = t.plan(list(zip(qs, outs)))
        for rep in range(3):
            for q in qs:  # new contents in the same buffers
                q.copy_(cuda(dg.gen_point_queries(keys, len(q), 0.5, seed=80 + rep + len(q))))
            plan.launch()
            torch.cuda.synchronize()
            exp = po.PortTree(sk, dg.values_for(sk))
            for q, o in zip(qs, outs):
                assert (o.cpu().numpy() == exp.search(q.cpu().numpy())).all()
        # a rebuild (overflowing upsert) moves the arena: the plan re-captures itself
        bk, bv = dg.gen_upserts(keys, 300000, 1.0, seed=90)
        t.upsert(bk, bv)
        ek, ev = po.upsert_set(sk, dg.values_for(sk), bk, bv)
        t.set_search_config(group_width=8)
        plan.launch()
        torch.cuda.synchronize()
        exp = po.PortTree(ek, ev)
        for q, o in zip(qs, outs):
            assert (o.cpu().numpy() == exp.search(q.cpu().numpy())).all()
        plan.close()


def bucket_edges(sk, n_leaf, count):
    """Keys at and next to the first `count` bucket boundaries of the join
    (top bits of key - key_min, as many bits as leave about 32 leaves per bucket)."""
    bits = 1
    while bits < 16 and (n_leaf >> bits) > 32:
        bits += 1
    lo, rng = int(sk[0]), (int(sk[-1]) - int(sk[0])) % (1 << 64)
    shift = max(rng.bit_length() - bits, 0)
    out = []
    for b in range(count):
        edge = lo + (b << shift)
        out += [edge - 1, edge, edge + 1]
    return np.array([min(max(x, -(2**63)), 2**63 - 1) for x in out], np.int64)


@pytest.mark.parametrize("nq", [(1 << 19) + 77, (1 << 21) + 333])  # about 256 / 1024 queries per bucket
@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_bucket_join_matches_oracle(fanout, leaf_cap, nq):
    keys = dg.gen_keys(1 << 20, seed=81)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), fanout=fanout, leaf_cap=leaf_cap) as t:
        t.set_search_config(join=1)
        q = dg.gen_point_queries(keys, nq, 0.7, seed=82)
        q[:6] = [sk[0], sk[-1], sk[0] - 1, sk[-1] + 1, -(2**63), 2**63 - 1]
        edges = bucket_edges(sk, t.info().n_leaf, 300)
        q[6:6 + len(edges)] = edges
        assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all()
        z = dg.gen_zipf_queries(sk, 1 << 21, 0.99, seed=83)  # hot buckets split into several runs
        assert (t.search(cuda(z)).cpu().numpy() == oracle.search(z)).all()
        t.set_search_config(join=-1)


@pytest.mark.parametrize("n", [1, 5, 16, 17, 100, 129, 1000, 5000])
@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_bucket_join_forced_on_small_trees(n, fanout, leaf_cap):
    """The join forced on trees of a few leaves (fewer than one 8-record TMA
    box, a last box reaching past the last leaf): exact against the oracle."""
    keys = dg.gen_keys(n, seed=500 + n)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), fanout=fanout, leaf_cap=leaf_cap) as t:
        t.set_search_config(join=1)
        q = dg.gen_point_queries(keys, 5000, 0.6, seed=600 + n)
        q[:4] = [sk[0], sk[-1], -(2**63), 2**63 - 1]
        assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all()


@pytest.mark.parametrize("ends", [(-(2**62), 2**62), (-(2**63), 2**63 - 2), (2**40, 2**63 - 2)])
def test_bucket_join_skewed_keys_fall_back(ends):
    # almost all keys in a narrow range: buckets over it hold too many leaves;
    # extreme ends put bucket boundaries past the largest key
    rng = np.random.default_rng(5)
    dense = np.unique(rng.integers(10**12, 10**12 + 10**8, 1 << 20))
    keys = np.unique(np.concatenate([dense, np.array(ends, np.int64)])).astype(np.int64)
    rng.shuffle(keys)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    with BPlusTree.bulk_load(keys, dg.values_for(keys)) as t:
        t.set_search_config(join=1)
        q = np.concatenate([sk[rng.integers(0, len(sk), 1 << 20)], rng.integers(10**12, 10**12 + 10**8, 1 << 19)])
        assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all()


def test_bucket_join_after_upserts(c1):
    keys, sk, _ = c1
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=12) as t:
        t.set_search_config(join=1)
        q0 = dg.gen_point_queries(keys, 1 << 18, 0.8, seed=90)
        assert (t.search(cuda(q0)).cpu().numpy() == po.PortTree(sk, dg.values_for(sk)).search(q0)).all()
        bk, bv = dg.gen_upserts(keys, 5000, 0.5, seed=91)
        bk[:2] = [int(sk[0]) - 12345, min(int(sk[-1]) + 12345, 2**63 - 2)]  # new smallest and largest keys
        t.upsert(bk, bv)
        ek, ev = po.upsert_set(sk, dg.values_for(sk), bk, bv)
        q = np.concatenate([bk, dg.gen_point_queries(ek, 1 << 20, 0.8, seed=92)])
        t.set_search_config(join=1)
        assert (t.search(cuda(q)).cpu().numpy() == po.PortTree(ek, ev).search(q)).all()


@pytest.mark.parametrize("fanout,leaf_cap", [(64, 16), (128, 64)])
def test_pointer_baseline_matches(fanout, leaf_cap):
    # the HB+-style comparison kernel answers like the product path, also
    # after a rebuild has replaced the arena
    keys = dg.gen_keys(1 << 18, 71)
    sk = np.sort(keys)
    with BPlusTree.bulk_load(keys, dg.values_for(keys), fanout=fanout, leaf_cap=leaf_cap) as t:
        q = dg.gen_point_queries(keys, 1 << 17, 0.7, seed=72)
        q[:3] = [2**63 - 1, -(2**63), sk[0]]
        dq = cuda(q)
        assert (t.search_pointer_baseline(dq).cpu().numpy() == po.PortTree(sk, dg.values_for(sk)).search(q)).all()
        bk, bv = dg.gen_upserts(keys, 60000, 0.9, seed=73)  # full leaves: a rebuild
        t.upsert(bk, bv)
        ek, ev = po.upsert_set(sk, dg.values_for(sk), bk, bv)
        assert (t.search_pointer_baseline(dq).cpu().numpy() == po.PortTree(ek, ev).search(q)).all()


def test_bounded_wait_gives_up_reports_timeout_and_recovers(c1):
    """With a wait limit of 0 every CTA's wait for its staged top levels gives
    up at once: the CTA records HM_ETIMEOUT (hm_sync reports it), waits with
    the default bound for its copy to land, and returns without writing
    results.  With the default limit the next search is exact again."""
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, 1 << 16, 0.5, seed=71)
    dq = cuda(q)
    t.set_search_config(sort_bits=0, join=2)
    try:
        assert t.info().smem_levels > 0
        out = torch.full_like(dq, -7)
        t.set_wait_limit(0)
        t.search(dq, out)
        with pytest.raises(HarmoniaError) as e:
            t.sync()
        assert e.value.code == -7  # HM_ETIMEOUT
        assert (out == -7).all()
        t.set_wait_limit(1 << 24)
        t.search(dq, out)
        t.sync()
        assert (out.cpu().numpy() == po.PortTree(sk, dg.values_for(sk)).search(q)).all()
    finally:
        t.set_wait_limit(1 << 24)
        t.set_search_config(sort_bits=-1, join=-1)


def test_bucket_join_bounded_wait_reports_timeout_and_recovers(c1):
    """The TMA-staged bucket join waits for each stage's loads with the same
    bound: at a limit of 0 every CTA gives up at its first stage, records
    HM_ETIMEOUT, waits (default bound) for the loads it issued and returns;
    hm_sync reports the timeout.  With the default limit the join is exact."""
    keys, sk, t = c1
    q = dg.gen_point_queries(keys, 1 << 20, 0.5, seed=72)
    dq = cuda(q)
    t.set_search_config(join=1)
    try:
        out = torch.empty_like(dq)
        t.set_wait_limit(0)
        t.search(dq, out)
        with pytest.raises(HarmoniaError) as e:
            t.sync()
        assert e.value.code == -7  # HM_ETIMEOUT
        t.set_wait_limit(1 << 24)
        t.search(dq, out)
        t.sync()
        assert (out.cpu().numpy() == po.PortTree(sk, dg.values_for(sk)).search(q)).all()
    finally:
        t.set_wait_limit(1 << 24)
        t.set_search_config(join=-1)


@pytest.mark.parametrize("smem,levels", [(256, 0), (49152, 2), (200 * 1024, 3)])
def test_staged_top_levels_budget(smem, levels):
    """2^18 keys: inner levels of 1, 4 and 256 rows; a 256-B budget stages
    none, the default two, 200 KiB all three (every inner row in shared
    memory).  Results equal the oracle at each depth, plain and pre-sorted."""
    keys = dg.gen_keys(1 << 18, seed=72)
    sk = np.sort(keys)
    oracle = po.PortTree(sk, dg.values_for(sk))
    q = dg.gen_point_queries(keys, 1 << 18, 0.6, seed=73)
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), smem_bytes=smem) as t:
        info = t.info()
        assert info.height == 3 and info.smem_levels == levels
        for bits in (0, 8):
            t.set_search_config(sort_bits=bits, join=2)
            assert (t.search(cuda(q)).cpu().numpy() == oracle.search(q)).all(), bits
