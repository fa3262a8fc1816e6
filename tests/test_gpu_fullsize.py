"""GPU parity at the benchmark's full sizes, pinned by the reference's own
digests: a 2^26-key tree at fanout 64 and 128, 2^24 point queries (90% hits,
unsorted and pre-sorted), 2^24 Zipf(0.99) queries, 2^20 ranges of 1..256
records and 2^20 inclusive ranges of about as many keys, 512 uneven batches
(1K..4M queries, uniform and Zipf) searched as one set, and one upsert epoch
of 4096K keys (5% new) (golden.json: c2_point, c3_zipf, c3_range,
c3_range_between, c4_batches, c2_upsert_4096k)."""
import numpy as np
import pytest

from harmonia_b200 import BPlusTree, datagen as dg
from tests.helpers import digest, load_golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
GOLD = load_golden()


@pytest.fixture(scope="module")
def big():
    g = GOLD["c2_point"]
    keys = dg.gen_keys(g["n"], g["key_seed"])
    return keys, np.sort(keys)


@pytest.mark.parametrize("fanout,leaf_cap,smem", [(64, 16, None), (128, 16, None), (64, 64, None),
                                                  (64, 16, 256), (64, 16, 200 * 1024)])
def test_c2_point_full_size(big, fanout, leaf_cap, smem):
    """smem: the budget for top levels staged in shared memory (None: the
    default, two levels at this size; 256 B: none; 200 KiB: still two, the
    third level alone is 600 KB)."""
    keys, sk = big
    g = GOLD["c2_point"]
    q = dg.gen_point_queries(keys, g["m"], g["hit"], g["q_seed"])
    dq = torch.from_numpy(q).cuda()
    with BPlusTree.bulk_load(torch.from_numpy(keys).cuda(), torch.from_numpy(dg.values_for(keys)).cuda(),
                             fanout=fanout, leaf_cap=leaf_cap, smem_bytes=smem) as t:
        if smem == 256:
            assert t.info().smem_levels == 0
        for bits, join in ((0, 2), (8, 2), (16, 2), (0, 1)):
            t.set_search_config(sort_bits=bits, join=join)
            out = t.search(dq).cpu().numpy()
            assert digest(out) == g["digest"], f"sort_bits={bits} join={join}"
        t.set_search_config(sort_bits=0, join=2)
        # the same batch partially sorted by its top 16 key bits: same results per key
        order = np.argsort(q >> np.int64(47), kind="stable")
        out = t.search(torch.from_numpy(q[order]).cuda()).cpu().numpy()
        back = np.empty_like(out)
        back[order] = out
        assert digest(back) == g["digest"]


def test_c3_zipf_and_range_full_size(big):
    keys, sk = big
    with BPlusTree.bulk_load(torch.from_numpy(keys).cuda(), torch.from_numpy(dg.values_for(keys)).cuda()) as t:
        g = GOLD["c3_zipf"]
        q = dg.gen_zipf_queries(sk, g["m"], g["theta"], g["q_seed"])
        assert digest(t.search(torch.from_numpy(q).cuda()).cpu().numpy()) == g["digest"]
        g = GOLD["c3_range"]
        st, ln = dg.gen_ranges(g["m"], g["lo"], g["hi"], g["seed"])
        off, k, v = t.range_search(torch.from_numpy(st).cuda(), torch.from_numpy(ln).cuda())
        assert len(k) == g["records"]
        assert digest(off.cpu().numpy(), k.cpu().numpy(), v.cpu().numpy()) == g["digest"]


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_c3_range_between_full_size(big):
    keys, sk = big
    g = GOLD["c3_range_between"]
    st, en = dg.gen_range_pairs(g["m"], g["n_keys"], g["lo"], g["hi"], g["seed"])
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys))) as t:
        off, k, v = t.range_between(cuda(st), cuda(en))
        assert len(k) == g["records"]
        assert digest(off.cpu().numpy(), k.cpu().numpy(), v.cpu().numpy()) == g["digest"]


def test_c4_uneven_batches_full_size(big):
    """The 512-batch set through a captured plan (two replays, the second
    after the outputs were overwritten) and through hm_search_batches; every
    batch's results against the reference's digest of that batch."""
    keys, sk = big
    g = GOLD["c4_batches"]
    sizes, q = dg.gen_uneven_batches(keys, sk, g["nb"], g["seed"])
    assert len(q) == g["queries"]
    ends = np.concatenate([[0], np.cumsum(sizes)])
    dq = cuda(q)
    out = torch.full_like(dq, -7)
    batches = [(dq[ends[b]:ends[b + 1]], out[ends[b]:ends[b + 1]]) for b in range(g["nb"])]

    def check(what):
        res = out.cpu().numpy()
        bad = [b for b in range(g["nb"]) if digest(res[ends[b]:ends[b + 1]]) != g["batch_digests"][b]]
        assert not bad, f"{what}: batches {bad[:8]} differ"
        assert digest(res) == g["digest"]

    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys))) as t:
        with t.plan(batches) as p:
            for rep in range(2):
                out.fill_(-7)
                p.launch()
                torch.cuda.synchronize()
                check(f"plan replay {rep}")
        out.fill_(-7)
        t.search_batches(batches)
        torch.cuda.synchronize()
        check("hm_search_batches")


@pytest.fixture(scope="module")
def upsert_4096k(big):
    keys, sk = big
    g = GOLD["c2_upsert_4096k"]
    bk, bv = dg.gen_upserts(keys, g["m"], g["new_frac"], g["seed"])
    return bk, bv


@pytest.mark.parametrize("leaf_fill,ref_rule", [(16, False), (12, True)])
def test_c2_upsert_epoch_4096k_full_size(big, upsert_4096k, leaf_fill, ref_rule):
    """One epoch at the paper's batch size (4096K keys, 5% new) on the 2^26-key
    tree: with full leaves every touched leaf overflows (subtree rebalance or
    rebuild); with 12 of 16 slots filled most new keys merge in place.  The
    contents, the batch's own keys and the C2 query batch afterwards against
    the reference's insert_parallel_Newupdate_batch."""
    keys, sk = big
    bk, bv = upsert_4096k
    g = GOLD["c2_upsert_4096k"]
    with BPlusTree.bulk_load(cuda(keys), cuda(dg.values_for(keys)), leaf_fill=leaf_fill) as t:
        t.upsert(cuda(bk), cuda(bv), ref_rule=ref_rule)
        ek, ev = t.export()
        assert len(ek) == g["n_after"] and digest(ek, ev) == g["export_digest"]
        assert digest(t.search(cuda(bk)).cpu().numpy()) == g["search_batch_digest"]
        gq = GOLD["c2_point"]
        q = dg.gen_point_queries(keys, gq["m"], gq["hit"], gq["q_seed"])
        assert digest(t.search(cuda(q)).cpu().numpy()) == g["search_c2_digest"]
