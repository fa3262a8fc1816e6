"""Generates the golden fixtures from the reference's own CPU B+tree.

Run in a container that has the reference sources (it builds
oracle/_ref/libhmref.so from them with `make -C oracle ref`):

    python tests/golden/make_golden.py          # 2^20-key cases + small arrays
    python tests/golden/make_golden.py --big    # adds the 2^26- and 2^25-key cases (~30 min)

Every input comes from harmonia_b200.datagen with the seeds recorded in
golden.json, so a test regenerates the inputs bit for bit and compares the
SHA-256 of its outputs with the reference's.  small.npz also stores the
reference's outputs of a 4096-key case as plain arrays.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from harmonia_b200 import datagen as dg  # noqa: E402
from oracle import pyoracle as po  # noqa: E402
from tests.helpers import GOLDEN_DIR, digest  # noqa: E402


def point_case(n, key_seed, m, hit, q_seed, zipf=False):
    keys = dg.gen_keys(n, key_seed)
    vals = dg.values_for(keys)
    t0 = time.time()
    ref = po.RefTree(keys, vals)
    build_s = time.time() - t0
    if zipf:
        q = dg.gen_zipf_queries(np.sort(keys), m, 0.99, q_seed)
    else:
        q = dg.gen_point_queries(keys, m, hit, q_seed)
    out = ref.search(q)
    return ref, keys, vals, {"n": n, "key_seed": key_seed, "m": m, "hit": hit, "q_seed": q_seed,
                             "zipf": zipf, "digest": digest(out), "hits": int((out >= 0).sum()),
                             "ref_height": ref.height, "ref_build_s": round(build_s, 1)}


def range_case(ref, m, lo, hi, seed):
    st, ln = dg.gen_ranges(m, lo, hi, seed)
    off, k, v = ref.range(st, ln)
    return {"m": m, "lo": lo, "hi": hi, "seed": seed, "digest": digest(off, k, v), "records": int(len(k))}


def range_between_case(ref, m, n_keys, lo, hi, seed):
    st, en = dg.gen_range_pairs(m, n_keys, lo, hi, seed)
    off, k, v = ref.range_between(st, en)
    return {"m": m, "n_keys": n_keys, "lo": lo, "hi": hi, "seed": seed, "digest": digest(off, k, v),
            "records": int(len(k))}


def batches_case(ref, keys, sk, nb, seed):
    """C4: per-batch digests of the uneven batch set (datagen.gen_uneven_batches)."""
    sizes, q = dg.gen_uneven_batches(keys, sk, nb, seed)
    res = ref.search(q)
    ends = np.concatenate([[0], np.cumsum(sizes)])
    return {"nb": nb, "seed": seed, "queries": int(len(q)), "digest": digest(res), "hits": int((res >= 0).sum()),
            "batch_digests": [digest(res[ends[b]:ends[b + 1]]) for b in range(nb)]}


def serving_replay_case(n, key_seed, count, seed):
    """C5: the seeded serving stream (datagen.gen_serving_stream) replayed on
    the reference in submission order: reads answered against the tree as
    the upserts before them left it, upserts applied by the reference's
    batched update."""
    keys = dg.gen_keys(n, key_seed)
    t0 = time.time()
    ref = po.RefTree(keys, dg.values_for(keys))
    build_s = time.time() - t0
    stream = dg.gen_serving_stream(keys, count, seed)
    reads = []
    for req in stream:
        if req[0] == "search":
            reads.append(digest(ref.search(req[1])))
        elif req[0] == "range":
            off, k, v = ref.range(req[1], req[2])
            reads.append(digest(off, k, v))
        else:
            ref.upsert(req[1], req[2])
    ek, ev = ref.export()
    return {"n": n, "key_seed": key_seed, "count": count, "seed": seed, "read_digests": reads,
            "kinds": "".join(r[0][0] for r in stream), "export_digest": digest(ek, ev), "n_after": int(len(ek)),
            "ref_build_s": round(build_s, 1)}


def upsert_case(ref, keys, m, new_frac, seed):
    bk, bv = dg.gen_upserts(keys, m, new_frac, seed)
    ref.upsert(bk, bv)
    ek, ev = ref.export()
    after = ref.search(bk)
    return {"m": m, "new_frac": new_frac, "seed": seed, "export_digest": digest(ek, ev),
            "n_after": int(len(ek)), "search_digest": digest(after)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    args = ap.parse_args()
    po.build(ref=True)
    path = os.path.join(GOLDEN_DIR, "golden.json")
    gold = json.load(open(path)) if os.path.exists(path) else {}
    gold["_about"] = ("SHA-256 digests of the reference CPU B+tree's outputs (open-harmonia/src, "
                      "built by oracle/Makefile) on harmonia_b200.datagen inputs; made by "
                      "tests/golden/make_golden.py")

    # C1: 2^20 keys, 2^20 queries, 50% hits; the same tree for Zipf, range and upsert.
    ref, keys, vals, c1 = point_case(1 << 20, 1, 1 << 20, 0.5, 2)
    gold["c1_point"] = c1
    q = dg.gen_zipf_queries(np.sort(keys), 1 << 20, 0.99, 3)
    gold["c1_zipf"] = {"m": 1 << 20, "theta": 0.99, "q_seed": 3, "digest": digest(ref.search(q))}
    gold["c1_range"] = range_case(ref, 1 << 16, 1, 256, 4)
    gold["c1_range_between"] = range_between_case(ref, 1 << 16, 1 << 20, 1, 256, 14)
    gold["c1_upsert"] = upsert_case(ref, keys, 1 << 14, 0.5, 5)
    # inclusive ranges again after the epoch (the reference walk over the updated tree)
    gold["c1_range_between_after"] = range_between_case(ref, 1 << 16, 1 << 20, 1, 256, 14)
    # a second epoch on the updated tree
    ek, _ = ref.export()
    gold["c1_upsert2"] = upsert_case(ref, ek, 1 << 14, 0.5, 6)

    # small: explicit arrays for a 4096-key tree
    n = 4096
    keys = dg.gen_keys(n, 7)
    vals = dg.values_for(keys)
    ref = po.RefTree(keys, vals)
    q = dg.gen_point_queries(keys, 8192, 0.5, 8)
    q[:4] = [np.sort(keys)[0], np.sort(keys)[-1], -5, 0]
    res = ref.search(q)
    st, ln = dg.gen_ranges(512, 1, 16, 9)
    st[:2] = [np.sort(keys)[10], np.sort(keys)[-3]]
    roff, rk, rv = ref.range(st, ln)
    bk, bv = dg.gen_upserts(keys, 256, 0.5, 10)
    ref.upsert(bk, bv)
    ek, ev = ref.export()
    np.savez_compressed(os.path.join(GOLDEN_DIR, "small.npz"), key_seed=7, n=n, q=q, res=res,
                        r_start=st, r_len=ln, r_off=roff, r_keys=rk, r_vals=rv, u_keys=bk,
                        u_vals=bv, after_keys=ek, after_vals=ev)
    gold["small"] = {"n": n, "key_seed": 7, "file": "small.npz"}

    if args.big:
        ref, keys, vals, c2 = point_case(1 << 26, 1, 1 << 24, 0.9, 2)
        gold["c2_point"] = c2
        q = dg.gen_zipf_queries(np.sort(keys), 1 << 24, 0.99, 3)
        gold["c3_zipf"] = {"m": 1 << 24, "theta": 0.99, "q_seed": 3, "digest": digest(ref.search(q))}
        gold["c3_range"] = range_case(ref, 1 << 20, 1, 256, 4)
        gold["c3_range_between"] = range_between_case(ref, 1 << 20, 1 << 26, 1, 256, 15)
        gold["c4_batches"] = batches_case(ref, keys, np.sort(keys), 512, 7)
        # one update epoch at the paper's batch size: 4096K keys, 5% new
        bk, bv = dg.gen_upserts(keys, 4 << 20, 0.05, 21)
        t0 = time.time()
        ref.upsert(bk, bv)
        up_s = time.time() - t0
        ek, ev = ref.export()
        q = dg.gen_point_queries(keys, 1 << 24, 0.9, 2)
        gold["c2_upsert_4096k"] = {"m": 4 << 20, "new_frac": 0.05, "seed": 21, "export_digest": digest(ek, ev),
                                   "n_after": int(len(ek)), "search_batch_digest": digest(ref.search(bk)),
                                   "search_c2_digest": digest(ref.search(q)), "ref_upsert_s": round(up_s, 1)}
        del ref, ek, ev
        gold["c5_serving_replay"] = serving_replay_case(1 << 25, 11, 400, 11)
    with open(path, "w") as f:
        json.dump(gold, f, indent=1, sort_keys=True)
    print(json.dumps(gold, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
