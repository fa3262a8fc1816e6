"""Benchmark of the batched B+tree point search on B200.

Workload (the headline): a 2^26-key tree at fanout 64 (keys uniform in
[0, 2^63), value = splitmix64(key) >> 1), one batch of 2^24 point queries
with 90% hits, seeded synthetic data.  A step is one batch through
BPlusTree.search (pre-sort + search + results in query order).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun each rank runs an independent
replica of the tree on its own GPU with its own query batch (the path does
not shard: replicas only); ``value`` is all ranks' queries over the slowest
rank's device time.

``--impl reference`` times the reference's own CPU B+tree
(open-harmonia/src, compiled into oracle/_ref/libhmref.so) on the same keys
and queries with all host threads: OpenMP over BPlusTree::search, the loop
of search_cpu_test (open-harmonia/src/main.cpp:772-812).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mqueries/s on 2^26-key tree (1 B200) vs plain batch; serving p50/p99 latency"
UNIT = "Mqueries/s"
FALLBACK_PEAK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--keys-log2", type=int, default=26)
    ap.add_argument("--queries-log2", type=int, default=24)
    ap.add_argument("--hit", type=float, default=0.9)
    ap.add_argument("--fanout", type=int, default=64)
    ap.add_argument("--leaf-cap", type=int, default=16)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (use the flags below)")
    ap.add_argument("--group-width", type=int, default=4)
    ap.add_argument("--qpg", type=int, default=1)
    ap.add_argument("--sort-bits", type=int, default=-1)
    ap.add_argument("--hints", type=int, default=1)
    ap.add_argument("--join", type=int, default=-1, help="1 bucket join, 2 never, -1 auto")
    ap.add_argument("--cpu-sample-log2", type=int, default=22)
    ap.add_argument("--extras", type=int, default=1, help="also time plain / pre-sorted input / e2e")
    ap.add_argument("--upsert-only", action="store_true",
                    help="time only the 4096K-key upsert epochs (one JSON line; each timed epoch is an NVTX "
                         "range named upsert_epoch)")
    return ap.parse_args()


def workload_name(args) -> str:
    """The workload both arms run, in words (the same string in both lines)."""
    return (f"point search, 2^{args.keys_log2} keys (uniform 63-bit, value = splitmix64(key)>>1), fanout "
            f"{args.fanout}, one 2^{args.queries_log2}-query batch, {int(args.hit * 100)}% hits")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_PEAK_GBS, "fallback"


def algorithmic_bytes_per_query(fanout: int) -> int:
    """Bytes a point query must move at 2^26 keys: 8 B key in + 8 B value out,
    the DRAM-resident level (the leaves: one 8-entry index + one 8-key slice,
    64 B + 64 B, or the 128-B row of a 16-key leaf), and one 32-B value sector.
    Inner levels are L2-resident.  Fanout 128 adds its 128-B index + 64-B
    slice for the last inner level, which no longer fits L2."""
    return 176 if fanout == 64 else 240


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
                self.lines = [l for l in out.splitlines() if l.strip()]
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args, ws, rank):
    """The reference's own CPU tree (oracle/_ref/libhmref.so, built from
    open-harmonia/src) on the same keys and the whole query batch per step:
    OpenMP over BPlusTree::search on all host threads, the loop of
    search_cpu_test (open-harmonia/src/main.cpp:772-812).  value = queries
    per step over the median step time."""
    if rank != 0:
        return 0
    from harmonia_b200 import datagen as dg
    from oracle import pyoracle as po

    if not po.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhmref.so is not built"}))
        return 0
    n = 1 << args.keys_log2
    keys = dg.gen_keys(n, 1)
    vals = dg.values_for(keys)
    t0 = time.time()
    ref = po.RefTree(keys, vals)
    build_s = time.time() - t0
    m = 1 << args.queries_log2
    q = dg.gen_point_queries(keys, m, args.hit, 2)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        ref.search(q, threads)
    times = []
    for _ in range(args.steps):
        a = time.perf_counter()
        ref.search(q, threads)
        times.append(time.perf_counter() - a)
    sec = statistics.median(times)
    v = m / sec / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded splitmix64 keys/queries)",
        "config": {"workload": workload_name(args), "queries_per_step": m, "statistic": "median of the steps",
                   "layout": "the reference's PPI tree (BPT_ORDER 64 inner nodes, 64-list big leaves)"},
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"the whole {m}-query batch per step, OpenMP BPlusTree::search over "
                                   f"{threads} threads, median of {args.steps} steps; tree build {build_s:.0f} s "
                                   "excluded"},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _cpu_reference_worker(conn, kind, keys_log2, queries_log2, hit):
    """Spawned helper process (no CUDA): builds one of the reference's CPU
    trees of the bench workload while the GPU legs run (the build is serial),
    then on "go" times it on all host threads and sends the figures back.
    kind "ppi": the reference's PPI tree (open-harmonia/src): point search
    (BPlusTree::search), range scans (the parallel walk of cpu-range.cpp) and
    one update epoch of 4096K keys (insert_parallel_Newupdate_batch).  kind
    "cfb": its pointer B+tree at order 128 (open-harmonia/regular_bpt):
    find()."""
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)  # the reference prints from its update path
    sys.path.insert(0, ROOT)
    from harmonia_b200 import datagen as dg
    from oracle import pyoracle as po

    n = 1 << keys_log2
    keys = dg.gen_keys(n, 1)
    vals = dg.values_for(keys)
    t0 = time.time()
    gpu = kind == "ppi" and po.gpu_ref_available()
    tree = po.RefTree(keys, vals, gpu=gpu) if kind == "ppi" else po.CfbTree(keys, vals)
    build_s = time.time() - t0
    conn.send({"built_s": build_s})
    if conn.recv() != "go":
        return
    threads = os.cpu_count() or 1
    m = 1 << queries_log2
    q = dg.gen_point_queries(keys, m, hit, 2)

    def median_s(fn, reps=5):
        ts = []
        for _ in range(reps):
            a = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - a)
        return statistics.median(ts)

    tree.search(q[: 1 << 20], threads)  # warm
    sec = median_s(lambda: tree.search(q, threads))
    cpu_out = tree.search(q, threads)
    res = {"build_s": round(build_s, 1), "cores": threads,
           "search": {"value": round(m / sec / 1e6, 3), "unit": UNIT, "ms_per_step": round(sec * 1e3, 1),
                      "sample": f"the whole {m}-query batch, median of 5"}}
    if kind == "ppi":
        # the reference's second CPU search: 16 queries per group, AVX2 child
        # search, each next node prefetched (search_cpu_prefetch_NTG_PPI)
        tree.search_prefetch(q[: 1 << 20], threads)
        sec = median_s(lambda: tree.search_prefetch(q, threads))
        same = bool((tree.search_prefetch(q, threads) == cpu_out).all())
        res["search_prefetch"] = {"value": round(m / sec / 1e6, 3), "unit": UNIT, "ms_per_step": round(sec * 1e3, 1),
                                  "same_results": same,
                                  "sample": f"the whole {m}-query batch, median of 5"}
        st, ln = dg.gen_ranges(1 << 20, 1, 256, seed=12)
        rec, _ = tree.range_timed(st, ln, threads)
        sec = median_s(lambda: tree.range_timed(st, ln, threads))
        res["range"] = {"value": round(len(st) / sec / 1e6, 3), "unit": "Mranges/s", "ms_per_step": round(sec * 1e3, 1),
                        "records_per_s_m": round(rec / sec / 1e6, 1),
                        "sample": "2^20 ranges of 1..256 records, the parallel walk of cpu-range.cpp, median of 5"}
        if gpu:  # the reference's own GPU search on this GPU, after every GPU leg of the bench
            try:
                g = po.RefGpuSearch(tree)
                out, md, mc = g.search(q, reps=5)
                g.close()
                wrong = int((out != cpu_out).sum())
                check = (f"{wrong} of {m} results differ from the reference's own CPU search "
                         f"({int(((out == -1) & (cpu_out >= 0)).sum())} hits returned as misses)")
                res["gpu"] = {"value": round(m / md / 1e3, 1), "unit": UNIT, "ms_per_step": round(md, 4),
                              "with_copies": {"value": round(m / mc / 1e3, 1), "unit": UNIT, "ms_per_step": round(mc, 3)},
                              "wrong_results": wrong, "check": check,
                              "what": "the reference's GPU search compiled for sm_100a (open-harmonia/src/full-multi-"
                                      "prefix-sort-8thread.cu: CUB SortPairs on bits [48,64) + the 8-thread kernel) "
                                      "on its own PPI tree, device-resident keys, mean of 5; with_copies adds the "
                                      "key upload and the result download (oracle/ref_gpu_driver.cu)"}
            except Exception as e:
                res["gpu"] = {"unavailable": repr(e)}
        bk, bv = dg.gen_upserts(keys, 4 << 20, 0.05, 21)
        a = time.perf_counter()
        tree.upsert(bk, bv)
        sec = time.perf_counter() - a
        res["upsert"] = {"value": round(len(bk) / sec / 1e6, 3), "unit": "Mkeys/s", "ms_per_step": round(sec * 1e3, 1),
                         "sample": "one insert_parallel_Newupdate_batch epoch of 4096K keys (5% new), once"}
    conn.send(res)


class CpuReference:
    """The spawned helpers of the reference CPU figures (see
    _cpu_reference_worker); started before any CUDA call."""

    def __init__(self, args):
        import multiprocessing as mp

        from oracle import pyoracle as po

        self.procs = {}
        ctx = mp.get_context("spawn")
        kinds = []
        if po.ref_available():
            kinds.append("ppi")
        if po.cfb_available() and args.fanout == 64:
            kinds.append("cfb")
        for kind in kinds:
            a, b = ctx.Pipe()
            p = ctx.Process(target=_cpu_reference_worker,
                            args=(b, kind, args.keys_log2, args.queries_log2, args.hit), daemon=True)
            p.start()
            self.procs[kind] = (p, a)

    def wait_built(self, timeout_s: float = 600.0) -> None:
        """Waits for the builds, so the host-bound legs (host-buffer search,
        serving) run with the host to themselves."""
        self.built = getattr(self, "built", {})
        for kind, (p, conn) in self.procs.items():
            if kind in self.built:
                continue
            try:
                if conn.poll(timeout_s):
                    self.built[kind] = conn.recv()
            except Exception:
                pass

    def run(self, timeout_s: float = 600.0) -> dict:
        """Waits for the builds, times every tree (one after another, so each
        has all host threads), returns {kind: figures}."""
        self.built = getattr(self, "built", {})
        out = {}
        for kind, (p, conn) in self.procs.items():
            try:
                if kind not in self.built:
                    if not conn.poll(timeout_s):
                        raise TimeoutError("reference build did not finish")
                    self.built[kind] = conn.recv()
                conn.send("go")
                if not conn.poll(timeout_s):
                    raise TimeoutError("reference timing did not finish")
                out[kind] = conn.recv()
            except Exception as e:  # reported in the line, the bench goes on
                out[kind] = {"unavailable": repr(e)}
            p.join(5)
            if p.is_alive():
                p.kill()
        return out


def cpu_baseline_port(keys_sorted, vals_sorted, q, seconds: float = 10.0):
    """The oracle's C restatement (OpenMP over the queries, as the reference's
    search_cpu_test) on a bounded sample of the batch."""
    from oracle import pyoracle as po

    t = po.PortTree(keys_sorted, vals_sorted)
    m = 1 << 20
    t.search(q[:m])  # warm
    a = time.perf_counter()
    done = 0
    while done < len(q) and time.perf_counter() - a < seconds:
        t.search(q[done:done + m])
        done += m
    sec = time.perf_counter() - a
    cores = os.cpu_count() or 1
    return {"value": round(min(done, len(q)) / sec / 1e6, 3), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{min(done, len(q))} queries of the batch in {sec:.1f} s, C restatement of the "
                      f"search (oracle/hm_oracle.c), OpenMP over {cores} threads"}


def _digest(*arrays) -> str:
    """SHA-256 over the little-endian int64 bytes of the arrays (the golden
    fixtures' digest)."""
    import hashlib

    h = hashlib.sha256()
    for x in arrays:
        h.update(np.ascontiguousarray(np.asarray(x), dtype="<i8").tobytes())
    return h.hexdigest()


def _golden(name):
    """An entry of tests/golden/golden.json (digests of the reference CPU
    tree's outputs on these seeded workloads), or None."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
            return json.load(f).get(name)
    except Exception:
        return None


def batched_uneven(tree, keys, sk, dev, timed, steps, warmup, seed=7):
    """512 batches with sizes log-uniform in [1K, 4M], half uniform (90% hits),
    half Zipf(0.99) over key rank (datagen.gen_uneven_batches): one untuned
    launch per batch, the tuned hm_search once per batch, and the whole set in
    one captured CUDA graph (joint pre-sort + bucket join or search).  Every
    batch's results are checked against the reference's digests."""
    import torch
    from harmonia_b200 import datagen as dg

    nb = 512
    sizes, hq = dg.gen_uneven_batches(keys, sk, nb, seed)
    total = int(sizes.sum())
    ends = np.concatenate([[0], np.cumsum(sizes)])
    allq = torch.from_numpy(hq).to(dev)
    allo = torch.empty_like(allq)
    del hq
    batches = [(allq[ends[b]:ends[b + 1]], allo[ends[b]:ends[b + 1]]) for b in range(nb)]
    cfg = tree.config()

    def per_batch():
        for q, out in batches:
            tree.search(q, out)

    tree.set_search_config(group_width=4, queries_per_group=1, sort_bits=0, join=2)
    for _ in range(warmup):
        per_batch()
    plain_ms = timed(steps, per_batch)
    tree.set_search_config(**{k: cfg[k] for k in ("group_width", "queries_per_group", "sort_bits", "cache_hints",
                                                   "join")})
    for _ in range(warmup):
        per_batch()
    tuned_ms = timed(steps, per_batch)
    plan = tree.plan(batches)
    for _ in range(warmup):
        plan.launch()
    plan_ms = timed(steps, plan.launch)
    g = _golden("c4_batches")
    res = allo.cpu().numpy()
    if g and g["nb"] == nb and g["seed"] == seed and g["queries"] == total:
        bad = [b for b in range(nb) if _digest(res[ends[b]:ends[b + 1]]) != g["batch_digests"][b]]
        assert not bad, f"batched results differ from the reference in batches {bad[:8]}"
        check = "every batch's results equal the reference's (golden c4_batches digests)"
    else:  # spot check: a loaded key's value is splitmix64(key) >> 1, a miss is -1
        for b in (0, 1, nb // 2, nb - 1):
            qq = batches[b][0][:2048].cpu().numpy()
            pos = np.searchsorted(sk, qq).clip(max=len(sk) - 1)
            exp = np.where(sk[pos] == qq, dg.values_for(qq), -1)
            assert (res[ends[b]:ends[b] + len(qq)] == exp).all(), "batched results are wrong"
        check = "spot check of 4 batches"
    plan.close()
    return {"batches": nb, "queries": total, "min_batch": int(sizes.min()), "max_batch": int(sizes.max()),
            "check": check,
            "plain_per_batch": {"value": round(total / plain_ms / 1e3, 1), "unit": UNIT,
                                "ms_per_step": round(plain_ms, 3),
                                "what": "one search launch per batch, unsorted, group width 4, 1 query per group (the default)"},
            "tuned_per_batch": {"value": round(total / tuned_ms / 1e3, 1), "unit": UNIT,
                                "ms_per_step": round(tuned_ms, 3),
                                "what": "hm_search with the tuned configuration once per batch (pre-sort and "
                                        "bucket join where the automatic choice takes them), no graph"},
            "graph": {"value": round(total / plan_ms / 1e3, 1), "unit": UNIT, "ms_per_step": round(plan_ms, 3),
                      "what": "the 512 batches in one captured CUDA graph: joint 16-bit pre-sort reading the "
                              "batches in place, bucket join, inverse pre-sort writing each batch's output"},
            "speedup": round(plain_ms / plan_ms, 3), "speedup_vs_tuned_per_batch": round(tuned_ms / plan_ms, 3)}


def upsert_epochs(keys, dev, steps, peak):
    """One update epoch of 4096K keys on the 2^26-key tree (5% new keys, the
    rest existing with value key-1: the paper's batched-update config),
    applied by hm_upsert_batch from device buffers to a freshly loaded tree per
    step (CUDA events around the call; the load is not timed).  Two layouts:
    12 of 16 leaf slots filled (new keys merge in place) and full leaves
    (overflowing leaves rebalance their subtree or the tree is rebuilt).
    Roofline of the in-place epoch: B_u = 16 + 128 + 2 x 256 B per touched
    leaf / updates per touched leaf (key and value in, the descent's leaf
    line, each touched leaf row read and written once)."""
    import torch
    from harmonia_b200 import BPlusTree, datagen as dg

    bk, bv = dg.gen_upserts(keys, 4 << 20, 0.05, 21)
    d_keys = torch.from_numpy(keys).to(dev)
    d_vals = torch.from_numpy(dg.values_for(keys)).to(dev)
    d_bk, d_bv = torch.from_numpy(bk).to(dev), torch.from_numpy(bv).to(dev)
    g = _golden("c2_upsert_4096k")
    out = {"keys_per_epoch": len(bk), "new_frac": 0.05}
    sk = np.sort(keys)
    for fill, name in ((12, "leaf_fill_12"), (16, "full_leaves")):
        times = []
        for i in range(1 + steps):
            t = BPlusTree.bulk_load(d_keys, d_vals, leaf_fill=fill)
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("upsert_epoch")
            a.record()
            t.upsert(d_bk, d_bv)
            b.record()
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
            if i > 0:
                times.append(a.elapsed_time(b))
            if i == steps and g:
                ek, ev = t.export()
                assert _digest(ek, ev) == g["export_digest"], "contents after the epoch differ from the reference"
            t.close()
        ms = statistics.median(times)
        r = {"value": round(len(bk) / ms / 1e3, 1), "unit": "Mkeys/s", "ms_per_step": round(ms, 3),
             "what": f"hm_upsert_batch, 4096K keys, tree bulk-loaded with {fill} keys per 16-key leaf, median of {steps}"}
        if fill == 12:
            n_leaf = -(-len(keys) // fill)
            qd, rem = divmod(len(keys), n_leaf)
            rank = np.searchsorted(sk, bk, side="right") - 1
            rank = rank.clip(min=0)
            cut = rem * (qd + 1)
            leaf = np.where(rank < cut, rank // (qd + 1), rem + (rank - cut) // max(qd, 1))
            touched = len(np.unique(leaf))
            bu = 16 + 128 + 2 * 256 * touched / len(bk)
            ach = bu * len(bk) / (ms * 1e-3) / 1e9
            r["roofline"] = {"bound": "hbm", "algorithmic_bytes_per_update": round(bu, 1), "touched_leaves": touched,
                             "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4)}
        out[name] = r
    out["check"] = "contents after the epoch equal the reference's (golden c2_upsert_4096k)" if g else "none"
    return out


def fanout_128(keys, q, d_q, dev, timed, steps, warmup, exp):
    """The same keys and batch on a fanout-128 tree: the descent unsorted, the
    descent on a batch pre-sorted by its top 16 key bits, and the tuned path.
    Algorithmic bytes of the descent at fanout 128: 240 B per query (the last
    inner level, 1 KiB rows, is no longer L2-resident)."""
    import torch
    from harmonia_b200 import BPlusTree, datagen as dg

    m = len(q)
    t = BPlusTree.bulk_load(torch.from_numpy(keys).to(dev), torch.from_numpy(dg.values_for(keys)).to(dev),
                            fanout=128)
    out = torch.empty_like(d_q)
    res = {"tree": {"height": int(t.info().height), "n_leaf": int(t.info().n_leaf)}}

    def run(name, qq, what, bq=None):
        for _ in range(warmup):
            t.search(qq, out)
        ms = timed(steps, lambda: t.search(qq, out))
        r = {"value": round(m / ms / 1e3, 1), "unit": UNIT, "ms_per_step": round(ms, 4), "what": what}
        if bq:
            r["algorithmic_gbs"] = round(bq * m / (ms * 1e-3) / 1e9, 1)
        res[name] = r

    t.set_search_config(group_width=4, queries_per_group=1, sort_bits=0, join=2)
    run("plain", d_q, "one descent launch on the unsorted batch, group width 4, 1 query per group (the default)", 240)
    assert (out[:4096].cpu().numpy() == exp).all(), "fanout-128 results are wrong"
    order = np.argsort(q >> np.int64(47), kind="stable")
    d_qs = torch.from_numpy(q[order]).to(dev)
    run("presorted_input", d_qs, "the same launch on the batch pre-sorted by its top 16 key bits", 240)
    del d_qs
    tuned = t.autotune(d_q)
    run("tuned", d_q, "the autotuned path (descent settings, and the bucket join where it wins)")
    assert (out[:4096].cpu().numpy() == exp).all(), "fanout-128 results are wrong"
    res["tuned"]["config"] = {k: tuned[k] for k in ("group_width", "queries_per_group", "sort_bits", "join")}
    t.close()
    return res


class _PinnedRing:
    """Page-locked result buffers for serving requests, handed out in ring
    order; a slice is reused only after the request that held it finished (a
    client with a bounded pool of registered buffers)."""

    def __init__(self, n):
        import collections
        import torch
        self.buf = torch.empty(n, dtype=torch.int64, pin_memory=True).numpy()
        self.n, self.at, self.live = n, 0, collections.deque()

    def take(self, m):
        if self.at + m > self.n:
            self.at = 0
        lo, hi = self.at, self.at + m
        while self.live and self.live[0][0] < hi and lo < self.live[0][1]:
            self.live.popleft()[2].wait()
        self.at = hi
        return lo, hi, self.buf[lo:hi]

    def hold(self, lo, hi, ticket):
        self.live.append((lo, hi, ticket))


def serving_loads(dev, loads=(0.25, 0.5, 0.9), seconds=2.0, seed=11, pinned=False):
    """Serving workload: a 2^25-key tree; Poisson arrivals, request sizes
    log-uniform in [64, 2^20]; 90% point search (80% hits), 5% range (length
    1..128), 5% upsert (half new, half existing keys) applied in epochs.
    Capacity is the mix with 64 requests kept outstanding; the offered loads
    are fractions of the highest Poisson rate the server keeps up with.
    Reports throughput and p50/p99 submit-to-completion latency at each load,
    and checks the seeded stream against the reference and a sample of the
    loads' answers."""
    import threading
    from harmonia_b200 import BPlusTree, datagen as dg
    from harmonia_b200.serving import Server

    n = 1 << 25
    keys = dg.gen_keys(n, seed)
    tree = BPlusTree.bulk_load(keys, dg.values_for(keys), leaf_fill=12)
    pool = dg.gen_point_queries(keys, 1 << 24, 0.8, seed + 1)
    ring = None
    if pinned:  # point requests in page-locked buffers: copied by DMA, no staging copy
        import torch
        pinned_pool = torch.empty(len(pool), dtype=torch.int64, pin_memory=True).numpy()
        pinned_pool[:] = pool
        pool = pinned_pool
        ring = _PinnedRing(1 << 26)
    rstart, rlen = dg.gen_ranges(1 << 16, 1, 128, seed + 2)
    rng = np.random.default_rng(seed)
    out = {}
    with Server(tree, streams=3, max_launch_queries=1 << 22, device_budget_bytes=2 << 30) as srv:
        def sizes(k):
            return np.exp(rng.uniform(np.log(64), np.log(1 << 20), k)).astype(np.int64)

        new_keys = dg.gen_keys(1 << 22, seed + 100)
        new_at = [0]

        def submit(kind_u, m):
            """One request of the mix: 90% point, 5% range, 5% upsert."""
            if kind_u < 0.90:
                o = int(rng.integers(0, len(pool) - m))
                if ring is None:
                    return ("s", srv.search(pool[o:o + m]), o, m)
                lo, hi, ob = ring.take(m)
                tk = srv.search(pool[o:o + m], out=ob)
                ring.hold(lo, hi, tk)
                return ("s", tk, o, m)
            if kind_u < 0.95:
                k = max(1, m // 64)
                o = int(rng.integers(0, len(rstart) - k))
                return ("r", srv.range(rstart[o:o + k], rlen[o:o + k]), o, k)
            k = max(2, min(m // 16, 64))
            nk = new_keys[new_at[0]:new_at[0] + k // 2]
            new_at[0] += k // 2
            ek = keys[rng.integers(0, n, k - k // 2)]
            bk = np.concatenate([nk, ek])
            bv = np.concatenate([dg.values_for(nk), ek - 1])
            return ("u", srv.upsert(bk, bv), 0, k)

        # capacity: the seeded request stream (datagen.gen_serving_stream, the
        # same mix) submitted back to back; every read and the contents after
        # it are checked against the reference replaying it in order
        stream = dg.gen_serving_stream(keys, 400, seed)
        cap_n = len(stream)
        t0 = time.perf_counter()
        tks = []
        for req in stream:
            if req[0] == "search":
                tks.append(srv.search(req[1]))
            elif req[0] == "range":
                tks.append(srv.range(req[1], req[2]))
            else:
                tks.append(srv.upsert(req[1], req[2]))
        for tk in tks:
            tk.wait()
        burst_wall = time.perf_counter() - t0
        burst = {"requests": cap_n, "req_per_s": round(cap_n / burst_wall, 1),
                 "mqps": round(srv.stats()["queries"] / burst_wall / 1e6, 1)}
        g = _golden("c5_serving_replay")
        if g and g["n"] == n and g["count"] == cap_n and g["seed"] == seed:
            reads = []
            for req, tk in zip(stream, tks):
                if req[0] == "search":
                    reads.append(_digest(tk._result()))
                elif req[0] == "range":
                    reads.append(_digest(*tk._result()))
            assert reads == g["read_digests"], "serving reads differ from the reference replay"
            ek, ev = tree.export()
            assert _digest(ek, ev) == g["export_digest"], "contents after the stream differ from the reference"
            out["check"] = ("the capacity stream's reads and the contents after it equal the reference replaying "
                            "it in order (golden c5_serving_replay)")
        del stream, tks
        # sustained capacity: a closed loop that keeps 64 requests of the mix
        # outstanding (a client with 64 requests in flight) for about two
        # seconds; a burst of thousands submitted at once lets the server
        # coalesce far more than Poisson arrivals at the same rate do, so
        # loads taken as fractions of it were not sustainable
        import collections
        srv.reset_stats()
        cap_n = max(2000, int(2.0 * burst["req_per_s"]))
        cap_kinds, cap_sizes = rng.random(cap_n), sizes(cap_n)
        window = collections.deque()
        t0 = time.perf_counter()
        for u, m in zip(cap_kinds, cap_sizes):
            if len(window) >= 64:
                window.popleft()[1].wait()
            window.append(submit(u, int(m)))
        while window:
            window.popleft()[1].wait()
        cap_wall = time.perf_counter() - t0
        cap_rps = cap_n / cap_wall
        cap_qps = srv.stats()["queries"] / cap_wall
        def poisson(rate, secs):
            """Poisson arrivals of the mix at `rate` requests/s for `secs`
            seconds; returns (tickets, wall seconds until the last finished)."""
            srv.reset_stats()
            count = int(rate * secs) + 1
            gaps = rng.exponential(1.0 / rate, count)
            kinds = rng.random(count)
            szs = sizes(count)
            tickets = []
            t_start = time.perf_counter()
            due = t_start
            for i in range(count):
                due += gaps[i]
                while time.perf_counter() < due:
                    pass
                tickets.append(submit(kinds[i], int(szs[i])))
            for kind, tk, o, m in tickets:
                tk.wait()
            return tickets, time.perf_counter() - t_start

        # sustainable rate: the highest Poisson rate (from 90 % of the
        # closed-loop capacity down in steps of 15 %) that the server keeps up
        # with over one second (every request done within 5 % of the window
        # after the last arrival); the offered loads are fractions of it
        rate, tries = 0.9 * cap_rps, []
        for _ in range(6):
            tk_s, wall = poisson(rate, 1.0)
            keeps_up = wall <= 1.05 * (len(tk_s) / rate) + 0.005
            tries.append({"req_per_s": round(rate, 1), "keeps_up": keeps_up,
                          "p99_ms": round(srv.stats()["p99_us"] / 1e3, 3)})
            if keeps_up:
                break
            rate *= 0.85
        sus_rps, sus_qps = rate, srv.stats()["queries"] / wall
        del tk_s
        for frac in loads:
            rate = frac * sus_rps  # requests per second
            tickets, wall = poisson(rate, seconds)
            count = len(tickets)
            st = srv.stats()
            out[f"load_{frac}"] = {"offered_req_per_s": round(rate, 1), "requests": count,
                                   "throughput_mqps": round(st["queries"] / wall / 1e6, 1),
                                   "p50_ms": round(st["p50_us"] / 1e3, 3), "p99_ms": round(st["p99_us"] / 1e3, 3),
                                   "max_ms": round(st["max_us"] / 1e3, 3), "launches": st["launches"],
                                   "epochs": st["epochs"], "failed": st["failed"],
                                   "split_ms": {k[:-3]: round(st[k] / 1e3, 3) for k in (
                                       "queue_p50_us", "queue_p99_us", "stage_p50_us", "stage_p99_us",
                                       "device_p50_us", "device_p99_us", "finish_p50_us", "finish_p99_us",
                                       "epoch_drain_mean_us", "epoch_apply_mean_us")}}
        # answers in the mix: a point request's hits return splitmix64(key)>>1 or key-1 (updated)
        s_hits = [t for t in tickets if t[0] == "s"][-20:]  # the newest: their result buffers are not reused yet
        for kind, tk, o, m in s_hits:
            q = pool[o:o + m]
            got = tk._result()
            ok = (got == -1) | (got == dg.values_for(q)) | (got == q - 1)
            assert ok.all(), "serving answer outside the possible values"
        out["capacity"] = {"req_per_s": round(cap_rps, 1), "mqps": round(cap_qps / 1e6, 1), "requests": cap_n,
                           "what": "the request mix with 64 requests kept outstanding for about 2 s"}
        out["sustainable"] = {"req_per_s": round(sus_rps, 1), "mqps": round(sus_qps / 1e6, 1), "tries": tries,
                              "what": "the highest Poisson arrival rate of the mix the server kept up with over 1 s "
                                      "(from 90 % of capacity down in 15 % steps); the loads are fractions of it"}
        out["request_buffers"] = ("page-locked (point searches copied by DMA, no staging)" if pinned
                                  else "pageable (copied through pinned staging)")
        out["burst"] = dict(burst, what="the 400-request seeded stream submitted back to back (the parity run)")
    tree.close()
    return out


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_init()
    if args.impl == "reference":
        return run_reference(args, ws, rank)
    # the reference's CPU trees build in helper processes while the GPU legs
    # run (spawned before any CUDA call)
    cpu_ref = CpuReference(args) if (rank == 0 and ws == 1 and args.extras and not args.upsert_only) else None

    import torch
    import torch.distributed as dist

    from harmonia_b200 import BPlusTree, datagen as dg, launch_count
    from harmonia_b200 import replicas

    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)

    n = 1 << args.keys_log2
    m = 1 << args.queries_log2
    keys = dg.gen_keys(n, 1)
    if args.upsert_only:
        peak, kind = peaks()
        if rank == 0:  # one GPU's epochs; other ranks only wait
            up = upsert_epochs(keys, dev, args.steps, peak)
            print(json.dumps({"leg": "upsert", "keys": n, "peak_kind": kind, **up}))
        if ws > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    vals = dg.values_for(keys)
    q = dg.gen_point_queries(keys, m, args.hit, replicas.query_seed(2, rank))
    d_keys = torch.from_numpy(keys).to(dev)
    d_vals = torch.from_numpy(vals).to(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tree = BPlusTree.bulk_load(d_keys, d_vals, fanout=args.fanout, leaf_cap=args.leaf_cap)
    torch.cuda.synchronize()
    bulk_ms = (time.perf_counter() - t0) * 1e3
    del d_keys, d_vals
    d_q = torch.from_numpy(q).to(dev)
    d_out = torch.empty_like(d_q)
    info = tree.info()

    def timed(steps, fn):
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(steps):
            fn()
        b.record()
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        ms = replicas.max_over_ranks(a.elapsed_time(b), dev if ws > 1 else None)
        return ms / steps

    extras = {}
    # plain single-batch launch: unsorted, default group width/depth, no tuning
    if args.extras:
        tree.set_search_config(group_width=4, queries_per_group=1, sort_bits=0, join=2)
        for _ in range(args.warmup):
            tree.search(d_q, d_out)
        plain_ms = timed(args.steps, lambda: tree.search(d_q, d_out))
        extras["plain"] = {"value": round(ws * m / plain_ms / 1e3, 1), "unit": UNIT, "ms_per_step": round(plain_ms, 4),
                           "what": "one launch of the search kernel on the unsorted batch, group width 4, "
                                   "1 query per group (the default configuration), no pre-sort"}
    tree.set_search_config(group_width=args.group_width, queries_per_group=args.qpg,
                           sort_bits=args.sort_bits, cache_hints=args.hints, join=args.join)
    tuned = tree.config()
    if not args.no_tune:
        tuned = tree.autotune(d_q)
    for _ in range(args.warmup):
        tree.search(d_q, d_out)
    # spot check outside the timed region: a loaded key's value is
    # splitmix64(key) >> 1 by construction of the workload, a miss is -1
    sk = np.sort(keys)
    qs = q[:4096]
    pos = np.searchsorted(sk, qs).clip(max=n - 1)
    exp = np.where(sk[pos] == qs, dg.values_for(qs), -1)
    assert (d_out[:4096].cpu().numpy() == exp).all(), "search results are wrong"

    # ---- headline timed region (no stage events inside it: an event between
    # two kernels of the path would stop the next one from launching early) ----
    l0 = launch_count()
    with ClockSampler(local) as clk:
        ms = timed(args.steps, lambda: tree.search(d_q, d_out))
    launches = launch_count() - l0
    # stage split: the same step again with CUDA events around each stage
    tree.profile(True)
    tree.profile_read()
    for _ in range(max(3, min(args.steps, 10))):
        tree.search(d_q, d_out)
    torch.cuda.synchronize()
    stages = tree.profile_read()
    tree.profile(False)
    value = replicas.job_throughput(m, ws, ms)  # Mqueries/s (m queries per rank per step)

    peak, peak_kind = peaks()
    info = tree.info()
    if stages.get("join"):
        # the bucket join dominates: it reads every query (8 B), writes every
        # result (8 B) and stages every leaf record once; for batches up to
        # 2^25 queries it also reads each result's 4-B place (the position
        # after the first pre-sort pass, where it writes the result)
        kernel, stage_key = "join_kernel", "join"
        bq = (20 if m <= (1 << 25) else 16) + info.n_leaf * info.leaf_row_words * 8 / m
    else:
        kernel, stage_key = "search_kernel", "search"
        bq = algorithmic_bytes_per_query(args.fanout)
    k_launches, k_total = stages.get(stage_key, (0, 0.0))
    kernel_ms = k_total / max(k_launches, 1)
    achieved = bq * m / (kernel_ms * 1e-3) / 1e9 if kernel_ms > 0 else None
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            key = "join" if kernel == "join_kernel" else f"bits{tuned['sort_bits']}"
            traffic = json.load(open(tf)).get(f"search_f{args.fanout}_lc{args.leaf_cap}_{key}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1) if achieved else None,
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_query": round(bq, 2), "queries_per_launch": m,
                "kernel_ms": round(kernel_ms, 4),
                "path_ms": round(sum(v[1] / max(v[0], 1) for v in stages.values()), 4)}

    # comparison kernel: HB+-style pointer-chasing descent (one thread per query)
    if args.extras:
        for _ in range(args.warmup):
            tree.search_pointer_baseline(d_q, d_out)
        pb_ms = timed(args.steps, lambda: tree.search_pointer_baseline(d_q, d_out))
        assert (d_out[:4096].cpu().numpy() == exp).all(), "pointer baseline results are wrong"
        extras["pointer_baseline"] = {"value": round(ws * m / pb_ms / 1e3, 1), "unit": UNIT,
                                      "ms_per_step": round(pb_ms, 4),
                                      "what": "HB+-style descent following per-node child ids, one thread per "
                                              "query, no prefix array, no pre-sort (comparison kernel)"}

    # pre-sorted input (the batch arrives partially sorted by its top 16 key bits)
    if args.extras:
        order = np.argsort(q >> np.int64(47), kind="stable")
        d_qs = torch.from_numpy(q[order]).to(dev)
        tree.set_search_config(sort_bits=0, join=2)
        for _ in range(args.warmup):
            tree.search(d_qs, d_out)
        ps_ms = timed(args.steps, lambda: tree.search(d_qs, d_out))
        extras["presorted_input"] = {"value": round(ws * m / ps_ms / 1e3, 1), "unit": UNIT,
                                     "what": "batch pre-sorted by its top 16 key bits before the timed region"}
        tree.set_search_config(**{k: tuned[k] for k in ("group_width", "queries_per_group", "sort_bits",
                                                       "cache_hints", "join")})
        del d_qs

    # skewed point queries and ranges (the skewed + range workload): the
    # tuned path on Zipf(0.99) queries, then 2^20 range queries with start
    # uniform and length uniform in [1, 256], output compacted by prefix sum
    if args.extras:
        z = dg.gen_zipf_queries(sk, m, 0.99, seed=11)
        d_z = torch.from_numpy(z).to(dev)
        for _ in range(args.warmup):
            tree.search(d_z, d_out)
        z_ms = timed(args.steps, lambda: tree.search(d_z, d_out))
        assert (d_out[:4096].cpu().numpy() == dg.values_for(z[:4096])).all(), "Zipf results are wrong"
        del d_z
        nr = 1 << 20
        rs, rl = dg.gen_ranges(nr, 1, 256, seed=12)
        d_rs, d_rl = torch.from_numpy(rs).to(dev), torch.from_numpy(rl.astype(np.int32)).to(dev)
        for _ in range(args.warmup):
            tree.range_search(d_rs, d_rl)
        r_ms = timed(args.steps, lambda: tree.range_search(d_rs, d_rl))
        off, rk, _ = tree.range_search(d_rs[:64], d_rl[:64])
        i0 = np.searchsorted(sk, rs[:64])
        exp_n = np.minimum(rl[:64].astype(np.int64), len(sk) - i0)
        assert (np.diff(off.cpu().numpy()) == exp_n).all(), "range counts are wrong"
        assert (rk[:int(exp_n[0])].cpu().numpy() == sk[i0[0]:i0[0] + exp_n[0]]).all(), "range keys are wrong"
        records = int(np.minimum(rl.astype(np.int64), len(sk) - np.searchsorted(sk, rs)).sum())
        extras["skewed_range"] = {
            "zipf_point": {"value": round(ws * m / z_ms / 1e3, 1), "unit": UNIT, "ms_per_step": round(z_ms, 4),
                           "what": "2^24 point queries, Zipf(0.99) over key rank, the tuned path"},
            "range": {"value": round(ws * nr / r_ms / 1e3, 1), "unit": "Mranges/s", "ms_per_step": round(r_ms, 4),
                      "records_per_s_m": round(ws * records / r_ms / 1e3, 1),
                      "what": "2^20 ranges, start uniform, length uniform in [1, 256], compacted output "
                              "(hm_range on device buffers, returns the total to the host)"}}
        del d_rs, d_rl

    if args.extras:
        extras["batched_uneven"] = batched_uneven(tree, keys, sk, dev, timed, max(3, args.steps // 3),
                                                  args.warmup)
    if args.extras and args.fanout == 64:
        extras["fanout_128"] = fanout_128(keys, q, d_q, dev, timed, args.steps, args.warmup, exp)

    if cpu_ref is not None:
        cpu_ref.wait_built()

    # ---- end to end through the public API with host (pinned) buffers ----
    h_q = torch.from_numpy(q).pin_memory()
    h_out = torch.empty_like(h_q).pin_memory()
    for _ in range(args.warmup):
        tree.search(h_q, h_out)
    e2e_ms = timed(args.steps, lambda: tree.search(h_q, h_out))
    assert (h_out[:4096].numpy() == exp).all()
    e2e = {"value": round(ws * m / e2e_ms / 1e3, 1), "unit": UNIT, "h2d_bytes_per_step": m * 8,
           "d2h_bytes_per_step": m * 8, "ms_per_step": round(e2e_ms, 3),
           "what": "BPlusTree.search on pinned host buffers: chunked H2D, search, D2H through the C ABI"}

    if args.extras and args.fanout == 64:
        extras["upsert"] = upsert_epochs(keys, dev, 3, peak)

    if args.extras and rank == 0:
        extras["serving"] = serving_loads(dev)
        # the same mix from a client whose point-search buffers are page-locked
        extras["serving_pinned"] = serving_loads(dev, pinned=True)

    cpu = cpu_port = None
    if rank == 0 and ws == 1:
        cpu_port = cpu_baseline_port(sk, dg.values_for(sk), q, seconds=5.0)
        cpu = cpu_port
    if cpu_ref is not None:
        figs = cpu_ref.run()
        ppi, cfb = figs.get("ppi", {}), figs.get("cfb", {})
        if "search" in ppi:
            f = ppi["search"]
            cpu = {"value": f["value"], "unit": UNIT, "cores": ppi["cores"], "kind": "reference",
                   "sample": f"{f['sample']}: OpenMP BPlusTree::search of the reference's PPI tree "
                             f"(oracle/_ref, open-harmonia/src) over {ppi['cores']} threads; tree build "
                             f"{ppi['build_s']} s excluded"}
        elif ppi:
            cpu_port["reference"] = ppi
        if "search_prefetch" in ppi:
            f = ppi["search_prefetch"]
            extras["cpu_reference_prefetch"] = dict(
                f, cores=ppi["cores"],
                what="the reference's software-pipelined CPU search (search_cpu_prefetch_NTG_PPI, "
                     "cpu-search-prefetch-avxNTG.cpp:480-535: 16 queries per group, AVX2 child search, "
                     "prefetch of each next node) on the same PPI tree, OpenMP over groups")
        if "range" in ppi and "skewed_range" in extras:
            extras["skewed_range"]["range"]["cpu_reference"] = dict(ppi["range"], cores=ppi["cores"])
        if "gpu" in ppi:
            extras["reference_gpu"] = ppi["gpu"]
        if "upsert" in ppi and "upsert" in extras:
            extras["upsert"]["cpu_reference"] = dict(ppi["upsert"], cores=ppi["cores"])
        if "fanout_128" in extras:
            extras["fanout_128"]["cpu_reference"] = (
                dict(cfb["search"], cores=cfb["cores"], build_s=cfb["build_s"],
                     what="find() of the reference's pointer B+tree at order 128 (open-harmonia/regular_bpt)")
                if "search" in cfb else cfb)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded splitmix64 keys/queries)",
            "config": {"workload": workload_name(args),
                       "layout": f"fanout {args.fanout} inner rows, {args.leaf_cap}-key leaf records",
                       "l2": "inputs larger than L2 (2^24 x 8 B queries + tree of "
                             f"{info.device_bytes / 2**30:.2f} GiB), no flush",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                       "tuned": {k: tuned[k] for k in ("group_width", "queries_per_group", "sort_bits",
                                                       "cache_hints", "join")},
                       "tree": {"height": info.height, "n_inner": info.n_inner, "n_leaf": info.n_leaf,
                                "smem_levels": info.smem_levels},
                       "bulk_load_ms": round(bulk_ms, 1)},
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "stages_ms_per_step": {k: round(v[1] / max(v[0], 1), 4) for k, v in stages.items()},
            "roofline": roofline,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "cpu_baseline_port": cpu_port,
        }
        line.update(extras)
        if "plain" in extras:
            line["vs_plain"] = round(value / extras["plain"]["value"], 3)
        print(json.dumps(line), flush=True)
    tree.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
