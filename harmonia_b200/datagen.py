"""Seeded synthetic workloads for the batched B+tree path.

The reference ships no datasets (its generator, open-harmonia/script/
generate-data/util.py:45-130, is unseeded numpy), so every workload here is
defined by a seed and reproduced exactly on any machine:

* keys: ``n`` distinct int64 in [0, 2^63 - 1): a 63-bit bijection of a seeded
  counter, so distinctness needs no dedup pass.  ``Max_Key`` (2^63 - 1, the
  reference's empty-slot sentinel, open-harmonia/src/bpt.h:26) is never
  produced.
* values: ``splitmix64(key) >> 1``, non-negative because the reference treats a
  negative value as "absent" (open-harmonia/src/bpt.cpp:374).
* point queries: a hit fraction sampled from the loaded keys, the rest uniform
  63-bit keys (misses with probability 1 - n/2^63).
* Zipf(theta) queries over key rank (rank 0 = smallest key is hottest), drawn
  with the closed-form sampler of Gray et al., "Quickly generating
  billion-record synthetic databases" (SIGMOD'94).
* range queries: start uniform, length uniform in [lo, hi]; inclusive ranges:
  start uniform, end = start + about L keys' spacing.

splitmix64 is the generator of Steele, Lea and Flood (OOPSLA'14).
"""
from __future__ import annotations

import numpy as np

MAX_KEY = np.int64(2**63 - 1)
_M63 = np.uint64(2**63 - 1)
_GOLD = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser of (x + golden gamma), elementwise on uint64."""
    with np.errstate(over="ignore"):
        z = np.asarray(x, dtype=np.uint64) + _GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _perm63(x: np.ndarray) -> np.ndarray:
    """A bijection of [0, 2^63): odd multiplies and xor-shifts mod 2^63."""
    with np.errstate(over="ignore"):
        x = np.asarray(x, dtype=np.uint64) & _M63
        x = (x * np.uint64(0x5851F42D4C957F2D)) & _M63
        x ^= x >> np.uint64(29)
        x = (x * np.uint64(0x14057B7EF767814F)) & _M63
        x ^= x >> np.uint64(31)
        x = (x * np.uint64(0x2545F4914F6CDD1D)) & _M63
        x ^= x >> np.uint64(27)
        return x


def gen_keys(n: int, seed: int = 1) -> np.ndarray:
    """n distinct keys in [0, 2^63 - 1), in generation (unsorted) order."""
    base = splitmix64(np.array([seed], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        ctr = (np.arange(n, dtype=np.uint64) + base) & _M63
    k = _perm63(ctr)
    bad = k == np.uint64(2**63 - 1)
    if bad.any():  # the single preimage of Max_Key: take the next counter value
        with np.errstate(over="ignore"):
            k[bad] = _perm63(np.array([(int(base) + n) & (2**63 - 1)], dtype=np.uint64))
    return k.astype(np.int64)


def values_for(keys: np.ndarray) -> np.ndarray:
    """Value of each key: splitmix64(key) >> 1 (always >= 0)."""
    return (splitmix64(keys.astype(np.uint64)) >> np.uint64(1)).astype(np.int64)


def gen_point_queries(keys: np.ndarray, m: int, hit_frac: float, seed: int = 2) -> np.ndarray:
    """m queries: a hit_frac share drawn from ``keys``, the rest uniform."""
    r = splitmix64(np.arange(m, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40))
    hit = (r % np.uint64(1_000_000)) < np.uint64(int(round(hit_frac * 1_000_000)))
    n = len(keys)
    q = (splitmix64(r ^ np.uint64(0x5BD1E995)) >> np.uint64(1)).astype(np.int64)
    q[q == MAX_KEY] = 0
    if n:
        idx = (splitmix64(r) % np.uint64(n)).astype(np.int64)
        q[hit] = keys[idx[hit]]
    return q


def _zeta(n: int, theta: float) -> float:
    acc = 0.0
    step = 1 << 22
    for s in range(1, n + 1, step):
        i = np.arange(s, min(n + 1, s + step), dtype=np.float64)
        acc += float(np.sum(i ** (-theta)))
    return acc


def zipf_ranks(n: int, m: int, theta: float = 0.99, seed: int = 3) -> np.ndarray:
    """m ranks in [0, n) with P(rank = i) ~ 1 / (i+1)^theta (Gray et al.)."""
    zetan = _zeta(n, theta)
    zeta2 = 1.0 + 2.0 ** (-theta)
    alpha = 1.0 / (1.0 - theta)
    eta = (1.0 - (2.0 / n) ** (1.0 - theta)) / (1.0 - zeta2 / zetan)
    u = (splitmix64(np.arange(m, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40))
         >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    uz = u * zetan
    r = (n * np.power(eta * u - eta + 1.0, alpha)).astype(np.int64)
    r = np.where(uz < 1.0, 0, np.where(uz < zeta2, 1, r))
    return np.clip(r, 0, n - 1)


def gen_zipf_queries(sorted_keys: np.ndarray, m: int, theta: float = 0.99, seed: int = 3) -> np.ndarray:
    """m point queries, Zipf(theta) over the rank of the loaded keys."""
    return sorted_keys[zipf_ranks(len(sorted_keys), m, theta, seed)]


def gen_ranges(m: int, lo: int, hi: int, seed: int = 4):
    """m range queries: start uniform in [0, 2^63 - 1), length uniform in [lo, hi]."""
    r = splitmix64(np.arange(m, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40))
    start = (splitmix64(r ^ np.uint64(0x27D4EB2F165667C5)) >> np.uint64(1)).astype(np.int64)
    start[start == MAX_KEY] = 0
    length = (lo + (r % np.uint64(hi - lo + 1)).astype(np.int64)).astype(np.int32)
    return start, length


def gen_range_pairs(m: int, n_keys: int, lo: int, hi: int, seed: int = 4):
    """m inclusive ranges (start, end) over a tree of about n_keys uniform
    keys: start as gen_ranges, end = start + L * gap - 1 with L uniform in
    [lo, hi] and gap = 2^63 / n_keys the mean key spacing, so a range holds
    about L keys.  Every 64th range is empty (end = start - 1).  end stays
    below Max_Key (the reference's descent asserts for that key)."""
    start, length = gen_ranges(m, lo, hi, seed)
    gap = np.uint64((2**63) // max(n_keys, 1))
    with np.errstate(over="ignore"):
        e = start.astype(np.uint64) + length.astype(np.uint64) * gap - np.uint64(1)
    e = np.minimum(e, np.uint64(2**63 - 2)).astype(np.int64)
    empty = (np.arange(m) % 64) == 63
    e[empty] = start[empty] - 1
    return start, e


def _first_unique(a: np.ndarray) -> np.ndarray:
    """Distinct elements of a in order of first appearance."""
    _, idx = np.unique(a, return_index=True)
    return a[np.sort(idx)]


def gen_upserts(keys: np.ndarray, m: int, new_frac: float = 0.5, seed: int = 5):
    """m distinct upsert keys: a new_frac share of new keys, the rest existing.

    Existing keys carry value key-1 and new keys splitmix64(key)>>1, so the
    product's supplied-value upsert and the reference's update rule (existing
    key -> key-1, open-harmonia/src/bpt-ppi-update-batch.cpp:47) give the same
    contents.  Keys are distinct within the batch (the reference inserts a
    repeated new key twice, open-harmonia/src/bpt-ppi-update-batch.cpp:59-66).
    """
    n = len(keys)
    n_new = int(round(m * new_frac))
    n_old = m - n_new
    r = splitmix64(np.arange(4 * m + 16, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40))
    old = _first_unique(keys[(r % np.uint64(max(n, 1))).astype(np.int64)])[:n_old] if n else keys[:0]
    kset = set(keys.tolist()) if n <= (1 << 22) else None
    cand = (splitmix64(r ^ np.uint64(0x1B873593)) >> np.uint64(1)).astype(np.int64)
    cand = cand[cand != MAX_KEY]
    if kset is not None:
        cand = np.array([c for c in cand.tolist() if c not in kset], dtype=np.int64)
    else:
        cand = cand[~np.isin(cand, keys)]
    new = _first_unique(cand)[:n_new]
    bk = np.concatenate([old, new])
    order = np.argsort(splitmix64(bk.astype(np.uint64) ^ np.uint64(seed)))
    bk = bk[order]
    is_old = np.isin(bk, old)
    bv = np.where(is_old, bk - 1, values_for(bk))
    return bk.astype(np.int64), bv.astype(np.int64)


def _unit(r: np.ndarray) -> np.ndarray:
    """Uniform doubles in [0, 1) from uint64 draws (top 53 bits)."""
    return (r >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def gen_uneven_batches(keys: np.ndarray, sorted_keys: np.ndarray, nb: int = 512, seed: int = 7,
                       lo: int = 1024, hi: int = 4 << 20, pool_n: int = 1 << 24):
    """The uneven multi-batch workload: nb batches with sizes log-uniform in
    [lo, hi]; even batches draw from a pool of uniform point queries (90%
    hits), odd ones from a pool of Zipf(0.99) queries over key rank; batch b is
    a wrapped run of its pool starting at a seeded offset.  Returns (sizes,
    queries): queries is one array holding the batches back to back."""
    r = splitmix64(np.arange(nb, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40))
    sizes = np.exp(np.log(lo) + _unit(r) * (np.log(hi) - np.log(lo))).astype(np.int64)
    pools = (gen_point_queries(keys, pool_n, 0.9, seed + 1), gen_zipf_queries(sorted_keys, pool_n, 0.99, seed + 2))
    out = np.empty(int(sizes.sum()), np.int64)
    o = 0
    for b in range(nb):
        m = int(sizes[b])
        start = int(r[b] % np.uint64(pool_n))
        idx = (np.arange(m, dtype=np.int64) + start) % pool_n
        out[o:o + m] = pools[b % 2][idx]
        o += m
    return sizes, out


def gen_serving_stream(keys: np.ndarray, count: int, seed: int = 11, lo: int = 64, hi: int = 1 << 20):
    """A seeded serving request stream over a tree holding ``keys``: sizes
    log-uniform in [lo, hi]; 90% point searches (80% hits), 5% range requests
    (size/64 ranges, length uniform in [1, 128]), 5% upserts (size/16 keys,
    2..64: half new keys with value splitmix64(key)>>1, half existing keys with
    value key-1, the reference's update rule).  Returns a list of
    ("search", q) / ("range", start, length) / ("upsert", keys, values)."""
    n = len(keys)
    r = splitmix64(np.arange(3 * count, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40)).reshape(count, 3)
    kind = _unit(r[:, 0])
    sizes = np.exp(np.log(lo) + _unit(r[:, 1]) * (np.log(hi) - np.log(lo))).astype(np.int64)
    fresh = gen_keys(1 << 20, seed + 100)
    fresh = fresh[~np.isin(fresh, keys)]
    at = 0
    out = []
    for i in range(count):
        m = int(sizes[i])
        sub = seed * 1_000_003 + i
        if kind[i] < 0.90:
            out.append(("search", gen_point_queries(keys, m, 0.8, sub)))
        elif kind[i] < 0.95:
            st, ln = gen_ranges(max(1, m // 64), 1, 128, sub)
            out.append(("range", st, ln))
        else:
            k = max(2, min(m // 16, 64))
            nk = fresh[at:at + k // 2]
            at += k // 2
            ek = keys[(splitmix64(np.arange(k - k // 2, dtype=np.uint64) + r[i, 2]) % np.uint64(n)).astype(np.int64)]
            out.append(("upsert", np.concatenate([nk, ek]), np.concatenate([values_for(nk), ek - 1])))
    return out

