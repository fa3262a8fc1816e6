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
* range queries: start uniform, length uniform in [lo, hi].

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
