// Batched point search: narrowed thread groups (NTG) of W lanes descend the
// breadth-first tree, two compare stages per node, top levels in shared
// memory staged by a bulk TMA copy.
//
// Reference: full_multi_prefix_sort_8thread_kernel
// (open-harmonia/src/full-multi-prefix-sort-8thread.cu:95-263) and the CFB
// kernel multi_prefix_sort_kernel (open-harmonia/regular_bpt/prefix-sort.cu:98-250).
// Same algorithm per node: compare the query with the node's index (every
// 8th key), then with the chosen 8-key slice; child = number of keys <= q;
// next node = prefix[node] + child; at the leaf an equality test.  What
// changes for sm_100a:
//   * one group of W lanes (W = 1..32) per query; each lane fetches 16 B
//     (two keys) per load, so W=4 reads one 64-B index or slice in one step;
//     group counts are summed with __shfl_xor_sync (no shared-memory flag
//     scan, no __syncthreads per level; the reference uses four);
//   * each group keeps Q queries in flight (the reference's GPU_SWP_SIZE
//     runs them one after another);
//   * the first levels (a BFS prefix of the rows plus their prefix entries)
//     are copied once per CTA into shared memory with cp.async.bulk
//     (1-D TMA, mbarrier completion, no multicast) and reused by a
//     persistent grid; the reference keeps them in __constant__ memory
//     (open-harmonia/src/ppi-bpt-v14-1.cu:128,290), which serialises
//     divergent indices;
//   * the leaf test compares all slots of the leaf row at once and only the
//     matching lane loads the value, which it writes straight to the output
//     (the reference returns a (leaf, slot) pair decoded on the host,
//     open-harmonia/src/full-multi-prefix-sort-8thread.cu:34-39,454-476).
#include "hm_internal.cuh"
#include "async_copy.cuh"

#include <cstdio>
#include <mutex>

namespace hm {

namespace {

constexpr int kThreads = 256;

struct Args {
  DevTree t;
  const int64_t *q;
  int64_t *out;
  const int32_t *pos;
  int64_t n;
  // multi-batch mode (nb > 0)
  const hm_batch *batches;
  const int64_t *tile_start;  // nb+1 prefix of tiles per batch
  int nb;
  int64_t total_tiles;
  unsigned long long *tile_counter;
  unsigned *err;
};

// L2 cache policies (createpolicy): inner rows are re-read by every query and
// should stay in L2; leaf rows are touched about once per batch.
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// 16-B read-only global load with an L2 cache policy.
__device__ __forceinline__ longlong2 ldg2(const int64_t *p, uint64_t pol) {
  longlong2 r;
  asm volatile("ld.global.nc.L2::cache_hint.v2.s64 {%0, %1}, [%2], %3;"
               : "=l"(r.x), "=l"(r.y)
               : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ int64_t ldg1(const int64_t *p, uint64_t pol) {
  int64_t r;
  asm volatile("ld.global.nc.L2::cache_hint.s64 %0, [%1], %2;" : "=l"(r) : "l"(p), "l"(pol));
  return r;
}
__device__ __forceinline__ int32_t ldg1(const int32_t *p, uint64_t pol) {
  int32_t r;
  asm volatile("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(r) : "l"(p), "l"(pol));
  return r;
}

template <bool SMEM>
__device__ __forceinline__ longlong2 load2(const int64_t *p, uint64_t pol) {
  if constexpr (SMEM) {
    return *reinterpret_cast<const longlong2 *>(p);
  } else {
    return ldg2(p, pol);
  }
}

// Sum over the W lanes of an aligned group.
template <int W>
__device__ __forceinline__ int group_sum(int v) {
#pragma unroll
  for (int o = W / 2; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Number of keys <= q among LEN sorted keys at p, counted by the W lanes of a
// group (lane `sub` reads vectors sub, sub+W, ...).
template <int W, int LEN, bool SMEM>
__device__ __forceinline__ int count_le(const int64_t *p, int64_t q, int sub, uint64_t pol) {
  constexpr int NV = LEN / 2;
  constexpr int VPL = (NV + W - 1) / W;
  longlong2 v[VPL];
#pragma unroll
  for (int i = 0; i < VPL; i++) {
    int vi = sub + i * W;
    if (NV % W == 0 || vi < NV)
      v[i] = load2<SMEM>(p + 2 * vi, pol);
    else
      v[i] = make_longlong2(kMaxKey, kMaxKey);
  }
  int c = 0;
#pragma unroll
  for (int i = 0; i < VPL; i++) c += (v[i].x <= q) + (v[i].y <= q);
  return group_sum<W>(c);
}

// Child position in an inner row: index stage then slice stage.
template <int W, int F, bool SMEM>
__device__ __forceinline__ int rank_inner(const int64_t *row, int64_t q, int sub, uint64_t pol) {
  int k = count_le<W, F / 8, SMEM>(row, q, sub, pol);
  k = min(k, F / 8 - 1);
  return 8 * k + count_le<W, 8, SMEM>(row + F / 8 + 8 * k, q, sub, pol);
}

// Equality test over LEN keys at p; returns the matching slot or -1 in the
// lane that holds it (other lanes return -1).
template <int W, int LEN>
__device__ __forceinline__ int match_slot(const int64_t *p, int64_t q, int sub, uint64_t pol) {
  constexpr int NV = LEN / 2;
  constexpr int VPL = (NV + W - 1) / W;
  longlong2 v[VPL];
#pragma unroll
  for (int i = 0; i < VPL; i++) {
    int vi = sub + i * W;
    if (NV % W == 0 || vi < NV)
      v[i] = ldg2(p + 2 * vi, pol);
    else
      v[i] = make_longlong2(kMaxKey, kMaxKey);
  }
  int slot = -1;
#pragma unroll
  for (int i = 0; i < VPL; i++) {
    int vi = sub + i * W;
    if (v[i].x == q) slot = 2 * vi;
    if (v[i].y == q) slot = 2 * vi + 1;
  }
  return slot;
}

// Equality test over a 16-key leaf record that also loads, in the same round
// trip, the values beside the lane's keys: the matching lane returns the
// value (others HM_NOT_FOUND), so no dependent load follows the compare.  It
// reads the whole 256-B record instead of 128 B of keys and one 32-B value
// sector, one DRAM round trip fewer.  Measured on 2^24 unsorted queries at
// 2^26 keys: 18.2 Gq/s at one query per group against 15.4 for the best
// setting without it; at two queries per group the extra registers cost more
// than the round trip saves (12.6), so only Q = 1 uses it.
#ifndef HM_LEAF_VALUES_WITH_KEYS
#define HM_LEAF_VALUES_WITH_KEYS 1
#endif
template <int W, int LC>
__device__ __forceinline__ int64_t match_value(const int64_t *p, int64_t q, int sub, uint64_t pol, bool *hit) {
  constexpr int NV = LC / 2;
  constexpr int VPL = (NV + W - 1) / W;
  longlong2 v[VPL], w[VPL];
#pragma unroll
  for (int i = 0; i < VPL; i++) {
    const int vi = sub + i * W;
    if (NV % W == 0 || vi < NV) {
      v[i] = ldg2(p + 2 * vi, pol);
      w[i] = ldg2(p + LC + 2 * vi, pol);
    } else {
      v[i] = make_longlong2(kMaxKey, kMaxKey);
      w[i] = make_longlong2(HM_NOT_FOUND, HM_NOT_FOUND);
    }
  }
  int64_t r = HM_NOT_FOUND;
  bool h = false;
#pragma unroll
  for (int i = 0; i < VPL; i++) {
    if (v[i].x == q) { r = w[i].x; h = true; }
    if (v[i].y == q) { r = w[i].y; h = true; }
  }
  *hit = h;
  return r;
}

// Processes one tile of up to G*Q queries: q_base[i] for i in [i0, i0+G*Q) ∩ [0, n).
template <int W, int F, int LC, int Q>
__device__ __forceinline__ void search_tile(const DevTree &t, const int64_t *srows,
                                            const int32_t *spref, const int64_t *__restrict__ qp,
                                            int64_t *__restrict__ outp,
                                            const int32_t *__restrict__ posp, int64_t n,
                                            int64_t i0) {
  constexpr int G = kThreads / W;   // groups per CTA
  constexpr int ROW = F / 8 + F;    // inner row words
  constexpr int LI = LC >= 32 ? LC / 8 : 0;
  constexpr int LROW = LI + 2 * LC;
  const int gid = threadIdx.x / W, sub = threadIdx.x % W;
  const int lane = threadIdx.x & 31;
  const uint64_t pol_inner = t.cache_hints == 1 ? policy_evict_last() : policy_evict_normal();
  const uint64_t pol_leaf = t.cache_hints == 1 ? policy_evict_first() : policy_evict_normal();

  int64_t key[Q], nav[Q];
  int64_t idx[Q];
  int32_t node[Q];
#pragma unroll
  for (int j = 0; j < Q; j++) {
    idx[j] = i0 + (int64_t)j * G + gid;
    key[j] = idx[j] < n ? __ldg(qp + idx[j]) : 0;
    nav[j] = key[j] == kMaxKey ? kMaxKey - 1 : key[j];  // never rank the sentinel
    node[j] = 0;
  }

  for (int lvl = 0; lvl < t.height; lvl++) {
    if (lvl < t.smem_levels) {
      int c[Q];
#pragma unroll
      for (int j = 0; j < Q; j++)
        c[j] = rank_inner<W, F, true>(srows + (int64_t)node[j] * ROW, nav[j], sub, pol_inner);
#pragma unroll
      for (int j = 0; j < Q; j++) node[j] = spref[node[j]] + c[j];
    } else {
      int32_t base[Q];
      int k[Q];
#pragma unroll
      for (int j = 0; j < Q; j++) {
        const int64_t *row = t.inner + (int64_t)node[j] * ROW;
        base[j] = ldg1(t.prefix + node[j], pol_inner);
        k[j] = min(count_le<W, F / 8, false>(row, nav[j], sub, pol_inner), F / 8 - 1);
      }
#pragma unroll
      for (int j = 0; j < Q; j++) {
        const int64_t *row = t.inner + (int64_t)node[j] * ROW;
        node[j] = base[j] + 8 * k[j] + count_le<W, 8, false>(row + F / 8 + 8 * k[j], nav[j], sub, pol_inner);
      }
    }
  }

  if constexpr (LI == 0 && Q == 1 && HM_LEAF_VALUES_WITH_KEYS) {
    int64_t val[Q];
    bool found[Q];
#pragma unroll
    for (int j = 0; j < Q; j++) {
      const int64_t *row = t.leaf_rows + (int64_t)(node[j] - t.n_inner) * LROW;
      val[j] = match_value<W, LC>(row, key[j], sub, pol_leaf, &found[j]);
      if (key[j] == kMaxKey) found[j] = false;
    }
    const unsigned gm = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(W - 1)));
#pragma unroll
    for (int j = 0; j < Q; j++) {
      const unsigned hit = __ballot_sync(0xffffffffu, found[j]) & gm;
      const int writer = hit ? (__ffs(hit) - 1) : (lane & ~(W - 1));
      if (lane == writer && idx[j] < n) {
        const int64_t o = posp ? (int64_t)__ldg(posp + idx[j]) : idx[j];
        outp[o] = found[j] ? val[j] : (int64_t)HM_NOT_FOUND;
      }
    }
    return;
  }

  int slot[Q];
  int32_t leaf[Q];
#pragma unroll
  for (int j = 0; j < Q; j++) {
    leaf[j] = node[j] - t.n_inner;
    const int64_t *row = t.leaf_rows + (int64_t)leaf[j] * LROW;
    if constexpr (LI == 0) {
      slot[j] = match_slot<W, LC>(row, key[j], sub, pol_leaf);
    } else {
      int kk = min(count_le<W, LI, false>(row, nav[j], sub, pol_leaf), LI - 1);
      int s8 = match_slot<W, 8>(row + LI + 8 * kk, key[j], sub, pol_leaf);
      slot[j] = s8 >= 0 ? 8 * kk + s8 : -1;
    }
    if (key[j] == kMaxKey) slot[j] = -1;
  }

  const unsigned gmask = (W == 32) ? 0xffffffffu : (((1u << W) - 1u) << (lane & ~(W - 1)));
#pragma unroll
  for (int j = 0; j < Q; j++) {
    unsigned hit = __ballot_sync(0xffffffffu, slot[j] >= 0) & gmask;
    int writer = hit ? (__ffs(hit) - 1) : (lane & ~(W - 1));
    if (lane == writer && idx[j] < n) {
      int64_t v = slot[j] >= 0 ? ldg1(t.leaf_rows + (int64_t)leaf[j] * LROW + LI + LC + slot[j], pol_leaf)
                               : (int64_t)HM_NOT_FOUND;
      int64_t o = posp ? (int64_t)__ldg(posp + idx[j]) : idx[j];
      outp[o] = v;
    }
  }
}

#ifndef HM_SEARCH_MINB
#define HM_SEARCH_MINB 6  // resident CTAs per SM the register budget must allow (measured: 6 beats 1 and 8)
#endif

template <int W, int F, int LC, int Q>
__global__ void __launch_bounds__(kThreads, (Q <= 2 ? HM_SEARCH_MINB : 1)) search_kernel(Args a) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int ROW = F / 8 + F;
  constexpr int TILE = (kThreads / W) * Q;
  const DevTree &t = a.t;
  const unsigned rows_bytes = (unsigned)t.smem_nodes * ROW * 8u;
  const unsigned pref_bytes = ((unsigned)t.smem_nodes * 4u + 15u) & ~15u;
  int64_t *srows = reinterpret_cast<int64_t *>(smem);
  int32_t *spref = reinterpret_cast<int32_t *>(smem + rows_bytes);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + rows_bytes + pref_bytes);
  __shared__ int64_t claimed;

  if (t.smem_nodes > 0) {
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
      mbar_expect_tx(bar, rows_bytes + pref_bytes);
      bulk_g2s(srows, t.inner, rows_bytes, bar);
      bulk_g2s(spref, t.prefix, pref_bytes, bar);
    }
    __syncthreads();
    if (!mbar_wait_bounded(bar, 0, t.wait_polls)) {
      if (threadIdx.x == 0) atomicOr(a.err, kErrTimeout);
      mbar_wait_bounded(bar);  // let the copy land (default bound) before the CTA exits
      return;
    }
  }

  if (a.nb == 0) {
    const int64_t tiles = (a.n + TILE - 1) / TILE;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x)
      search_tile<W, F, LC, Q>(t, srows, spref, a.q, a.out, a.pos, a.n, tile * TILE);
    return;
  }
  // Multi-batch: tiles handed out by a global counter, batch found by binary search.
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) claimed = (int64_t)atomicAdd(a.tile_counter, 1ull);
    __syncthreads();
    int64_t tile = claimed;
    if (tile >= a.total_tiles) return;
    int lo = 0, hi = a.nb - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (__ldg(a.tile_start + mid) <= tile) lo = mid; else hi = mid - 1;
    }
    const hm_batch b = a.batches[lo];
    int64_t local = tile - __ldg(a.tile_start + lo);
    search_tile<W, F, LC, Q>(t, srows, spref, b.q, b.out, nullptr, b.n, local * TILE);
  }
}

using KernelFn = void (*)(Args);

template <int W, int F, int LC>
KernelFn pick_q(int qpg) {
  switch (qpg) {
    case 1: return search_kernel<W, F, LC, 1>;
    case 2: return search_kernel<W, F, LC, 2>;
    case 4: return search_kernel<W, F, LC, 4>;
    default: return nullptr;
  }
}

template <int W, int F>
KernelFn pick_lc(int lc, int qpg) {
  switch (lc) {
    case 16: return pick_q<W, F, 16>(qpg);
    case 64: return pick_q<W, F, 64>(qpg);
    default: return nullptr;
  }
}

template <int W>
KernelFn pick_f(int f, int lc, int qpg) {
  switch (f) {
    case 64: return pick_lc<W, 64>(lc, qpg);
    case 128: return pick_lc<W, 128>(lc, qpg);
    default: return nullptr;
  }
}

KernelFn pick_kernel(int w, int f, int lc, int qpg) {
  switch (w) {
    case 1: return pick_f<1>(f, lc, qpg);
    case 2: return pick_f<2>(f, lc, qpg);
    case 4: return pick_f<4>(f, lc, qpg);
    case 8: return pick_f<8>(f, lc, qpg);
    case 16: return pick_f<16>(f, lc, qpg);
    case 32: return pick_f<32>(f, lc, qpg);
    default: return nullptr;
  }
}

struct GridCache {
  KernelFn fn = nullptr;
  size_t smem = 0;
  int device = 0;
  int blocks_per_sm = 0;
};

// Resident CTAs per SM of a search kernel variant, looked up once per process
// (any thread) and device: later launches make no occupancy query.
int grid_for(const hm_tree *t, KernelFn fn, size_t smem, int *blocks) {
  static std::mutex mu;
  static GridCache cache[64];
  std::lock_guard<std::mutex> lk(mu);
  for (auto &c : cache)
    if (c.fn == fn && c.smem == smem && c.device == t->device) {
      *blocks = c.blocks_per_sm * t->num_sms;
      return HM_OK;
    }
  if (smem > 48 * 1024) {
    int rc = opt_in_smem((const void *)fn, (int)smem);
    if (rc) return rc;
  }
  int per = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kThreads, smem);
  if (e != cudaSuccess) return cuda_err(e);
  if (per < 1) return HM_EINVAL;
  for (auto &c : cache)
    if (c.fn == nullptr) {
      c.fn = fn;
      c.device = t->device;
      c.smem = smem;
      c.blocks_per_sm = per;
      break;
    }
  *blocks = per * t->num_sms;
  return HM_OK;
}

}  // namespace

size_t search_smem_bytes(const hm_tree *t) {
  size_t rows = (size_t)t->smem_nodes * t->inner_row * 8;
  size_t pref = ((size_t)t->smem_nodes * 4 + 15) & ~(size_t)15;
  return rows + pref + 16;
}

int search_tile_queries(int group_width, int qpg) { return (kThreads / group_width) * qpg; }

int launch_search_warm(const hm_tree *t, int group_width, int qpg) {
  KernelFn fn = pick_kernel(group_width, t->cfg.fanout, t->cfg.leaf_cap, qpg);
  if (!fn) return HM_EINVAL;
  int blocks = 0;
  return grid_for(t, fn, search_smem_bytes(t), &blocks);
}

int launch_search(const hm_tree *t, const SearchLaunch &l, int group_width, int qpg,
                  cudaStream_t s) {
  if (l.n <= 0) return HM_OK;
  KernelFn fn = pick_kernel(group_width, t->cfg.fanout, t->cfg.leaf_cap, qpg);
  if (!fn) return HM_EINVAL;
  size_t smem = search_smem_bytes(t);
  int blocks = 0;
  int rc = grid_for(t, fn, smem, &blocks);
  if (rc) return rc;
  int64_t tiles = (l.n + search_tile_queries(group_width, qpg) - 1) / search_tile_queries(group_width, qpg);
  if (tiles < blocks) blocks = (int)tiles;
  Args a{};
  a.t = t->view();
  a.q = l.q;
  a.out = l.out;
  a.pos = l.pos;
  a.n = l.n;
  a.nb = 0;
  a.err = t->d_err;
  fn<<<blocks, kThreads, smem, s>>>(a);
  note_launch();
  return cuda_err(cudaGetLastError());
}

int launch_search_batches(const hm_tree *t, const hm_batch *d_batches, const int64_t *d_tile_start,
                          int nb, int64_t total_tiles, int group_width, int qpg, cudaStream_t s) {
  if (nb <= 0 || total_tiles <= 0) return HM_OK;
  KernelFn fn = pick_kernel(group_width, t->cfg.fanout, t->cfg.leaf_cap, qpg);
  if (!fn) return HM_EINVAL;
  size_t smem = search_smem_bytes(t);
  int blocks = 0;
  int rc = grid_for(t, fn, smem, &blocks);
  if (rc) return rc;
  if (total_tiles < blocks) blocks = (int)total_tiles;
  Args a{};
  a.t = t->view();
  a.nb = nb;
  a.batches = d_batches;
  a.tile_start = d_tile_start;
  a.total_tiles = total_tiles;
  a.tile_counter = reinterpret_cast<unsigned long long *>(const_cast<int64_t *>(d_tile_start + nb + 1));
  a.err = t->d_err;
  fn<<<blocks, kThreads, smem, s>>>(a);
  note_launch();
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
