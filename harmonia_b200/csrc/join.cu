// Bucket join: point search for a pre-sorted batch that is large relative to
// the tree.
//
// After the query pre-sort (partition.cu) the queries of one bucket form a
// contiguous run and the bucket's keys lie in a contiguous range of leaves.
// Instead of one descent per query (search.cu), a CTA takes a run of one
// bucket, copies the bucket's leaf records (keys and values, 256 B per
// 16-key leaf) from HBM into shared memory in order (2-D tiled TMA loads for
// 16-key leaves, per-thread cp.async otherwise), and
// answers every query of the run from shared memory: a binary search over the
// leaves' first keys (or, for batches of many queries per bucket, a 64-slot
// directory of them built once per run) picks the leaf, a binary search of
// its keys the slot.  The leaf range of each bucket comes from one descent per
// bucket boundary (a separate kernel, one thread per boundary; kept per tree
// shape between calls).  Leaves are read once per run
// and sequentially, so the DRAM traffic of a batch with more queries than
// leaves falls from a random 160 B per query to the size of the touched leaf
// region.  A bucket whose leaves do not fit shared memory (very skewed keys)
// falls back to a scalar descent per query.  For batches up to 2^25 queries
// the results go straight to the queries' positions after the first pre-sort
// pass (recorded by the second), so only the first pass is undone.
//
// The per-query semantics are the reference's (child = number of separators
// <= key, open-harmonia/src/avx.cpp:2-54; equality in the leaf,
// open-harmonia/src/bpt.h:252-274): a key routed to leaf j lies between
// leaf j's first key and leaf j+1's first key, so the largest leaf of the
// range whose first key is <= q is the leaf the descent would reach.
#include "hm_internal.cuh"
#include "async_copy.cuh"

#include <cuda.h>  // CUtensorMap and its enums; the encoder is fetched through the runtime

#include <mutex>

#include <algorithm>

namespace hm {

namespace {

constexpr int kThreads = 256;
#ifndef HM_JOIN_PER_THREAD
#define HM_JOIN_PER_THREAD 1  // queries a thread answers per step (measured: 1 beats 2, 4 and 8)
#endif
constexpr int kPerThread = HM_JOIN_PER_THREAD;
constexpr int kRun = kThreads * kPerThread;  // queries a CTA answers per step
#ifndef HM_JOIN_ITEM_RUNS
#define HM_JOIN_ITEM_RUNS 64
#endif
// Steps of one work item: a bucket with more queries is cut into items of
// kItemMax (hot buckets of a skewed batch); each item stages its bucket's
// leaves once, so larger items re-read a hot bucket's leaves less often
// (measured on the 217 M-query batch set, half Zipf: join 1.60 ms with
// 4096-query items, 1.48 with 8192, 1.44 with 16384).
constexpr int kItemRuns = HM_JOIN_ITEM_RUNS;
constexpr int kItemMax = kRun * kItemRuns;  // queries per work item, at most
static_assert(kItemMax < 65536, "an item's query count is kept in 16 bits");
#ifndef HM_JOIN_STAGES
#define HM_JOIN_STAGES 2  // shared-memory ring of the join kernel
#endif
#ifndef HM_JOIN_MINB
#define HM_JOIN_MINB 4  // resident join CTAs per SM the register budget allows
#endif
#ifndef HM_JOIN_SLACK
#define HM_JOIN_SLACK 4  // a stage holds mean + mean / HM_JOIN_SLACK + 8 leaves
#endif
constexpr int kStages = HM_JOIN_STAGES;
constexpr int kStageMax = (216 / kStages) * 1024;  // shared memory of one stage, at most

#ifndef HM_JOIN_MAX_BITS
#define HM_JOIN_MAX_BITS 16
#endif
static_assert(HM_JOIN_MAX_BITS <= 16, "a bucket number is kept in 16 bits");

// A work item: at most kItemMax queries of one bucket, grouped queries
// [qa, qa + len), and the bucket's leaves [l0, l0 + nl); the leaves are
// staged once for all of them.
struct __align__(16) Item {
  int32_t qa, l0, b;  // first query, first leaf, bucket
  uint32_t len_nl;    // queries (at most kItemMax) << 16 | leaves (capped at 65535)
  __host__ __device__ int len() const { return (int)(len_nl >> 16); }
  __host__ __device__ int nl() const { return (int)(len_nl & 0xffffu); }
};

// Per bucket b in [0, nb]: cnt[b] = its work items (0 for b = nb) and, with
// want_leafb, leafb[b] = leaf holding the smallest key of bucket b (bucket
// b's keys lie in leaves [leafb[b], leafb[b+1]]).  leafb depends only on the
// inner nodes, the key range and the bucket bits, so the launcher keeps it
// per tree shape and skips the descents while that holds.
__global__ void bucket_prep_kernel(DevTree t, int f, int64_t lo, int shift, int nb,
                                   const int64_t *__restrict__ bstart, int32_t *__restrict__ leafb,
                                   int32_t *__restrict__ cnt, bool want_leafb) {
  pdl_enter();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nb; b += gridDim.x * blockDim.x) {
    if (cnt) cnt[b] = b < nb ? (int32_t)((bstart[b + 1] - bstart[b] + kItemMax - 1) / kItemMax) : 0;
    if (!want_leafb) continue;
    if (b == 0) {
      leafb[0] = 0;
      continue;
    }
    if (b == nb) {
      leafb[nb] = t.n_leaf - 1;
      continue;
    }
    const uint64_t off = (uint64_t)b << shift;
    if (off >= (uint64_t)kMaxKey - (uint64_t)lo) {  // boundary at or past Max_Key: no key above it
      leafb[b] = t.n_leaf - 1;
      continue;
    }
    leafb[b] = descend_leaf(t, f, (int64_t)((uint64_t)lo + off));
  }
}

// Bucket b's items start at first[b] (exclusive scan of cnt).
__global__ void expand_items_kernel(int nb, const int64_t *__restrict__ bstart, const int32_t *__restrict__ leafb,
                                    const int32_t *__restrict__ cnt, const int64_t *__restrict__ first,
                                    Item *__restrict__ items) {
  pdl_enter();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int c = cnt[b];
    if (c == 0) continue;
    const int64_t s = bstart[b], e = bstart[b + 1];
    const int32_t l0 = leafb[b], nl = leafb[b + 1] - l0 + 1;
    int64_t o = first[b];
    for (int r = 0; r < c; r++) {
      Item it;
      it.qa = (int32_t)(s + (int64_t)r * kItemMax);
      const int32_t len = (int32_t)min((int64_t)kItemMax, e - (s + (int64_t)r * kItemMax));
      it.l0 = l0;
      it.b = b;
      it.len_nl = (uint32_t)len << 16 | (uint32_t)min(nl, 65535);  // a capped count is never staged
      items[o + r] = it;
    }
  }
}

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Words of one leaf in a stage: its keys at a stride of LC + 1 (leaf m's key s
// at m * (LC + 1) + s, so lanes reading different leaves fall in different
// banks), then, after all keys, its values densely (m * LC + s).
template <int LC>
__host__ __device__ constexpr int stage_leaf_bytes() {
  return (2 * LC + 1) * 8;
}

template <int LC>
struct Stage {
  int64_t *kp, *vp;
  __device__ Stage(int64_t *base, int ml) : kp(base), vp(base + ml * (LC + 1)) {}
  __device__ __forceinline__ int64_t first(int m) const { return kp[m * (LC + 1)]; }
  __device__ __forceinline__ int64_t key(int m, int c) const { return kp[m * (LC + 1) + c]; }
  __device__ __forceinline__ int64_t val(int m, int c) const { return vp[m * LC + c]; }
};

// A stage filled by 2-D tiled TMA loads of 16-key leaf records (LC = 16):
// the keys of leaf m in 128-B row m of the key block, the values in row m of
// the value block, both in the TMA's 128-B swizzle (16-B chunk j of row m at
// chunk j ^ (m mod 8); the blocks start on 1024-B boundaries), and the
// leaves' first keys copied densely once the loads land (the binary search
// over them then reads consecutive words).
struct StageTma {
  const unsigned char *kb, *vb;
  const int64_t *firsts;
  __device__ StageTma(const unsigned char *k, const unsigned char *v, const int64_t *f) : kb(k), vb(v), firsts(f) {}
  __device__ __forceinline__ static int off(int m, int c) {
    return m * 128 + ((((c >> 1) ^ m) & 7) << 4) + ((c & 1) << 3);
  }
  __device__ __forceinline__ int64_t first(int m) const { return firsts[m]; }
  __device__ __forceinline__ int64_t key(int m, int c) const {
    return *reinterpret_cast<const int64_t *>(kb + off(m, c));
  }
  __device__ __forceinline__ int64_t val(int m, int c) const {
    return *reinterpret_cast<const int64_t *>(vb + off(m, c));
  }
};

// Asynchronous copy of an item's leaf records into a stage (nothing when the
// leaves do not fit; such an item takes the scalar path).
template <int LC>
__device__ __forceinline__ void stage_leaves(const DevTree &t, const Item &it, Stage<LC> st, int ml) {
  constexpr int LI = LC >= 32 ? LC / 8 : 0;
  constexpr int ROW = LI + 2 * LC;
  constexpr int KS = LC + 1;
  if (it.nl() < 1 || it.nl() > ml) return;
  const longlong2 *src = reinterpret_cast<const longlong2 *>(t.leaf_rows + (int64_t)it.l0 * ROW);
  const int nvec = it.nl() * (ROW / 2);
  for (int v = threadIdx.x; v < nvec; v += kThreads) {
    const int m = v / (ROW / 2), w = 2 * (v - m * (ROW / 2));
    if (w < LI) continue;
    if (w < LI + LC) {
      cp_async8(st.kp + m * KS + (w - LI), reinterpret_cast<const int64_t *>(src + v));
      cp_async8(st.kp + m * KS + (w - LI) + 1, reinterpret_cast<const int64_t *>(src + v) + 1);
    } else {
      cp_async16(st.vp + m * LC + (w - LI - LC), src + v);
    }
  }
}

template <int LC, typename ST>
__device__ __forceinline__ int64_t lookup_staged(const ST &st, int nl, int span, int64_t q) {
  // leaf: the last of [1, nl) whose first key is <= q, else 0
  int m = 0;
  for (int step = span >> 1; step > 0; step >>= 1)
    if (m + step < nl && st.first(m + step) <= q) m += step;
  // slot: the last key <= q among the leaf's sorted keys (Max_Key pads the
  // tail), else slot 0
  int c = 0;
#pragma unroll
  for (int step = LC / 2; step > 0; step >>= 1)
    if (st.key(m, c + step) <= q) c += step;
  return st.key(m, c) == q ? st.val(m, c) : HM_NOT_FOUND;
}

// Directory of the staged leaves of one item (bucket b): slot j covers the
// keys [s_j, s_j+1) with s_j = bucket low + j << dshift, and dir[j] is the
// last leaf whose first key is <= s_j (0 if none), so a query of slot j lies
// in a leaf of [dir[j], dir[j+1]] (dir[D] = nl - 1).  Keys are compared in the
// biased unsigned order (k ^ sign bit), which is the signed order.
#ifndef HM_JOIN_DIR_BITS
#define HM_JOIN_DIR_BITS 6
#endif
constexpr int kDirBits = HM_JOIN_DIR_BITS;
constexpr int kDir = 1 << kDirBits;
#ifndef HM_JOIN_DIR_MIN
#define HM_JOIN_DIR_MIN 768  // mean queries per bucket from which the directory kernel runs
#endif

__host__ __device__ __forceinline__ uint64_t biased(int64_t k) { return (uint64_t)k ^ kSign; }

template <typename ST>
__device__ __forceinline__ void build_dir(const ST &st, int nl, int span, uint64_t lo_u, int dshift,
                                          int32_t *dir) {
  for (int j = threadIdx.x; j <= kDir; j += kThreads) {
    if (j == kDir) {
      dir[j] = nl - 1;
      continue;
    }
    uint64_t sj = lo_u + ((uint64_t)j << dshift);
    if (sj < lo_u) sj = ~0ull;  // past the top of the key space
    int m = 0;
    for (int step = span >> 1; step > 0; step >>= 1)
      if (m + step < nl && biased(st.first(m + step)) <= sj) m += step;
    dir[j] = m;
  }
}

template <int LC, typename ST>
__device__ __forceinline__ int64_t lookup_dir(const ST &st, int nl, const int32_t *dir, uint64_t lo_u, int dshift,
                                              int64_t q) {
  const uint64_t qu = biased(q);
  int m, hi;
  if (qu < lo_u) {  // below the bucket (bucket 0 only: not a loaded key)
    m = 0;
    hi = dir[0];
  } else {
    const uint64_t j = (qu - lo_u) >> dshift;
    const int jj = j < (uint64_t)kDir ? (int)j : kDir - 1;
    m = dir[jj];
    hi = dir[jj + 1];
  }
  while (m < hi && st.first(m + 1) <= q) m++;
  int c = 0;
#pragma unroll
  for (int step = LC / 2; step > 0; step >>= 1)
    if (st.key(m, c + step) <= q) c += step;
  (void)nl;
  return st.key(m, c) == q ? st.val(m, c) : HM_NOT_FOUND;
}

template <int LC>
__device__ __noinline__ int64_t lookup_scalar(const DevTree &t, int f, int64_t q) {
  constexpr int LI = LC >= 32 ? LC / 8 : 0;
  constexpr int ROW = LI + 2 * LC;
  const int32_t leaf = descend_leaf(t, f, q);
  const int64_t *kr = t.leaf_rows + (int64_t)leaf * ROW + LI;
  int64_t v = HM_NOT_FOUND;
#pragma unroll 4
  for (int s = 0; s < LC; s++)
    if (__ldg(kr + s) == q) v = __ldg(kr + LC + s);
  return v;
}

// Answers the queries of the current item kRun at a time (results to out in
// grouped order, or to out[place[i]]) while loading the next step's queries:
// this item's next run, else the first run of the next item.
template <int LC, bool DIR, bool PLACED, typename ST>
__device__ __forceinline__ void answer_item(const DevTree &t, int f, const ST &st, const Item &cur, const Item &next,
                                            bool staged, int span, uint64_t lo_u, int dshift, const int32_t *dir,
                                            const int64_t *__restrict__ qs, const int32_t *__restrict__ place,
                                            int64_t *__restrict__ out, int64_t (&q)[kPerThread],
                                            int32_t (&qo)[kPerThread]) {
  for (int r0 = 0; r0 < cur.len(); r0 += kRun) {
    // the next step's queries: this item's next run, else the next item's first
    const bool more = r0 + kRun < cur.len();
    const int32_t na = more ? cur.qa + r0 + kRun : next.qa;
    const int32_t nlen = more ? cur.len() - r0 - kRun : next.len();
    int64_t qn[kPerThread];
    int32_t on[kPerThread];
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
      const int r = j * kThreads + threadIdx.x;
      const bool in = r < nlen;
      qn[j] = in ? __ldg(qs + na + r) : 0;
      on[j] = PLACED ? (in ? __ldg(place + na + r) : 0) : na + r;
    }
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
      const int r = r0 + j * kThreads + threadIdx.x;
      if (r >= cur.len()) continue;
      int64_t v = HM_NOT_FOUND;
      if (q[j] != kMaxKey) {
        if (!staged)
          v = lookup_scalar<LC>(t, f, q[j]);
        else if (DIR)
          v = lookup_dir<LC>(st, cur.nl(), dir, lo_u, dshift, q[j]);
        else
          v = lookup_staged<LC>(st, cur.nl(), span, q[j]);
      }
      out[qo[j]] = v;  // grouped order: consecutive threads, consecutive slots
    }
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
      q[j] = qn[j];
      qo[j] = on[j];
    }
  }
}

// Persistent CTAs walk the items with a stride of the grid through a ring of
// kStages shared-memory stages: the leaves of the next kStages - 1 items are
// in flight (cp.async) while the current one is answered from shared memory,
// kRun queries per step.  Item descriptors are loaded kStages items ahead and
// the queries of the next step (of this item or the next) one step ahead.
// DIR: each staged item first builds its directory (batches with many queries
// per bucket); otherwise a query binary-searches the staged first keys.
// PLACED: grouped query i's result goes to out[place[i]] (its position before
// the last pre-sort pass, which the pass recorded), else to out[i].
template <int LC, bool DIR, bool PLACED>
__global__ void __launch_bounds__(kThreads, HM_JOIN_MINB) join_kernel(DevTree t, int f, const Item *__restrict__ items,
                                                        const int64_t *__restrict__ nitems,
                                                        const int64_t *__restrict__ qs,
                                                        const int32_t *__restrict__ place, int64_t *__restrict__ out,
                                                        int ml, uint64_t key_lo_u, int shift) {
  pdl_enter();
  static_assert(kStages >= 2, "a ring of at least two stages");
  extern __shared__ __align__(16) int64_t smem[];
  const int stage_words = ml * (2 * LC + 1);
  const int64_t n_items = *nitems;
  const int64_t g = gridDim.x;
  int64_t it = blockIdx.x;
  if (it >= n_items) return;
  const Item none{0, 0, 0, 0};
  __shared__ int32_t dir[DIR ? kDir + 1 : 1];
  const int dshift = shift > kDirBits ? shift - kDirBits : 0;
  Item d[kStages];  // items it, it + g, ..., it + (kStages - 1) g
#pragma unroll
  for (int x = 0; x < kStages; x++) d[x] = it + x * g < n_items ? items[it + x * g] : none;
#pragma unroll
  for (int x = 0; x < kStages - 1; x++) {
    stage_leaves<LC>(t, d[x], Stage<LC>(smem + x * stage_words, ml), ml);
    cp_async_commit();
  }
  int64_t q[kPerThread];
  int32_t qo[kPerThread];  // where each result goes
#pragma unroll
  for (int j = 0; j < kPerThread; j++) {
    const int r = j * kThreads + threadIdx.x;
    const bool in = r < d[0].len();
    q[j] = in ? __ldg(qs + d[0].qa + r) : 0;
    qo[j] = PLACED ? (in ? __ldg(place + d[0].qa + r) : 0) : d[0].qa + r;
  }
  int cur_stage = 0;
  for (; it < n_items; it += g) {
    const int fill = cur_stage == 0 ? kStages - 1 : cur_stage - 1;  // (cur + kStages - 1) % kStages
    stage_leaves<LC>(t, d[kStages - 1], Stage<LC>(smem + fill * stage_words, ml), ml);
    cp_async_commit();
    const Item dn = it + kStages * g < n_items ? items[it + kStages * g] : none;
    asm volatile("cp.async.wait_group %0;" ::"n"(kStages - 1) : "memory");  // the current item's group is done
    __syncthreads();
    const Item cur = d[0];
    const Stage<LC> st(smem + cur_stage * stage_words, ml);
    const bool staged = cur.nl() >= 1 && cur.nl() <= ml;
    int span = 1;
    while (span < cur.nl()) span <<= 1;
    const uint64_t lo_u = key_lo_u + ((uint64_t)cur.b << shift);
    if (DIR && staged) {  // uniform across the CTA
      build_dir(st, cur.nl(), span, lo_u, dshift, dir);
      __syncthreads();
    }
    answer_item<LC, DIR, PLACED>(t, f, st, cur, d[1], staged, span, lo_u, dshift, dir, qs, place, out, q, qo);
    __syncthreads();  // this stage is refilled in the next iteration
#pragma unroll
    for (int x = 0; x < kStages - 1; x++) d[x] = d[x + 1];
    d[kStages - 1] = dn;
    cur_stage = cur_stage == kStages - 1 ? 0 : cur_stage + 1;
  }
  cp_async_wait_all();
}

// The join for 16-key leaf records with the stages filled by the tensor
// memory accelerator: one thread issues, per item, 2-D tiled loads of 8
// records at a time (one box for their keys, one for their values, 1 KiB
// each, 128-B swizzle) that complete on the stage's mbarrier; the other
// threads do no address work for the staging.  An item's last box may bring
// up to 7 records past its range (the next bucket's leaves, or zeros past the
// last leaf), which are never searched.  Every wait is bounded: on a timeout
// the CTA records HM_ETIMEOUT in err, waits (bounded) for the loads it issued
// and returns.
template <bool DIR, bool PLACED>
__global__ void __launch_bounds__(kThreads, HM_JOIN_MINB) join_tma_kernel(
    const __grid_constant__ CUtensorMap tmap, DevTree t, int f, const Item *__restrict__ items,
    const int64_t *__restrict__ nitems, const int64_t *__restrict__ qs, const int32_t *__restrict__ place,
    int64_t *__restrict__ out, int ml, uint64_t key_lo_u, int shift, unsigned *err) {
  constexpr int LC = 16;
  pdl_enter();
  static_assert(kStages >= 2, "a ring of at least two stages");
  extern __shared__ __align__(16) unsigned char dyn[];
  __shared__ __align__(8) uint64_t bars[kStages];
  __shared__ int32_t dir[DIR ? kDir + 1 : 1];
  const int64_t n_items = *nitems;
  const int64_t g = gridDim.x;
  int64_t it = blockIdx.x;
  if (it >= n_items) return;
  const int rb = (ml + 7) & ~7;  // rows of a stage's key block (and value block)
  const int block = rb * 128;
  unsigned char *base = dyn + ((1024u - (smem_addr(dyn) & 1023u)) & 1023u);  // 1024-B aligned
  int64_t *firsts = reinterpret_cast<int64_t *>(base + (size_t)kStages * 2 * block);  // [kStages][rb]
  if (threadIdx.x == 0) {
    for (int x = 0; x < kStages; x++) mbar_init(&bars[x], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // thread 0: the loads of item `itm` into stage x (none for an item that is
  // not staged: the arrival alone completes the phase)
  auto issue = [&](const Item &itm, int x) {
    const bool stg = itm.nl() >= 1 && itm.nl() <= ml;
    const int boxes = stg ? (itm.nl() + 7) >> 3 : 0;
    fence_proxy_async_smem();  // the stage's earlier reads come before these writes
    mbar_expect_tx(&bars[x], (unsigned)boxes * 2048u);
    unsigned char *kb = base + (size_t)x * 2 * block;
    for (int b = 0; b < boxes; b++) {
      tma_load_2d(kb + b * 1024, &tmap, 0, itm.l0 + 8 * b, &bars[x]);
      tma_load_2d(kb + block + b * 1024, &tmap, 16, itm.l0 + 8 * b, &bars[x]);
    }
  };
  const Item none{0, 0, 0, 0};
  const int dshift = shift > kDirBits ? shift - kDirBits : 0;
  Item d[kStages];  // items it, it + g, ..., it + (kStages - 1) g
#pragma unroll
  for (int x = 0; x < kStages; x++) d[x] = it + x * g < n_items ? items[it + x * g] : none;
  if (threadIdx.x == 0)
    for (int x = 0; x < kStages - 1; x++) issue(d[x], x);
  unsigned phase = 0;  // bit x: parity of stage x's next phase
  unsigned pending = (1u << (kStages - 1)) - 1;  // bit x: stage x has loads issued and not waited for
  int64_t q[kPerThread];
  int32_t qo[kPerThread];
#pragma unroll
  for (int j = 0; j < kPerThread; j++) {
    const int r = j * kThreads + threadIdx.x;
    const bool in = r < d[0].len();
    q[j] = in ? __ldg(qs + d[0].qa + r) : 0;
    qo[j] = PLACED ? (in ? __ldg(place + d[0].qa + r) : 0) : d[0].qa + r;
  }
  int cur_stage = 0;
  for (; it < n_items; it += g) {
    const int fill = cur_stage == 0 ? kStages - 1 : cur_stage - 1;  // (cur + kStages - 1) % kStages
    if (threadIdx.x == 0) issue(d[kStages - 1], fill);
    pending |= 1u << fill;
    const Item dn = it + kStages * g < n_items ? items[it + kStages * g] : none;
    const bool ok = mbar_wait_bounded(&bars[cur_stage], (phase >> cur_stage) & 1u, t.wait_polls);
    phase ^= 1u << cur_stage;
    pending &= ~(1u << cur_stage);
    if (__syncthreads_or(!ok)) {  // a load that never landed: report, drain, stop
      if (threadIdx.x == 0) {
        atomicOr(err, kErrTimeout);
        for (int x = 0; x < kStages; x++)
          if ((pending >> x) & 1u) mbar_wait_bounded(&bars[x], (phase >> x) & 1u);
        if (!ok) mbar_wait_bounded(&bars[cur_stage], ((phase >> cur_stage) & 1u) ^ 1u);
      }
      __syncthreads();
      return;
    }
    const Item cur = d[0];
    const unsigned char *kb = base + (size_t)cur_stage * 2 * block;
    int64_t *fs = firsts + (size_t)cur_stage * rb;
    const bool staged = cur.nl() >= 1 && cur.nl() <= ml;
    if (staged)
      for (int m = threadIdx.x; m < cur.nl(); m += kThreads)
        fs[m] = *reinterpret_cast<const int64_t *>(kb + StageTma::off(m, 0));
    __syncthreads();
    const StageTma st(kb, kb + block, fs);
    int span = 1;
    while (span < cur.nl()) span <<= 1;
    const uint64_t lo_u = key_lo_u + ((uint64_t)cur.b << shift);
    if (DIR && staged) {  // uniform across the CTA
      build_dir(st, cur.nl(), span, lo_u, dshift, dir);
      __syncthreads();
    }
    answer_item<LC, DIR, PLACED>(t, f, st, cur, d[1], staged, span, lo_u, dshift, dir, qs, place, out, q, qo);
    __syncthreads();  // this stage is refilled in the next iteration
#pragma unroll
    for (int x = 0; x < kStages - 1; x++) d[x] = d[x + 1];
    d[kStages - 1] = dn;
    cur_stage = cur_stage == kStages - 1 ? 0 : cur_stage + 1;
  }
  // loads issued for items past the end (none are staged, but their phases
  // must complete before the CTA's shared memory is released)
  if (threadIdx.x == 0)
    for (int x = 0; x < kStages; x++)
      if ((pending >> x) & 1u) mbar_wait_bounded(&bars[x], (phase >> x) & 1u);
}

int64_t max_items(int64_t n, int nb) { return n / kItemMax + nb + 1; }

int leaf_bytes(int lc) { return lc == 16 ? stage_leaf_bytes<16>() : stage_leaf_bytes<64>(); }

// Leaves one stage holds: room for the mean leaves per bucket, a quarter more
// and a margin, as an even count (keeps the value part 16-B aligned).  A
// bucket of more leaves takes the scalar path.
int stage_leaves_for(const hm_tree *t, int bits) {
  const int64_t mean = (t->n_leaf + ((int64_t)1 << bits) - 1) >> bits;
  int64_t ml = mean + mean / HM_JOIN_SLACK + 8;
  ml = std::min<int64_t>(ml, kStageMax / leaf_bytes(t->cfg.leaf_cap));
  return (int)(ml & ~int64_t(1));
}

}  // namespace

int join_bits(const hm_tree *t) {
  // HM_JOIN_MAX_BITS bits, or fewer while buckets still average at most 32 leaves
  int b = 1;
  while (b < HM_JOIN_MAX_BITS && (t->n_leaf >> b) > 32) b++;
  return b;
}

bool join_fits(const hm_tree *t) {
  if (t->cfg.leaf_cap != 16 && t->cfg.leaf_cap != 64) return false;
  const int bits = join_bits(t);
  const int64_t mean = (t->n_leaf + ((int64_t)1 << bits) - 1) >> bits;
  return mean + mean / HM_JOIN_SLACK + 8 <= stage_leaves_for(t, bits) + 1;
}

size_t join_scratch_bytes(int64_t n, int bits) {
  const int64_t nb = (int64_t)1 << bits;
  return (size_t)(2 * align_up(4 * (nb + 1), 256) + align_up(8 * (nb + 2), 256) +
                  align_up((int64_t)scan_scratch_bytes(nb + 1), 256) +
                  align_up((int64_t)sizeof(Item) * max_items(n, (int)nb), 256)) +
         256;
}

namespace {

// Bucket geometry, as the partition computes it: bucket of k = (k - key_min) >> shift.
int bucket_shift(const hm_tree *t, int bits) {
  uint64_t range = (uint64_t)t->key_max - (uint64_t)t->key_min;
  int len = 0;
  while (len < 64 && (range >> len) != 0) len++;
  return len > bits ? len - bits : 0;
}

// The leaf of each bucket boundary (nb + 1 entries): kept per tree shape in
// the tree, else computed into leafb_scratch.  With bstart (contiguous
// buckets) the same launch writes each bucket's item count into cnt; without
// it the launch is skipped when the kept boundaries are valid.
const int32_t *bucket_bounds(const hm_tree *t, int bits, int shift, const int64_t *bstart, int32_t *leafb_scratch,
                             int32_t *cnt, cudaStream_t s) {
  const int nb = 1 << bits;
  const unsigned gb = (unsigned)((nb + 1 + 255) / 256);
  int32_t *leafb = leafb_scratch;
  // kept per tree shape (not inside a graph capture, whose replays must
  // follow later changes of the tree)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;
  }
  bool want_leafb = true;
  bool fill_cache = false;
  // Held until the fill (if any) is enqueued and its event recorded: another
  // caller then finds the cache valid and waits on that event.  Once filled
  // the cache is only read, until a write to the tree changes its shape.
  std::unique_lock<std::mutex> cache_lock(t->mu, std::defer_lock);
  if (cap == cudaStreamCaptureStatusNone) {
    cache_lock.lock();
    const bool same = t->join_leafb_valid && t->join_leafb_gen == t->generation &&
                      t->join_leafb_shape == t->shape_version && t->join_leafb_lo == t->key_min &&
                      t->join_leafb_hi == t->key_max && t->join_leafb_nleaf == t->n_leaf && t->join_leafb_bits == bits;
    if (same) {
      leafb = t->join_leafb;
      want_leafb = false;
      cudaStreamWaitEvent(s, t->join_leafb_ready, 0);
    } else {
      t->join_leafb_valid = false;
      bool ok = true;
      if (t->join_leafb_cap < nb + 1) {
        if (t->join_leafb) cudaFree(t->join_leafb);
        t->join_leafb = nullptr;
        t->join_leafb_cap = 0;
        ok = cudaMalloc(&t->join_leafb, 4 * (size_t)(nb + 1)) == cudaSuccess;
        if (ok) t->join_leafb_cap = nb + 1;
      }
      if (ok && !t->join_leafb_ready)
        ok = cudaEventCreateWithFlags(&t->join_leafb_ready, cudaEventDisableTiming) == cudaSuccess;
      if (ok) {
        leafb = t->join_leafb;
        fill_cache = true;
      } else {
        cudaGetLastError();  // no cache: the boundaries are computed into scratch as in a capture
      }
    }
  }
  if (want_leafb || bstart) {
    launch_pdl(bucket_prep_kernel, gb, 256, 0, s, t->view(), t->cfg.fanout, t->key_min, shift, nb, bstart, leafb,
               bstart ? cnt : nullptr, want_leafb);
    note_launch();
  }
  if (fill_cache && cudaEventRecord(t->join_leafb_ready, s) == cudaSuccess) {
    t->join_leafb_valid = true;
    t->join_leafb_gen = t->generation;
    t->join_leafb_shape = t->shape_version;
    t->join_leafb_lo = t->key_min;
    t->join_leafb_hi = t->key_max;
    t->join_leafb_nleaf = t->n_leaf;
    t->join_leafb_bits = bits;
  }
  return leafb;
}

using JoinKernel = void (*)(DevTree, int, const Item *, const int64_t *, const int64_t *, const int32_t *, int64_t *,
                            int, uint64_t, int);

template <bool PLACED>
JoinKernel pick_join(int lc, bool dir) {
  if (lc == 16) return dir ? join_kernel<16, true, PLACED> : join_kernel<16, false, PLACED>;
  if (lc == 64) return dir ? join_kernel<64, true, PLACED> : join_kernel<64, false, PLACED>;
  return nullptr;
}

#ifndef HM_JOIN_TMA
#define HM_JOIN_TMA 1  // 16-key leaves: stages filled by 2-D tiled TMA loads
#endif

using TmaJoinKernel = void (*)(const CUtensorMap, DevTree, int, const Item *, const int64_t *, const int64_t *,
                               const int32_t *, int64_t *, int, uint64_t, int, unsigned *);

// The TMA join serves the binary-search variant only: with the directory
// (thousands of queries per item) the per-lookup cost of the swizzled
// addressing outweighs the staging work it saves (measured on 217 M queries:
// join 1.80 against 1.58 ms; at 2^24 queries without the directory 0.336
// against 0.347 ms).
template <bool PLACED>
TmaJoinKernel pick_tma_join(bool dir) {
  return dir ? nullptr : join_tma_kernel<false, PLACED>;
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's tensor-map encoder, looked up once per process (nullptr if
// the driver does not provide it: the join then stages with cp.async).
EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
    cudaGetLastError();
  });
  return fn;
}

// The leaf records of a 16-key tree as a 2-D tensor for TMA: n_leaf rows of
// 32 int64 (keys, then values; 256-B rows), boxes of 16 words x 8 rows
// (128-B inner extent, the 128-B swizzle's limit).
bool leaf_tensor_map(const hm_tree *t, CUtensorMap *m) {
  EncodeTiled enc = encoder();
  if (!enc || t->cfg.leaf_cap != 16 || t->leaf_index != 0 || t->n_leaf < 8) return false;  // a box's rows exist
  const cuuint64_t dim[2] = {32, (cuuint64_t)t->n_leaf};
  const cuuint64_t stride[1] = {32 * sizeof(int64_t)};
  const cuuint32_t box[2] = {16, 8};
  const cuuint32_t estride[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_INT64, 2, t->leaf_rows, dim, stride, box, estride,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Shared memory of the TMA join: alignment slack, per stage a key block and a
// value block of rb 128-B rows and rb first keys.
size_t tma_join_smem(int ml) {
  const size_t rb = (size_t)((ml + 7) & ~7);
  return 1024 + (size_t)kStages * (2 * rb * 128 + rb * 8);
}

// Launches the join over the items (their count at nitems).
int run_join(const hm_tree *t, JoinKernel k, TmaJoinKernel tk, int bits, int64_t n_items_max, const Item *items,
             const int64_t *nitems, const int64_t *qs, const int32_t *place, int64_t *out, int shift,
             cudaStream_t s) {
  if (!k) return HM_EINVAL;
  const int lc = t->cfg.leaf_cap;
  const int ml = stage_leaves_for(t, bits);
  CUtensorMap tmap;
  if (HM_JOIN_TMA && tk && leaf_tensor_map(t, &tmap)) {
    const size_t smem = tma_join_smem(ml);
    const int per_sm = std::max(1, std::min(8, (int)((227 * 1024) / (smem + 1024))));
    const unsigned grid = (unsigned)std::min<int64_t>(n_items_max, (int64_t)t->num_sms * per_sm);
    int rc = opt_in_smem((const void *)tk, (int)tma_join_smem(kStageMax / leaf_bytes(16)));
    if (rc) return rc;
    launch_pdl(tk, grid, kThreads, smem, s, tmap, t->view(), t->cfg.fanout, items, nitems, qs, place, out, ml,
               biased(t->key_min), shift, t->d_err);
    note_launch();
    return HM_OK;
  }
  const size_t smem = (size_t)kStages * ml * leaf_bytes(lc);
  const int per_sm = std::max(1, std::min(8, (int)((227 * 1024) / (smem + 1024))));
  const unsigned grid = (unsigned)std::min<int64_t>(n_items_max, (int64_t)t->num_sms * per_sm);
  int rc = opt_in_smem((const void *)k, kStages * kStageMax);
  if (rc) return rc;
  launch_pdl(k, grid, kThreads, smem, s, t->view(), t->cfg.fanout, items, nitems, qs, place, out, ml,
             biased(t->key_min), shift);
  note_launch();
  return HM_OK;
}

// measured: the directory pays from about three queries per thread and item
bool use_dir(int64_t n, int nb) { return HM_JOIN_DIR_BITS > 0 && n >= (int64_t)HM_JOIN_DIR_MIN * nb; }

}  // namespace

int launch_join(const hm_tree *t, const int64_t *qs, const int64_t *bstart, int bits, int64_t n, int64_t *out,
                void *scratch, cudaStream_t s, const int32_t *place) {
  if (n <= 0) return HM_OK;
  const int nb = 1 << bits;
  char *p = static_cast<char *>(scratch);
  int32_t *leafb_s = reinterpret_cast<int32_t *>(p);
  p += align_up(4 * (nb + 1), 256);
  int32_t *cnt = reinterpret_cast<int32_t *>(p);
  p += align_up(4 * (nb + 1), 256);
  int64_t *first = reinterpret_cast<int64_t *>(p);
  p += align_up(8 * (nb + 2), 256);
  void *scan = p;
  p += align_up((int64_t)scan_scratch_bytes(nb + 1), 256);  // keeps the 16-B items aligned
  Item *items = reinterpret_cast<Item *>(p);
  const int shift = bucket_shift(t, bits);
  const unsigned gb = (unsigned)((nb + 1 + 255) / 256);
  const int32_t *leafb = bucket_bounds(t, bits, shift, bstart, leafb_s, cnt, s);
  exclusive_scan_i32(cnt, first, nb + 1, scan, s);
  launch_pdl(expand_items_kernel, gb, 256, 0, s, nb, bstart, leafb, cnt, first, items);
  note_launch();
  const bool dir = use_dir(n, nb);
  const JoinKernel k = place ? pick_join<true>(t->cfg.leaf_cap, dir) : pick_join<false>(t->cfg.leaf_cap, dir);
  const TmaJoinKernel tk = place ? pick_tma_join<true>(dir) : pick_tma_join<false>(dir);
  int rc = run_join(t, k, tk, bits, max_items(n, nb), items, first + nb, qs, place, out, shift, s);
  if (rc) return rc;
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
