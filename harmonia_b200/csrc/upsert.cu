// One epoch of batched upserts applied on the GPU.
//
// Reference: BPlusTree::insert_parallel_Newupdate_batch
// (open-harmonia/src/bpt-ppi-update-batch.cpp:86-200): 56 CPU threads
// descend per key, update an existing key under the leaf mutex
// (value = key-1, :47) or insert into the record list if it has room
// (:59-67), a leaf inner split otherwise (:71-76), a serial insert for the
// rest (:151-170) and a periodic re-BFS of the inner nodes
// (rebuild_without_leaf, open-harmonia/src/bpt-ppi-update.cpp:320-463).  The
// reference never refreshes the GPU copy.
//
// Here the epoch runs on the device tree itself (an epoch of at most 1024
// keys whose new keys all fit their leaves in one CTA, see small_epoch_kernel;
// otherwise in these steps):
//   1. sort the batch by key (stable, payload = input index) and keep the
//      last occurrence of each key;
//   2. one thread per key descends; a hit overwrites the value in place
//      (supplied value, or key-1 under HM_UPSERT_REF_KEY_MINUS_1);
//   3. the misses, still in key order, are grouped by leaf; if every touched
//      leaf has room, one warp per leaf merges its new keys into the sorted
//      row (separators stay valid: a key routed to leaf j lies in
//      [separator_j, separator_j+1)), and leaf_base is rescanned;
//   4. otherwise the tree is rebuilt: the current contents and the misses
//      are merged (each element's output slot = own rank + rank in the other
//      run) and bulk-loaded into a fresh arena with the same parameters.
#include "hm_internal.cuh"

#include <algorithm>
#include <cstring>

namespace hm {

void scan_counts(int64_t *counts, int64_t m, cudaStream_t s);
void exclusive_scan_i32(const int32_t *in, int64_t *out, int64_t n, void *scratch, cudaStream_t s);
void export_contents(const hm_tree *t, int64_t *d_keys, int64_t *d_vals, cudaStream_t s);

namespace {

constexpr int kThreads = 256;

unsigned grid_for(int64_t items) {
  int64_t b = (items + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)b;
}

// keep[i] = 1 for the last occurrence of each key in the sorted batch;
// flags bit1 if a key equals Max_Key.
__global__ void last_occurrence_kernel(const uint64_t *__restrict__ uk, int64_t n,
                                       int32_t *__restrict__ keep, unsigned *flags) {
  unsigned f = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    keep[i] = (i == n - 1 || uk[i] != uk[i + 1]) ? 1 : 0;
    if ((int64_t)(uk[i] ^ kSign) == kMaxKey) f |= 2u;
  }
  if (f) atomicOr(flags, f);
}

__global__ void compact_batch_kernel(const uint64_t *__restrict__ uk, const int32_t *__restrict__ idx,
                                     const int64_t *__restrict__ vals, const int32_t *__restrict__ keep,
                                     const int64_t *__restrict__ at, int64_t n,
                                     int64_t *__restrict__ bk, int64_t *__restrict__ bv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (keep[i]) {
      int64_t o = at[i];
      bk[o] = (int64_t)(uk[i] ^ kSign);
      bv[o] = vals[idx[i]];
    }
  }
}

// Small batches (the serving loop's epochs) skip the multi-pass radix sort:
// Keys in one upsert or delete epoch, at most: the batch sort carries each
// key's input position as an int32 (such a batch would need about 200 GB of
// scratch anyway).
constexpr int64_t kMaxEpochKeys = 0x7fffffff;

// one CTA sorts (key, input index) pairs in shared memory with a bitonic
// network, keeps each key's last occurrence and writes the kept keys (and
// values) in key order to bk/bv and their number to *count; flags bit1 if a
// key equals Max_Key.
constexpr int kSmallSort = 2048;

__global__ void __launch_bounds__(1024) small_sort_unique_kernel(const int64_t *__restrict__ keys,
                                                                 const int64_t *__restrict__ vals, int n,
                                                                 int64_t *__restrict__ bk, int64_t *__restrict__ bv,
                                                                 int64_t *__restrict__ count, unsigned *flags) {
  __shared__ uint64_t sk[kSmallSort];
  __shared__ int32_t si[kSmallSort];
  __shared__ int32_t wsum[32];
  const int tid = threadIdx.x;
  int P = 1;
  while (P < n) P <<= 1;
  unsigned f = 0;
  for (int i = tid; i < P; i += blockDim.x) {
    const bool real = i < n;
    const int64_t k = real ? keys[i] : 0;
    if (real && k == kMaxKey) f |= 2u;
    sk[i] = real ? (uint64_t)k ^ kSign : ~0ull;  // padding sorts after every real key
    si[i] = real ? i : INT32_MAX;
  }
  if (f) atomicOr(flags, f);
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool asc = (i & k) == 0;
          const bool gt = sk[i] > sk[ixj] || (sk[i] == sk[ixj] && si[i] > si[ixj]);
          if (gt == asc) {
            const uint64_t tk = sk[i];
            sk[i] = sk[ixj];
            sk[ixj] = tk;
            const int32_t ti = si[i];
            si[i] = si[ixj];
            si[ixj] = ti;
          }
        }
      }
      __syncthreads();
    }
  }
  // keep the last occurrence of each key; two elements per thread, block scan
  int kept[2], mine = 0;
  for (int h = 0; h < 2; h++) {
    const int i = 2 * tid + h;
    kept[h] = i < n && (i == n - 1 || sk[i] != sk[i + 1]);
    mine += kept[h];
  }
  int incl = mine;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((tid & 31) >= o) incl += y;
  }
  if ((tid & 31) == 31) wsum[tid >> 5] = incl;
  __syncthreads();
  int before = incl - mine;
  for (int w = 0; w < (tid >> 5); w++) before += wsum[w];
  for (int h = 0; h < 2; h++) {
    const int i = 2 * tid + h;
    if (kept[h]) {
      bk[before] = (int64_t)(sk[i] ^ kSign);
      if (bv) bv[before] = vals[si[i]];
      before++;
    }
  }
  if (tid == blockDim.x - 1) *count = before;
}

// ---- small epochs in one kernel ----
//
// An epoch of at most kSmallEpoch keys (the serving loop's write requests)
// whose new keys all fit their leaves is applied by one CTA: bitonic sort of
// (key, input index) in shared memory, last occurrence kept, a descent per
// key, hits written in place, each leaf's new keys merged into its sorted row
// from the back; a second kernel adds the new keys to leaf_base.  The CTA
// checks everything (Max_Key, room in every touched leaf) before it writes
// anything, so an epoch it cannot apply leaves the tree untouched for the
// general path.  Same results as the general path, one host synchronisation
// instead of four.
constexpr int kSmallEpoch = 1024;

struct SmallEpochResult {
  int32_t applied;   // 1: applied in place; 0: nothing changed
  int32_t maxkey;    // a key equals Max_Key (nothing changed)
  int32_t inserted;  // new keys
  int32_t runs;      // leaves that received new keys
  int64_t new_min, new_max;  // smallest and largest new key
};

__global__ void __launch_bounds__(kSmallEpoch) small_epoch_kernel(
    DevTree t, int f, int lc, int li, int flags, const int64_t *__restrict__ keys, const int64_t *__restrict__ vals,
    int n, int64_t *leaf_rows, int32_t *leaf_cnt, int32_t *__restrict__ run_leaf, int32_t *__restrict__ run_pre,
    SmallEpochResult *__restrict__ res) {
  __shared__ uint64_t sk[kSmallEpoch];
  __shared__ int32_t si[kSmallEpoch];
  __shared__ int64_t kk[kSmallEpoch], kv[kSmallEpoch];  // kept keys and values, key order
  __shared__ int32_t lf[kSmallEpoch];                     // their leaves; then the misses' leaves
  __shared__ int32_t wsum[32];
  __shared__ int32_t total;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // exclusive block scan of one int per thread; total of all in `total`
  auto scan = [&](int v) {
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    __syncthreads();
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = incl - v;
    for (int w = 0; w < warp; w++) before += wsum[w];
    if (tid == blockDim.x - 1) total = before + v;
    __syncthreads();
    return before;
  };
  int P = 1;
  while (P < n) P <<= 1;
  bool mx = false;
  for (int i = tid; i < P; i += blockDim.x) {
    const bool real = i < n;
    const int64_t k = real ? keys[i] : 0;
    mx |= real && k == kMaxKey;
    sk[i] = real ? (uint64_t)k ^ kSign : ~0ull;  // padding sorts after every real key
    si[i] = real ? i : INT32_MAX;
  }
  if (__syncthreads_or(mx)) {
    if (tid == 0) res->maxkey = 1;
    return;
  }
  for (int k = 2; k <= P; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const bool asc = (i & k) == 0;
          const bool gt = sk[i] > sk[ixj] || (sk[i] == sk[ixj] && si[i] > si[ixj]);
          if (gt == asc) {
            const uint64_t tk = sk[i];
            sk[i] = sk[ixj];
            sk[ixj] = tk;
            const int32_t ti = si[i];
            si[i] = si[ixj];
            si[ixj] = ti;
          }
        }
      }
      __syncthreads();
    }
  }
  // keep each key's last occurrence (thread i owns sorted element i)
  const bool keep = tid < n && (tid == n - 1 || sk[tid] != sk[tid + 1]);
  const int at = scan(keep);
  const int m = total;
  if (keep) {
    kk[at] = (int64_t)(sk[tid] ^ kSign);
    kv[at] = vals[si[tid]];
  }
  __syncthreads();
  // descend: hit slot or miss, per kept key (thread i owns kept key i)
  int64_t key = 0, val = 0;
  int32_t leaf = -1, slot = -1;
  const int stride = li + 2 * lc;
  if (tid < m) {
    key = kk[tid];
    val = kv[tid];
    leaf = descend_leaf(t, f, key);
    const int64_t *kr = t.leaf_rows + (int64_t)leaf * stride + li;
    const int cnt = t.leaf_cnt[leaf];
    for (int x = 0; x < cnt; x++)
      if (kr[x] == key) slot = x;
  }
  const bool miss = tid < m && slot < 0;
  const int mi = scan(miss);
  const int nm = total;
  if (miss) {  // the misses, still in key order, compacted
    kk[mi] = key;
    kv[mi] = val;
    lf[mi] = leaf;
  }
  __syncthreads();
  // runs of misses per leaf, and room for each run
  bool start = false, fits = true;
  int rl = 0;
  if (tid < nm) {
    start = tid == 0 || lf[tid] != lf[tid - 1];
    if (start) {
      int e = tid + 1;
      while (e < nm && lf[e] == lf[tid]) e++;
      rl = e - tid;
      fits = t.leaf_cnt[lf[tid]] + rl <= lc;
    }
  }
  if (!__syncthreads_and(fits)) return;  // res->applied stays 0: nothing changed
  // hits in place (before the merges, which move the rows' values)
  if (tid < m && slot >= 0)
    leaf_rows[(int64_t)leaf * stride + li + lc + slot] = (flags & HM_UPSERT_REF_KEY_MINUS_1) ? key - 1 : val;
  __syncthreads();
  const int r = scan(start);
  const int runs = total;
  if (start) {
    // merge the run [tid, tid + rl) into the leaf's sorted row from the back
    const int32_t L = lf[tid];
    int64_t *kr = leaf_rows + (int64_t)L * stride + li;
    int64_t *vr = kr + lc;
    int a = leaf_cnt[L], b = rl;
    for (int o = a + b - 1; o >= 0 && b > 0; o--) {
      if (a > 0 && kr[a - 1] > kk[tid + b - 1]) {
        kr[o] = kr[a - 1];
        vr[o] = vr[a - 1];
        a--;
      } else {
        kr[o] = kk[tid + b - 1];
        vr[o] = kv[tid + b - 1];
        b--;
      }
    }
    const int nc = leaf_cnt[L] + rl;
    if (li > 0) {
      int64_t *ir = leaf_rows + (int64_t)L * stride;
      for (int x = 0; x < li; x++) ir[x] = (8 * (x + 1) < nc) ? kr[8 * (x + 1)] : kMaxKey;
    }
    leaf_cnt[L] = nc;
    run_leaf[r] = L;
    run_pre[r] = tid;  // new keys in earlier runs (the misses before this run)
  }
  if (tid == 0) {
    res->applied = 1;
    res->inserted = nm;
    res->runs = runs;
    if (nm > 0) {
      res->new_min = kk[0];
      res->new_max = kk[nm - 1];
    }
  }
}

// leaf_base[l] += new keys in leaves before l, after an applied small epoch.
__global__ void small_epoch_base_kernel(int64_t *leaf_base, int64_t n_leaf, const int32_t *__restrict__ run_leaf,
                                        const int32_t *__restrict__ run_pre, const SmallEpochResult *__restrict__ res) {
  if (!res->applied || res->inserted == 0) return;
  const int runs = res->runs, inserted = res->inserted;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n_leaf; l += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = runs;  // first run whose leaf >= l
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (run_leaf[mid] < l) lo = mid + 1; else hi = mid;
    }
    const int add = lo < runs ? run_pre[lo] : inserted;
    if (add) leaf_base[l] += add;
  }
}

// Hits are updated in place; misses get miss[i] = 1 and their leaf.
__global__ void apply_kernel(DevTree t, int f, int lc, int li, int flags,
                             const int64_t *__restrict__ bk, const int64_t *__restrict__ bv, int64_t m,
                             int64_t *leaf_rows, int32_t *__restrict__ miss,
                             int32_t *__restrict__ leaf_of) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = bk[i];
    int32_t leaf = descend_leaf(t, f, k);
    const int64_t *kr = t.leaf_rows + (int64_t)leaf * (li + 2 * lc) + li;
    int cnt = t.leaf_cnt[leaf];
    int slot = -1;
    for (int s = 0; s < cnt; s++)
      if (kr[s] == k) slot = s;
    leaf_of[i] = leaf;
    if (slot >= 0) {
      leaf_rows[(int64_t)leaf * (li + 2 * lc) + li + lc + slot] =
          (flags & HM_UPSERT_REF_KEY_MINUS_1) ? k - 1 : bv[i];
      miss[i] = 0;
    } else {
      miss[i] = 1;
    }
  }
}

__global__ void compact_miss_kernel(const int64_t *__restrict__ bk, const int64_t *__restrict__ bv,
                                    const int32_t *__restrict__ leaf_of, const int32_t *__restrict__ miss,
                                    const int64_t *__restrict__ at, int64_t m, int64_t *__restrict__ mk,
                                    int64_t *__restrict__ mv, int32_t *__restrict__ ml) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (miss[i]) {
      int64_t o = at[i];
      mk[o] = bk[i];
      mv[o] = bv[i];
      ml[o] = leaf_of[i];
    }
  }
}

// For each run of misses on one leaf (misses are in key order, so leaves are
// non-decreasing): seg_start[leaf] = first miss index, add[leaf] = run length;
// flags bit0 if the leaf would overflow.
__global__ void miss_runs_kernel(const int32_t *__restrict__ ml, int64_t nm,
                                 const int32_t *__restrict__ leaf_cnt, int lc,
                                 int64_t *__restrict__ run_start, int32_t *__restrict__ run_len,
                                 int32_t *__restrict__ run_leaf, int32_t *__restrict__ is_start,
                                 unsigned *flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nm;
       i += (int64_t)gridDim.x * blockDim.x) {
    bool st = (i == 0) || ml[i] != ml[i - 1];
    is_start[i] = st ? 1 : 0;
    if (st) {
      int64_t e = i + 1;
      while (e < nm && ml[e] == ml[i]) e++;
      run_start[i] = i;
      run_len[i] = (int32_t)(e - i);
      run_leaf[i] = ml[i];
      if (leaf_cnt[ml[i]] + (e - i) > lc) atomicOr(flags, 1u);
    }
  }
}

// One warp per run: merge the run's new keys into the leaf row.
__global__ void merge_leaf_kernel(int64_t *leaf_rows, int32_t *leaf_cnt, int lc,
                                  int li, const int64_t *__restrict__ mk, const int64_t *__restrict__ mv,
                                  const int32_t *__restrict__ is_start,
                                  const int64_t *__restrict__ run_start,
                                  const int32_t *__restrict__ run_len,
                                  const int32_t *__restrict__ run_leaf, int64_t nm,
                                  const int32_t *__restrict__ run_parent = nullptr,
                                  const int32_t *__restrict__ mark = nullptr) {
  __shared__ int64_t sk[kThreads / 32][128];
  __shared__ int64_t sv[kThreads / 32][128];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = blockIdx.x * (int64_t)(blockDim.x / 32) + w; i < nm; i += warps) {
    if (!is_start[i]) continue;
    if (mark && mark[run_parent[i]]) continue;  // its subtree is rebalanced instead
    const int32_t leaf = run_leaf[i];
    const int64_t r0 = run_start[i];
    const int rl = run_len[i];
    int64_t *kr = leaf_rows + (int64_t)leaf * (li + 2 * lc) + li;
    int64_t *vr = kr + lc;
    const int cnt = leaf_cnt[leaf];
    // existing key a goes to a + #(new < key); new key b to b + #(existing < key)
    for (int a = lane; a < cnt; a += 32) {
      int64_t k = kr[a];
      int below = 0;
      for (int b = 0; b < rl; b++) below += (mk[r0 + b] < k);
      sk[w][a + below] = k;
      sv[w][a + below] = vr[a];
    }
    for (int b = lane; b < rl; b += 32) {
      int64_t k = mk[r0 + b];
      int below = 0;
      for (int a = 0; a < cnt; a++) below += (kr[a] < k);
      sk[w][b + below] = k;
      sv[w][b + below] = mv[r0 + b];
    }
    __syncwarp();
    const int nc = cnt + rl;
    for (int x = lane; x < lc; x += 32) {
      kr[x] = x < nc ? sk[w][x] : kMaxKey;
      vr[x] = x < nc ? sv[w][x] : (int64_t)HM_NOT_FOUND;
    }
    __syncwarp();
    if (li > 0) {
      int64_t *ir = leaf_rows + (int64_t)leaf * (li + 2 * lc);
      for (int x = lane; x < li; x += 32) ir[x] = (8 * (x + 1) < lc) ? kr[8 * (x + 1)] : kMaxKey;
    }
    if (lane == 0) leaf_cnt[leaf] = nc;
    __syncwarp();
  }
}

// ---- subtree rebalancing (an epoch whose new keys overflow a leaf) ----
//
// The subtree of a last-level inner node p is its children leaves [a, b].
// When a leaf overflows but p's subtree still has room for its keys and all
// the epoch's new keys routed into it, the subtree's keys are re-spread
// evenly over the same leaves and p's separators rewritten; nothing outside
// the subtree changes (p's own separator in its parent stays a valid fence,
// because every new key routed here is at least that separator).  Only when
// some subtree has no room is the whole tree rebuilt.

struct Subtree {
  int64_t lvl0, lvl1;  // last inner level: nodes [lvl0, lvl1); lvl1 == n_inner
  int64_t n_inner, n_leaf;
};

__device__ __forceinline__ int64_t first_miss_at_or_after(const int32_t *__restrict__ ml, int64_t nm, int64_t leaf) {
  int64_t lo = 0, hi = nm;  // first miss whose leaf >= leaf
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (ml[mid] < leaf) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void subtree_leaves(const int32_t *__restrict__ prefix, const Subtree &g, int64_t p,
                                               int64_t *a, int64_t *b) {
  const int64_t c0 = prefix[p];
  const int64_t c1 = p + 1 < g.lvl1 ? prefix[p + 1] : g.n_inner + g.n_leaf;
  *a = c0 - g.n_inner;
  *b = c1 - 1 - g.n_inner;
}

// One thread per run of misses: its leaf's parent (run_parent, as an index
// into the last level); an overflowing leaf marks its parent when the
// subtree has room, else flags bit2 (rebuild the tree).
__global__ void subtree_mark_kernel(const int32_t *__restrict__ prefix, const int32_t *__restrict__ leaf_cnt,
                                    const int64_t *__restrict__ leaf_base, int lc, Subtree g,
                                    const int32_t *__restrict__ is_start, const int32_t *__restrict__ run_len,
                                    const int32_t *__restrict__ run_leaf, const int32_t *__restrict__ ml,
                                    int64_t nm, int32_t *__restrict__ run_parent, int32_t *__restrict__ mark,
                                    unsigned *flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nm;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!is_start[i]) continue;
    const int64_t leaf = run_leaf[i];
    int64_t lo = g.lvl0, hi = g.lvl1 - 1;  // last node p with prefix[p] <= the leaf's id
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= g.n_inner + leaf) lo = mid; else hi = mid - 1;
    }
    run_parent[i] = (int32_t)(lo - g.lvl0);
    if (leaf_cnt[leaf] + run_len[i] <= lc) continue;
    int64_t a, b;
    subtree_leaves(prefix, g, lo, &a, &b);
    const int64_t keys = leaf_base[b] + leaf_cnt[b] - leaf_base[a];
    const int64_t adds = first_miss_at_or_after(ml, nm, b + 1) - first_miss_at_or_after(ml, nm, a);
    if (keys + adds <= (b - a + 1) * (int64_t)lc) {
      mark[lo - g.lvl0] = 1;
    } else {
      atomicOr(flags, 4u);
    }
  }
}

// One CTA per last-level node; marked ones are rebalanced.  The existing
// records are gathered into shared memory first, then every element (old or
// new) is written to its place in the merged order, spread evenly over the
// subtree's leaves (leaf jj gets positions [part_start(jj), part_start(jj+1))).
__global__ void subtree_rebalance_kernel(int64_t *inner, const int32_t *__restrict__ prefix, int64_t *leaf_rows,
                                         int32_t *leaf_cnt, const int64_t *__restrict__ leaf_base, int f, int lc,
                                         int li, Subtree g, const int32_t *__restrict__ mark,
                                         const int64_t *__restrict__ mk, const int64_t *__restrict__ mv,
                                         const int32_t *__restrict__ ml, int64_t nm) {
  extern __shared__ __align__(16) longlong2 staged[];  // the subtree's existing records
  if (!mark[blockIdx.x]) return;
  const int64_t p = g.lvl0 + blockIdx.x;
  int64_t a, b;
  subtree_leaves(prefix, g, p, &a, &b);
  const int64_t nl = b - a + 1, row = li + 2 * lc;
  const int64_t base = leaf_base[a];
  const int64_t K = leaf_base[b] + leaf_cnt[b] - base;
  const int64_t m0 = first_miss_at_or_after(ml, nm, a), m1 = first_miss_at_or_after(ml, nm, b + 1);
  const int64_t M = m1 - m0, T = K + M;
  for (int64_t x = threadIdx.x; x < nl * lc; x += blockDim.x) {
    const int64_t j = a + x / lc, sl = x % lc;
    if (sl < leaf_cnt[j]) {
      const int64_t *r = leaf_rows + j * row + li;
      staged[leaf_base[j] - base + sl] = make_longlong2(r[sl], r[lc + sl]);
    }
  }
  __syncthreads();
  const int64_t q = T / nl, rem = T % nl;
  auto put = [&](int64_t pos, int64_t k, int64_t v) {
    const int64_t jj = pos < rem * (q + 1) ? pos / (q + 1) : rem + (pos - rem * (q + 1)) / q;
    const int64_t sl = pos - part_start(jj, T, nl);
    int64_t *r = leaf_rows + (a + jj) * row + li;
    r[sl] = k;
    r[lc + sl] = v;
  };
  for (int64_t e = threadIdx.x; e < K; e += blockDim.x) {  // old record: own index + new keys below it
    const int64_t k = staged[e].x;
    int64_t lo = m0, hi = m1;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (mk[mid] < k) lo = mid + 1; else hi = mid;
    }
    put(e + (lo - m0), k, staged[e].y);
  }
  for (int64_t i = threadIdx.x; i < M; i += blockDim.x) {  // new key: own index + old keys below it
    const int64_t k = mk[m0 + i];
    int64_t lo = 0, hi = K;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (staged[mid].x < k) lo = mid + 1; else hi = mid;
    }
    put(i + lo, k, mv[m0 + i]);
  }
  for (int64_t x = threadIdx.x; x < nl * lc; x += blockDim.x) {  // padding and counts
    const int64_t jj = x / lc, sl = x % lc;
    const int64_t len = part_start(jj + 1, T, nl) - part_start(jj, T, nl);
    if (sl >= len) {
      int64_t *r = leaf_rows + (a + jj) * row + li;
      r[sl] = kMaxKey;
      r[lc + sl] = HM_NOT_FOUND;
    }
    if (sl == 0) leaf_cnt[a + jj] = (int32_t)len;
  }
  __syncthreads();
  for (int64_t x = threadIdx.x; x < nl * li; x += blockDim.x) {  // 64-key leaves: index words
    const int64_t jj = x / li, w = x % li;
    int64_t *r = leaf_rows + (a + jj) * row;
    r[w] = 8 * (w + 1) < lc ? r[li + 8 * (w + 1)] : kMaxKey;
  }
  int64_t *pr = inner + p * (f / 8 + f);
  for (int sidx = threadIdx.x; sidx < f; sidx += blockDim.x)  // separators: first key of child s + 1
    pr[f / 8 + sidx] = sidx < nl - 1 ? leaf_rows[(a + sidx + 1) * row + li] : kMaxKey;
  __syncthreads();
  for (int w = threadIdx.x; w < f / 8; w += blockDim.x) pr[w] = 8 * (w + 1) < f ? pr[f / 8 + 8 * (w + 1)] : kMaxKey;
}

// Merge of two sorted, disjoint runs: out slot = own index + rank in the other run.
__global__ void merge_rank_kernel(const int64_t *__restrict__ a, const int64_t *__restrict__ av, int64_t na,
                                  const int64_t *__restrict__ b, int64_t nb, bool strict,
                                  uint64_t *__restrict__ ok, int64_t *__restrict__ ov) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t k = a[i];
    int64_t lo = 0, hi = nb;  // first b >= k (strict) or > k
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      bool before = strict ? (b[mid] < k) : (b[mid] <= k);
      if (before) lo = mid + 1; else hi = mid;
    }
    ok[i + lo] = (uint64_t)k ^ kSign;
    ov[i + lo] = av[i];
  }
}

// ---- delete epochs ----

__global__ void compact_keys_kernel(const uint64_t *__restrict__ uk, const int32_t *__restrict__ keep,
                                    const int64_t *__restrict__ at, int64_t n, int64_t *__restrict__ bk) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (keep[i]) bk[at[i]] = (int64_t)(uk[i] ^ kSign);
}

// One thread per distinct key: descend; a stored key's slot is overwritten
// with Max_Key (the leaf is compacted next); route[i] = the key's leaf.
__global__ void delete_mark_kernel(DevTree t, int f, int lc, int li, const int64_t *__restrict__ bk, int64_t m,
                                   int64_t *leaf_rows, int32_t *__restrict__ route) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = bk[i];
    const int32_t leaf = descend_leaf(t, f, k == kMaxKey ? kMaxKey - 1 : k);  // never rank the sentinel
    route[i] = leaf;
    if (k == kMaxKey) continue;  // never stored
    int64_t *kr = leaf_rows + (int64_t)leaf * (li + 2 * lc) + li;
    const int cnt = t.leaf_cnt[leaf];
    for (int s = 0; s < cnt; s++)
      if (kr[s] == k) kr[s] = kMaxKey;
  }
}

// One thread per leaf the batch routed to (keys are sorted, so each leaf's
// keys are one run of route[]): squeeze out the marked slots keeping key
// order, refresh the leaf index words, count what went; flags bit0 when a
// leaf that held keys is left empty (the tree is then rebuilt).
__global__ void delete_compact_kernel(int64_t *leaf_rows, int32_t *leaf_cnt, int lc, int li,
                                      const int32_t *__restrict__ route, int64_t m,
                                      unsigned long long *removed, unsigned *flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i > 0 && route[i - 1] == route[i]) continue;
    const int32_t leaf = route[i];
    int64_t *row = leaf_rows + (int64_t)leaf * (li + 2 * lc);
    int64_t *kr = row + li, *vr = kr + lc;
    const int cnt = leaf_cnt[leaf];
    int live = 0;
    for (int s = 0; s < cnt; s++) {
      if (kr[s] == kMaxKey) continue;
      kr[live] = kr[s];
      vr[live] = vr[s];
      live++;
    }
    if (live == cnt) continue;
    for (int s = live; s < cnt; s++) {
      kr[s] = kMaxKey;
      vr[s] = HM_NOT_FOUND;
    }
    for (int x = 0; x < li; x++) row[x] = (8 * (x + 1) < lc) ? kr[8 * (x + 1)] : kMaxKey;
    leaf_cnt[leaf] = live;
    atomicAdd(removed, (unsigned long long)(cnt - live));
    if (live == 0) atomicOr(flags, 1u);
  }
}

size_t al(int64_t bytes) { return (size_t)align_up(bytes, 256); }

}  // namespace

// Bulk-loads n1 sorted (sign-flipped) keys and their values into a fresh arena
// with the tree's parameters and swaps it in; the old arena is freed.
int rebuild_from_sorted(hm_tree *t, const uint64_t *ck, const int64_t *cv, int64_t n1, cudaStream_t s) {
  BuildTarget nt = t->target();  // new shape; the arena is swapped in at the end
  int rc = shape(n1, t->cfg, &nt.height, nt.lvl_start, &nt.n_inner, &nt.n_leaf);
  if (rc) return rc;
  size_t off_prefix = al(nt.n_inner * nt.inner_row * 8);
  size_t off_lrows = off_prefix + al(align_up(nt.n_inner, 4) * 4);
  size_t off_lcnt = off_lrows + al(nt.n_leaf * nt.leaf_row * 8);
  size_t off_lbase = off_lcnt + al(nt.n_leaf * 4);
  size_t total = off_lbase + al(nt.n_leaf * 8);
  int64_t tn = std::max<int64_t>(std::max<int64_t>(n1, nt.n_leaf), 1);
  char *tmp = nullptr;
  void *arena = nullptr;
  cudaError_t e = dev_alloc(&arena, total);
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void **>(&tmp), 2 * al(8 * tn));
  if (e != cudaSuccess) {
    dev_release(arena);
    dev_release(tmp);
    return cuda_err(e);
  }
  int64_t *tmp_a = reinterpret_cast<int64_t *>(tmp);
  int64_t *tmp_b = reinterpret_cast<int64_t *>(tmp + al(8 * tn));
  char *base = static_cast<char *>(arena);
  cudaMemsetAsync(base, 0, total, s);
  nt.inner = reinterpret_cast<int64_t *>(base);
  nt.prefix = reinterpret_cast<int32_t *>(base + off_prefix);
  nt.leaf_rows = reinterpret_cast<int64_t *>(base + off_lrows);
  nt.leaf_cnt = reinterpret_cast<int32_t *>(base + off_lcnt);
  nt.leaf_base = reinterpret_cast<int64_t *>(base + off_lbase);
  rc = build_from_sorted(nt, ck, cv, n1, tmp_a, tmp_b, s);
  e = cudaStreamSynchronize(s);
  dev_release(tmp);
  if (rc == HM_OK && e != cudaSuccess) rc = cuda_err(e);
  if (rc) {
    dev_release(arena);
    return rc;
  }
  cudaDeviceSynchronize();  // no call of any stream may still read the old arena
  dev_release(t->arena);
  t->arena = arena;
  t->arena_bytes = total;
  t->inner = nt.inner;
  t->prefix = nt.prefix;
  t->leaf_rows = nt.leaf_rows;
  t->leaf_cnt = nt.leaf_cnt;
  t->leaf_base = nt.leaf_base;
  t->height = nt.height;
  std::memcpy(t->lvl_start, nt.lvl_start, sizeof(t->lvl_start));
  t->n_inner = nt.n_inner;
  t->n_leaf = nt.n_leaf;
  t->n_keys = n1;
  t->generation++;
  return HM_OK;
}

int upsert_epoch(hm_tree *t, const int64_t *d_keys, const int64_t *d_vals, int64_t n, int flags,
                 cudaStream_t s) {
  if (n <= 0) return HM_OK;
  if (n > kMaxEpochKeys) return HM_ETOOLARGE;
  const int lc = t->cfg.leaf_cap, li = t->leaf_index, f = t->cfg.fanout;
  if (n <= kSmallEpoch && t->n_keys > 0) {  // one kernel, one synchronisation, if every new key fits
    ScratchLease lease(t, s);
    const size_t rb = al(4 * n);
    int rc = lease.acquire(2 * rb + al(sizeof(SmallEpochResult)) + 256);
    if (rc) return rc;
    char *p = static_cast<char *>(lease.ptr());
    int32_t *run_leaf = reinterpret_cast<int32_t *>(p);
    int32_t *run_pre = reinterpret_cast<int32_t *>(p + rb);
    SmallEpochResult *dres = reinterpret_cast<SmallEpochResult *>(p + 2 * rb);
    SmallEpochResult hres{};
    cudaError_t e = cudaMemsetAsync(dres, 0, sizeof(SmallEpochResult), s);
    if (e != cudaSuccess) return cuda_err(e);
    small_epoch_kernel<<<1, kSmallEpoch, 0, s>>>(t->view(), f, lc, li, flags, d_keys, d_vals, (int)n, t->leaf_rows,
                                                 t->leaf_cnt, run_leaf, run_pre, dres);
    small_epoch_base_kernel<<<grid_for(t->n_leaf), kThreads, 0, s>>>(t->leaf_base, t->n_leaf, run_leaf, run_pre,
                                                                     dres);
    note_launch(2);
    e = cudaMemcpyAsync(&hres, dres, sizeof(hres), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(e);
    if (hres.maxkey) return HM_EMAXKEY;
    if (hres.applied) {
      t->n_keys += hres.inserted;
      if (hres.inserted > 0) {
        if (hres.new_min < t->key_min) t->key_min = hres.new_min;
        if (hres.new_max > t->key_max) t->key_max = hres.new_max;
      }
      return HM_OK;
    }
    // some leaf has no room: nothing was changed; the general path below
  }
  // scratch: uk, uk_alt, idx, idx_alt (n each, 8 B), keep/miss/leaf_of/is_start (4 B),
  // at (8 B, n+1), bk, bv, mk, mv, run_start (8 B), run_len/run_leaf/ml (4 B), sort scratch, flags
  const size_t s8 = al(8 * (n + 1)), s4 = al(4 * (n + 1));
  // the leaf_base rescan covers every leaf, not just the batch
  const int64_t scan_n = std::max<int64_t>(n, t->n_leaf) + 1;
  const size_t lb8 = al(8 * (t->n_leaf + 1));
  const size_t mk4 = al(4 * (t->n_inner + 1));  // subtree marks, one per last-level node
  size_t need = 9 * s8 + 7 * s4 + lb8 + mk4 + al((int64_t)radix_scratch_bytes(n)) +
                al((int64_t)scan_scratch_bytes(scan_n)) + 256;
  ScratchLease lease(t, s);
  int rc = lease.acquire(need);
  if (rc) return rc;
  char *p = static_cast<char *>(lease.ptr());
  auto take8 = [&](void) { char *r = p; p += s8; return r; };
  auto take4 = [&](void) { char *r = p; p += s4; return r; };
  uint64_t *uk = reinterpret_cast<uint64_t *>(take8());
  uint64_t *uk_alt = reinterpret_cast<uint64_t *>(take8());
  int32_t *idx = reinterpret_cast<int32_t *>(take8());  // input positions (8-B slots: run_start reuses one)
  int32_t *idx_alt = reinterpret_cast<int32_t *>(take8());
  int64_t *at = reinterpret_cast<int64_t *>(take8());
  int64_t *bk = reinterpret_cast<int64_t *>(take8());
  int64_t *bv = reinterpret_cast<int64_t *>(take8());
  int64_t *mk = reinterpret_cast<int64_t *>(take8());
  int64_t *mv = reinterpret_cast<int64_t *>(take8());
  int32_t *keep = reinterpret_cast<int32_t *>(take4());
  int32_t *miss = reinterpret_cast<int32_t *>(take4());
  int32_t *leaf_of = reinterpret_cast<int32_t *>(take4());
  int32_t *ml = reinterpret_cast<int32_t *>(take4());
  int32_t *is_start = reinterpret_cast<int32_t *>(take4());
  int32_t *run_len = reinterpret_cast<int32_t *>(take4());
  int32_t *run_leaf = reinterpret_cast<int32_t *>(take4());
  int64_t *run_start = nullptr;  // the position buffer the sort leaves free
  void *sort_scratch = p;
  p += al((int64_t)radix_scratch_bytes(n));
  int64_t *lbase_tmp = reinterpret_cast<int64_t *>(p);  // n_leaf + 1 entries
  p += lb8;
  void *scan_scratch = p;
  p += al((int64_t)scan_scratch_bytes(scan_n));
  int32_t *marks = reinterpret_cast<int32_t *>(p);
  p += mk4;
  unsigned *dflags = reinterpret_cast<unsigned *>(p);

  cudaMemsetAsync(dflags, 0, 8, s);
  if (n <= kSmallSort) {
    small_sort_unique_kernel<<<1, 1024, 0, s>>>(d_keys, d_vals, (int)n, bk, bv, at + n, dflags);
    note_launch();
  } else {
    transform_keys_in(d_keys, uk, n, s);
    if (radix_sort_positions(uk, idx, uk_alt, idx_alt, n, 0, 64, sort_scratch, s)) {
      std::swap(uk, uk_alt);
      std::swap(idx, idx_alt);
    }
    last_occurrence_kernel<<<grid_for(n), kThreads, 0, s>>>(uk, n, keep, dflags);
    exclusive_scan_i32(keep, at, n, scan_scratch, s);
    compact_batch_kernel<<<grid_for(n), kThreads, 0, s>>>(uk, idx, d_vals, keep, at, n, bk, bv);
    note_launch(2);
  }
  run_start = reinterpret_cast<int64_t *>(idx_alt);
  int64_t hm_[2] = {0, 0};
  unsigned hf = 0;
  cudaMemcpyAsync(&hm_[0], at + n, 8, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&hf, dflags, 4, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);
  if (hf & 2u) return HM_EMAXKEY;
  const int64_t m = hm_[0];

  apply_kernel<<<grid_for(m), kThreads, 0, s>>>(t->view(), f, lc, li, flags, bk, bv, m, t->leaf_rows,
                                                miss, leaf_of);
  exclusive_scan_i32(miss, at, m, scan_scratch, s);
  compact_miss_kernel<<<grid_for(m), kThreads, 0, s>>>(bk, bv, leaf_of, miss, at, m, mk, mv, ml);
  note_launch(2);
  cudaMemcpyAsync(&hm_[1], at + m, 8, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);
  const int64_t nm = hm_[1];
  if (nm == 0) return HM_OK;

  cudaMemsetAsync(dflags, 0, 4, s);
  miss_runs_kernel<<<grid_for(nm), kThreads, 0, s>>>(ml, nm, t->leaf_cnt, lc, run_start, run_len,
                                                      run_leaf, is_start, dflags);
  note_launch();
  cudaMemcpyAsync(&hf, dflags, 4, cudaMemcpyDeviceToHost, s);
  int64_t new_ends[2];
  cudaMemcpyAsync(&new_ends[0], mk, 8, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&new_ends[1], mk + nm - 1, 8, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);

  // Some leaf overflows: rebalance the subtrees (last-level nodes) that have
  // room; if one has none, rebuild the tree.
  int32_t *mark = nullptr, *run_parent = nullptr;
  const Subtree g{t->lvl_start[t->height - 1], t->n_inner, t->n_inner, t->n_leaf};
  const int64_t last_nodes = g.lvl1 - g.lvl0;
  if (hf & 1u) {
    run_parent = keep;  // free after the batch compaction; nm <= n entries
    mark = marks;
    cudaMemsetAsync(mark, 0, 4 * last_nodes, s);
    subtree_mark_kernel<<<grid_for(nm), kThreads, 0, s>>>(t->prefix, t->leaf_cnt, t->leaf_base, lc, g, is_start,
                                                           run_len, run_leaf, ml, nm, run_parent, mark, dflags);
    note_launch();
    e = cudaMemcpyAsync(&hf, dflags, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(e);
  }
  if (!(hf & 4u)) {
    // Every touched leaf has room, or its subtree does: merge in place.
    int64_t blocks = (nm + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    merge_leaf_kernel<<<(unsigned)blocks, kThreads, 0, s>>>(t->leaf_rows, t->leaf_cnt, lc,
                                                            li, mk, mv, is_start, run_start, run_len,
                                                            run_leaf, nm, run_parent, mark);
    note_launch();
    if (hf & 1u) {
      const size_t smem = (size_t)t->cfg.fanout * lc * sizeof(longlong2);
      rc = opt_in_smem((const void *)subtree_rebalance_kernel, 128 * 64 * (int)sizeof(longlong2));  // up to 128 KiB
      if (rc) return rc;
      subtree_rebalance_kernel<<<(unsigned)last_nodes, kThreads, smem, s>>>(
          t->inner, t->prefix, t->leaf_rows, t->leaf_cnt, t->leaf_base, t->cfg.fanout, lc, li, g, mark, mk, mv, ml,
          nm);
      note_launch();
      t->shape_version++;  // separators of the last inner level changed
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_err(e);
    }
    exclusive_scan_i32(t->leaf_cnt, lbase_tmp, t->n_leaf, scan_scratch, s);
    cudaMemcpyAsync(t->leaf_base, lbase_tmp, 8 * t->n_leaf, cudaMemcpyDeviceToDevice, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(e);
    t->n_keys += nm;
  } else {
    // Rebuild: contents (already carrying this epoch's in-place updates)
    // merged with the misses, then a bulk load into a fresh arena.
    const int64_t n0 = t->n_keys, n1 = n0 + nm;
    const int64_t tn = std::max<int64_t>(n1, 1);
    char *tmp = nullptr;
    e = dev_alloc(reinterpret_cast<void **>(&tmp), 4 * al(8 * tn));
    if (e != cudaSuccess) return cuda_err(e);
    int64_t *ek = reinterpret_cast<int64_t *>(tmp);
    int64_t *ev = reinterpret_cast<int64_t *>(tmp + al(8 * tn));
    uint64_t *ck = reinterpret_cast<uint64_t *>(tmp + 2 * al(8 * tn));
    int64_t *cv = reinterpret_cast<int64_t *>(tmp + 3 * al(8 * tn));
    export_contents(t, ek, ev, s);
    merge_rank_kernel<<<grid_for(n0), kThreads, 0, s>>>(ek, ev, n0, mk, nm, true, ck, cv);
    merge_rank_kernel<<<grid_for(nm), kThreads, 0, s>>>(mk, mv, nm, ek, n0, true, ck, cv);
    note_launch(2);
    rc = rebuild_from_sorted(t, ck, cv, n1, s);
    release_after(tmp, s);
    if (rc) return rc;
  }
  if (t->n_keys == nm || new_ends[0] < t->key_min) t->key_min = new_ends[0];
  if (t->n_keys == nm || new_ends[1] > t->key_max) t->key_max = new_ends[1];
  return HM_OK;
}

// One epoch of deletes (no counterpart in the reference, whose
// BPlusTree::remove is an empty stub, open-harmonia/src/bpt.cpp:771-773):
// sort the batch and drop repeats, mark each stored key's slot, compact the
// touched leaves in place and rescan leaf_base.  Separators stay valid (the
// remaining keys of leaf j still lie between its separators), so the inner
// levels are untouched.  A leaf left empty would break the invariant that
// every leaf's first key is a key of the leaf (the bucket join searches
// leaves by first key), so such an epoch ends in a rebuild of the remaining
// contents instead.
int delete_epoch(hm_tree *t, const int64_t *d_keys, int64_t n, int64_t *removed_out, cudaStream_t s) {
  if (removed_out) *removed_out = 0;
  if (n <= 0) return HM_OK;
  if (n > kMaxEpochKeys) return HM_ETOOLARGE;
  const int lc = t->cfg.leaf_cap, li = t->leaf_index, f = t->cfg.fanout;
  const size_t s8 = al(8 * (n + 1)), s4 = al(4 * (n + 1));
  const int64_t scan_n = std::max<int64_t>(n, t->n_leaf) + 1;
  const size_t lb8 = al(8 * (t->n_leaf + 1));
  size_t need = 6 * s8 + 2 * s4 + lb8 + al((int64_t)radix_scratch_bytes(n)) +
                al((int64_t)scan_scratch_bytes(scan_n)) + 256;
  ScratchLease lease(t, s);
  int rc = lease.acquire(need);
  if (rc) return rc;
  char *p = static_cast<char *>(lease.ptr());
  auto take8 = [&](void) { char *r = p; p += s8; return r; };
  auto take4 = [&](void) { char *r = p; p += s4; return r; };
  uint64_t *uk = reinterpret_cast<uint64_t *>(take8());
  uint64_t *uk_alt = reinterpret_cast<uint64_t *>(take8());
  int32_t *idx = reinterpret_cast<int32_t *>(take8());
  int32_t *idx_alt = reinterpret_cast<int32_t *>(take8());
  int64_t *at = reinterpret_cast<int64_t *>(take8());
  int64_t *bk = reinterpret_cast<int64_t *>(take8());
  int32_t *keep = reinterpret_cast<int32_t *>(take4());
  int32_t *route = reinterpret_cast<int32_t *>(take4());
  void *sort_scratch = p;
  p += al((int64_t)radix_scratch_bytes(n));
  int64_t *lbase_tmp = reinterpret_cast<int64_t *>(p);  // n_leaf + 1 entries
  p += lb8;
  void *scan_scratch = p;
  p += al((int64_t)scan_scratch_bytes(scan_n));
  unsigned long long *dremoved = reinterpret_cast<unsigned long long *>(p);
  unsigned *dflags = reinterpret_cast<unsigned *>(p + 8);

  cudaMemsetAsync(p, 0, 16, s);
  if (n <= kSmallSort) {
    small_sort_unique_kernel<<<1, 1024, 0, s>>>(d_keys, nullptr, (int)n, bk, nullptr, at + n, dflags);
    note_launch();
  } else {
    transform_keys_in(d_keys, uk, n, s);
    if (radix_sort_positions(uk, idx, uk_alt, idx_alt, n, 0, 64, sort_scratch, s)) std::swap(uk, uk_alt);
    last_occurrence_kernel<<<grid_for(n), kThreads, 0, s>>>(uk, n, keep, dflags);
    exclusive_scan_i32(keep, at, n, scan_scratch, s);
    compact_keys_kernel<<<grid_for(n), kThreads, 0, s>>>(uk, keep, at, n, bk);
    note_launch(2);
  }
  int64_t m = 0;
  cudaMemcpyAsync(&m, at + n, 8, cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);

  delete_mark_kernel<<<grid_for(m), kThreads, 0, s>>>(t->view(), f, lc, li, bk, m, t->leaf_rows, route);
  cudaMemsetAsync(dflags, 0, 4, s);  // the Max_Key bit of the dedup pass is not an error here
  delete_compact_kernel<<<grid_for(m), kThreads, 0, s>>>(t->leaf_rows, t->leaf_cnt, lc, li, route, m, dremoved,
                                                          dflags);
  note_launch(2);
  unsigned long long removed = 0;
  unsigned hf = 0;
  cudaMemcpyAsync(&removed, dremoved, 8, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&hf, dflags, 4, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);
  if (removed_out) *removed_out = (int64_t)removed;
  if (removed == 0) return HM_OK;
  exclusive_scan_i32(t->leaf_cnt, lbase_tmp, t->n_leaf, scan_scratch, s);
  cudaMemcpyAsync(t->leaf_base, lbase_tmp, 8 * t->n_leaf, cudaMemcpyDeviceToDevice, s);
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);
  t->n_keys -= (int64_t)removed;
  if (!(hf & 1u)) return HM_OK;
  // a leaf emptied: rebuild from the remaining contents
  const int64_t n1 = t->n_keys, tn = std::max<int64_t>(n1, 1);
  char *tmp = nullptr;
  e = dev_alloc(reinterpret_cast<void **>(&tmp), 3 * al(8 * tn));
  if (e != cudaSuccess) return cuda_err(e);
  int64_t *ek = reinterpret_cast<int64_t *>(tmp);
  int64_t *ev = reinterpret_cast<int64_t *>(tmp + al(8 * tn));
  uint64_t *ck = reinterpret_cast<uint64_t *>(tmp + 2 * al(8 * tn));
  export_contents(t, ek, ev, s);
  if (n1 > 0) transform_keys_in(ek, ck, n1, s);
  rc = rebuild_from_sorted(t, ck, ev, n1, s);
  release_after(tmp, s);
  return rc;
}

}  // namespace hm
