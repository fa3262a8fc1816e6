// Device-wide exclusive scan, export of the tree contents, and the range scan
// with prefix-sum output compaction.
//
// Range reference: range_prefix_sort_1thread_search_1_thread_scan_kernel
// (open-harmonia/src/range.cu:101-227) descends with the start key and copies
// up to Range_Size = 8 records into fixed per-query slots (no compaction),
// with the end key forced to Max_Key (open-harmonia/src/range.cu:349-355).
// Here a query asks for the first len[i] records with key >= start[i], or
// (inclusive form) every record with start[i] <= key <= end[i]; a locate pass
// descends and computes each query's count, an exclusive scan
// turns counts into offsets, and a copy pass (one warp per query) writes the
// records contiguously: leaves are ordered, so the records of a query are the
// key-ordered run that starts at (leaf, slot) and continues in leaf+1, ...
#include "hm_internal.cuh"

namespace hm {

namespace {

constexpr int kThreads = 256;

int scan_ctas(int64_t n) {
  int64_t c = (n + 4095) / 4096;
  if (c > 148 * 4) c = 148 * 4;
  if (c < 1) c = 1;
  return (int)c;
}

constexpr int kScanPer = 8;                    // elements per thread per scan step
constexpr int kScanStep = kThreads * kScanPer;  // elements per CTA per scan step

template <typename T>
__global__ void __launch_bounds__(kThreads) seg_sum_kernel(const T *__restrict__ in, int64_t n,
                                                           int64_t seg, int64_t *__restrict__ part) {
  pdl_enter();
  __shared__ int64_t red[kThreads / 32];
  int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  int64_t s = 0;
  for (int64_t base = b0; base < b1; base += kScanStep) {
    T v[kScanPer];
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {  // all loads first
      const int64_t i = base + j * kThreads + threadIdx.x;
      v[j] = i < b1 ? in[i] : (T)0;
    }
#pragma unroll
    for (int j = 0; j < kScanPer; j++) s += (int64_t)v[j];
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += red[w];
    part[blockIdx.x] = t;
  }
}

// Exclusive scan of each segment, offset by the sum of the segments before it
// (each CTA adds up those of the at most 592 segment sums itself).  A step
// stages kScanStep elements in shared memory (coalesced), each thread scans
// kScanPer consecutive ones (index i at i + i / 8: one pad word per 8 keeps
// the threads' runs in different banks), one block scan of the thread sums.
template <typename T>
__global__ void __launch_bounds__(kThreads) seg_scan_kernel(const T *__restrict__ in, int64_t n,
                                                            int64_t seg, const int64_t *__restrict__ part,
                                                            int64_t *__restrict__ out, int nctas) {
  pdl_enter();
  __shared__ int64_t buf[kScanStep + kScanStep / 8];
  __shared__ int64_t wsum[kThreads / 32];
  __shared__ int64_t carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  {
    int64_t before = 0;
    for (int i = tid; i < (int)blockIdx.x; i += kThreads) before += part[i];
    for (int o = 16; o; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
    if (lane == 0) wsum[warp] = before;
    __syncthreads();
    if (tid == 0) {
      int64_t c = 0;
      for (int w = 0; w < kThreads / 32; w++) c += wsum[w];
      carry = c;
    }
    __syncthreads();
  }
  for (int64_t base = b0; base < b1; base += kScanStep) {
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
      const int e = j * kThreads + tid;
      const int64_t i = base + e;
      buf[e + (e >> 3)] = i < b1 ? (int64_t)in[i] : 0;
    }
    __syncthreads();
    int64_t x[kScanPer], local = 0;
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
      x[j] = buf[tid * (kScanPer + 1) + j];
      local += x[j];
    }
    int64_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int64_t run = carry + incl - local;
    for (int w = 0; w < warp; w++) run += wsum[w];
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
      buf[tid * (kScanPer + 1) + j] = run;
      run += x[j];
    }
    __syncthreads();
    if (tid == kThreads - 1) carry = run;
#pragma unroll
    for (int j = 0; j < kScanPer; j++) {
      const int e = j * kThreads + tid;
      const int64_t i = base + e;
      if (i < b1) out[i] = buf[e + (e >> 3)];
    }
    __syncthreads();
  }
  if (blockIdx.x == nctas - 1 && tid == 0) out[n] = carry;
}

__global__ void export_kernel(DevTree t, int lc, int li, int64_t *__restrict__ keys,
                              int64_t *__restrict__ vals) {
  const int64_t total = (int64_t)t.n_leaf * lc;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = x / lc;
    int s = (int)(x - j * lc);
    if (s < t.leaf_cnt[j]) {
      int64_t o = t.leaf_base[j] + s;
      const int64_t *r = t.leaf_rows + j * (li + 2 * lc) + li;
      keys[o] = r[s];
      vals[o] = r[lc + s];
    }
  }
}

// One thread per query: descend with the start key, take its lower bound in
// the leaf (global rank g through leaf_base).  Length form (end == nullptr):
// count = min(len, keys from g to the end).  Inclusive form: a second descent
// with the end key gives the global rank of its upper bound (keys <= end: the
// leaves before the end key's leaf hold only smaller keys, the ones after only
// larger, because separators fence the leaves), count = that rank - g, and
// nothing when end < start (BPlusTree::range_search,
// open-harmonia/src/bpt.cpp:695-769).  The end key Max_Key reaches the end of
// the key space without a descent.
__global__ void range_locate_kernel(DevTree t, int f, int lc, int li, const int64_t *__restrict__ start,
                                    const int32_t *__restrict__ len, const int64_t *__restrict__ end,
                                    int64_t n, int32_t *__restrict__ first_leaf,
                                    int32_t *__restrict__ first_slot, int64_t *__restrict__ count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = __ldg(start + i);
    const int64_t e = end ? __ldg(end + i) : 0;
    const bool empty = end ? (e < s) : (__ldg(len + i) <= 0);
    if (empty || s == kMaxKey || t.n_keys == 0) {
      first_leaf[i] = 0;
      first_slot[i] = 0;
      count[i] = 0;
      continue;
    }
    int32_t leaf = descend_leaf(t, f, s);
    const int64_t *kr = t.leaf_rows + (int64_t)leaf * (li + 2 * lc) + li;
    int cnt = __ldg(t.leaf_cnt + leaf);
    int lb = 0;  // first slot with key >= start
    while (lb < cnt && __ldg(kr + lb) < s) lb++;
    int64_t g = __ldg(t.leaf_base + leaf) + lb;
    first_leaf[i] = leaf;
    first_slot[i] = lb;
    if (end) {
      int64_t g_end = t.n_keys;  // global rank of the first key > end
      if (e != kMaxKey) {
        const int32_t le = descend_leaf(t, f, e);
        const int64_t *ke = t.leaf_rows + (int64_t)le * (li + 2 * lc) + li;
        const int ce = __ldg(t.leaf_cnt + le);
        int ub = 0;
        while (ub < ce && __ldg(ke + ub) <= e) ub++;
        g_end = __ldg(t.leaf_base + le) + ub;
      }
      count[i] = g_end > g ? g_end - g : 0;
    } else {
      const int64_t want = __ldg(len + i), rem = t.n_keys - g;
      count[i] = want < rem ? want : rem;
    }
  }
}

// One warp per query.  The records of a query are the global ranks
// [g0, g0 + count) in key order (g0 = leaf_base[first leaf] + first slot).
// Per window of 32 leaves the warp loads their leaf_base entries (one
// coalesced load); each lane finds the leaf of its record by a 5-step shuffle
// search (the last leaf of the window whose base is <= the rank), so the
// loads of all records are independent (no walk leaf by leaf).
__global__ void range_copy_kernel(DevTree t, int lc, int li, const int32_t *__restrict__ first_leaf,
                                  const int32_t *__restrict__ first_slot,
                                  const int64_t *__restrict__ offsets, int64_t n,
                                  int64_t *__restrict__ okeys, int64_t *__restrict__ ovals) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  const int row = li + 2 * lc;
  int64_t i = blockIdx.x * (int64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
  // the next query's header is loaded while the current one is copied
  int64_t o_n = 0, e_n = 0, L_n = 0, s_n = 0;
  if (i < n) {
    o_n = offsets[i];
    e_n = offsets[i + 1];
    L_n = first_leaf[i];
    s_n = first_slot[i];
  }
  for (; i < n; i += warps) {
    const int64_t o = o_n, rem = e_n - o_n, s0 = s_n;
    int64_t L = L_n;
    if (i + warps < n) {
      o_n = offsets[i + warps];
      e_n = offsets[i + warps + 1];
      L_n = first_leaf[i + warps];
      s_n = first_slot[i + warps];
    }
    if (rem <= 0) continue;  // uniform across the warp
    const int64_t g0 = __ldg(t.leaf_base + L) + s0;
    int64_t x0 = 0;
    while (x0 < rem) {
      const int64_t lb = L + lane < t.n_leaf ? __ldg(t.leaf_base + L + lane) : t.n_keys;
      const int64_t wend = L + 32 < t.n_leaf ? __ldg(t.leaf_base + L + 32) : t.n_keys;
      const int64_t xe = min(rem, wend - g0);  // this window holds records [x0, xe)
      for (int64_t xb = x0; xb < xe; xb += 32) {
        const int64_t x = xb + lane;
        const int64_t r = g0 + x;
        int j = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const int64_t v = __shfl_sync(0xffffffffu, lb, j + step);
          if (v <= r) j += step;
        }
        const int64_t base = __shfl_sync(0xffffffffu, lb, j);
        if (x < xe) {
          const int64_t *kr = t.leaf_rows + (L + j) * row + li + (r - base);
          okeys[o + x] = __ldg(kr);
          ovals[o + x] = __ldg(kr + lc);
        }
      }
      x0 = xe;
      L += 32;
    }
  }
}

unsigned grid_for_items(int64_t items, unsigned cap) {
  int64_t b = (items + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

}  // namespace

size_t scan_scratch_bytes(int64_t n) { return sizeof(int64_t) * (scan_ctas(n) + 8); }

template <typename T>
void exclusive_scan(const T *in, int64_t *out, int64_t n, void *scratch, cudaStream_t s) {
  const int nctas = scan_ctas(n);
  const int64_t seg = (n + nctas - 1) / nctas;
  int64_t *part = static_cast<int64_t *>(scratch);
  if (n == 0) {
    cudaMemsetAsync(out, 0, sizeof(int64_t), s);
    return;
  }
  launch_pdl(seg_sum_kernel<T>, nctas, kThreads, 0, s, in, n, seg, part);
  launch_pdl(seg_scan_kernel<T>, nctas, kThreads, 0, s, in, n, seg, part, out, nctas);
  note_launch(2);
}


void exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *scratch, cudaStream_t s) {
  exclusive_scan<int64_t>(in, out, n, scratch, s);
}

void exclusive_scan_i32(const int32_t *in, int64_t *out, int64_t n, void *scratch, cudaStream_t s) {
  exclusive_scan<int32_t>(in, out, n, scratch, s);
}

void export_contents(const hm_tree *t, int64_t *d_keys, int64_t *d_vals, cudaStream_t s) {
  if (t->n_keys == 0) return;
  export_kernel<<<grid_for_items(t->n_leaf * t->cfg.leaf_cap, 148u * 32), kThreads, 0, s>>>(
      t->view(), t->cfg.leaf_cap, t->leaf_index, d_keys, d_vals);
  note_launch();
}

size_t range_scratch_bytes(int64_t n) {
  return (size_t)align_up(n * 4, 256) * 2 + (size_t)align_up(n * 8, 256) + scan_scratch_bytes(n) + 256;
}

int range_locate(const hm_tree *t, const int64_t *start, const int32_t *len, const int64_t *end, int64_t n,
                 int32_t *first_leaf, int32_t *first_slot, int64_t *count, cudaStream_t s) {
  range_locate_kernel<<<grid_for_items(n, 148u * 16), kThreads, 0, s>>>(
      t->view(), t->cfg.fanout, t->cfg.leaf_cap, t->leaf_index, start, len, end, n, first_leaf,
      first_slot, count);
  note_launch();
  return cuda_err(cudaGetLastError());
}

int range_copy_out(const hm_tree *t, const int32_t *first_leaf, const int32_t *first_slot,
                   const int64_t *offsets, int64_t n, int64_t *okeys, int64_t *ovals, cudaStream_t s) {
  int64_t warps = n;
  int64_t blocks = (warps + (kThreads / 32) - 1) / (kThreads / 32);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  range_copy_kernel<<<(unsigned)blocks, kThreads, 0, s>>>(t->view(), t->cfg.leaf_cap, t->leaf_index,
                                                         first_leaf, first_slot, offsets, n, okeys,
                                                         ovals);
  note_launch();
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
