// Comparison kernel, not the product path: a pointer-chasing descent in the
// style of the reference's HB+ GPU search (open-harmonia/src/gbpt.cu:30-113,
// open-harmonia/regular_bpt/noprefix-nosort.cu:89).  Every inner node keeps
// its children's ids and a query follows them, one dependent load per level
// after the node's compare, with no prefix-sum child array and no pre-sort.
// It reads the same key rows and leaves as the product kernels, so the
// difference in a report is the layout and the search, not the data.
#include "hm_internal.cuh"

#include <mutex>

#include <algorithm>

namespace hm {

namespace {

constexpr int kThreads = 256;

struct Levels {
  int64_t start[kMaxLevels + 1];
  int height;
  int64_t n_inner, n_leaf;
};

// child_ids[p * f + c] = id of child c of inner node p, -1 past its last.
__global__ void child_ids_kernel(const int32_t *__restrict__ prefix, Levels lv, int f, int32_t *__restrict__ ids) {
  const int64_t total = lv.n_inner * f;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total;
       x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = x / f;
    const int c = (int)(x - p * f);
    int l = 0;
    while (l + 1 < lv.height && lv.start[l + 1] <= p) l++;
    const int64_t level_end = lv.start[l + 1];
    const int64_t next_end = l + 2 <= lv.height ? lv.start[l + 2] : lv.n_inner + lv.n_leaf;
    const int64_t c0 = prefix[p], c1 = p + 1 < level_end ? prefix[p + 1] : next_end;
    ids[x] = c < c1 - c0 ? (int32_t)(c0 + c) : -1;
  }
}

// One thread per query: index compare, slice compare, then the child id.
__global__ void __launch_bounds__(kThreads) pointer_search_kernel(const int64_t *__restrict__ inner,
                                                                  const int32_t *__restrict__ ids,
                                                                  const int64_t *__restrict__ leaf_rows, int height,
                                                                  int64_t n_inner, int f, int lc, int li,
                                                                  const int64_t *__restrict__ q, int64_t n,
                                                                  int64_t *__restrict__ out) {
  const int ix = f / 8, row = ix + f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t key = __ldg(q + i);
    if (key == kMaxKey) {
      out[i] = HM_NOT_FOUND;
      continue;
    }
    int64_t node = 0;
    for (int l = 0; l < height; l++) {
      const int64_t *r = inner + node * row;
      int k = 0;
      for (int v = 0; v < ix / 2; v++) {
        const longlong2 p = __ldg(reinterpret_cast<const longlong2 *>(r + 2 * v));
        k += (p.x <= key) + (p.y <= key);
      }
      k = min(k, ix - 1);
      int c = 8 * k;
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const longlong2 p = __ldg(reinterpret_cast<const longlong2 *>(r + ix + 8 * k + 2 * v));
        c += (p.x <= key) + (p.y <= key);
      }
      node = __ldg(ids + node * f + c);  // the pointer chase
    }
    const int64_t *kr = leaf_rows + (node - n_inner) * (li + 2 * lc) + li;
    int64_t v = HM_NOT_FOUND;
    for (int s = 0; s < lc; s++)
      if (__ldg(kr + s) == key) v = __ldg(kr + lc + s);
    out[i] = v;
  }
}

}  // namespace

}  // namespace hm

using namespace hm;

extern "C" int hm_search_baseline(hm_tree *t, int kind, const int64_t *q, size_t n_, int64_t *out, hm_stream hs) {
  if (!t || kind != HM_BASELINE_POINTER || (n_ > 0 && (!q || !out))) return HM_EINVAL;
  const int64_t n = (int64_t)n_;
  if (n == 0) return HM_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(hs);
  const int f = t->cfg.fanout;
  // The child ids are built once per arena, under the tree's lock; a caller on
  // another stream that finds them built waits for the build's event.
  std::unique_lock<std::mutex> lk(t->mu);
  if (t->child_ids && t->child_ids_generation == t->generation) {
    cudaError_t e = cudaStreamWaitEvent(s, t->child_ids_ready, 0);
    if (e != cudaSuccess) return cuda_err(e);
  } else {
    if (t->child_ids) cudaFree(t->child_ids);
    t->child_ids = nullptr;
    cudaError_t e = cudaSuccess;
    if (!t->child_ids_ready) e = cudaEventCreateWithFlags(&t->child_ids_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&t->child_ids, (size_t)std::max<int64_t>(t->n_inner * f, 1) * 4);
    if (e != cudaSuccess) {
      t->child_ids = nullptr;
      return cuda_err(e);
    }
    Levels lv;
    for (int l = 0; l <= kMaxLevels; l++) lv.start[l] = t->lvl_start[l];
    lv.height = t->height;
    lv.n_inner = t->n_inner;
    lv.n_leaf = t->n_leaf;
    const int64_t total = t->n_inner * f;
    const unsigned grid = (unsigned)std::min<int64_t>((total + kThreads - 1) / kThreads + 1, 148 * 32);
    child_ids_kernel<<<grid, kThreads, 0, s>>>(t->prefix, lv, f, t->child_ids);
    note_launch();
    e = cudaEventRecord(t->child_ids_ready, s);
    if (e != cudaSuccess) {
      cudaFree(t->child_ids);
      t->child_ids = nullptr;
      return cuda_err(e);
    }
    t->child_ids_generation = t->generation;
  }
  lk.unlock();
  const unsigned grid = (unsigned)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)t->num_sms * 8);
  pointer_search_kernel<<<grid, kThreads, 0, s>>>(t->inner, t->child_ids, t->leaf_rows, t->height, t->n_inner, f,
                                                  t->cfg.leaf_cap, t->leaf_index, q, n, out);
  note_launch();
  return cuda_err(cudaGetLastError());
}
