// Query pre-sort (the reference's PSA, "partially sorted aggregation"):
// partition a batch of queries by the top `bits` bits of their key, relative
// to the tree's key range, and carry each query's original position along.
//
// The reference runs cub::DeviceRadixSort::SortPairs on bits [48,64) of
// (key, pos) before every search launch
// (open-harmonia/src/full-multi-prefix-sort-8thread.cu:305-309,
// open-harmonia/regular_bpt/prefix-sort.cu:288-293) and scatters results back
// through the permutation on the host.  Here it is one histogram pass and one
// scatter pass; the order inside a bucket is not kept (the search writes each
// result to out[pos], so it does not matter), which lets the scatter take its
// slots with shared-memory atomics instead of a stable rank.  The digit is
// taken relative to [key_min, key_max] of the tree so that all 2^bits buckets
// cover loaded keys (the reference's fixed bits [48,64) leave half of them
// empty for non-negative keys).
#include "hm_internal.cuh"

namespace hm {

void scan_counts(int64_t *counts, int64_t m, cudaStream_t s);

namespace {

constexpr int kThreads = 256;

struct Digit {
  int64_t lo, hi;
  int shift;
  int maxd;
  __device__ __forceinline__ int operator()(int64_t k) const {
    if (k <= lo) return 0;
    if (k >= hi) return maxd;
    return (int)((uint64_t)(k - lo) >> shift);
  }
};

int part_ctas(int64_t n) {
  int64_t c = (n + 8191) / 8192;
  if (c > 148 * 4) c = 148 * 4;
  if (c < 1) c = 1;
  return (int)c;
}

__global__ void __launch_bounds__(kThreads) hist_kernel(const int64_t *__restrict__ q, int64_t n,
                                                        int64_t seg, Digit dg, int nb,
                                                        int64_t *__restrict__ counts, int nctas) {
  extern __shared__ unsigned hist[];
  for (int i = threadIdx.x; i < nb; i += kThreads) hist[i] = 0;
  __syncthreads();
  int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kThreads) atomicAdd(&hist[dg(__ldg(q + i))], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < nb; d += kThreads) counts[(int64_t)d * nctas + blockIdx.x] = hist[d];
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(const int64_t *__restrict__ q, int64_t n,
                                                           int64_t seg, Digit dg, int nb,
                                                           const int64_t *__restrict__ offsets,
                                                           int nctas, int64_t *__restrict__ q_out,
                                                           int32_t *__restrict__ pos_out) {
  extern __shared__ unsigned long long cursor[];
  for (int d = threadIdx.x; d < nb; d += kThreads)
    cursor[d] = (unsigned long long)offsets[(int64_t)d * nctas + blockIdx.x];
  __syncthreads();
  int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kThreads) {
    int64_t k = __ldg(q + i);
    unsigned long long o = atomicAdd(&cursor[dg(k)], 1ull);
    q_out[o] = k;
    pos_out[o] = (int32_t)i;
  }
}

Digit make_digit(const hm_tree *t, int bits) {
  Digit d;
  d.lo = t->key_min;
  d.hi = t->key_max;
  d.maxd = (1 << bits) - 1;
  uint64_t range = (uint64_t)t->key_max - (uint64_t)t->key_min;
  int len = 0;
  while (len < 64 && (range >> len) != 0) len++;
  d.shift = len > bits ? len - bits : 0;
  return d;
}

}  // namespace

size_t partition_scratch_bytes(int64_t n, int bits) {
  return sizeof(int64_t) * ((size_t)1 << bits) * part_ctas(n) + 256;
}

int partition_queries(const hm_tree *t, const int64_t *q, int64_t n, int bits, int64_t *q_out,
                      int32_t *pos_out, void *scratch, cudaStream_t s) {
  if (bits < 1 || bits > 12 || n > INT32_MAX) return HM_EINVAL;
  const int nb = 1 << bits;
  const int nctas = part_ctas(n);
  const int64_t seg = (n + nctas - 1) / nctas;
  int64_t *counts = static_cast<int64_t *>(scratch);
  Digit dg = make_digit(t, bits);
  hist_kernel<<<nctas, kThreads, nb * sizeof(unsigned), s>>>(q, n, seg, dg, nb, counts, nctas);
  scan_counts(counts, (int64_t)nb * nctas, s);
  scatter_kernel<<<nctas, kThreads, nb * sizeof(unsigned long long), s>>>(q, n, seg, dg, nb, counts,
                                                                        nctas, q_out, pos_out);
  note_launch(2);
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
