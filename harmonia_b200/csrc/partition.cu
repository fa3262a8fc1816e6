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

// Scatter with shared-memory staging: each 4096-query tile is first grouped
// by digit in shared memory, then written out so that consecutive threads
// write consecutive slots of one bucket (coalesced runs instead of one
// scattered 8-B store per query).
constexpr int kTile = 4096;
constexpr int kPerThread = kTile / kThreads;

__global__ void __launch_bounds__(kThreads) scatter_kernel(const int64_t *__restrict__ q, int64_t n,
                                                           int64_t seg, Digit dg, int nb,
                                                           const int64_t *__restrict__ offsets,
                                                           int nctas, int64_t *__restrict__ q_out,
                                                           int32_t *__restrict__ pos_out) {
  extern __shared__ __align__(16) unsigned char sm[];
  int64_t *sk = reinterpret_cast<int64_t *>(sm);                     // kTile keys
  int32_t *sp = reinterpret_cast<int32_t *>(sm + kTile * 8);         // kTile positions
  unsigned *cursor = reinterpret_cast<unsigned *>(sm + kTile * 12);  // nb: global next slot
  unsigned *tcount = cursor + nb;                                    // nb: tile histogram
  unsigned *tstart = tcount + nb;                                    // nb: tile scan / rank cursor
  unsigned *tbase = tstart + nb;                                     // nb: tile scan (kept)
  __shared__ unsigned wsum[kThreads / 32];
  for (int d = threadIdx.x; d < nb; d += kThreads) {
    cursor[d] = (unsigned)offsets[(int64_t)d * nctas + blockIdx.x];
    tcount[d] = 0;
  }
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t t0 = b0; t0 < b1; t0 += kTile) {
    int64_t k[kPerThread];
    int dig[kPerThread];
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
      int64_t i = t0 + j * kThreads + threadIdx.x;
      k[j] = i < b1 ? __ldg(q + i) : 0;
      dig[j] = i < b1 ? dg(k[j]) : -1;
      if (dig[j] >= 0) atomicAdd(&tcount[dig[j]], 1u);
    }
    __syncthreads();
    // exclusive scan of the tile histogram (nb <= 4096 bins, kThreads threads)
    const int per = (nb + kThreads - 1) / kThreads;
    unsigned run = 0;
    for (int x = 0; x < per; x++) {
      int d = threadIdx.x * per + x;
      if (d < nb) run += tcount[d];
    }
    unsigned incl = run;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    unsigned before = incl - run;
    for (int x = 0; x < w; x++) before += wsum[x];
    for (int x = 0; x < per; x++) {
      int d = threadIdx.x * per + x;
      if (d < nb) {
        tstart[d] = before;
        tbase[d] = before;
        before += tcount[d];
      }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPerThread; j++) {
      if (dig[j] >= 0) {
        unsigned slot = atomicAdd(&tstart[dig[j]], 1u);
        sk[slot] = k[j];
        sp[slot] = (int32_t)(t0 + j * kThreads + threadIdx.x);
      }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kTile, b1 - t0);
    for (int i = threadIdx.x; i < cnt; i += kThreads) {
      int64_t key = sk[i];
      int d = dg(key);
      unsigned o = cursor[d] + (unsigned)i - tbase[d];
      q_out[o] = key;
      pos_out[o] = sp[i];
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nb; d += kThreads) {
      cursor[d] += tcount[d];
      tcount[d] = 0;
    }
    __syncthreads();
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
  const int64_t m = ((int64_t)1 << bits) * part_ctas(n);
  return sizeof(int64_t) * (size_t)(m + 1) + scan_scratch_bytes(m) + 256;
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
  const size_t smem = (size_t)kTile * 12 + (size_t)nb * 16;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_err(e);
  }
  scatter_kernel<<<nctas, kThreads, smem, s>>>(q, n, seg, dg, nb, counts, nctas, q_out, pos_out);
  note_launch(2);
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
