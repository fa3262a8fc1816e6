// One stable counting-sort pass over 8-bit digits: the building block of the
// radix sort (bulk load, upsert epochs) and of the query pre-sort.
//
//   hist_kernel     each CTA counts the digits of its contiguous segment
//                   -> counts[digit][cta]
//   (scan)          exclusive scan of counts in digit-major order
//   scatter_kernel  each CTA re-reads its segment in 2048-element tiles:
//                   ranks every element inside the tile (per-warp
//                   __match_any_sync + per-warp digit counters + a cross-warp
//                   prefix), stages the tile in shared memory grouped by
//                   digit, then writes it out so that consecutive threads
//                   store consecutive slots of one digit's run.
// Elements of one digit keep their input order (warp, round, lane order is
// element order), so passes compose into an LSD radix sort.
#pragma once

#include "hm_internal.cuh"

namespace hm {
namespace radix {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRounds = 8;                       // rounds of 32 per warp per tile
constexpr int kTile = kWarps * 32 * kRounds;     // 2048 elements
constexpr int kBins = 256;
constexpr int kMaxCtas = 148 * 8;

inline int ctas_for(int64_t n) {
  int64_t c = (n + kTile - 1) / kTile;
  if (c > kMaxCtas) c = kMaxCtas;
  if (c < 1) c = 1;
  return (int)c;
}

template <typename K, typename Digit>
__global__ void __launch_bounds__(kThreads) hist_kernel(const K *__restrict__ keys, int64_t n, int64_t seg,
                                                        Digit dg, int64_t *__restrict__ counts, int nctas) {
  pdl_enter();
  __shared__ unsigned hist[kWarps][kBins];
  const int w = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWarps * kBins; i += kThreads) (&hist[0][0])[i] = 0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kThreads) atomicAdd(&hist[w][dg(keys[i])], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < kBins; d += kThreads) {
    unsigned c = 0;
#pragma unroll
    for (int x = 0; x < kWarps; x++) c += hist[x][d];
    counts[(int64_t)d * nctas + blockIdx.x] = c;
  }
}

// GEN_VAL: the payload is the element's input position (vals is ignored).
template <typename K, typename V, typename Digit, bool GEN_VAL>
__global__ void __launch_bounds__(kThreads) scatter_kernel(const K *__restrict__ keys, const V *__restrict__ vals,
                                                           K *__restrict__ keys_out, V *__restrict__ vals_out,
                                                           int64_t n, int64_t seg, Digit dg,
                                                           const int64_t *__restrict__ offsets, int nctas) {
  pdl_enter();
  __shared__ unsigned wcnt[kWarps][kBins + 1];  // bin kBins collects invalid lanes
  __shared__ unsigned tstart[kBins];
  __shared__ unsigned dcount[kBins];
  __shared__ unsigned wsum[kWarps];
  __shared__ int64_t gcur[kBins];
  __shared__ K sk[kTile];
  __shared__ V sv[kTile];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int d = tid; d < kBins; d += kThreads) gcur[d] = offsets[(int64_t)d * nctas + blockIdx.x];
  for (int i = tid; i < kWarps * (kBins + 1); i += kThreads) (&wcnt[0][0])[i] = 0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t tile = b0; tile < b1; tile += kTile) {
    K k[kRounds];
    V v[kRounds];
    int dig[kRounds];
    unsigned loc[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      const int64_t e = tile + w * (32 * kRounds) + r * 32 + lane;
      const bool valid = e < b1;
      k[r] = valid ? keys[e] : K(0);
      if constexpr (GEN_VAL) {
        v[r] = (V)e;
      } else {
        v[r] = valid ? vals[e] : V(0);
      }
      dig[r] = valid ? dg(k[r]) : kBins;
    }
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      const unsigned peers = __match_any_sync(0xffffffffu, dig[r]);
      const unsigned base = wcnt[w][dig[r]];
      __syncwarp();
      if ((peers & lt_mask) == 0) wcnt[w][dig[r]] = base + __popc(peers);
      __syncwarp();
      loc[r] = base + __popc(peers & lt_mask);
    }
    __syncthreads();
    // per digit: exclusive offsets of the warps and the tile count
    unsigned cnt_d = 0;
    if (tid < kBins) {
#pragma unroll
      for (int x = 0; x < kWarps; x++) {
        const unsigned c = wcnt[x][tid];
        wcnt[x][tid] = cnt_d;
        cnt_d += c;
      }
      dcount[tid] = cnt_d;
    }
    // exclusive scan of the tile counts over the 256 digits
    unsigned incl = cnt_d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (tid < kBins) {
      unsigned before = incl - cnt_d;
      for (int x = 0; x < w; x++) before += wsum[x];
      tstart[tid] = before;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
      if (dig[r] < kBins) {
        const unsigned p = tstart[dig[r]] + wcnt[w][dig[r]] + loc[r];
        sk[p] = k[r];
        sv[p] = v[r];
      }
    }
    __syncthreads();
    const int cnt = (int)min((int64_t)kTile, b1 - tile);
    for (int p = tid; p < cnt; p += kThreads) {
      const K key = sk[p];
      const int d = dg(key);
      const int64_t o = gcur[d] + (p - (int)tstart[d]);
      keys_out[o] = key;
      vals_out[o] = sv[p];
    }
    __syncthreads();
    if (tid < kBins) {
      gcur[tid] += dcount[tid];
#pragma unroll
      for (int x = 0; x < kWarps; x++) wcnt[x][tid] = 0;
    }
    if (tid < kWarps) wcnt[tid][kBins] = 0;
    __syncthreads();
  }
}

// Scratch for one pass over n elements: counts (kBins * ctas + 1) + scan scratch.
inline size_t pass_scratch_bytes(int64_t n) {
  const int64_t m = (int64_t)kBins * ctas_for(n);
  return sizeof(int64_t) * (size_t)(m + 1) + scan_scratch_bytes(m) + 256;
}

template <typename K, typename V, typename Digit, bool GEN_VAL>
void stable_pass(const K *keys, const V *vals, K *keys_out, V *vals_out, int64_t n, Digit dg,
                 void *scratch, cudaStream_t s) {
  if (n <= 0) return;
  const int nctas = ctas_for(n);
  const int64_t seg = (n + nctas - 1) / nctas;
  int64_t *counts = static_cast<int64_t *>(scratch);
  // dependent launches: each kernel waits for its predecessor's results
  // before touching memory, but is scheduled while that one finishes
  launch_pdl(hist_kernel<K, Digit>, nctas, kThreads, 0, s, keys, n, seg, dg, counts, nctas);
  note_launch();
  scan_counts(counts, (int64_t)kBins * nctas, s);
  launch_pdl(scatter_kernel<K, V, Digit, GEN_VAL>, nctas, kThreads, 0, s, keys, vals, keys_out, vals_out, n, seg,
             dg, static_cast<const int64_t *>(counts), nctas);
  note_launch();
}

}  // namespace radix
}  // namespace hm
