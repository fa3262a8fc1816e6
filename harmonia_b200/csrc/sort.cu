// Stable LSD radix sort of (uint64 key, payload) pairs, 8-bit digits.
//
// Used by the bulk loader (full 64-bit sort of the input keys) and the upsert
// epoch (sort of the batch).  The reference sorts with vendored CUB
// (cub::DeviceRadixSort::SortPairs, open-harmonia/src/full-multi-prefix-sort-8thread.cu:305-309);
// this is a self-contained reduce-then-scan sort:
//   upsweep   each CTA histograms its contiguous segment (256 bins)
//   scan      one CTA turns the digit-major [digit][cta] counts into offsets
//   downsweep each CTA re-reads its segment in 1024-element tiles, ranks every
//             element stably inside the tile (warp __match_any_sync + a
//             cross-warp prefix in shared memory) and scatters it to
//             offset[digit][cta] + running rank.
// Stability comes from ranking in (warp, iteration, lane) order, which is the
// element order of the tile.
#include "hm_internal.cuh"

namespace hm {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItemsPerWarp = 128;  // 4 iterations of 32
constexpr int kTile = kWarps * kItemsPerWarp;
constexpr int kBins = 256;
constexpr int kMaxCtas = 148 * 8;

int sort_ctas(int64_t n) {
  int64_t c = (n + kTile - 1) / kTile;
  if (c > kMaxCtas) c = kMaxCtas;
  if (c < 1) c = 1;
  return (int)c;
}

__global__ void __launch_bounds__(kThreads) upsweep_kernel(const uint64_t *__restrict__ keys, int64_t n,
                                                           int64_t seg, int shift,
                                                           int64_t *__restrict__ counts, int nctas) {
  __shared__ unsigned hist[kBins];
  for (int i = threadIdx.x; i < kBins; i += kThreads) hist[i] = 0;
  __syncthreads();
  int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t i = b0 + threadIdx.x; i < b1; i += kThreads)
    atomicAdd(&hist[(keys[i] >> shift) & 0xff], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < kBins; d += kThreads)
    counts[(int64_t)d * nctas + blockIdx.x] = hist[d];
}

// Exclusive scan of counts[0..m) in place by one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) scan_counts_kernel(int64_t *counts, int64_t m) {
  __shared__ int64_t part[1024];
  int64_t per = (m + 1023) / 1024;
  int64_t b0 = (int64_t)threadIdx.x * per, b1 = min(m, b0 + per);
  int64_t s = 0;
  for (int64_t i = b0; i < b1; i++) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of 1024 partial sums
  for (int o = 1; o < 1024; o <<= 1) {
    int64_t v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int64_t run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int64_t i = b0; i < b1; i++) {
    int64_t c = counts[i];
    counts[i] = run;
    run += c;
  }
}

template <typename V>
__global__ void __launch_bounds__(kThreads) downsweep_kernel(
    const uint64_t *__restrict__ keys, const V *__restrict__ vals, uint64_t *__restrict__ keys_out,
    V *__restrict__ vals_out, int64_t n, int64_t seg, int shift,
    const int64_t *__restrict__ offsets, int nctas) {
  __shared__ unsigned warp_cnt[kWarps][kBins + 1];  // +1: bin 256 collects invalid lanes
  __shared__ int64_t warp_base[kWarps][kBins];
  __shared__ int64_t cursor[kBins];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int d = threadIdx.x; d < kBins; d += kThreads)
    cursor[d] = offsets[(int64_t)d * nctas + blockIdx.x];
  for (int i = threadIdx.x; i < kWarps * (kBins + 1); i += kThreads) (&warp_cnt[0][0])[i] = 0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * seg, b1 = min(n, b0 + seg);
  for (int64_t tile = b0; tile < b1; tile += kTile) {
    uint64_t k[4];
    V v[4];
    int dig[4];
    unsigned local[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      int64_t e = tile + warp * kItemsPerWarp + j * 32 + lane;
      bool valid = e < b1;
      k[j] = valid ? keys[e] : 0;
      v[j] = valid ? vals[e] : V(0);
      dig[j] = valid ? (int)((k[j] >> shift) & 0xff) : kBins;
      unsigned peers = __match_any_sync(0xffffffffu, dig[j]);
      unsigned base = warp_cnt[warp][dig[j]];
      __syncwarp();
      if ((peers & lt_mask) == 0) warp_cnt[warp][dig[j]] = base + __popc(peers);
      __syncwarp();
      local[j] = base + __popc(peers & lt_mask);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kBins; d += kThreads) {
      int64_t run = cursor[d];
#pragma unroll
      for (int w = 0; w < kWarps; w++) {
        warp_base[w][d] = run;
        run += warp_cnt[w][d];
        warp_cnt[w][d] = 0;
      }
      cursor[d] = run;
    }
    if (threadIdx.x < kWarps) warp_cnt[threadIdx.x][kBins] = 0;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (dig[j] < kBins) {
        int64_t o = warp_base[warp][dig[j]] + local[j];
        keys_out[o] = k[j];
        vals_out[o] = v[j];
      }
    }
    __syncthreads();
  }
}

}  // namespace

// In-place exclusive scan of counts[0..m) (digit-major histograms).  Large
// arrays go through the multi-CTA scan; the caller's buffer has room for
// m + 1 entries plus scan_scratch_bytes(m) bytes after them.
void scan_counts(int64_t *counts, int64_t m, cudaStream_t s) {
  if (m <= 4096) {
    scan_counts_kernel<<<1, 1024, 0, s>>>(counts, m);
    note_launch();
    return;
  }
  exclusive_scan_i64(counts, counts, m, counts + m + 1, s);
}

size_t radix_scratch_bytes(int64_t n) {
  (void)n;
  const int64_t m = (int64_t)kBins * kMaxCtas;
  return sizeof(int64_t) * (size_t)(m + 1) + scan_scratch_bytes(m) + 256;
}

template <typename V>
bool radix_sort_pairs(uint64_t *ukeys, V *vals, uint64_t *ukeys_alt, V *vals_alt, int64_t n,
                      int begin_bit, int end_bit, void *scratch, cudaStream_t s) {
  if (n <= 1) return false;
  int nctas = sort_ctas(n);
  int64_t seg = (n + nctas - 1) / nctas;
  int64_t *counts = static_cast<int64_t *>(scratch);
  uint64_t *ka = ukeys, *kb = ukeys_alt;
  V *va = vals, *vb = vals_alt;
  bool flipped = false;
  for (int bit = begin_bit; bit < end_bit; bit += 8) {
    upsweep_kernel<<<nctas, kThreads, 0, s>>>(ka, n, seg, bit, counts, nctas);
    note_launch(1);
    scan_counts(counts, (int64_t)kBins * nctas, s);
    downsweep_kernel<V><<<nctas, kThreads, 0, s>>>(ka, va, kb, vb, n, seg, bit, counts, nctas);
    note_launch(1);
    uint64_t *tk = ka;
    ka = kb;
    kb = tk;
    V *tv = va;
    va = vb;
    vb = tv;
    flipped = !flipped;
  }
  return flipped;
}

template bool radix_sort_pairs<int64_t>(uint64_t *, int64_t *, uint64_t *, int64_t *, int64_t, int,
                                        int, void *, cudaStream_t);
template bool radix_sort_pairs<int32_t>(uint64_t *, int32_t *, uint64_t *, int32_t *, int64_t, int,
                                        int, void *, cudaStream_t);

}  // namespace hm
