// Stable LSD radix sort of (uint64 key, payload) pairs, 8-bit digits, built
// from the counting-sort pass in radix_pass.cuh.
//
// Used by the bulk loader (full 64-bit sort of the input keys) and by the
// upsert epoch (sort of the batch).  The reference sorts with vendored CUB
// (cub::DeviceRadixSort::SortPairs,
// open-harmonia/src/full-multi-prefix-sort-8thread.cu:305-309); this sort is
// self-contained.
#include "radix_pass.cuh"

namespace hm {

namespace {

// One-CTA in-place exclusive scan (small arrays).
__global__ void __launch_bounds__(1024) scan_counts_kernel(int64_t *counts, int64_t m) {
  pdl_enter();
  __shared__ int64_t part[1024];
  int64_t per = (m + 1023) / 1024;
  int64_t b0 = (int64_t)threadIdx.x * per, b1 = min(m, b0 + per);
  int64_t s = 0;
  for (int64_t i = b0; i < b1; i++) s += counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
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

struct RadixDigit {
  int shift;
  __device__ __forceinline__ int operator()(uint64_t k) const { return (int)((k >> shift) & 0xff); }
};

}  // namespace

// In-place exclusive scan of counts[0..m) (digit-major histograms).  Large
// arrays go through the multi-CTA scan; the caller's buffer has room for
// m + 1 entries plus scan_scratch_bytes(m) bytes after them.
void scan_counts(int64_t *counts, int64_t m, cudaStream_t s) {
  if (m <= 4096) {
    launch_pdl(scan_counts_kernel, 1, 1024, 0, s, counts, m);
    note_launch();
    return;
  }
  exclusive_scan_i64(counts, counts, m, counts + m + 1, s);
}

size_t radix_scratch_bytes(int64_t n) { return radix::pass_scratch_bytes(n); }

template <typename V>
bool radix_sort_pairs(uint64_t *ukeys, V *vals, uint64_t *ukeys_alt, V *vals_alt, int64_t n,
                      int begin_bit, int end_bit, void *scratch, cudaStream_t s) {
  if (n <= 1) return false;
  uint64_t *ka = ukeys, *kb = ukeys_alt;
  V *va = vals, *vb = vals_alt;
  bool flipped = false;
  for (int bit = begin_bit; bit < end_bit; bit += 8) {
    radix::stable_pass<uint64_t, V, RadixDigit, false>(ka, va, kb, vb, n, RadixDigit{bit}, scratch, s);
    std::swap(ka, kb);
    std::swap(va, vb);
    flipped = !flipped;
  }
  return flipped;
}

bool radix_sort_positions(uint64_t *ukeys, int32_t *pos, uint64_t *ukeys_alt, int32_t *pos_alt, int64_t n,
                          int begin_bit, int end_bit, void *scratch, cudaStream_t s) {
  if (n <= 0 || begin_bit >= end_bit) return false;
  // the first pass writes each element's input position as its payload
  radix::stable_pass<uint64_t, int32_t, RadixDigit, true>(ukeys, nullptr, ukeys_alt, pos_alt, n,
                                                          RadixDigit{begin_bit}, scratch, s);
  if (begin_bit + 8 >= end_bit) return true;
  return !radix_sort_pairs<int32_t>(ukeys_alt, pos_alt, ukeys, pos, n, begin_bit + 8, end_bit, scratch, s);
}

template bool radix_sort_pairs<int64_t>(uint64_t *, int64_t *, uint64_t *, int64_t *, int64_t, int,
                                        int, void *, cudaStream_t);
template bool radix_sort_pairs<int32_t>(uint64_t *, int32_t *, uint64_t *, int32_t *, int64_t, int,
                                        int, void *, cudaStream_t);

}  // namespace hm
