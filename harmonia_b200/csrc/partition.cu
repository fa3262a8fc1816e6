// Query pre-sort (the reference's PSA, "partially sorted aggregation"):
// order a batch of queries by the top `bits` bits of their key, relative to
// the tree's key range, and carry each query's original position along.
//
// The reference runs cub::DeviceRadixSort::SortPairs on bits [48,64) of
// (key, pos) before every search launch
// (open-harmonia/src/full-multi-prefix-sort-8thread.cu:305-309,
// open-harmonia/regular_bpt/prefix-sort.cu:288-293) and scatters results back
// through the permutation on the host.  Here the digit is taken relative to
// [key_min, key_max] of the tree so that all 2^bits buckets cover loaded keys
// (fixed bits [48,64) leave half of them empty for non-negative keys); up to
// 8 bits take one stable counting-sort pass, up to 16 bits two (LSD: low
// part first).  The search then writes each result to out[pos].
#include "radix_pass.cuh"

#include <algorithm>

namespace hm {

namespace {

// Bits [sub_shift, sub_shift + 8) of the clamped bucket of a key.
struct KeyDigit {
  int64_t lo, hi;
  int shift;
  int maxd;
  int sub_shift;
  int sub_mask;
  __device__ __forceinline__ int operator()(int64_t k) const {
    int full;
    if (k <= lo)
      full = 0;
    else if (k >= hi)
      full = maxd;
    else
      full = (int)((uint64_t)(k - lo) >> shift);
    return (full >> sub_shift) & sub_mask;
  }
};

KeyDigit make_digit(const hm_tree *t, int bits) {
  KeyDigit d;
  d.lo = t->key_min;
  d.hi = t->key_max;
  d.maxd = (1 << bits) - 1;
  uint64_t range = (uint64_t)t->key_max - (uint64_t)t->key_min;
  int len = 0;
  while (len < 64 && (range >> len) != 0) len++;
  d.shift = len > bits ? len - bits : 0;
  d.sub_shift = 0;
  d.sub_mask = 0xff;
  return d;
}

}  // namespace

size_t partition_scratch_bytes(int64_t n, int bits) {
  size_t b = radix::pass_scratch_bytes(n);
  if (bits > 8) b += (size_t)align_up(n * 8, 256) + (size_t)align_up(n * 4, 256);
  return b;
}

int partition_queries(const hm_tree *t, const int64_t *q, int64_t n, int bits, int64_t *q_out,
                      int32_t *pos_out, void *scratch, cudaStream_t s) {
  if (bits < 1 || bits > 16 || n > INT32_MAX) return HM_EINVAL;
  KeyDigit dg = make_digit(t, bits);
  if (bits <= 8) {
    dg.sub_mask = (1 << bits) - 1;
    radix::stable_pass<int64_t, int32_t, KeyDigit, true>(q, nullptr, q_out, pos_out, n, dg, scratch, s);
    return cuda_err(cudaGetLastError());
  }
  // two stable passes: low (bits-8) bits of the bucket, then its high 8 bits
  char *p = static_cast<char *>(scratch) + radix::pass_scratch_bytes(n);
  int64_t *q_tmp = reinterpret_cast<int64_t *>(p);
  int32_t *pos_tmp = reinterpret_cast<int32_t *>(p + align_up(n * 8, 256));
  KeyDigit lo = dg;
  lo.sub_shift = 0;
  lo.sub_mask = (1 << (bits - 8)) - 1;
  radix::stable_pass<int64_t, int32_t, KeyDigit, true>(q, nullptr, q_tmp, pos_tmp, n, lo, scratch, s);
  KeyDigit hi = dg;
  hi.sub_shift = bits - 8;
  hi.sub_mask = 0xff;
  radix::stable_pass<int64_t, int32_t, KeyDigit, false>(q_tmp, pos_tmp, q_out, pos_out, n, hi, scratch, s);
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
