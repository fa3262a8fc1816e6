// Query pre-sort (the reference's PSA, "partially sorted aggregation"):
// group a batch of queries by the top `bits` bits of their key, relative to
// the tree's key range, report where each bucket starts, and afterwards move
// per-query results from the grouped order back to the caller's order.
//
// The reference runs cub::DeviceRadixSort::SortPairs on bits [48,64) of
// (key, pos) before every search launch
// (open-harmonia/src/full-multi-prefix-sort-8thread.cu:305-309,
// open-harmonia/regular_bpt/prefix-sort.cu:288-293) and scatters results back
// through the permutation on the host.  Here:
//   * the bucket is taken relative to [key_min, key_max] of the tree so every
//     bucket holds loaded keys (fixed bits [48,64) leave half of them empty for
//     non-negative keys);
//   * order inside a bucket does not matter, so the passes are unstable and
//     take their slots with shared-memory atomics;
//   * up to 8 bits take one pass; more take two, most significant first: the
//     second pass partitions every first-pass bucket on its own, in chunks that
//     never straddle a bucket, with offsets from one global scan of counts laid
//     out as [bucket][digit][chunk];
//   * each pass stages an 8192-query tile in shared memory grouped by digit
//     (12 B per query: key, digit and position) and writes it out so
//     consecutive threads store consecutive slots;
//   * the payload is either the query's input position (int32, for callers
//     that scatter results themselves) or its offset inside its 8192-query
//     input chunk (uint16).  With offsets, unpermute_results undoes the passes
//     in reverse: per input chunk one CTA reads the chunk's digit runs (each
//     contiguous), places every result at its offset in shared memory and
//     writes the chunk out in order, so no pass writes single 8-byte values
//     at random addresses.
#include "hm_internal.cuh"

#include <algorithm>

namespace hm {

namespace {

constexpr int kThreads = 256;
#ifndef HM_PSA_CHUNK
#define HM_PSA_CHUNK 8192
#endif
constexpr int64_t kChunk = HM_PSA_CHUNK;  // queries per CTA chunk (offsets inside a chunk fit 16 bits)
static_assert(kChunk <= 65536, "offsets inside a chunk are kept in 16 bits");
#ifndef HM_PSA_TILE
#define HM_PSA_TILE 8192  // queries a scatter CTA stages at a time (a divisor of kChunk)
#endif
constexpr int kTile = HM_PSA_TILE;

// Launch shapes (compile-time tunables, measured on B200 at 2^24 queries).
#ifndef HM_PSA_REV_THREADS
#define HM_PSA_REV_THREADS 512
#endif
#ifndef HM_PSA_REV_MINB
#define HM_PSA_REV_MINB 3
#endif
#ifndef HM_PSA_REV_BATCH
#define HM_PSA_REV_BATCH 2  // digit runs a warp of the inverse reads at once
#endif
constexpr int kRevThreads = HM_PSA_REV_THREADS;

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Bucket of a key: top `bits` bits of (k - lo) over the tree's key range.
struct Bucket {
  int64_t lo, hi;
  int shift;
  int maxd;
  __device__ __forceinline__ int operator()(int64_t k) const {
    if (k <= lo) return 0;
    if (k >= hi) return maxd;
    return (int)(((uint64_t)k - (uint64_t)lo) >> shift);
  }
};

// A chunk: a contiguous input range inside one first-pass bucket.
struct Chunk {
  int64_t begin, end;
  int32_t bucket;   // first-pass bucket (0 in the first pass)
  int32_t idx;      // chunk index inside its bucket
  int32_t nchunks;  // chunks of its bucket
  int32_t base;     // global index of the bucket's first chunk
};

// Counts of a pass are laid out [bucket][digit][chunk in bucket]: chunk c of
// bucket b, digit d at base_b * 256 + d * nchunks_b + c.  One global exclusive
// scan turns them into output offsets grouped by bucket, then digit.
__device__ __forceinline__ int64_t count_index(const Chunk &c, int d) {
  return (int64_t)c.base * 256 + (int64_t)d * c.nchunks + c.idx;
}

// For a batch set, the first pass cuts each batch into its own chunks (a chunk
// never straddles two batches), numbered globally as one bucket's chunks, so
// the counts stay laid out [digit][chunk] and the output is one partition of
// the whole set.  Each chunk carries its batch's pointers shifted by the
// batch's start: element i of the set is qbase[i] (queries), obase[i]
// (results).
struct ChunkIO {
  const int64_t *qbase;
  int64_t *obase;
};

// One CTA: the batch set's first-pass chunks and their ChunkIO.
__global__ void __launch_bounds__(1024) batch_chunk_kernel(BatchView bv, Chunk *__restrict__ chunks,
                                                            int32_t *__restrict__ nchunks_total,
                                                            int32_t *__restrict__ bfirst, ChunkIO *__restrict__ cio) {
  pdl_enter();
  __shared__ int32_t pre[1024];
  const int tid = threadIdx.x, nb = bv.nb;
  const int per = (nb + 1023) / 1024;
  int32_t mine = 0;
  for (int x = 0; x < per; x++) {
    const int b = tid * per + x;
    if (b < nb) mine += (int32_t)((bv.qpre[b + 1] - bv.qpre[b] + kChunk - 1) / kChunk);
  }
  pre[tid] = mine;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan
    const int32_t v = tid >= o ? pre[tid - o] : 0;
    __syncthreads();
    pre[tid] += v;
    __syncthreads();
  }
  const int32_t total = pre[1023];
  int32_t at = pre[tid] - mine;
  for (int x = 0; x < per; x++) {
    const int b = tid * per + x;
    if (b >= nb) break;
    const int64_t s = bv.qpre[b], e = bv.qpre[b + 1];
    const hm_batch bt = bv.batches[b];
    for (int64_t c0 = s; c0 < e; c0 += kChunk, at++) {
      Chunk c;
      c.begin = c0;
      c.end = min(e, c0 + kChunk);
      c.bucket = 0;
      c.idx = at;
      c.nchunks = total;
      c.base = 0;
      chunks[at] = c;
      ChunkIO io;
      io.qbase = bt.q - s;  // only indexed inside the batch
      io.obase = bt.out - s;
      cio[at] = io;
    }
  }
  if (tid == 1023) {
    nchunks_total[0] = total;
    nchunks_total[1] = 0;  // work counter of the persistent scatter
    bfirst[0] = total > 0 ? 0 : -1;
  }
}

#ifndef HM_PSA_HIST_PER
#define HM_PSA_HIST_PER 8  // keys a histogram thread loads before counting them
#endif
constexpr int kHistPer = HM_PSA_HIST_PER;

// Digit counts of one chunk per CTA.  whole_n >= 0: the input is one bucket
// of whole_n queries cut into kChunk pieces, and this kernel writes that
// chunk table itself (no chunk kernel before it).
template <bool BATCHED>
__global__ void __launch_bounds__(kThreads) psa_hist_kernel(const int64_t *__restrict__ q, BatchView bv, const ChunkIO *__restrict__ cio,
                                                        Chunk *__restrict__ chunks,
                                                        int32_t *__restrict__ nchunks_total,
                                                        int32_t *__restrict__ bfirst, int64_t whole_n, Bucket bk,
                                                        int shift2, int mask2, int64_t *__restrict__ counts) {
  pdl_enter();
  __shared__ unsigned hist[256];
  const int nct = whole_n >= 0 ? (int)((whole_n + kChunk - 1) / kChunk) : *nchunks_total;
  if ((int)blockIdx.x >= nct) {
    // the counts of the chunks this launch does not have stay zero for the scan
    for (int d = threadIdx.x; d < 256; d += kThreads) counts[(int64_t)blockIdx.x * 256 + d] = 0;
    return;
  }
  Chunk c;
  if (whole_n >= 0) {
    c.begin = (int64_t)blockIdx.x * kChunk;
    c.end = min(whole_n, c.begin + kChunk);
    c.bucket = 0;
    c.idx = (int32_t)blockIdx.x;
    c.nchunks = nct;
    c.base = 0;
    if (threadIdx.x == 0) {
      chunks[blockIdx.x] = c;
      if (blockIdx.x == 0) {
        nchunks_total[0] = nct;
        nchunks_total[1] = 0;  // work counter of the persistent scatter
        bfirst[0] = 0;
      }
    }
  } else {
    c = chunks[blockIdx.x];
  }
  const int64_t *src = BATCHED ? cio[blockIdx.x].qbase : q;  // a chunk lies inside one batch
  for (int i = threadIdx.x; i < 256; i += kThreads) hist[i] = 0;
  __syncthreads();
  for (int64_t base = c.begin; base < c.end; base += kHistPer * kThreads) {
    int64_t k[kHistPer];
#pragma unroll
    for (int j = 0; j < kHistPer; j++) {  // all loads first
      const int64_t i = base + j * kThreads + threadIdx.x;
      k[j] = i < c.end ? __ldg(src + i) : 0;
    }
#pragma unroll
    for (int j = 0; j < kHistPer; j++)
      if (base + j * kThreads + threadIdx.x < c.end) atomicAdd(&hist[(bk(k[j]) >> shift2) & mask2], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += kThreads) counts[count_index(c, d)] = hist[d];  // 0 past mask2
}

// Scatter of one pass.  A grid of resident CTAs takes chunks from a counter
// (the first one by block index).  Per tile: rank every query inside its
// digit with shared-memory atomics, scan the 256 tile counts, stage the tile
// grouped by digit as keys (8 B) plus an aux word (digit << 16 | position in
// the tile), then write it out so consecutive threads store consecutive slots
// of one digit run.  The loads of the next tile -- the next chunk's first tile
// at a chunk's end -- are issued before the write-out.  The payload is derived
// from the position at write-out: the input position (int32), the offset
// inside the chunk (uint16), or loaded from pay_in (LOAD).
#ifndef HM_PSA_SCATTER_THREADS
#define HM_PSA_SCATTER_THREADS 512
#endif
#ifndef HM_PSA_SCATTER_MINB
#define HM_PSA_SCATTER_MINB 2  // resident CTAs per SM (shared memory holds 2 at 8192-query tiles)
#endif
constexpr int kSc = HM_PSA_SCATTER_THREADS;
constexpr int kPer = kTile / kSc;
static_assert(kSc >= 256 && kTile % kSc == 0 && kChunk % kTile == 0, "a thread per digit; positions in 16 bits");
// Ranking inside a tile: a shared-memory atomic per key on the tile's 256
// digit counters (measured faster than warp-level __match_any_sync ranking
// into per-warp counters).
constexpr int stage_bytes() { return kTile * 12; }

template <typename T, bool LOAD, bool BATCHED>
__global__ void __launch_bounds__(kSc, HM_PSA_SCATTER_MINB) psa_scatter_kernel(
    const int64_t *__restrict__ q, const ChunkIO *__restrict__ cio, const T *__restrict__ pay_in,
    const Chunk *__restrict__ chunks, int32_t *__restrict__ nchunks_total, Bucket bk, int shift2, int mask2,
    const int64_t *__restrict__ offs, int64_t *__restrict__ q_out, T *__restrict__ pay_out) {
  pdl_enter();
  extern __shared__ __align__(16) unsigned char dyn[];
  int64_t *skey = reinterpret_cast<int64_t *>(dyn);                 // grouped keys
  uint32_t *saux = reinterpret_cast<uint32_t *>(dyn + 8 * kTile);  // digit << 16 | tile position
  __shared__ unsigned cnt[256];
  __shared__ unsigned tstart[256];
  __shared__ int64_t gcur[256];
  __shared__ int64_t adj[256];
  __shared__ unsigned wsum[8];
  __shared__ int next_chunk;
  const int nct = nchunks_total[0];
  int ci = blockIdx.x;
  if (ci >= nct) return;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const bool digit_thread = tid < 256;  // threads 0..255 own a digit's counters
  Chunk c = chunks[ci];
  const int64_t *src = BATCHED ? cio[ci].qbase : q;  // a chunk lies inside one batch
  int64_t k[kPer];
  auto load_tile = [&](const int64_t *sp, int64_t t0, int64_t end) {
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int64_t i = t0 + j * kSc + tid;
      k[j] = i < end ? __ldg(sp + i) : 0;
    }
  };
  load_tile(src, c.begin, c.end);
  if (digit_thread) gcur[tid] = tid <= mask2 ? offs[count_index(c, tid)] : 0;
  int64_t t0 = c.begin;
  for (;;) {
    const bool last_tile = t0 + kTile >= c.end;
    if (digit_thread) cnt[tid] = 0;
    if (tid == 0 && last_tile) next_chunk = (int)gridDim.x + atomicAdd(&nchunks_total[1], 1);
    __syncthreads();
    const int n = (int)min((int64_t)kTile, c.end - t0);
    unsigned dr[kPer];  // digit << 16 | rank inside the tile's digit run; ~0u past the end
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      if (j * kSc + tid < n) {
        const unsigned d = (unsigned)((bk(k[j]) >> shift2) & mask2);
        dr[j] = d << 16 | atomicAdd(&cnt[d], 1u);
      } else {
        dr[j] = ~0u;
      }
    }
    __syncthreads();
    // exclusive scan of the 256 tile counts (one per digit thread)
    unsigned mine = 0, incl = 0;
    if (digit_thread) {
      mine = cnt[tid];
      incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[w] = incl;
    }
    __syncthreads();
    if (digit_thread) {
      unsigned before = incl - mine;
      for (int x = 0; x < w; x++) before += wsum[x];
      tstart[tid] = before;
      adj[tid] = gcur[tid] - (int64_t)before;  // slot sl of digit d goes to adj[d] + sl
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      if (dr[j] != ~0u) {
        const unsigned d = dr[j] >> 16;
        const unsigned sl = tstart[d] + (dr[j] & 0xffffu);
        skey[sl] = k[j];
        saux[sl] = d << 16 | (unsigned)(j * kSc + tid);
      }
    }
    __syncthreads();
    // issue the next tile's loads (this chunk's next tile, or the next chunk's first)
    const int64_t cur_t0 = t0, cur_off = t0 - c.begin;
    bool more = true;
    if (!last_tile) {
      t0 += kTile;
      load_tile(src, t0, c.end);
    } else {
      ci = next_chunk;
      more = ci < nct;
      if (more) {
        c = chunks[ci];
        src = BATCHED ? cio[ci].qbase : q;
        t0 = c.begin;
        load_tile(src, t0, c.end);
      }
    }
    for (int sl = tid; sl < n; sl += kSc) {
      const int64_t key = skey[sl];
      const unsigned a = saux[sl];
      const int64_t o = adj[a >> 16] + sl;
      const unsigned e = a & 0xffffu;
      q_out[o] = key;
      if constexpr (LOAD)
        pay_out[o] = __ldg(pay_in + cur_t0 + e);
      else if constexpr (sizeof(T) == 2)
        pay_out[o] = (T)(cur_off + e);
      else
        pay_out[o] = (T)(cur_t0 + e);
    }
    __syncthreads();
    if (!more) break;
    if (digit_thread) {
      if (last_tile)
        gcur[tid] = tid <= mask2 ? offs[count_index(c, tid)] : 0;
      else
        gcur[tid] += cnt[tid];
    }
  }
}

// Inverse of one pass for 64-bit results, per input chunk.  The chunk's
// elements sit in one contiguous run per digit (offs gives the run starts, in
// [bucket][digit][chunk] order, so the next entry ends the run); each carries
// its offset inside the chunk.  The results are placed by offset in shared
// memory, then written to the chunk's input range in order.  The runs are cut
// into units of 64 elements (a skewed batch can put most of a chunk in one
// run); warps take units round-robin, a lane per element so every load is
// one coalesced request, kRevBatch units at a time: the offsets are loaded
// first, then each result is copied from global memory straight to its slot
// with cp.async.  The chunk is written out with 16-B stores when aligned.
constexpr int kRevWarps = kRevThreads / 32;
constexpr int kRevBatch = HM_PSA_REV_BATCH;
#ifndef HM_PSA_REV_UNIT
#define HM_PSA_REV_UNIT 64  // elements of a unit of the inverse (a multiple of 32)
#endif
constexpr int kUnit = HM_PSA_REV_UNIT;
constexpr int kUnitPer = kUnit / 32;

// Persistent CTAs take chunks blockIdx.x, blockIdx.x + gridDim.x, ...; the
// next chunk's descriptor, run table and output pointer are loaded into
// registers while the current chunk's result copies are in flight, which
// takes two dependent round trips off every chunk but the first (measured:
// both inverse passes 0.178 -> 0.169 ms at 2^24 queries against one CTA per
// chunk).
template <bool BATCHED>
__global__ void __launch_bounds__(kRevThreads, HM_PSA_REV_MINB) psa_unpermute_persist_kernel(
    const Chunk *__restrict__ chunks, const int32_t *__restrict__ nchunks_total, const int64_t *__restrict__ offs,
    int nd, const int64_t *__restrict__ res_in, const uint16_t *__restrict__ loc, int64_t *__restrict__ res_out,
    BatchView bv, const ChunkIO *__restrict__ cio) {
  pdl_enter();
  extern __shared__ __align__(16) int64_t staged[];  // kChunk results
  __shared__ int64_t rs[256];
  __shared__ int32_t rl[256];
  __shared__ int32_t up[257];
  __shared__ uint8_t unit_run[kChunk / kUnit + 256];
  __shared__ int32_t wsum[8];
  const int nct = *nchunks_total;
  int ci = blockIdx.x;
  if (ci >= nct) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  (void)bv;
  // this thread's run (digit tid) of the current chunk, and the chunk
  Chunk c = chunks[ci];
  int64_t ra = 0;
  int32_t rn = 0;
  int64_t *dst = BATCHED ? cio[ci].obase : res_out;
  if (tid < nd) {
    const int64_t k = count_index(c, tid);
    ra = offs[k];
    rn = (int32_t)(offs[k + 1] - ra);
  }
  for (;;) {
    const int len = (int)(c.end - c.begin);
    if (tid < 256) {  // runs and the exclusive scan of their units
      int32_t u = 0;
      if (tid < nd) {
        rs[tid] = ra;
        rl[tid] = rn;
        u = (rn + kUnit - 1) / kUnit;
      }
      int32_t incl = u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) wsum[wid] = incl;
      up[tid] = incl - u;
    }
    __syncthreads();
    if (tid < 256) {
      int32_t add = 0;
      for (int x = 0; x < wid; x++) add += wsum[x];
      up[tid] += add;
      if (tid == 255) up[256] = up[255] + (255 < nd ? (rl[255] + kUnit - 1) / kUnit : 0);
    }
    __syncthreads();
    const int units = up[nd];
    for (int d = tid; d < nd; d += kRevThreads)
      for (int u = up[d]; u < up[d + 1]; u++) unit_run[u] = (uint8_t)d;
    __syncthreads();
    for (int u0 = wid; u0 < units; u0 += kRevWarps * kRevBatch) {
      uint16_t l[kRevBatch][kUnitPer];
      int64_t a[kRevBatch];
      int cnt[kRevBatch];
#pragma unroll
      for (int x = 0; x < kRevBatch; x++) {
        const int u = u0 + x * kRevWarps;
        cnt[x] = 0;
        a[x] = 0;
        if (u < units) {
          const int d = unit_run[u];
          const int e0 = (u - up[d]) * kUnit;
          a[x] = rs[d] + e0;
          cnt[x] = min(kUnit, rl[d] - e0);
#pragma unroll
          for (int h = 0; h < kUnitPer; h++)
            if (lane + 32 * h < cnt[x]) l[x][h] = __ldg(loc + a[x] + lane + 32 * h);
        }
      }
#pragma unroll
      for (int x = 0; x < kRevBatch; x++)
#pragma unroll
        for (int h = 0; h < kUnitPer; h++)
          if (lane + 32 * h < cnt[x]) cp_async8(staged + l[x][h], res_in + a[x] + lane + 32 * h);
    }
    // the next chunk's descriptor, run and output pointer, while the copies fly
    const int cn = ci + (int)gridDim.x;
    Chunk c_next = c;
    int64_t ra_n = 0;
    int32_t rn_n = 0;
    int64_t *dst_n = dst;
    if (cn < nct) {
      c_next = chunks[cn];
      if (BATCHED) dst_n = cio[cn].obase;
      if (tid < nd) {
        const int64_t k = count_index(c_next, tid);
        ra_n = offs[k];
        rn_n = (int32_t)(offs[k + 1] - ra_n);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    int64_t *o = dst + c.begin;
    if ((reinterpret_cast<uintptr_t>(o) & 15) == 0) {
      const int pairs = len >> 1;
      const longlong2 *sv = reinterpret_cast<const longlong2 *>(staged);
      longlong2 *ov = reinterpret_cast<longlong2 *>(o);
      for (int x = tid; x < pairs; x += kRevThreads) ov[x] = sv[x];
      if ((len & 1) && tid == 0) o[len - 1] = staged[len - 1];
    } else {
      for (int x = tid; x < len; x += kRevThreads) o[x] = staged[x];
    }
    if (cn >= nct) break;
    __syncthreads();  // staged, rs, rl, up and unit_run are refilled next
    ci = cn;
    c = c_next;
    ra = ra_n;
    rn = rn_n;
    dst = dst_n;
  }
}

// One CTA: chunk descriptors for a pass.  bstart == nullptr: the whole input
// as one bucket (nb = 1).  Otherwise every bucket [bstart[b], bstart[b+1]) of nb is
// split into chunks of at most kChunk queries; chunks are ordered by bucket.
__global__ void __launch_bounds__(1024) chunk_kernel(const int64_t *__restrict__ bstart, int nb, int64_t n,
                                                     Chunk *__restrict__ chunks, int32_t *__restrict__ nchunks_total,
                                                     int32_t *__restrict__ bfirst) {
  pdl_enter();
  __shared__ int32_t pre[1024];
  const int tid = threadIdx.x;
  if (!bstart) {  // one bucket: the whole input
    const int32_t nc = (int32_t)((n + kChunk - 1) / kChunk);
    for (int32_t i = tid; i < nc; i += 1024) {
      Chunk c;
      c.begin = (int64_t)i * kChunk;
      c.end = min(n, c.begin + kChunk);
      c.bucket = 0;
      c.idx = i;
      c.nchunks = nc;
      c.base = 0;
      chunks[i] = c;
    }
    if (tid == 0) {
      nchunks_total[0] = nc;
      nchunks_total[1] = 0;  // work counter of the persistent scatter
      bfirst[0] = nc > 0 ? 0 : -1;
    }
    return;
  }
  const int per = (nb + 1023) / 1024;
  int32_t mine = 0;
  for (int x = 0; x < per; x++) {
    const int b = tid * per + x;
    if (b < nb) mine += (int32_t)((bstart[b + 1] - bstart[b] + kChunk - 1) / kChunk);
  }
  pre[tid] = mine;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan
    const int32_t v = tid >= o ? pre[tid - o] : 0;
    __syncthreads();
    pre[tid] += v;
    __syncthreads();
  }
  int32_t base = pre[tid] - mine;
  for (int x = 0; x < per; x++) {
    const int b = tid * per + x;
    if (b >= nb) break;
    const int64_t s = bstart[b], e = bstart[b + 1];
    const int32_t nc = (int32_t)((e - s + kChunk - 1) / kChunk);
    bfirst[b] = nc > 0 ? base : -1;
    for (int32_t i = 0; i < nc; i++) {
      Chunk c;
      c.begin = s + (int64_t)i * kChunk;
      c.end = min(e, c.begin + kChunk);
      c.bucket = b;
      c.idx = i;
      c.nchunks = nc;
      c.base = base;
      chunks[base + i] = c;
    }
    base += nc;
  }
  if (tid == 1023) {
    nchunks_total[0] = pre[1023];
    nchunks_total[1] = 0;
  }
}

// Starts of the pass's output buckets: bucket (b, d) starts at the offset of
// digit d in b's first chunk (bfirst, from the chunk kernel); an empty input
// bucket b starts where it did.
__global__ void bucket_starts_kernel(const Chunk *__restrict__ chunks, const int32_t *__restrict__ bfirst,
                                     const int64_t *__restrict__ offs, int nb, int nd, int64_t n,
                                     const int64_t *__restrict__ bstart_in, int64_t *__restrict__ bstart) {
  pdl_enter();
  const int total = nb * nd;
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x <= total; x += gridDim.x * blockDim.x) {
    if (x == total) {
      bstart[total] = n;
      continue;
    }
    const int b = x / nd, d = x % nd;
    const int first = bfirst[b];
    bstart[x] = first >= 0 ? offs[count_index(chunks[first], d)] : (bstart_in ? bstart_in[b] : 0);
  }
}

Bucket make_bucket(const hm_tree *t, int bits) {
  Bucket d;
  d.lo = t->key_min;
  d.hi = t->key_max;
  d.maxd = (1 << bits) - 1;
  uint64_t range = (uint64_t)t->key_max - (uint64_t)t->key_min;
  int len = 0;
  while (len < 64 && (range >> len) != 0) len++;
  d.shift = len > bits ? len - bits : 0;
  return d;
}

int64_t max_chunks(int64_t n, int nb) { return (n + kChunk - 1) / kChunk + nb + 1; }

// One pass's chunk descriptors and scanned counts (kept for the inverse).
struct Pass {
  Chunk *chunks;
  int32_t *nchunks;
  int32_t *bfirst;  // first chunk of each input bucket, -1 for an empty one (at most 256)
  int64_t *offs;    // 256 * mc + 1
  int64_t mc;
};

struct Work {
  Pass p1, p2;
  void *scan;
  int64_t *bstart1;  // first-pass bucket starts (257)
  int64_t *bstart;   // final bucket starts (2^bits + 1)
  int64_t *q_tmp;    // first-pass keys (two passes); the inverse's temporary
  void *pay1;        // first-pass payloads (two passes)
  uint16_t *loc;     // final offsets (offset mode)
  ChunkIO *cio;      // batch sets: the batches of each first-pass chunk
};

size_t work_layout(int64_t n, int bits, bool offsets, Work *w, char *base, int batches = 1) {
  const bool two = bits > 8;
  const int64_t mc1 = max_chunks(n, batches), mc2 = two ? max_chunks(n, 256) : 0;
  const size_t pay = offsets ? 2 : 4;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *p = base ? base + off : nullptr;
    off += (size_t)align_up((int64_t)bytes, 256);
    return p;
  };
  Work x{};
  x.p1.mc = mc1;
  x.p1.chunks = reinterpret_cast<Chunk *>(take(sizeof(Chunk) * mc1));
  x.p1.nchunks = reinterpret_cast<int32_t *>(take(16));
  x.p1.bfirst = reinterpret_cast<int32_t *>(take(4 * 256));
  x.p1.offs = reinterpret_cast<int64_t *>(take(8 * (256 * mc1 + 1)));
  if (two) {
    x.p2.mc = mc2;
    x.p2.chunks = reinterpret_cast<Chunk *>(take(sizeof(Chunk) * mc2));
    x.p2.nchunks = reinterpret_cast<int32_t *>(take(16));
    x.p2.bfirst = reinterpret_cast<int32_t *>(take(4 * 256));
    x.p2.offs = reinterpret_cast<int64_t *>(take(8 * (256 * mc2 + 1)));
  }
  x.scan = take(scan_scratch_bytes(256 * std::max(mc1, mc2)));
  x.bstart1 = reinterpret_cast<int64_t *>(take(8 * 258));
  x.bstart = reinterpret_cast<int64_t *>(take(8 * (((size_t)1 << bits) + 1)));
  x.q_tmp = two ? reinterpret_cast<int64_t *>(take(8 * n)) : nullptr;
  x.pay1 = two ? take(pay * n) : nullptr;
  x.loc = offsets ? reinterpret_cast<uint16_t *>(take(2 * n)) : nullptr;
  x.cio = reinterpret_cast<ChunkIO *>(take(sizeof(ChunkIO) * mc1));
  if (w) *w = x;
  return off;
}

template <typename T, bool LOAD, bool BATCHED = false>
void one_pass(const Bucket &bk, const int64_t *q, const T *pay_in, int64_t n, const int64_t *bstart_in, int nb,
              int shift2, int mask2, int64_t *q_out, T *pay_out, int64_t *bstart_out, const Pass &ps, void *scan,
              int sms, cudaStream_t s, const BatchView &bv = BatchView(), const ChunkIO *cio = nullptr) {
  // a single unbatched input: the histogram kernel writes the chunk table
  const bool whole = !BATCHED && bstart_in == nullptr;
  if (BATCHED)
    launch_pdl(batch_chunk_kernel, 1, 1024, 0, s, bv, ps.chunks, ps.nchunks, ps.bfirst, const_cast<ChunkIO *>(cio));
  else if (!whole)
    launch_pdl(chunk_kernel, 1, 1024, 0, s, bstart_in, nb, n, ps.chunks, ps.nchunks, ps.bfirst);
  launch_pdl(psa_hist_kernel<BATCHED>, (unsigned)ps.mc, kThreads, 0, s, q, bv, cio, ps.chunks, ps.nchunks, ps.bfirst,
             whole ? n : (int64_t)-1, bk, shift2,
                                                                 mask2, ps.offs);
  exclusive_scan_i64(ps.offs, ps.offs, 256 * ps.mc, scan, s);
  opt_in_smem((const void *)psa_scatter_kernel<T, LOAD, BATCHED>, stage_bytes());
  const unsigned grid = (unsigned)std::min<int64_t>(ps.mc, (int64_t)sms * HM_PSA_SCATTER_MINB);
  launch_pdl(psa_scatter_kernel<T, LOAD, BATCHED>, grid, kSc, stage_bytes(), s, q, cio, pay_in, ps.chunks, ps.nchunks, bk,
                                                                         shift2, mask2, ps.offs, q_out, pay_out);
  const int nd = mask2 + 1;
  launch_pdl(bucket_starts_kernel, (unsigned)((nb * nd + 256) / 256), 256, 0, s, ps.chunks, ps.bfirst, ps.offs, nb, nd, n,
                                                                         bstart_in, bstart_out);
  note_launch(whole ? 3 : 4);  // [chunk,] histogram, scatter, bucket starts (the scan counts its own)
}

int device_sms() {
  static int sms[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!sms[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    sms[dev] = v;
  }
  return sms[dev];
}

template <bool BATCHED = false>
void unpermute_pass(const Pass &ps, int nd, const int64_t *res_in, const uint16_t *loc, int64_t *res_out,
                    cudaStream_t s, const BatchView &bv = BatchView(), const ChunkIO *cio = nullptr) {
  opt_in_smem((const void *)psa_unpermute_persist_kernel<BATCHED>, (int)(8 * kChunk));
  const unsigned grid = (unsigned)std::min<int64_t>(ps.mc, (int64_t)device_sms() * HM_PSA_REV_MINB);
  launch_pdl(psa_unpermute_persist_kernel<BATCHED>, grid, kRevThreads, 8 * kChunk, s, ps.chunks, ps.nchunks, ps.offs,
             nd, res_in, loc, res_out, bv, cio);
  note_launch();
}

}  // namespace

size_t partition_scratch_bytes(int64_t n, int bits, bool offsets, int batches) {
  return work_layout(n, bits, offsets, nullptr, nullptr, batches) + 256;
}

int partition_queries(const hm_tree *t, const int64_t *q, int64_t n, int bits, int64_t *q_out, int32_t *pos_out,
                      void *scratch, cudaStream_t s, const int64_t **bucket_start, const BatchView *bv) {
  if (n == 0) return HM_OK;
  if (bits < 1 || bits > 16 || n > INT32_MAX || n < 0) return HM_EINVAL;
  const bool offsets = pos_out == nullptr;
  if (bv && !offsets) return HM_EINVAL;
  Work w;
  work_layout(n, bits, offsets, &w, static_cast<char *>(scratch), bv ? bv->nb : 1);
  const Bucket bk = make_bucket(t, bits);
  const int sms = t->num_sms;
  if (bits <= 8) {
    if (bv)
      one_pass<uint16_t, false, true>(bk, nullptr, nullptr, n, nullptr, 1, 0, (1 << bits) - 1, q_out, w.loc,
                                      w.bstart, w.p1, w.scan, sms, s, *bv, w.cio);
    else if (offsets)
      one_pass<uint16_t, false>(bk, q, nullptr, n, nullptr, 1, 0, (1 << bits) - 1, q_out, w.loc, w.bstart, w.p1,
                                w.scan, sms, s);
    else
      one_pass<int32_t, false>(bk, q, nullptr, n, nullptr, 1, 0, (1 << bits) - 1, q_out, pos_out, w.bstart, w.p1,
                               w.scan, sms, s);
  } else {
    const int low = bits - 8;
    if (offsets) {
      uint16_t *loc1 = static_cast<uint16_t *>(w.pay1);
      if (bv)
        one_pass<uint16_t, false, true>(bk, nullptr, nullptr, n, nullptr, 1, low, 0xff, w.q_tmp, loc1, w.bstart1,
                                        w.p1, w.scan, sms, s, *bv, w.cio);
      else
        one_pass<uint16_t, false>(bk, q, nullptr, n, nullptr, 1, low, 0xff, w.q_tmp, loc1, w.bstart1, w.p1, w.scan,
                                  sms, s);
      one_pass<uint16_t, false>(bk, w.q_tmp, nullptr, n, w.bstart1, 256, 0, (1 << low) - 1, q_out, w.loc, w.bstart,
                                w.p2, w.scan, sms, s);
    } else {
      int32_t *pos1 = static_cast<int32_t *>(w.pay1);
      one_pass<int32_t, false>(bk, q, nullptr, n, nullptr, 1, low, 0xff, w.q_tmp, pos1, w.bstart1, w.p1, w.scan, sms, s);
      one_pass<int32_t, true>(bk, w.q_tmp, pos1, n, w.bstart1, 256, 0, (1 << low) - 1, q_out, pos_out, w.bstart, w.p2,
                              w.scan, sms, s);
    }
  }
  if (bucket_start) *bucket_start = w.bstart;
  return cuda_err(cudaGetLastError());
}

int partition_queries_placed(const hm_tree *t, const int64_t *q, int64_t n, int bits, int64_t *q_out,
                             int32_t *place, void *scratch, cudaStream_t s, const int64_t **bucket_start,
                             const BatchView *bv) {
  if (n == 0) return HM_OK;
  if (bits <= 8 || bits > 16 || n > INT32_MAX || n < 0 || !place) return HM_EINVAL;
  Work w;
  work_layout(n, bits, true, &w, static_cast<char *>(scratch), bv ? bv->nb : 1);
  const Bucket bk = make_bucket(t, bits);
  const int sms = t->num_sms;
  const int low = bits - 8;
  uint16_t *loc1 = static_cast<uint16_t *>(w.pay1);
  if (bv)
    one_pass<uint16_t, false, true>(bk, nullptr, nullptr, n, nullptr, 1, low, 0xff, w.q_tmp, loc1, w.bstart1, w.p1,
                                    w.scan, sms, s, *bv, w.cio);
  else
    one_pass<uint16_t, false>(bk, q, nullptr, n, nullptr, 1, low, 0xff, w.q_tmp, loc1, w.bstart1, w.p1, w.scan, sms,
                              s);
  one_pass<int32_t, false>(bk, w.q_tmp, nullptr, n, w.bstart1, 256, 0, (1 << low) - 1, q_out, place, w.bstart, w.p2,
                           w.scan, sms, s);
  if (bucket_start) *bucket_start = w.bstart;
  return cuda_err(cudaGetLastError());
}

int unpermute_first_pass(int64_t n, int bits, const int64_t *res1, int64_t *out, void *scratch, cudaStream_t s,
                         const BatchView *bv) {
  if (n == 0) return HM_OK;
  if (bits <= 8 || bits > 16 || n > INT32_MAX || n < 0) return HM_EINVAL;
  Work w;
  work_layout(n, bits, true, &w, static_cast<char *>(scratch), bv ? bv->nb : 1);
  const uint16_t *loc1 = static_cast<const uint16_t *>(w.pay1);
  if (bv)
    unpermute_pass<true>(w.p1, 256, res1, loc1, nullptr, s, *bv, w.cio);
  else
    unpermute_pass(w.p1, 256, res1, loc1, out, s);
  return cuda_err(cudaGetLastError());
}

int unpermute_results(int64_t n, int bits, int64_t *res_sorted, int64_t *out, void *scratch, cudaStream_t s,
                      const BatchView *bv) {
  if (n == 0) return HM_OK;
  if (bits < 1 || bits > 16 || n > INT32_MAX || n < 0) return HM_EINVAL;
  Work w;
  work_layout(n, bits, true, &w, static_cast<char *>(scratch), bv ? bv->nb : 1);
  const int64_t *res1 = res_sorted;  // results in first-pass order
  const uint16_t *loc1 = w.loc;
  if (bits > 8) {
    unpermute_pass(w.p2, 1 << (bits - 8), res_sorted, w.loc, w.q_tmp, s);
    res1 = w.q_tmp;
    loc1 = static_cast<const uint16_t *>(w.pay1);
  }
  const int nd1 = bits <= 8 ? 1 << bits : 256;
  if (bv)
    unpermute_pass<true>(w.p1, nd1, res1, loc1, nullptr, s, *bv, w.cio);
  else
    unpermute_pass(w.p1, nd1, res1, loc1, out, s);
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
