// C-ABI entry points (include/harmonia.h) and the host-side orchestration:
// argument checks, device/host pointer handling, the chunked copy pipeline
// for host buffers, scratch management and error reporting.  The reference
// drivers this replaces exit on any CUDA error
// (CUDA_ERROR_HANDLER, open-harmonia/src/cuda_utils.h:3-12); every path here
// returns an HM_E* code instead.
#include "hm_internal.cuh"

#include <algorithm>
#include <mutex>
#include <set>
#include <tuple>
#include <unordered_map>
#include <vector>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace hm {

static std::atomic<uint64_t> g_launches{0};
static thread_local bool t_capturing = false;
void note_launch(int n) {
  if (!t_capturing) g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed);
}
void set_capturing(bool on) { t_capturing = on; }

static std::atomic<int> g_last_cuda{0};

int cuda_err(cudaError_t e) {
  if (e == cudaSuccess) return HM_OK;
  g_last_cuda.store((int)e);
  if (e == cudaErrorMemoryAllocation) return HM_ENOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return HM_ENODEVICE;
  return HM_ECUDA;
}

// ---- device block cache ----
// Large device blocks (tree arenas, bulk-load and rebuild temporaries,
// scratch blocks) are kept when their owner releases them and handed to later
// requests on the same device: a cudaMalloc of a GiB-sized block maps it anew
// (milliseconds, and variable) and cudaFree synchronises the whole device.
// A request takes the smallest cached block of at least its size and at most
// half again as large (plus 64 MiB).  A block is released only once no work
// is in flight on it (every caller releases after a synchronisation).  At
// most kCacheCap bytes stay cached (the oldest are freed first);
// hm_trim_memory frees them all.
namespace {
struct CachedBlock {
  void *p;
  size_t bytes;
  int dev;
};
std::mutex g_cache_mu;
std::vector<CachedBlock> g_cache;                           // free blocks, oldest first
std::unordered_map<void *, std::pair<size_t, int>> g_live;  // blocks handed out by dev_alloc
size_t g_cached = 0;
constexpr size_t kCacheCap = (size_t)16 << 30;

void free_block(const CachedBlock &b) {
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != b.dev) cudaSetDevice(b.dev);
  cudaFree(b.p);
  if (cur != b.dev) cudaSetDevice(cur);
}

// Frees the cached blocks of device dev (-1: every device); returns the bytes freed.
size_t trim_cache(int dev) {
  std::vector<CachedBlock> out;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    std::vector<CachedBlock> keep;
    for (const CachedBlock &b : g_cache) (dev < 0 || b.dev == dev ? out : keep).push_back(b);
    g_cache.swap(keep);
    for (const CachedBlock &b : out) g_cached -= b.bytes;
  }
  size_t freed = 0;
  for (const CachedBlock &b : out) {
    free_block(b);
    freed += b.bytes;
  }
  return freed;
}
}  // namespace

cudaError_t dev_alloc(void **p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    int best = -1;
    for (int i = 0; i < (int)g_cache.size(); i++) {
      const CachedBlock &b = g_cache[i];
      if (b.dev == dev && b.bytes >= bytes && b.bytes <= bytes + bytes / 2 + ((size_t)64 << 20) &&
          (best < 0 || b.bytes < g_cache[best].bytes))
        best = i;
    }
    if (best >= 0) {
      const CachedBlock b = g_cache[best];
      g_cache.erase(g_cache.begin() + best);
      g_cached -= b.bytes;
      g_live[b.p] = {b.bytes, b.dev};
      *p = b.p;
      return cudaSuccess;
    }
  }
  e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation && trim_cache(dev) > 0) {  // cached blocks stand in the way
    cudaGetLastError();
    e = cudaMalloc(p, bytes);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  std::lock_guard<std::mutex> lk(g_cache_mu);
  g_live[*p] = {bytes, dev};
  return cudaSuccess;
}

void dev_release(void *p) {
  if (!p) return;
  std::vector<CachedBlock> evict;
  bool ours = false;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_live.find(p);
    if (it != g_live.end()) {
      ours = true;
      g_cache.push_back({p, it->second.first, it->second.second});
      g_cached += it->second.first;
      g_live.erase(it);
      while (g_cached > kCacheCap && !g_cache.empty()) {
        evict.push_back(g_cache.front());
        g_cached -= g_cache.front().bytes;
        g_cache.erase(g_cache.begin());
      }
    }
  }
  if (!ours) cudaFree(p);
  for (const CachedBlock &b : evict) free_block(b);
}

void release_after(void *p, cudaStream_t s) {
  if (!p) return;
  cudaStreamSynchronize(s);
  dev_release(p);
}

// Scratch blocks come from the block cache above and grow by half again when
// a call needs more.  An outgrown block is retired, not released: its last
// use may still run on another stream, and waiting for it would stall that
// stream's reads.  Retired blocks go back to the cache with the tree (after
// its device-wide synchronisation); with growth by half again they add up to
// at most about twice the largest block.  (A stream-ordered pool that returns
// memory to the system at every synchronisation, like the device's default
// pool, maps it anew for each fresh tree: measured 4.6 against 2.1 ms for a
// 4096K-key upsert epoch on a fresh 2^26-key tree.)
// Idle blocks kept per tree before a busy stream's block is reused instead of
// adding one (each holds as much as its largest call needed).
constexpr size_t kPoolBlocks = 8;

int ScratchLease::acquire(size_t bytes) {
  if (idx_ >= 0) return HM_EINVAL;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s_, &cs) != cudaSuccess) {
    cudaGetLastError();
    return HM_EINVAL;
  }
  if (cs != cudaStreamCaptureStatusNone) return HM_EINVAL;
  std::lock_guard<std::mutex> lk(t_->mu);
  auto &pool = t_->pool;
  int pick = -1;
  for (size_t i = 0; i < pool.size() && pick < 0; i++)  // last used on this stream
    if (!pool[i].leased && pool[i].stream == s_) pick = (int)i;
  for (size_t i = 0; i < pool.size() && pick < 0; i++) {  // last use finished
    if (pool[i].leased) continue;
    if (!pool[i].recorded) {
      pick = (int)i;
    } else {
      const cudaError_t q = cudaEventQuery(pool[i].done);
      if (q == cudaSuccess) pick = (int)i;
      else cudaGetLastError();  // not ready (or an earlier failure reported elsewhere)
    }
  }
  bool any_idle = false;
  for (auto &b : pool) any_idle |= !b.leased;
  if (pick < 0 && (pool.size() < kPoolBlocks || !any_idle)) {  // a new block
    hm_tree::ScratchBlock b;
    cudaError_t e = cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_err(e);
    pool.push_back(b);
    pick = (int)pool.size() - 1;
  }
  if (pick < 0) {  // the block idle longest; s waits for its last use
    for (size_t i = 0; i < pool.size(); i++)
      if (!pool[i].leased && (pick < 0 || pool[i].tick < pool[pick].tick)) pick = (int)i;
  }
  hm_tree::ScratchBlock &b = pool[pick];
  if (b.recorded) {
    cudaError_t e = cudaStreamWaitEvent(s_, b.done, 0);
    if (e != cudaSuccess) return cuda_err(e);
  }
  if (b.bytes < bytes) {
    if (b.ptr) t_->retired.push_back(b.ptr);  // its previous use may still run: released with the tree
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t want = (size_t)align_up((int64_t)std::max(bytes, bytes / 2 + bytes), 1 << 20);
    cudaError_t e = dev_alloc(&b.ptr, want);
    if (e != cudaSuccess) {
      b.ptr = nullptr;
      return cuda_err(e);
    }
    b.bytes = want;
  }
  b.stream = s_;
  b.leased = true;
  idx_ = pick;
  return HM_OK;
}

ScratchLease::~ScratchLease() {
  if (idx_ < 0) return;
  std::lock_guard<std::mutex> lk(t_->mu);
  hm_tree::ScratchBlock &b = t_->pool[idx_];
  if (cudaEventRecord(b.done, s_) == cudaSuccess) {
    b.recorded = true;
  } else {
    cudaGetLastError();
  }
  b.leased = false;
  b.tick = ++t_->pool_tick;
}

void *ScratchLease::ptr() const { return idx_ < 0 ? nullptr : t_->pool[idx_].ptr; }
size_t ScratchLease::bytes() const { return idx_ < 0 ? 0 : t_->pool[idx_].bytes; }

void free_scratch_pool(hm_tree *t) {
  for (auto &b : t->pool) {
    dev_release(b.ptr);
    if (b.done) cudaEventDestroy(b.done);
  }
  t->pool.clear();
  for (void *p : t->retired) dev_release(p);
  t->retired.clear();
}

static const char *kStageNames[kStageCount] = {"partition", "search", "search_batches", "range",
                                               "upsert", "join", "unpermute", "delete"};

static cudaEvent_t prof_event(hm_tree *t) {
  if (!t->prof_pool.empty()) {
    cudaEvent_t e = t->prof_pool.back();
    t->prof_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

int prof_begin(hm_tree *t, cudaStream_t s) {
  if (!t->prof) return -1;
  std::lock_guard<std::mutex> lk(t->mu);
  hm_tree::ProfRec r{-1, prof_event(t), prof_event(t)};
  cudaEventRecord(r.a, s);
  t->prof_recs.push_back(r);
  return (int)t->prof_recs.size() - 1;
}

void prof_end(hm_tree *t, int stage, int token, cudaStream_t s) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(t->mu);
  if (token >= (int)t->prof_recs.size()) return;
  t->prof_recs[token].stage = stage;
  cudaEventRecord(t->prof_recs[token].b, s);
}

}  // namespace hm

using namespace hm;

namespace {

// Chunks of the host-buffer pipeline: the first and last ones small (the
// first copy in and the last search + copy out run alone), the middle ones
// large (each chunk costs a few microseconds of copy setup and stream waits).
#ifndef HM_HOST_CHUNK
#define HM_HOST_CHUNK (1 << 21)
#endif
#ifndef HM_HOST_CHUNK_MIN
#define HM_HOST_CHUNK_MIN (1 << 18)
#endif
constexpr int64_t kChunk = HM_HOST_CHUNK;
constexpr int64_t kChunkMin = HM_HOST_CHUNK_MIN;

// Chunk sizes for n queries: doubling from kChunkMin up to kChunk, kChunk
// while the ramp down still fits, then halving back to kChunkMin.
std::vector<int64_t> chunk_schedule(int64_t n) {
  std::vector<int64_t> up, down;
  int64_t left = n;
  for (int64_t c = kChunkMin; c < kChunk && left > 0; c *= 2) {  // ramp up
    const int64_t m = std::min(c, left);
    up.push_back(m);
    left -= m;
  }
  for (int64_t c = kChunkMin; c < kChunk && left > 0; c *= 2) {  // ramp down, built from the end
    const int64_t m = std::min(c, left);
    down.push_back(m);
    left -= m;
  }
  while (left > 0) {
    const int64_t m = std::min(kChunk, left);
    up.push_back(m);
    left -= m;
  }
  up.insert(up.end(), down.rbegin(), down.rend());
  return up;
}

bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_pinned_host(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int check_config(const hm_config &c) {
  if (c.fanout != 64 && c.fanout != 128) return HM_EINVAL;
  if (c.leaf_cap != 16 && c.leaf_cap != 64) return HM_EINVAL;
  if (c.inner_fill < 2 || c.inner_fill > c.fanout) return HM_EINVAL;
  if (c.leaf_fill < 1 || c.leaf_fill > c.leaf_cap) return HM_EINVAL;
  switch (c.group_width) {
    case 1: case 2: case 4: case 8: case 16: case 32: break;
    default: return HM_EINVAL;
  }
  if (c.queries_per_group != 1 && c.queries_per_group != 2 && c.queries_per_group != 4)
    return HM_EINVAL;
  if (c.sort_bits < -1 || c.sort_bits > 16) return HM_EINVAL;
  if (c.smem_bytes < 0 || c.smem_bytes > 200 * 1024) return HM_EINVAL;
  if (c.cache_hints != 1 && c.cache_hints != 2) return HM_EINVAL;
  if (c.join != -1 && c.join != 1 && c.join != 2) return HM_EINVAL;
  return HM_OK;
}

void fill_defaults(hm_config *c) {
  if (c->fanout == 0) c->fanout = 64;
  if (c->leaf_cap == 0) c->leaf_cap = 16;
  if (c->inner_fill == 0) c->inner_fill = c->fanout;
  if (c->leaf_fill == 0) c->leaf_fill = c->leaf_cap;
  if (c->group_width == 0) c->group_width = 4;
  if (c->queries_per_group == 0) c->queries_per_group = 1;
  if (c->smem_bytes == 0) c->smem_bytes = 48 * 1024;
  if (c->cache_hints == 0) c->cache_hints = 1;
  if (c->join == 0) c->join = -1;
}

void choose_smem_levels(hm_tree *t) {
  t->smem_levels = 0;
  t->smem_nodes = 0;
  for (int l = 1; l <= t->height; l++) {
    int64_t nodes = t->lvl_start[l];
    int64_t bytes = nodes * t->inner_row * 8 + align_up(nodes * 4, 16) + 16;
    if (bytes > t->cfg.smem_bytes) break;
    t->smem_levels = l;
    t->smem_nodes = (int)nodes;
  }
}

cudaStream_t as_stream(hm_stream s) { return reinterpret_cast<cudaStream_t>(s); }

int free_tree(hm_tree *t) {
  if (!t) return HM_OK;
  cudaDeviceSynchronize();
  dev_release(t->arena);
  if (t->child_ids) cudaFree(t->child_ids);
  if (t->join_leafb) cudaFree(t->join_leafb);
  if (t->join_leafb_ready) cudaEventDestroy(t->join_leafb_ready);
  if (t->child_ids_ready) cudaEventDestroy(t->child_ids_ready);
  free_scratch_pool(t);
  if (t->d_err) cudaFree(t->d_err);
  if (t->pinned) cudaFreeHost(t->pinned);
  for (auto &s : t->io_stream)
    if (s) cudaStreamDestroy(s);
  for (auto &e : t->io_event)
    if (e) cudaEventDestroy(e);
  for (auto &r : t->prof_recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto &e : t->prof_pool) cudaEventDestroy(e);
  delete t;
  return HM_OK;
}

int ensure_io(hm_tree *t) {
  if (t->io_stream[0]) return HM_OK;
  for (auto &s : t->io_stream) {
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_err(e);
  }
  for (auto &e : t->io_event) {
    cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if (r != cudaSuccess) return cuda_err(r);
  }
  return HM_OK;
}

int ensure_pinned(hm_tree *t, size_t bytes) {
  if (bytes <= t->pinned_bytes) return HM_OK;
  if (t->pinned) cudaFreeHost(t->pinned);
  t->pinned = nullptr;
  t->pinned_bytes = 0;
  cudaError_t e = cudaMallocHost(&t->pinned, bytes);
  if (e != cudaSuccess) return cuda_err(e);
  t->pinned_bytes = bytes;
  return HM_OK;
}

// Search of device-resident queries on stream s by the plan for n queries.
int search_device(hm_tree *t, const int64_t *d_q, int64_t n, int64_t *d_out, cudaStream_t s,
                  void *scratch_base, size_t scratch_avail) {
  const SearchPlan p = plan_search(t, n);
  if (p.scratch > scratch_avail) return HM_ENOMEM;
  return run_planned_search(t, p, d_q, n, d_out, s, scratch_base);
}

size_t search_scratch_need(const hm_tree *t, int64_t n) { return plan_search(t, n).scratch; }

}  // namespace

// The join writes its results in first-pass order (no second inverse pass)
// for batches up to HM_JOIN_PLACED_MAX queries.  Its writes then scatter over
// one first-pass bucket's range of the result array (n / 256 results) while
// the CTAs work through that bucket; measured at 2^26 keys: 0.783 against
// 0.837 ms at 2^24 queries, 1.300 against 1.370 ms at 2^25, even at 2^26
// (2.315 / 2.327 ms) and 6.6 against 1.6 ms of join at 217 M queries, where
// the written ranges no longer stay in L2 until complete.
#ifndef HM_JOIN_PLACED
#define HM_JOIN_PLACED 1
#endif
#ifndef HM_JOIN_PLACED_MAX
#define HM_JOIN_PLACED_MAX (int64_t(1) << 25)
#endif

namespace hm {

SearchPlan plan_search(const hm_tree *t, int64_t n, int batches) {
  SearchPlan p;
  p.batches = std::max(batches, 1);
  if (n <= 0 || n > INT32_MAX) return p;  // positions are carried as int32
  const hm_config &c = t->cfg;
  const bool join = (c.join == 1 && (c.leaf_cap == 16 || c.leaf_cap == 64)) ||
                    (c.join == -1 && t->n_leaf >= 1024 && join_fits(t) &&
                     // measured: the join wins from about 4 queries per leaf
                     n >= std::min(t->join_tuned_min, std::max<int64_t>((int64_t)1 << 22, 4 * (int64_t)t->n_leaf)));
  if (join) {
    p.join = true;
    p.bits = join_bits(t);
    p.placed = HM_JOIN_PLACED && p.bits > 8 && n <= HM_JOIN_PLACED_MAX;
  } else {
    p.bits = (c.sort_bits > 0 && n >= t->presort_min) ? c.sort_bits : 0;
  }
  if (p.bits > 0) {  // grouped queries, grouped results, partition (offset mode), join
    p.scratch = 2 * (size_t)align_up(n * 8, 256) + partition_scratch_bytes(n, p.bits, true, p.batches);
    if (p.join) p.scratch += join_scratch_bytes(n, p.bits);
    if (p.placed) p.scratch += (size_t)align_up(n * 4, 256);
  }
  return p;
}

int run_planned_search(hm_tree *t, const SearchPlan &p, const int64_t *d_q, int64_t n, int64_t *d_out,
                       cudaStream_t s, void *scratch, const BatchView *bv) {
  if (n <= 0) return HM_OK;
  if (bv && p.bits <= 0) return HM_EINVAL;  // a batch set is searched through the pre-sort
  if (p.bits <= 0) {
    SearchLaunch l{d_q, d_out, nullptr, n};
    int tok = prof_begin(t, s);
    int rc = launch_search(t, l, t->cfg.group_width, t->cfg.queries_per_group, s);
    prof_end(t, kStageSearch, tok, s);
    return rc;
  }
  char *b = static_cast<char *>(scratch);
  int64_t *qs = reinterpret_cast<int64_t *>(b);
  int64_t *res = reinterpret_cast<int64_t *>(b + align_up(n * 8, 256));
  char *ps = b + 2 * align_up(n * 8, 256);
  char *js = ps + partition_scratch_bytes(n, p.bits, true, p.batches);
  const int64_t *bstart = nullptr;
  if (p.placed) {  // the join places results in first-pass order: one inverse pass
    int32_t *place = reinterpret_cast<int32_t *>(js + join_scratch_bytes(n, p.bits));
    int tok = prof_begin(t, s);
    int rc = partition_queries_placed(t, d_q, n, p.bits, qs, place, ps, s, &bstart, bv);
    prof_end(t, kStagePartition, tok, s);
    if (rc) return rc;
    tok = prof_begin(t, s);
    rc = launch_join(t, qs, bstart, p.bits, n, res, js, s, place);
    prof_end(t, kStageJoin, tok, s);
    if (rc) return rc;
    tok = prof_begin(t, s);
    rc = unpermute_first_pass(n, p.bits, res, d_out, ps, s, bv);
    prof_end(t, kStageUnpermute, tok, s);
    return rc;
  }
  int tok = prof_begin(t, s);
  int rc = partition_queries(t, d_q, n, p.bits, qs, nullptr, ps, s, &bstart, bv);
  prof_end(t, kStagePartition, tok, s);
  if (rc) return rc;
  tok = prof_begin(t, s);
  if (p.join) {
    rc = launch_join(t, qs, bstart, p.bits, n, res, js, s);
    prof_end(t, kStageJoin, tok, s);
  } else {
    SearchLaunch l{qs, res, nullptr, n};
    rc = launch_search(t, l, t->cfg.group_width, t->cfg.queries_per_group, s);
    prof_end(t, kStageSearch, tok, s);
  }
  if (rc) return rc;
  tok = prof_begin(t, s);
  rc = unpermute_results(n, p.bits, res, d_out, ps, s, bv);
  prof_end(t, kStageUnpermute, tok, s);
  return rc;
}

int opt_in_smem(const void *fn, int bytes) {
  static std::mutex mu;
  static std::set<std::tuple<const void *, int, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_err(e);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({fn, dev, bytes})) return HM_OK;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  if (e != cudaSuccess) return cuda_err(e);
  done.insert({fn, dev, bytes});
  return HM_OK;
}

// Entry points into this file's helpers for the other host sources.
int run_search(hm_tree *t, const int64_t *d_q, int64_t n, int64_t *d_out, cudaStream_t s,
               void *scratch, size_t scratch_bytes) {
  return search_device(t, d_q, n, d_out, s, scratch, scratch_bytes);
}
size_t run_search_scratch(const hm_tree *t, int64_t n) { return search_scratch_need(t, n); }
void refresh_smem_levels(hm_tree *t) { choose_smem_levels(t); }
}  // namespace hm

extern "C" {

int hm_config_default(hm_config *cfg) {
  if (!cfg) return HM_EINVAL;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->sort_bits = -1;
  fill_defaults(cfg);
  return HM_OK;
}

const char *hm_strerror(int code) {
  switch (code) {
    case HM_OK: return "ok";
    case HM_EINVAL: return "invalid argument or configuration";
    case HM_ENOMEM: return "out of device or pinned host memory";
    case HM_EDUPLICATE: return "bulk load: duplicate key";
    case HM_EMAXKEY: return "key equals the sentinel INT64_MAX";
    case HM_ECUDA: return "CUDA runtime error";
    case HM_ECAPACITY: return "output capacity too small";
    case HM_ETIMEOUT: return "a bounded device-side wait gave up";
    case HM_ENODEVICE: return "no usable CUDA device";
    case HM_EBUSY: return "busy: queue full or memory budget exhausted";
    case HM_ECANCELLED: return "request cancelled or server stopped";
    case HM_ETOOLARGE: return "size exceeds a documented maximum";
    case HM_EIO: return "file missing, unreadable, unwritable or malformed";
    default: return "unknown error";
  }
}

uint64_t hm_launch_count(void) { return g_launches.load(); }

int hm_last_cuda_error(char *buf, size_t cap) {
  const int e = g_last_cuda.load();
  if (buf && cap > 0) {
    std::snprintf(buf, cap, "%s: %s", cudaGetErrorName((cudaError_t)e), cudaGetErrorString((cudaError_t)e));
  }
  return e;
}

int hm_bulk_load(const int64_t *keys, const int64_t *vals, size_t n_, const hm_config *cfg_in,
                 hm_tree **out) {
  if (!out || (n_ > 0 && (!keys || !vals))) return HM_EINVAL;
  *out = nullptr;
  hm_config cfg;
  if (cfg_in) {
    cfg = *cfg_in;
    fill_defaults(&cfg);
  } else {
    hm_config_default(&cfg);
  }
  int rc = check_config(cfg);
  if (rc) return rc;
  const int64_t n = (int64_t)n_;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_err(e);

  hm_tree *t = new (std::nothrow) hm_tree();
  if (!t) return HM_ENOMEM;
  t->device = dev;
  t->cfg = cfg;
  cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, dev);
  rc = shape(n, cfg, &t->height, t->lvl_start, &t->n_inner, &t->n_leaf);
  if (rc) {
    delete t;
    return rc;
  }
  t->n_keys = n;
  t->inner_row = cfg.fanout / 8 + cfg.fanout;
  t->leaf_index = cfg.leaf_cap >= 32 ? cfg.leaf_cap / 8 : 0;
  t->leaf_row = t->leaf_index + 2 * cfg.leaf_cap;

  // Arena: every array 256-B aligned; prefix padded to a multiple of 4.
  size_t off_inner = 0;
  size_t off_prefix = off_inner + align_up(t->n_inner * t->inner_row * 8, 256);
  size_t off_lrows = off_prefix + align_up(align_up(t->n_inner, 4) * 4, 256);
  size_t off_lcnt = off_lrows + align_up(t->n_leaf * t->leaf_row * 8, 256);
  size_t off_lbase = off_lcnt + align_up(t->n_leaf * 4, 256);
  size_t total = off_lbase + align_up(t->n_leaf * 8, 256);

  // Temporaries: two key and two value buffers for the sort, sort scratch, flags.
  int64_t tn = std::max<int64_t>(std::max<int64_t>(n, t->n_leaf), 1);
  size_t tb = align_up(tn * 8, 256);
  size_t temp_bytes = 4 * tb + align_up((int64_t)radix_scratch_bytes(n), 256) + 256;
  char *temp = nullptr;
  e = dev_alloc(&t->arena, total);
  if (e == cudaSuccess) e = dev_alloc(reinterpret_cast<void **>(&temp), temp_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&t->d_err, 256);
  if (e != cudaSuccess) {
    dev_release(temp);
    free_tree(t);
    return cuda_err(e);
  }
  t->arena_bytes = total;
  char *base = static_cast<char *>(t->arena);
  t->inner = reinterpret_cast<int64_t *>(base + off_inner);
  t->prefix = reinterpret_cast<int32_t *>(base + off_prefix);
  t->leaf_rows = reinterpret_cast<int64_t *>(base + off_lrows);
  t->leaf_cnt = reinterpret_cast<int32_t *>(base + off_lcnt);
  t->leaf_base = reinterpret_cast<int64_t *>(base + off_lbase);

  uint64_t *uk = reinterpret_cast<uint64_t *>(temp);
  uint64_t *uk_alt = reinterpret_cast<uint64_t *>(temp + tb);
  int64_t *vv = reinterpret_cast<int64_t *>(temp + 2 * tb);
  int64_t *vv_alt = reinterpret_cast<int64_t *>(temp + 3 * tb);
  void *sort_scratch = temp + 4 * tb;
  unsigned *flags = reinterpret_cast<unsigned *>(temp + temp_bytes - 256);
  cudaStream_t s = 0;
  cudaMemsetAsync(t->arena, 0, total, s);
  cudaMemsetAsync(t->d_err, 0, 256, s);
  cudaMemsetAsync(flags, 0, 4, s);
  if (n > 0) {
    // keys land in uk_alt as int64, are sign-flipped into uk, values go to vv
    e = cudaMemcpyAsync(uk_alt, keys, n * 8, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(vv, vals, n * 8, cudaMemcpyDefault, s);
    if (e != cudaSuccess) {
      release_after(temp, s);
      free_tree(t);
      return cuda_err(e);
    }
    transform_keys_in(reinterpret_cast<int64_t *>(uk_alt), uk, n, s);
    bool alt = radix_sort_pairs<int64_t>(uk, vv, uk_alt, vv_alt, n, 0, 64, sort_scratch, s);
    if (alt) {
      std::swap(uk, uk_alt);
      std::swap(vv, vv_alt);
    }
    check_sorted_keys(uk, n, flags, s);
  }
  unsigned hflags = 0;
  e = cudaMemcpyAsync(&hflags, flags, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess || hflags) {
    release_after(temp, s);
    free_tree(t);
    if (e != cudaSuccess) return cuda_err(e);
    return (hflags & 2u) ? HM_EMAXKEY : HM_EDUPLICATE;
  }
  rc = build_from_sorted(t->target(), uk, vv, n, reinterpret_cast<int64_t *>(uk_alt), vv_alt, s);
  if (rc == HM_OK && n > 0) {
    uint64_t ends[2] = {0, 0};
    cudaMemcpyAsync(&ends[0], uk, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&ends[1], uk + n - 1, 8, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    t->key_min = (int64_t)(ends[0] ^ kSign);
    t->key_max = (int64_t)(ends[1] ^ kSign);
    if (e != cudaSuccess) rc = cuda_err(e);
  } else if (rc == HM_OK) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_err(e);
  }
  release_after(temp, s);
  if (rc) {
    free_tree(t);
    return rc;
  }
  choose_smem_levels(t);
  *out = t;
  return HM_OK;
}

int hm_free(hm_tree *t) { return free_tree(t); }

int hm_tree_get_info(const hm_tree *t, hm_tree_info *info) {
  if (!t || !info) return HM_EINVAL;
  std::memset(info, 0, sizeof(*info));
  info->fanout = t->cfg.fanout;
  info->leaf_cap = t->cfg.leaf_cap;
  info->height = t->height;
  info->inner_row_words = t->inner_row;
  info->leaf_row_words = t->leaf_row;
  info->leaf_index_words = t->leaf_index;
  info->smem_levels = t->smem_levels;
  info->n_keys = t->n_keys;
  info->n_inner = t->n_inner;
  info->n_leaf = t->n_leaf;
  for (int i = 0; i <= t->height && i <= kMaxLevels; i++) info->lvl_start[i] = t->lvl_start[i];
  info->inner = t->inner;
  info->prefix = t->prefix;
  info->leaf_rows = t->leaf_rows;
  info->leaf_cnt = t->leaf_cnt;
  info->leaf_base = t->leaf_base;
  info->device_bytes = t->arena_bytes;
  return HM_OK;
}

int hm_get_config(const hm_tree *t, hm_config *cfg) {
  if (!t || !cfg) return HM_EINVAL;
  *cfg = t->cfg;
  return HM_OK;
}

int hm_set_search_config(hm_tree *t, const hm_config *cfg) {
  if (!t || !cfg) return HM_EINVAL;
  hm_config c = t->cfg;
  if (cfg->group_width) c.group_width = cfg->group_width;
  if (cfg->queries_per_group) c.queries_per_group = cfg->queries_per_group;
  c.sort_bits = cfg->sort_bits;
  if (cfg->smem_bytes) c.smem_bytes = cfg->smem_bytes;
  if (cfg->cache_hints) c.cache_hints = cfg->cache_hints;
  if (cfg->join) c.join = cfg->join;
  int rc = check_config(c);
  if (rc) return rc;
  t->cfg = c;
  t->presort_min = 0;  // an explicit pre-sort applies at every batch size
  choose_smem_levels(t);
  return HM_OK;
}

int hm_search(hm_tree *t, const int64_t *q, size_t n_, int64_t *out, hm_stream hs) {
  if (!t || (n_ > 0 && (!q || !out))) return HM_EINVAL;
  const int64_t n = (int64_t)n_;
  if (n == 0) return HM_OK;
  cudaStream_t s = as_stream(hs);
  bool dq = is_device_ptr(q), dout = is_device_ptr(out);
  if (dq && dout) {
    const size_t need = search_scratch_need(t, n);
    ScratchLease lease(t, s);
    if (need > 0) {
      int rc = lease.acquire(need);
      if (rc) return rc;
    }
    return search_device(t, q, n, out, s, lease.ptr(), lease.bytes());
  }
  if (dq != dout) return HM_EINVAL;  // mixed host/device buffers are not supported
  // Host buffers: chunked pipeline over a ring of kIoRing device buffers, copies
  // in and out on their own streams overlapping the search of other chunks.
  // One host-buffer search at a time per tree (copy streams, events, staging).
  std::lock_guard<std::mutex> io_lock(t->io_mu);
  int rc = ensure_io(t);
  if (rc) return rc;
  constexpr int R = kIoRing;
  const std::vector<int64_t> sizes = chunk_schedule(n);
  int64_t chunk = 0;
  size_t sneed = 0;
  for (int64_t m : sizes) {
    chunk = std::max(chunk, m);
    sneed = std::max(sneed, search_scratch_need(t, m));
  }
  const size_t cbytes = (size_t)align_up(chunk * 8, 256);
  ScratchLease lease(t, s);  // its previous use is ordered before s, which the pipeline waits for
  rc = lease.acquire(2 * R * cbytes + sneed);
  if (rc) return rc;
  char *sb = static_cast<char *>(lease.ptr());
  int64_t *dqb[R], *dob[R];
  for (int b = 0; b < R; b++) {
    dqb[b] = reinterpret_cast<int64_t *>(sb + (size_t)b * cbytes);
    dob[b] = reinterpret_cast<int64_t *>(sb + (size_t)(R + b) * cbytes);
  }
  void *search_scratch = sb + 2 * R * cbytes;
  const bool pinned = is_pinned_host(q) && is_pinned_host(out);
  int64_t *hq[R] = {}, *ho[R] = {};
  if (!pinned) {
    rc = ensure_pinned(t, 2 * R * cbytes);
    if (rc) return rc;
    char *pb = static_cast<char *>(t->pinned);
    for (int b = 0; b < R; b++) {
      hq[b] = reinterpret_cast<int64_t *>(pb + (size_t)b * cbytes);
      ho[b] = reinterpret_cast<int64_t *>(pb + (size_t)(R + b) * cbytes);
    }
  }
  cudaStream_t sin = t->io_stream[0], scomp = t->io_stream[1], sout = t->io_stream[2];
  cudaEvent_t *ev_in = t->io_event, *ev_comp = t->io_event + R, *ev_out = t->io_event + 2 * R;
  cudaEvent_t ev_order = t->io_event[3 * R];
  // Order the pipeline after prior work on the caller's stream.
  cudaEventRecord(ev_order, s);
  cudaStreamWaitEvent(sin, ev_order, 0);
  cudaStreamWaitEvent(scomp, ev_order, 0);
  const int64_t nchunks = (int64_t)sizes.size();
  std::vector<int64_t> starts(nchunks + 1, 0);
  for (int64_t c = 0; c < nchunks; c++) starts[c + 1] = starts[c] + sizes[c];
  cudaError_t e = cudaSuccess;
  for (int64_t c = 0; c < nchunks && e == cudaSuccess; c++) {
    const int b = (int)(c % R);
    const bool reuse = c >= R;  // ring slot b held chunk c - R
    const int64_t o = starts[c], m = sizes[c];
    if (reuse) cudaStreamWaitEvent(sin, ev_comp[b], 0);  // dqb[b] no longer read
    if (pinned) {
      e = cudaMemcpyAsync(dqb[b], q + o, m * 8, cudaMemcpyHostToDevice, sin);
    } else {
      if (reuse) cudaEventSynchronize(ev_in[b]);  // staging hq[b] consumed
      std::memcpy(hq[b], q + o, m * 8);
      e = cudaMemcpyAsync(dqb[b], hq[b], m * 8, cudaMemcpyHostToDevice, sin);
    }
    cudaEventRecord(ev_in[b], sin);
    cudaStreamWaitEvent(scomp, ev_in[b], 0);
    if (reuse) cudaStreamWaitEvent(scomp, ev_out[b], 0);  // dob[b] drained
    rc = search_device(t, dqb[b], m, dob[b], scomp, search_scratch, sneed);
    if (rc) break;
    cudaEventRecord(ev_comp[b], scomp);
    cudaStreamWaitEvent(sout, ev_comp[b], 0);
    if (pinned) {
      e = cudaMemcpyAsync(out + o, dob[b], m * 8, cudaMemcpyDeviceToHost, sout);
    } else {
      if (reuse) {
        // drain chunk c - R from staging before reusing ho[b]
        cudaEventSynchronize(ev_out[b]);
        std::memcpy(out + starts[c - R], ho[b], sizes[c - R] * 8);
      }
      e = cudaMemcpyAsync(ho[b], dob[b], m * 8, cudaMemcpyDeviceToHost, sout);
    }
    cudaEventRecord(ev_out[b], sout);
  }
  if (rc == HM_OK && e == cudaSuccess) e = cudaStreamSynchronize(sout);
  if (rc == HM_OK && e == cudaSuccess && !pinned) {
    for (int64_t c = std::max<int64_t>(0, nchunks - R); c < nchunks; c++) {
      std::memcpy(out + starts[c], ho[(int)(c % R)], sizes[c] * 8);
    }
  }
  cudaStreamSynchronize(scomp);
  cudaStreamSynchronize(sin);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_err(e);
  return hm_sync(t, hs);
}

int hm_trim_memory(size_t *released) {
  const size_t freed = trim_cache(-1);
  if (released) *released = freed;
  return HM_OK;
}

int hm_sync(hm_tree *t, hm_stream hs) {
  if (!t) return HM_EINVAL;
  cudaError_t e = cudaStreamSynchronize(as_stream(hs));
  if (e != cudaSuccess) return cuda_err(e);
  // the error word is read on the caller's stream (the legacy default stream
  // would also wait for other streams' work on this device)
  unsigned err = 0;
  e = cudaMemcpyAsync(&err, t->d_err, 4, cudaMemcpyDeviceToHost, as_stream(hs));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(hs));
  if (e != cudaSuccess) return cuda_err(e);
  if (err) {
    cudaMemsetAsync(t->d_err, 0, 4, as_stream(hs));
    cudaStreamSynchronize(as_stream(hs));
    return (err & kErrTimeout) ? HM_ETIMEOUT : HM_ECUDA;
  }
  return HM_OK;
}

int hm_export(hm_tree *t, int64_t *keys, int64_t *vals, size_t cap, size_t *n) {
  if (!t) return HM_EINVAL;
  if (n) *n = (size_t)t->n_keys;
  if ((size_t)t->n_keys > cap) return HM_ECAPACITY;
  if (t->n_keys == 0) return HM_OK;
  if (!keys || !vals) return HM_EINVAL;
  cudaStream_t s = 0;
  bool dk = is_device_ptr(keys), dv = is_device_ptr(vals);
  if (dk && dv) {
    export_contents(t, keys, vals, s);
    return cuda_err(cudaStreamSynchronize(s));
  }
  const size_t b = (size_t)align_up(t->n_keys * 8, 256);
  ScratchLease lease(t, s);
  int rc = lease.acquire(2 * b);
  if (rc) return rc;
  int64_t *ek = static_cast<int64_t *>(lease.ptr());
  int64_t *ev = reinterpret_cast<int64_t *>(static_cast<char *>(lease.ptr()) + b);
  export_contents(t, ek, ev, s);
  cudaError_t e = cudaMemcpyAsync(keys, ek, t->n_keys * 8, cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vals, ev, t->n_keys * 8, cudaMemcpyDefault, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return cuda_err(e);
}

}  // extern "C"

namespace {

// Body of hm_range (len given, end == nullptr) and hm_range_between (end
// given, len == nullptr): locate, scan of the counts into offsets, total to
// the host, compacted copy.
int range_impl(hm_tree *t, const int64_t *start, const int32_t *len, const int64_t *end, size_t n_,
               int64_t *offsets, int64_t *okeys, int64_t *ovals, size_t cap, size_t *total, hm_stream hs) {
  const int64_t n = (int64_t)n_;
  cudaStream_t s = as_stream(hs);
  if (total) *total = 0;
  const void *second = end ? static_cast<const void *>(end) : static_cast<const void *>(len);
  const bool dev_in = n == 0 || (is_device_ptr(start) && is_device_ptr(second));
  const bool dev_out = is_device_ptr(offsets);
  const size_t b8 = (size_t)align_up((n + 1) * 8, 256), b4 = (size_t)align_up(n * 4 + 4, 256);
  size_t need = 2 * b4 + b8 + (size_t)align_up((int64_t)scan_scratch_bytes(n + 1), 256);
  if (!dev_in) need += b8 + (end ? b8 : b4);
  if (!dev_out) need += b8;
  ScratchLease lease(t, s);
  int rc = lease.acquire(need);
  if (rc) return rc;
  char *p = static_cast<char *>(lease.ptr());
  int32_t *fl = reinterpret_cast<int32_t *>(p);
  p += b4;
  int32_t *fs = reinterpret_cast<int32_t *>(p);
  p += b4;
  int64_t *cnt = reinterpret_cast<int64_t *>(p);
  p += b8;
  void *scan_scratch = p;
  p += align_up((int64_t)scan_scratch_bytes(n + 1), 256);
  const int64_t *d_start = start;
  const int32_t *d_len = len;
  const int64_t *d_end = end;
  cudaError_t e = cudaSuccess;
  if (!dev_in) {
    int64_t *ds = reinterpret_cast<int64_t *>(p);
    p += b8;
    e = cudaMemcpyAsync(ds, start, n * 8, cudaMemcpyHostToDevice, s);
    d_start = ds;
    if (end) {
      int64_t *de = reinterpret_cast<int64_t *>(p);
      p += b8;
      if (e == cudaSuccess) e = cudaMemcpyAsync(de, end, n * 8, cudaMemcpyHostToDevice, s);
      d_end = de;
    } else {
      int32_t *dl = reinterpret_cast<int32_t *>(p);
      p += b4;
      if (e == cudaSuccess) e = cudaMemcpyAsync(dl, len, n * 4, cudaMemcpyHostToDevice, s);
      d_len = dl;
    }
    if (e != cudaSuccess) return cuda_err(e);
  }
  int64_t *d_off = dev_out ? offsets : reinterpret_cast<int64_t *>(p);
  const int tok = prof_begin(t, s);
  if (n > 0) {
    rc = range_locate(t, d_start, d_len, d_end, n, fl, fs, cnt, s);
    if (rc) return rc;
  }
  exclusive_scan_i64(cnt, d_off, n, scan_scratch, s);
  int64_t tot = 0;
  e = cudaMemcpyAsync(&tot, d_off + n, 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_err(e);
  if (total) *total = (size_t)tot;
  if (!dev_out) {
    e = cudaMemcpyAsync(offsets, d_off, (n + 1) * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(e);
  }
  if ((size_t)tot > cap) return HM_ECAPACITY;
  if (tot == 0) return HM_OK;
  if (!okeys || !ovals) return HM_EINVAL;
  const bool dev_rec = is_device_ptr(okeys) && is_device_ptr(ovals);
  if (dev_rec) {
    rc = range_copy_out(t, fl, fs, d_off, n, okeys, ovals, s);
    prof_end(t, kStageRange, tok, s);
    if (rc) return rc;
    return hm_sync(t, hs);
  }
  // host record buffers: a stream-ordered temporary (no device-wide
  // synchronisation, unlike cudaMalloc/cudaFree)
  int64_t *tk = nullptr;
  e = cudaMallocAsync(reinterpret_cast<void **>(&tk), 2 * (size_t)align_up(tot * 8, 256), s);
  if (e != cudaSuccess) return cuda_err(e);
  int64_t *tv = reinterpret_cast<int64_t *>(reinterpret_cast<char *>(tk) + align_up(tot * 8, 256));
  rc = range_copy_out(t, fl, fs, d_off, n, tk, tv, s);
  prof_end(t, kStageRange, tok, s);
  if (rc == HM_OK) {
    e = cudaMemcpyAsync(okeys, tk, tot * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ovals, tv, tot * 8, cudaMemcpyDeviceToHost, s);
  }
  cudaFreeAsync(tk, s);
  if (rc == HM_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (rc == HM_OK) rc = cuda_err(e);
  return rc ? rc : hm_sync(t, hs);
}

}  // namespace

extern "C" {

int hm_range(hm_tree *t, const int64_t *start, const int32_t *len, size_t n, int64_t *offsets,
             int64_t *okeys, int64_t *ovals, size_t cap, size_t *total, hm_stream hs) {
  if (total) *total = 0;
  if (!t || (n > 0 && (!start || !len)) || !offsets) return HM_EINVAL;
  return range_impl(t, start, len, nullptr, n, offsets, okeys, ovals, cap, total, hs);
}

int hm_range_between(hm_tree *t, const int64_t *start, const int64_t *end, size_t n, int64_t *offsets,
                     int64_t *okeys, int64_t *ovals, size_t cap, size_t *total, hm_stream hs) {
  if (total) *total = 0;
  if (!t || (n > 0 && (!start || !end)) || !offsets) return HM_EINVAL;
  return range_impl(t, start, nullptr, end, n, offsets, okeys, ovals, cap, total, hs);
}

int hm_delete_batch(hm_tree *t, const int64_t *keys, size_t n_, size_t *removed, hm_stream hs) {
  if (removed) *removed = 0;
  if (!t || (n_ > 0 && !keys)) return HM_EINVAL;
  if (n_ > (size_t)0x7fffffff) return HM_ETOOLARGE;  // before anything is copied
  const int64_t n = (int64_t)n_;
  if (n == 0) return HM_OK;
  cudaStream_t s = as_stream(hs);
  const int64_t *dk = keys;
  ScratchLease staging(t, s);  // host batches are copied into a leased block (no cudaFree)
  if (!is_device_ptr(keys)) {
    int rc = staging.acquire((size_t)align_up(n * 8, 256));
    if (rc) return rc;
    int64_t *tk = static_cast<int64_t *>(staging.ptr());
    cudaError_t e = cudaMemcpyAsync(tk, keys, n * 8, cudaMemcpyDefault, s);
    if (e != cudaSuccess) return cuda_err(e);
    dk = tk;
  }
  int64_t gone = 0;
  int tok = prof_begin(t, s);
  int rc = delete_epoch(t, dk, n, &gone, s);
  prof_end(t, kStageDelete, tok, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (rc == HM_OK && e != cudaSuccess) rc = cuda_err(e);
  if (removed) *removed = (size_t)gone;
  choose_smem_levels(t);
  return rc ? rc : hm_sync(t, hs);
}

int hm_upsert_batch(hm_tree *t, const int64_t *keys, const int64_t *vals, size_t n_, int flags,
                    hm_stream hs) {
  if (!t || (n_ > 0 && (!keys || !vals))) return HM_EINVAL;
  if (flags != HM_UPSERT_SUPPLIED && flags != HM_UPSERT_REF_KEY_MINUS_1) return HM_EINVAL;
  if (n_ > (size_t)0x7fffffff) return HM_ETOOLARGE;  // before anything is copied
  const int64_t n = (int64_t)n_;
  if (n == 0) return HM_OK;
  cudaStream_t s = as_stream(hs);
  const int64_t *dk = keys, *dv = vals;
  ScratchLease staging(t, s);  // host batches are copied into a leased block (no cudaFree)
  if (!(is_device_ptr(keys) && is_device_ptr(vals))) {
    int rc = staging.acquire(2 * (size_t)align_up(n * 8, 256));
    if (rc) return rc;
    int64_t *tk = static_cast<int64_t *>(staging.ptr());
    int64_t *tv = reinterpret_cast<int64_t *>(static_cast<char *>(staging.ptr()) + align_up(n * 8, 256));
    cudaError_t e = cudaMemcpyAsync(tk, keys, n * 8, cudaMemcpyDefault, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tv, vals, n * 8, cudaMemcpyDefault, s);
    if (e != cudaSuccess) return cuda_err(e);
    dk = tk;
    dv = tv;
  }
  int tok = prof_begin(t, s);
  int rc = upsert_epoch(t, dk, dv, n, flags, s);
  prof_end(t, kStageUpsert, tok, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (rc == HM_OK && e != cudaSuccess) rc = cuda_err(e);
  choose_smem_levels(t);
  return rc ? rc : hm_sync(t, hs);
}

int hm_autotune(hm_tree *t, const int64_t *sample_q, size_t n_, hm_config *best) {
  if (!t || (n_ > 0 && !sample_q)) return HM_EINVAL;
  const int64_t n = (int64_t)n_;
  if (n == 0 || !is_device_ptr(sample_q)) return HM_EINVAL;
  int64_t *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_out, n * 8);
  if (e != cudaSuccess) return cuda_err(e);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const hm_config orig = t->cfg;
  hm_config best_cfg = orig;
  float best_ms = 1e30f;
  const int widths[] = {2, 4, 8, 16, 32};
  const int qpgs[] = {1, 2, 4};
  const int bits_list[] = {0, 8, 12, 16};
  const int hints_list[] = {1, 2};
  std::vector<hm_config> cands;
  for (int w : widths)
    for (int q : qpgs)
      for (int bits : bits_list)
        for (int hints : hints_list) {
          hm_config c = orig;
          c.group_width = w;
          c.queries_per_group = q;
          c.sort_bits = bits;
          c.cache_hints = hints;
          c.join = 2;
          cands.push_back(c);
        }
  {
    hm_config c = orig;  // the bucket join (its own bucket bits), timed last
    c.join = 1;
    cands.push_back(c);
  }
  int rc = HM_OK;
  float join_ms = 1e30f;
  for (const hm_config &c : cands) {
    t->cfg = c;
    choose_smem_levels(t);
    ScratchLease lease(t, 0);
    const size_t need = search_scratch_need(t, n);
    if (need > 0) rc = lease.acquire(need);
    if (rc) break;
    float ms = 1e30f;
    for (int rep = 0; rep < 3 && rc == HM_OK; rep++) {
      cudaEventRecord(a, 0);
      rc = search_device(t, sample_q, n, d_out, 0, lease.ptr(), lease.bytes());
      cudaEventRecord(b, 0);
      cudaEventSynchronize(b);
      float x = 0;
      cudaEventElapsedTime(&x, a, b);
      if (rep > 0 && x < ms) ms = x;
    }
    if (rc) break;
    if (c.join == 1) {
      join_ms = ms;
    } else if (ms < best_ms) {
      best_ms = ms;
      best_cfg = c;
    }
  }
  // The descent settings serve every batch, a pre-sort only batches at least
  // as large as the sample (it wins there; its fixed cost of about ten
  // launches loses on small batches); the join, where it won, serves batches
  // at least as large as the sample (the automatic choice).
  t->presort_min = best_cfg.sort_bits > 0 ? n : 0;
  if (join_ms < best_ms) {
    best_cfg.join = -1;
    t->join_tuned_min = std::min<int64_t>(t->join_tuned_min, n);
  } else {
    best_cfg.join = 2;
  }
  t->cfg = rc ? orig : best_cfg;
  choose_smem_levels(t);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d_out);
  if (best) *best = t->cfg;
  return rc ? rc : hm_sync(t, 0);
}

int hm_set_wait_limit(hm_tree *t, int64_t polls) {
  if (!t || polls < 0) return HM_EINVAL;
  t->wait_polls = polls;
  return HM_OK;
}

int hm_profile(hm_tree *t, int enable) {
  if (!t) return HM_EINVAL;
  t->prof = enable != 0;
  return HM_OK;
}

int hm_profile_read(hm_tree *t, hm_stage_time *out, int cap, int *n) {
  if (!t || (cap > 0 && !out)) return HM_EINVAL;
  double ms[kStageCount] = {};
  uint64_t cnt[kStageCount] = {};
  int rc = HM_OK;
  std::vector<hm_tree::ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(t->mu);
    recs.swap(t->prof_recs);
  }
  std::vector<cudaEvent_t> back;
  for (auto &r : recs) {
    if (r.stage >= 0) {
      cudaError_t e = cudaEventSynchronize(r.b);
      float x = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&x, r.a, r.b);
      if (e != cudaSuccess) rc = cuda_err(e);
      ms[r.stage] += x;
      cnt[r.stage]++;
    }
    back.push_back(r.a);
    back.push_back(r.b);
  }
  {
    std::lock_guard<std::mutex> lk(t->mu);
    t->prof_pool.insert(t->prof_pool.end(), back.begin(), back.end());
  }
  int k = 0;
  for (int i = 0; i < kStageCount; i++) {
    if (!cnt[i]) continue;
    if (k < cap) {
      std::memset(&out[k], 0, sizeof(out[k]));
      std::strncpy(out[k].name, kStageNames[i], sizeof(out[k].name) - 1);
      out[k].launches = cnt[i];
      out[k].total_ms = ms[i];
    }
    k++;
  }
  if (n) *n = k;
  return rc;
}

}  // extern "C"
