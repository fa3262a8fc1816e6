// Internal definitions shared by the harmonia-b200 CUDA sources.
//
// Device layout of a tree (all in one HBM arena, every array 256-B aligned):
//   inner     n_inner rows of (F/8 + F) int64: an index of every 8th key
//             (index[j] = key[8(j+1)], Max_Key past the end) followed by F
//             key slots, <= F-1 separators, Max_Key in unused slots.  Rows are
//             numbered breadth-first, the root is row 0.  This is the
//             reference's Inner_node key part (inner_index + inner_key,
//             open-harmonia/src/bpt.h:76-80) in the CFB's BFS order
//             (open-harmonia/regular_bpt/traversal.cpp:36-78).
//   prefix    n_inner int32 (padded to a multiple of 4): id of the node's first
//             child; children are contiguous, so child c of node i is
//             prefix[i] + c.  Children of the last inner level are numbered
//             from n_inner, leaf j = id - n_inner (CFB prefix[] and
//             idx - internal_node_num, open-harmonia/regular_bpt/cfb.cpp:21-32).
//   leaf_rows n_leaf rows of (LI + 2*LC) int64: LI = LC/8 index words when
//             LC >= 32 (else 0), LC key slots (Max_Key when unused), then the
//             LC values of those keys (-1 when unused).  Keys and values of a
//             leaf share one 256-B aligned record for LC = 16, so a hit reads
//             its value from the DRAM page its keys came from (the reference's
//             Record_list also keeps key and value together,
//             open-harmonia/src/bpt.h:206-239).
//   leaf_cnt  n_leaf int32 keys per leaf; leaf_base n_leaf int64 exclusive scan.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <utility>
#include <vector>

#include "../../include/harmonia.h"

namespace hm {

constexpr int64_t kMaxKey = INT64_MAX;
constexpr uint64_t kSign = 0x8000000000000000ull;
constexpr int kMaxLevels = 32;
#ifndef HM_HOST_RING
#define HM_HOST_RING 4
#endif
constexpr int kIoRing = HM_HOST_RING;  // chunks of the host-buffer pipeline in flight

// Error word bits a kernel may set (read back by hm_sync).
enum : unsigned {
  kErrTimeout = 1u,   // a bounded mbarrier wait gave up
  kErrBadNode = 2u,   // a node id fell outside the tree (corrupt layout)
};

struct DevTree {
  const int64_t *inner;
  const int32_t *prefix;
  const int64_t *leaf_rows;
  const int32_t *leaf_cnt;
  const int64_t *leaf_base;
  int64_t n_keys;
  int32_t n_inner;
  int32_t n_leaf;
  int32_t height;      // inner levels
  int32_t smem_nodes;  // top nodes staged in shared memory (a BFS prefix)
  int32_t smem_levels;
  int32_t cache_hints; // 1: L2 evict_last for inner rows, evict_first for leaves
  int64_t wait_polls;  // polls of the first bounded wait for the staged top levels
};

#ifdef __CUDACC__
// One thread's descent to the leaf whose key range holds q: at each inner row
// count the index words <= q (index word w mirrors key slot 8(w+1)) to pick an
// 8-key slice, then the slice's keys <= q; child = first child + count
// (open-harmonia/src/avx.cpp:2-54 counts separators <= key the same way).
// Inner rows are read-only while any caller runs.
__device__ __forceinline__ int32_t descend_leaf(const DevTree &t, int f, int64_t q) {
  const int ix = f / 8, row = ix + f;
  int32_t node = 0;
  for (int l = 0; l < t.height; l++) {
    const int64_t *r = t.inner + (int64_t)node * row;
    int k = 0;
    for (int v = 0; v < ix / 2; v++) {
      const longlong2 p = __ldg(reinterpret_cast<const longlong2 *>(r + 2 * v));
      k += (p.x <= q) + (p.y <= q);
    }
    k = min(k, ix - 1);
    int c = 8 * k;
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const longlong2 p = __ldg(reinterpret_cast<const longlong2 *>(r + ix + 8 * k + 2 * v));
      c += (p.x <= q) + (p.y <= q);
    }
    node = __ldg(t.prefix + node) + c;
  }
  return node - t.n_inner;
}
#endif

__host__ __device__ inline int64_t part_start(int64_t j, int64_t total, int64_t parts) {
  int64_t q = total / parts, r = total % parts;
  return j * q + (j < r ? j : r);
}

inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// The shape and arrays a bulk build writes: a tree's own arena, or a new one
// being built for a rebuild before it is swapped in.
struct BuildTarget {
  int fanout = 0, leaf_cap = 0;
  int height = 0, inner_row = 0, leaf_row = 0, leaf_index = 0;
  int64_t n_inner = 0, n_leaf = 0;
  int64_t lvl_start[kMaxLevels + 1] = {};
  int64_t *inner = nullptr;
  int32_t *prefix = nullptr;
  int64_t *leaf_rows = nullptr;
  int32_t *leaf_cnt = nullptr;
  int64_t *leaf_base = nullptr;
};

// Counts kernel launches issued by this library (hm_launch_count); launches
// recorded into a CUDA graph are counted when the graph is replayed.
void note_launch(int n = 1);
void set_capturing(bool on);

}  // namespace hm

struct hm_tree {
  int device = 0;
  hm_config cfg{};
  int height = 0;
  int inner_row = 0, leaf_row = 0, leaf_index = 0;
  int64_t n_keys = 0, n_inner = 0, n_leaf = 0;
  int64_t lvl_start[hm::kMaxLevels + 1] = {};
  int smem_levels = 0;
  int smem_nodes = 0;
  int num_sms = 148;
  int64_t key_min = 0, key_max = 0;  // for the pre-sort digit
  uint64_t generation = 0;           // bumped when the arena is rebuilt
  uint64_t shape_version = 0;        // bumped when inner nodes change in place (subtree rebalance)
  // bucket join: the leaf of every bucket boundary, kept for the current
  // shape, key range and bucket bits (join.cu); written on the stream of the
  // search that filled it, join_leafb_ready recorded after it
  mutable int32_t *join_leafb = nullptr;
  mutable int64_t join_leafb_cap = 0;
  mutable bool join_leafb_valid = false;
  mutable uint64_t join_leafb_gen = 0, join_leafb_shape = 0;
  mutable int64_t join_leafb_lo = 0, join_leafb_hi = 0, join_leafb_nleaf = 0;
  mutable int join_leafb_bits = 0;
  mutable cudaEvent_t join_leafb_ready = nullptr;
  int64_t join_tuned_min = INT64_MAX;  // smallest batch the autotuner saw the join win
  int64_t presort_min = 0;  // a tuned pre-sort applies from this batch size (0: any size)
  int64_t wait_polls = int64_t(1) << 24;  // hm_set_wait_limit
  // comparison baseline (hm_search_baseline): children ids per inner node,
  // child_ids_ready recorded after the kernel that filled them
  int32_t *child_ids = nullptr;
  uint64_t child_ids_generation = ~0ull;
  cudaEvent_t child_ids_ready = nullptr;
  // arena
  void *arena = nullptr;
  size_t arena_bytes = 0;
  int64_t *inner = nullptr;
  int32_t *prefix = nullptr;
  int64_t *leaf_rows = nullptr;
  int32_t *leaf_cnt = nullptr;
  int64_t *leaf_base = nullptr;
  // Scratch pool: blocks of working memory leased to one call at a time
  // (ScratchLease).  A block is ordered on the device after its previous use
  // by the event recorded at the end of that use, so reads enqueued on
  // different streams (or from different host threads) never share a block
  // while either runs.  A block that is too small is replaced by one half
  // again as large and retired (freed with the tree, never during a call:
  // cudaFree synchronises the device).
  struct ScratchBlock {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;  // stream of the last use
    cudaEvent_t done = nullptr;     // recorded at the end of the last use
    bool recorded = false;
    bool leased = false;
    uint64_t tick = 0;  // release order, for reuse of the block idle longest
  };
  std::vector<ScratchBlock> pool;
  uint64_t pool_tick = 0;
  std::vector<void *> retired;  // outgrown blocks, freed with the tree
  // guards the host-side state that concurrent calls share: the scratch pool,
  // the join boundary cache, the comparison kernel's child ids and the
  // profiling records
  mutable std::mutex mu;
  // held for a whole host-buffer search: its copy streams, events and pinned
  // staging serve one call at a time
  std::mutex io_mu;
  unsigned *d_err = nullptr;
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  cudaStream_t io_stream[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t io_event[3 * hm::kIoRing + 1] = {};  // per ring slot: copied in, searched, copied out; + order
  // stage timing (hm_profile): event pairs recorded around each stage
  struct ProfRec {
    int stage;
    cudaEvent_t a, b;
  };
  bool prof = false;
  std::vector<ProfRec> prof_recs;
  std::vector<cudaEvent_t> prof_pool;

  hm::BuildTarget target() const {
    hm::BuildTarget b;
    b.fanout = cfg.fanout;
    b.leaf_cap = cfg.leaf_cap;
    b.height = height;
    b.inner_row = inner_row;
    b.leaf_row = leaf_row;
    b.leaf_index = leaf_index;
    b.n_inner = n_inner;
    b.n_leaf = n_leaf;
    for (int i = 0; i <= hm::kMaxLevels; i++) b.lvl_start[i] = lvl_start[i];
    b.inner = inner;
    b.prefix = prefix;
    b.leaf_rows = leaf_rows;
    b.leaf_cnt = leaf_cnt;
    b.leaf_base = leaf_base;
    return b;
  }

  hm::DevTree view() const {
    hm::DevTree d;
    d.inner = inner;
    d.prefix = prefix;
    d.leaf_rows = leaf_rows;
    d.leaf_cnt = leaf_cnt;
    d.leaf_base = leaf_base;
    d.n_keys = n_keys;
    d.n_inner = (int32_t)n_inner;
    d.n_leaf = (int32_t)n_leaf;
    d.height = height;
    d.smem_nodes = smem_nodes;
    d.smem_levels = smem_levels;
    d.cache_hints = cfg.cache_hints;
    d.wait_polls = wait_polls;
    return d;
  }
};

namespace hm {

// ---- programmatic dependent launch ----
// Kernels of the search path are launched with programmatic stream
// serialization: a kernel may be scheduled while its predecessor on the
// stream drains, and waits for it (griddepcontrol.wait, a no-op for a normal
// launch) before touching memory.  Each such kernel calls pdl_enter() first;
// it also lets its own successor be scheduled (launch_dependents), which
// happens once every CTA of this grid has started.
#ifndef HM_PDL
#define HM_PDL 1
#endif
__device__ __forceinline__ void pdl_enter() {
#if HM_PDL
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// Launches kernel k on stream s with the programmatic-serialization
// attribute (the kernel must call pdl_enter() before any memory access).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = HM_PDL;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// ---- radix sort (sort.cu) ----
// Stable LSD sort of (ukeys, vals) by bits [begin_bit, end_bit) of the
// unsigned key.  Buffers ping-pong; returns true if the result ends in the
// *_alt buffers.  Scratch needs radix_scratch_bytes(n).
size_t radix_scratch_bytes(int64_t n);
template <typename V>
bool radix_sort_pairs(uint64_t *ukeys, V *vals, uint64_t *ukeys_alt, V *vals_alt,
                      int64_t n, int begin_bit, int end_bit, void *scratch,
                      cudaStream_t s);
// The same sort of ukeys with each element's input position (int32, so n <
// 2^31) as the payload, generated by the first pass; true if the sorted
// keys and positions ended in the *_alt buffers.
bool radix_sort_positions(uint64_t *ukeys, int32_t *pos, uint64_t *ukeys_alt, int32_t *pos_alt, int64_t n,
                          int begin_bit, int end_bit, void *scratch, cudaStream_t s);

// ---- bulk build (build.cu) ----
int shape(int64_t n, const hm_config &c, int *height, int64_t *lvl_start,
          int64_t *n_inner, int64_t *n_leaf);
// Builds the arrays of b (already sized and allocated) from sorted
// unsigned-transformed keys.
int build_from_sorted(const BuildTarget &b, const uint64_t *ukeys, const int64_t *vals,
                      int64_t n, int64_t *tmp_a, int64_t *tmp_b, cudaStream_t s);
void check_sorted_keys(const uint64_t *ukeys, int64_t n, unsigned *d_flags, cudaStream_t s);
void transform_keys_in(const int64_t *keys, uint64_t *ukeys, int64_t n, cudaStream_t s);
void transform_keys_out(const uint64_t *ukeys, int64_t *keys, int64_t n, cudaStream_t s);

// ---- search (search.cu) ----
struct SearchLaunch {
  const int64_t *q;
  int64_t *out;
  const int32_t *pos;  // optional: out[pos[i]] = result of q[i]
  int64_t n;
};
int launch_search(const hm_tree *t, const SearchLaunch &l, int group_width, int qpg,
                  cudaStream_t s);
int launch_search_batches(const hm_tree *t, const hm_batch *d_batches, const int64_t *d_tile_start,
                          int nb, int64_t total_tiles, int group_width, int qpg,
                          cudaStream_t s);
int search_tile_queries(int group_width, int qpg);  // queries per CTA tile
// Resolves (and caches) the kernel's launch configuration without launching,
// so that a later launch can be captured in a CUDA graph.
int launch_search_warm(const hm_tree *t, int group_width, int qpg);
size_t search_smem_bytes(const hm_tree *t);

// ---- query pre-sort (partition.cu) ----
// A batch set on the device: batches[b] holds queries [qpre[b], qpre[b+1])
// of the set's concatenation (qpre has nb + 1 entries).
struct BatchView {
  const hm_batch *batches = nullptr;
  const int64_t *qpre = nullptr;
  int nb = 0;
};

// Pre-sort for a consumer that places its results itself (bits in 9..16):
// the first pass as partition_queries (offset mode), the second records in
// place[i] the position grouped query i had after the first pass.  Results
// written to res1[place[i]] are in first-pass order, which
// unpermute_first_pass takes back to the input order.
int partition_queries_placed(const hm_tree *t, const int64_t *q, int64_t n, int bits, int64_t *q_out,
                             int32_t *place, void *scratch, cudaStream_t s, const int64_t **bucket_start,
                             const BatchView *bv = nullptr);
int unpermute_first_pass(int64_t n, int bits, const int64_t *res1, int64_t *out, void *scratch, cudaStream_t s,
                         const BatchView *bv = nullptr);

// offsets: the partition keeps chunk offsets in the scratch for
// unpermute_results (pos_out == nullptr); else it writes input positions.
size_t partition_scratch_bytes(int64_t n, int bits, bool offsets, int batches = 1);  // batches: of a batch set
// Groups queries by the top `bits` bits of their key (relative to the tree's
// key range); *bucket_start (if given) receives a device pointer, inside the
// scratch, to the 2^bits + 1 bucket starts.  pos_out: original position of
// each grouped query, or nullptr for the offset mode.
// With bv, the queries are read from the batch set instead of q.
int partition_queries(const hm_tree *t, const int64_t *q, int64_t n, int bits,
                      int64_t *q_out, int32_t *pos_out, void *scratch, cudaStream_t s,
                      const int64_t **bucket_start = nullptr, const BatchView *bv = nullptr);
// Offset mode: out[i] = result of input query i, given the results in grouped
// order (res_sorted, clobbered) and the scratch of the matching partition.
// With bv, the results go to the batch set's outputs instead of out.
int unpermute_results(int64_t n, int bits, int64_t *res_sorted, int64_t *out, void *scratch, cudaStream_t s,
                      const BatchView *bv = nullptr);

// ---- scan, export, range (misc.cu) ----
void scan_counts(int64_t *counts, int64_t m, cudaStream_t s);  // one-CTA in-place exclusive scan
size_t scan_scratch_bytes(int64_t n);
void exclusive_scan_i64(const int64_t *in, int64_t *out, int64_t n, void *scratch,
                        cudaStream_t s);  // out has n+1 entries
void exclusive_scan_i32(const int32_t *in, int64_t *out, int64_t n, void *scratch, cudaStream_t s);
void export_contents(const hm_tree *t, int64_t *d_keys, int64_t *d_vals, cudaStream_t s);
size_t range_scratch_bytes(int64_t n);
// Counts per query: the first len[i] records >= start[i] (end == nullptr), or
// every record in [start[i], end[i]] (len unused).
int range_locate(const hm_tree *t, const int64_t *start, const int32_t *len, const int64_t *end, int64_t n,
                 int32_t *first_leaf, int32_t *first_slot, int64_t *count, cudaStream_t s);
int range_copy_out(const hm_tree *t, const int32_t *first_leaf, const int32_t *first_slot,
                   const int64_t *offsets, int64_t n, int64_t *okeys, int64_t *ovals, cudaStream_t s);

// ---- upsert (upsert.cu) ----
int delete_epoch(hm_tree *t, const int64_t *d_keys, int64_t n, int64_t *removed, cudaStream_t s);
int rebuild_from_sorted(hm_tree *t, const uint64_t *ck, const int64_t *cv, int64_t n1, cudaStream_t s);
int upsert_epoch(hm_tree *t, const int64_t *d_keys, const int64_t *d_vals, int64_t n,
                 int flags, cudaStream_t s);

// ---- stage timing ----
enum Stage { kStagePartition = 0, kStageSearch, kStageBatches, kStageRange, kStageUpsert, kStageJoin,
             kStageUnpermute, kStageDelete, kStageCount };
// Records the start event of a stage on stream s (no-op unless profiling).
int prof_begin(hm_tree *t, cudaStream_t s);
void prof_end(hm_tree *t, int stage, int token, cudaStream_t s);

// ---- bucket join (join.cu) ----
int join_bits(const hm_tree *t);   // bucket bits for the join (leaves per bucket fit shared memory)
bool join_fits(const hm_tree *t);  // the join supports this leaf size and its buckets fit on average
size_t join_scratch_bytes(int64_t n, int bits);
// place: nullptr = results in grouped order (out[i] for grouped query i);
// else out[place[i]].
int launch_join(const hm_tree *t, const int64_t *qs, const int64_t *bstart, int bits, int64_t n, int64_t *out,
                void *scratch, cudaStream_t s, const int32_t *place = nullptr);

// Opts kernel fn in to `bytes` of dynamic shared memory (and the largest
// shared-memory carveout) on the current device; once per device, kernel and
// size, from any thread.
int opt_in_smem(const void *fn, int bytes);

// ---- search plan (harmonia.cu) ----
// How a batch of n queries is searched: NTG descent on the batch as given
// (bits = 0), after a pre-sort (bits > 0, join = false), or pre-sort +
// bucket join; scratch = bytes of working memory it needs.
struct SearchPlan {
  int bits = 0;
  bool join = false;
  bool placed = false;  // the join writes its results in first-pass order (two-pass pre-sort)
  int batches = 1;  // batches of a batch set (its first pre-sort pass cuts each batch apart)
  size_t scratch = 0;
};
SearchPlan plan_search(const hm_tree *t, int64_t n, int batches = 1);
int run_planned_search(hm_tree *t, const SearchPlan &p, const int64_t *d_q, int64_t n, int64_t *d_out,
                       cudaStream_t s, void *scratch, const BatchView *bv = nullptr);

// ---- host helpers (harmonia.cu) ----
// Point search of device-resident queries on s, with the configured pre-sort;
// scratch must hold run_search_scratch(t, n) bytes.
int run_search(hm_tree *t, const int64_t *d_q, int64_t n, int64_t *d_out, cudaStream_t s,
               void *scratch, size_t scratch_bytes);
size_t run_search_scratch(const hm_tree *t, int64_t n);
void refresh_smem_levels(hm_tree *t);

// ---- scratch pool (harmonia.cu) ----
// A lease on one block of t's scratch pool for the work one call enqueues on
// stream s.  acquire(bytes) picks an idle block (the one last used on s, else
// one whose last use has finished, else a new one while the pool is small,
// else the one idle longest), makes s wait for the block's previous use and
// replaces it by a larger one if needed.  The destructor records the end of this use on s
// and returns the block to the pool, so the caller must have enqueued all
// work that touches the block by then.  A stream under graph capture gets
// HM_EINVAL: captured work uses memory the graph owns (hm_plan_create).
class ScratchLease {
 public:
  ScratchLease(hm_tree *t, cudaStream_t s) : t_(t), s_(s) {}
  ~ScratchLease();
  ScratchLease(const ScratchLease &) = delete;
  ScratchLease &operator=(const ScratchLease &) = delete;
  int acquire(size_t bytes);
  void *ptr() const;
  size_t bytes() const;

 private:
  hm_tree *t_;
  cudaStream_t s_;
  int idx_ = -1;
};
void free_scratch_pool(hm_tree *t);  // after the device is idle

// Large device blocks through the process's block cache (harmonia.cu):
// dev_alloc reuses a cached block of the device when one fits, else
// cudaMalloc; dev_release keeps the block for reuse (no work may still be in
// flight on it; blocks not from dev_alloc are freed); release_after first
// waits for stream s.
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_release(void *p);
void release_after(void *p, cudaStream_t s);

// ---- misc ----
int cuda_err(cudaError_t e);

}  // namespace hm
