/* harmonia-b200: batched B+tree search, range scan and batched upsert on one
 * NVIDIA B200 (sm_100a), behind a C ABI.
 *
 * The reference (fudan-ppi/harmonia, open-harmonia/) has no library API: each
 * experiment is `void fn(BPlusTree &tree, std::ifstream &search_file)`
 * (open-harmonia/src/ppi-bpt.h:4-98, open-harmonia/regular_bpt/gpu-cfb.h:2-8)
 * that builds, uploads, searches and frees inside one call, and errors end
 * the process (open-harmonia/src/cuda_utils.h:3-12).  The entry points below
 * replace those calls one to one; each names the reference code it stands in
 * for.  All functions return HM_OK (0) or a negative HM_E* code; none exits.
 *
 * Keys and values are int64 compared as signed integers.  INT64_MAX is the
 * empty-slot sentinel (Max_Key, open-harmonia/src/bpt.h:26) and cannot be
 * stored; a search for it returns "not found".  Not found is -1
 * (open-harmonia/src/bpt.h:272).
 *
 * Pointers passed as query/result buffers may be host or device memory
 * (detected per call).  With device buffers a call only enqueues work on the
 * given stream and returns; with host buffers it copies in chunks through
 * pinned staging, overlapping copies with the search, and returns when the
 * results are in host memory.
 *
 * Concurrency.  Read-only calls on one tree (hm_search, hm_range,
 * hm_search_batches, hm_export, hm_search_baseline) may be issued from any
 * host threads on any streams, and their work may overlap on the device: each
 * call leases a scratch block of its own from the tree's pool, ordered on the
 * device after that block's previous use; a block that is too small is
 * replaced by one half again as large and the old one is released only with
 * the tree, so no call frees device memory (which would synchronise the
 * device).
 * Host-buffer searches of one tree take turns (they share the tree's copy
 * streams and pinned staging).  Calls that change the tree or its settings
 * (hm_upsert_batch, hm_delete_batch, hm_set_search_config, hm_autotune,
 * hm_free) must not overlap any other call on the same tree, on the host or
 * on the device.  Calls that need scratch return HM_EINVAL on a stream under
 * graph capture; hm_plan_create captures searches with memory of its own.
 * hm_search_noalloc has its own rule (one shared array per device).
 */
#ifndef HARMONIA_H
#define HARMONIA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default) /* the library builds with -fvisibility=hidden */
#endif

#define HM_MAX_KEY INT64_MAX
#define HM_NOT_FOUND (-1)

enum {
  HM_OK = 0,
  HM_EINVAL = -1,      /* bad argument or configuration */
  HM_ENOMEM = -2,      /* device or pinned-host allocation failed */
  HM_EDUPLICATE = -3,  /* bulk load: a key occurs twice */
  HM_EMAXKEY = -4,     /* a key equals the sentinel INT64_MAX */
  HM_ECUDA = -5,       /* a CUDA runtime call failed */
  HM_ECAPACITY = -6,   /* range: output capacity too small */
  HM_ETIMEOUT = -7,    /* a bounded device-side wait gave up */
  HM_ENODEVICE = -8,   /* no usable CUDA device */
  HM_EBUSY = -9,       /* serving: queue full or budget exhausted */
  HM_ECANCELLED = -10, /* serving: request cancelled or server stopped */
  HM_ETOOLARGE = -11,  /* a size exceeds a documented maximum */
  HM_EIO = -12         /* a file could not be opened, read or written, or is malformed */
};

typedef void *hm_stream; /* a cudaStream_t; NULL = the legacy default stream */
typedef struct hm_tree hm_tree;

/* Layout and search parameters.  The reference fixes these at compile time:
 * BPT_ORDER 64 (open-harmonia/src/bpt.h:15), DEFAULT_ORDER / Narrow_Rate from
 * CMake (open-harmonia/CMakeLists.txt:55-57), Thread_Per_Query and
 * GPU_SWP_SIZE per file (open-harmonia/src/full-multi-prefix-sort-8thread.cu:19-29),
 * sort bits [48,64) (same file :305-309).  Zero means "default" everywhere. */
typedef struct {
  int fanout;            /* inner-node key slots: 64 or 128 (default 64) */
  int leaf_cap;          /* leaf key slots: 16 or 64 (default 16) */
  int inner_fill;        /* children per inner node at bulk load, 2..fanout (default fanout) */
  int leaf_fill;         /* keys per leaf at bulk load, 1..leaf_cap (default leaf_cap) */
  int group_width;       /* lanes cooperating on one query: 1,2,4,8,16,32 (default 4) */
  int queries_per_group; /* queries a group keeps in flight: 1,2,4 (default 1; at 1 a 16-key leaf's
                            values load with its keys) */
  int sort_bits;         /* query pre-sort: top bits, 0 = off, 1..16, -1 = auto (default -1) */
  int smem_bytes;        /* budget for top levels staged in shared memory (default 49152) */
  int cache_hints;       /* L2 policy: 1 = inner rows evict_last, leaves evict_first; 2 = none
                            (default 1) */
  int join;              /* large batches: 1 = pre-sort + bucket join, 2 = never, -1 = when the
                            batch has at least 4 queries per leaf and 2^22 queries, or at least
                            the sample size at which hm_autotune saw the join win (default -1) */
} hm_config;

/* Read-only description of a loaded tree. */
typedef struct {
  int fanout, leaf_cap, height; /* height = number of inner levels */
  int inner_row_words;          /* int64 words per inner row: fanout/8 index + fanout keys */
  int leaf_row_words;           /* int64 words per leaf row: index, leaf_cap keys, leaf_cap values */
  int leaf_index_words;         /* index words at the start of a leaf row (leaf_cap >= 32) */
  int smem_levels;              /* top levels staged in shared memory by the search kernel */
  int64_t n_keys, n_inner, n_leaf;
  int64_t lvl_start[33];        /* BFS id of each inner level's first node */
  /* device pointers into the tree's HBM arena */
  const int64_t *inner;     /* n_inner rows */
  const int32_t *prefix;    /* n_inner first-child ids (leaves count from n_inner) */
  const int64_t *leaf_rows; /* n_leaf rows */
  const int32_t *leaf_cnt;  /* n_leaf */
  const int64_t *leaf_base; /* n_leaf, exclusive scan of leaf_cnt */
  size_t device_bytes;      /* bytes of the tree arena */
} hm_tree_info;

/* Fills *cfg with the defaults. */
int hm_config_default(hm_config *cfg);

/* Builds a device-resident tree from n (key, value) pairs on the GPU: sort,
 * duplicate/sentinel check, leaves, then inner levels with the prefix-sum
 * child array.  Keys need not be sorted.
 * Replaces: the serial BPlusTree::insert loop + BPlusTree::sort + the upload
 * (open-harmonia/src/main.cpp:50-67,151-152; open-harmonia/src/traversal.cpp:35-195;
 * prepareGPU_v2 / prepareGPU_leaf, open-harmonia/src/prepareGPU.cu:140-163;
 * CFB generateCFB + prepareGPU, open-harmonia/regular_bpt/traversal.cpp:81-99,
 * open-harmonia/regular_bpt/helper.cu:12-28). */
int hm_bulk_load(const int64_t *keys, const int64_t *vals, size_t n,
                 const hm_config *cfg, hm_tree **out);

/* Batched point search: out[i] = value of q[i], or -1.
 * Replaces: full_multi_prefix_sort_8thread (+ its kernel and the CUB
 * pre-sort), open-harmonia/src/full-multi-prefix-sort-8thread.cu:95-495, and
 * multi_prefix_sort, open-harmonia/regular_bpt/prefix-sort.cu:98-478; the
 * result decode of the same file :454-476 is done on the device. */
int hm_search(hm_tree *t, const int64_t *q, size_t n, int64_t *out, hm_stream s);

/* One query batch of a multi-batch launch. */
typedef struct {
  const int64_t *q; /* device pointer */
  int64_t *out;     /* device pointer */
  int64_t n;
} hm_batch;

/* Searches nb independent batches (device buffers) together: small sets in
 * one persistent kernel that hands out tiles of all batches, large sets
 * gathered, pre-sorted together, searched and scattered back.  Returns when
 * done.
 * Replaces: the per-bucket launch loop of launch_kernel_thread,
 * open-harmonia/src/full-multi-prefix-sort-8thread.cu:276-327. */
int hm_search_batches(hm_tree *t, const hm_batch *batches, int nb, hm_stream s);

/* A batch set captured once as a CUDA graph and replayed: the batch buffers
 * are fixed, their contents may change between launches.  The plan owns its
 * work memory; it re-captures itself after the tree is rebuilt or retuned.
 * hm_plan_launch only enqueues on s.  (No reference counterpart: the
 * reference re-issues every launch from its launcher thread.) */
typedef struct hm_plan hm_plan;
int hm_plan_create(hm_tree *t, const hm_batch *batches, int nb, hm_plan **out);
int hm_plan_launch(hm_plan *p, hm_stream s);
int hm_plan_free(hm_plan *p);

/* Range scan: for query i the first len[i] records with key >= start[i], in
 * key order (fewer if the key space ends), compacted: query i's records are
 * okeys/ovals[offsets[i] .. offsets[i+1]).  offsets has n+1 entries; *total
 * receives offsets[n].  Returns HM_ECAPACITY (with *total set) when cap is
 * too small.
 * Replaces: range_prefix_sort_1thread_search_and_1thread_scan and its kernel,
 * open-harmonia/src/range.cu:101-227,312-360 (fixed Range_Size=8 slots, end
 * key forced to Max_Key), and traverse_PPItree, open-harmonia/src/cpu-range.cpp:129-183. */
int hm_range(hm_tree *t, const int64_t *start, const int32_t *len, size_t n,
             int64_t *offsets, int64_t *okeys, int64_t *ovals, size_t cap,
             size_t *total, hm_stream s);

/* Inclusive range scan: for query i every record with start[i] <= key <=
 * end[i], in key order (none when end[i] < start[i]; end[i] = INT64_MAX runs
 * to the end of the key space), compacted as hm_range: offsets has n+1
 * entries, *total receives offsets[n], HM_ECAPACITY (with *total set) when
 * cap is too small.  start and end may be host or device memory, as may the
 * outputs.  Pairs read by hm_read_ranges from a reference range file can be
 * passed as they are.
 * Replaces: BPlusTree::range_search(start_key, end_key, &records)
 * (open-harmonia/src/bpt.cpp:695-769) and the CFB find_range
 * (open-harmonia/regular_bpt/regular_bpt.cpp:320-340). */
int hm_range_between(hm_tree *t, const int64_t *start, const int64_t *end, size_t n,
                     int64_t *offsets, int64_t *okeys, int64_t *ovals, size_t cap,
                     size_t *total, hm_stream s);

#define HM_UPSERT_SUPPLIED 0        /* an existing key takes the supplied value */
#define HM_UPSERT_REF_KEY_MINUS_1 1 /* an existing key takes key-1, as the reference does */

/* Applies one epoch of upserts on the GPU: existing keys are updated in
 * place, new keys are merged into their leaves, and leaves that overflow
 * trigger a rebuild.  Within one batch the last occurrence of a key wins.
 * At most 2^31 - 1 keys per batch (HM_ETOOLARGE beyond).
 * Replaces: BPlusTree::insert_parallel_Newupdate_batch and its worker
 * (open-harmonia/src/bpt-ppi-update-batch.cpp:10-200), insert_Newupdate and
 * rebuild_without_leaf (open-harmonia/src/bpt-ppi-update.cpp:99-138,320-463). */
int hm_upsert_batch(hm_tree *t, const int64_t *keys, const int64_t *vals,
                    size_t n, int flags, hm_stream s);

/* Sorted contents of the tree into host or device buffers; *n receives the
 * key count.  Returns HM_ECAPACITY if cap < count.
 * Replaces: the ENABLE_TEST decode/print loops of the reference drivers
 * (open-harmonia/src/full-multi-prefix-sort-8thread.cu:454-476). */
int hm_export(hm_tree *t, int64_t *keys, int64_t *vals, size_t cap, size_t *n);

int hm_tree_get_info(const hm_tree *t, hm_tree_info *info);

/* Changes the search parameters of a loaded tree (group_width,
 * queries_per_group, sort_bits, smem_bytes); layout fields are ignored. */
int hm_set_search_config(hm_tree *t, const hm_config *cfg);
int hm_get_config(const hm_tree *t, hm_config *cfg);

/* Times candidate search parameters on a sample of queries (device buffer)
 * and keeps the fastest: group width {2,4,8,16,32} x queries per group
 * x sort bits.  Writes the chosen config to *best (may be NULL).
 * Replaces: the recompile-per-point sweeps open-harmonia/tests/multi-regular-narrow.sh
 * and open-harmonia/tests/bit-prefix-sort-8thread.sh. */
int hm_autotune(hm_tree *t, const int64_t *sample_q, size_t n, hm_config *best);

/* Polls a search kernel makes while it waits for the top levels it stages in
 * shared memory (and the bucket join for the leaf records its TMA loads
 * stage), before it gives up, records HM_ETIMEOUT (reported by hm_sync) and
 * returns without results (default 2^24, far above the microseconds a copy
 * takes).  A CTA that gave up still waits, with the default bound, for its
 * copies to land before it exits.  For tests of the timeout path: 0 makes
 * every staged wait give up at once.  Not thread-safe
 * with calls in flight on the tree.  No counterpart in the reference, whose
 * kernels have no bounded waits. */
int hm_set_wait_limit(hm_tree *t, int64_t polls);

/* Waits for the tree's outstanding work on stream s and returns any error a
 * kernel recorded (HM_ETIMEOUT for a bounded wait that gave up). */
int hm_sync(hm_tree *t, hm_stream s);

int hm_free(hm_tree *t);
const char *hm_strerror(int code);

/* Device memory the library keeps for reuse: the arena, build temporaries
 * and scratch blocks of freed trees and finished rebuilds (up to 16 GiB per
 * process; a cudaMalloc of a GiB-sized block maps it anew, and cudaFree
 * synchronises the device).  Later trees and calls on the same device take
 * blocks from it.  hm_trim_memory frees all of it and reports the bytes in
 * *released (may be NULL).  No counterpart in the reference, whose
 * experiments cudaMalloc and cudaFree their buffers per run. */
int hm_trim_memory(size_t *released);

/* ---- Serving loop ----
 * A request queue in front of one tree.  Callers submit point-search, range
 * and upsert requests with host buffers and wait on the returned ticket.  A
 * dispatcher thread admits requests in submission order while their device
 * bytes fit the budget, coalesces consecutive reads of one kind into one
 * launch, and keeps up to `streams` launches in flight (requests arriving
 * while others run are admitted as slots and memory free up).  An upsert or
 * a delete is an epoch barrier: it applies after every earlier request and
 * before every later one, so a read returns what it would return alone
 * against the writes submitted before it.  Every device wait is bounded
 * (device_wait_limit_ms).  No counterpart in the reference, which only runs
 * offline experiments (open-harmonia/src/main.cpp:160-417). */
enum { HM_REQ_SEARCH = 0, HM_REQ_RANGE = 1, HM_REQ_UPSERT = 2, HM_REQ_DELETE = 3 };

typedef struct {
  int kind;              /* HM_REQ_* */
  const int64_t *keys;   /* search: queries; range: start keys; upsert, delete: keys (host) */
  const int32_t *lens;   /* range: record counts */
  const int64_t *vals;   /* upsert: values */
  size_t n;
  int64_t *out;          /* search: n values or -1.  A search's keys and out may
                            also be page-locked host memory (cudaHostAlloc,
                            cudaHostRegister) or device memory: those are
                            copied by DMA with no host staging copy */
  int64_t *offsets;      /* range: n+1 offsets into out_keys/out_vals */
  int64_t *out_keys, *out_vals;
  size_t out_cap;        /* range: record capacity; HM_ECAPACITY if exceeded */
  int flags;             /* upsert: HM_UPSERT_* */
} hm_request;

typedef struct {
  size_t device_budget_bytes;  /* device bytes of admitted, unfinished requests (default 1 GiB) */
  int max_queue;               /* pending requests before HM_EBUSY (default 65536) */
  int streams;                 /* launches in flight (default 3) */
  int64_t max_launch_queries;  /* coalescing cap per launch (default 2^22) */
  int64_t device_wait_limit_ms; /* a launch unfinished after this fails with HM_ETIMEOUT and its slot
                                   is retired; while any slot is retired, upserts and deletes fail
                                   with HM_ETIMEOUT (its kernels may still read the tree) (default 30000) */
} hm_server_config;

typedef struct {
  uint64_t completed, failed, rejected, launches, epochs, queries, pending;
  double p50_us, p99_us, max_us, mean_us; /* submit-to-completion latency */
  double elapsed_s;
  /* Where a read's time goes (searches and ranges completed since the last
   * reset, p50 and p99 of each part): queue = submitted until taken into a
   * launch (waits for slots, the memory budget and write epochs ahead of it);
   * stage = inputs copied to pinned staging (page-locked and device buffers
   * skip it) and the launch enqueued; device =
   * enqueued until the launch is seen finished (copies and kernels); finish =
   * results copied to the caller's buffers.  Per write epoch, the mean wait
   * for the kernels of the reads before it to finish (drain; their result
   * copies may still run during the epoch) and the mean time to apply it. */
  double queue_p50_us, queue_p99_us, stage_p50_us, stage_p99_us;
  double device_p50_us, device_p99_us, finish_p50_us, finish_p99_us;
  double epoch_drain_mean_us, epoch_apply_mean_us;
} hm_server_stats;

typedef struct hm_server hm_server;
int hm_server_config_default(hm_server_config *cfg);
int hm_server_start(hm_tree *t, const hm_server_config *cfg, hm_server **out);
/* Copies the request descriptor (not the buffers, which must stay valid until
 * the request completes).  HM_EBUSY when the queue is full or the request
 * alone exceeds the budget; HM_ECANCELLED after stop. */
int hm_server_submit(hm_server *sv, const hm_request *r, uint64_t *ticket);
/* Waits up to timeout_us (< 0: no limit) for the ticket; *status receives the
 * request's HM_* result.  Returns HM_ETIMEOUT if still running. */
int hm_server_wait(hm_server *sv, uint64_t ticket, int64_t timeout_us, int *status);
int hm_server_get_stats(hm_server *sv, hm_server_stats *st);
int hm_server_reset_stats(hm_server *sv);
/* Cancels queued requests (their status becomes HM_ECANCELLED), lets those in
 * flight finish and joins the dispatcher; tickets can still be waited on. */
int hm_server_stop(hm_server *sv);
/* Stops if needed and frees the server and every uncollected request. */
int hm_server_free(hm_server *sv);

/* Point search that allocates nothing.  Some callers cannot allocate device
 * memory at the moment they search: a host runtime that reserves all device
 * memory up front and hands the library only its input and output buffers (a
 * database's GPU buffer manager, a framework's caching allocator), a serving
 * loop held to a fixed device-memory budget, or a latency-bound caller that
 * cannot afford the device-wide synchronisation cudaFree implies.  This entry
 * point runs the same pre-sort (8 bits) and search as hm_search, with its
 * working space in one fixed array the library keeps in device memory
 * (HM_NOALLOC_SCRATCH_BYTES on every GPU that loads the library, held until
 * the process exits).  q and out must be device memory, n at most
 * HM_NOALLOC_MAX_QUERIES (HM_ETOOLARGE otherwise, HM_EINVAL for host
 * buffers).  Only enqueues on s.  The first call on each device looks the
 * array's device address up and resolves the kernels' launch shapes (both
 * kept for the whole process, whichever thread calls next); make that first
 * call before any stream capture.  All calls on a device share the array,
 * which keeps whatever the last call left in it: calls that overlap on the
 * GPU (other streams, threads or trees) race, so serialise them.  It has no
 * counterpart in the reference. */
#define HM_NOALLOC_MAX_QUERIES (1 << 20)
#define HM_NOALLOC_SCRATCH_BYTES (14u << 20)
int hm_search_noalloc(hm_tree *t, const int64_t *q, size_t n, int64_t *out, hm_stream s);

/* The last CUDA runtime error any call of this library turned into HM_ECUDA,
 * HM_ENOMEM or HM_ENODEVICE (0 if none); its name and description go to buf.
 * Replaces: the printf of CUDA_ERROR_HANDLER (open-harmonia/src/cuda_utils.h:3-12). */
int hm_last_cuda_error(char *buf, size_t cap);

/* Kernel launches this library has issued since load (for launch counting). */
uint64_t hm_launch_count(void);

/* Per-stage device time, measured with CUDA events recorded on the stream
 * each stage's kernels run on.  Stages: "partition" (query pre-sort),
 * "search" (descent + leaf test), "search_batches", "range", "upsert".
 * Replaces: the cudaEvent timing of the reference drivers
 * (open-harmonia/src/full-multi-prefix-sort-8thread.cu:279-325,446-452). */
typedef struct {
  char name[32];
  uint64_t launches;
  double total_ms;
} hm_stage_time;

/* Turns stage timing on (1) or off (0) for tree t; off by default. */
int hm_profile(hm_tree *t, int enable);
/* Waits for the recorded events, writes up to cap stage totals to out,
 * sets *n, and clears the record. */
int hm_profile_read(hm_tree *t, hm_stage_time *out, int cap, int *n);

/* Comparison kernels for reports, not the product path.  HM_BASELINE_POINTER:
 * a pointer-chasing descent in the style of the reference's HB+ GPU search
 * (open-harmonia/src/gbpt.cu:30-113): every inner node stores its children's
 * ids and each query follows them (one dependent load per level, one thread
 * per query, no prefix-sum child array, no pre-sort).  Device buffers; the
 * child-id array (4 B per child slot) is built on the first call after a
 * rebuild.  Results equal hm_search's. */
#define HM_BASELINE_POINTER 1
int hm_search_baseline(hm_tree *t, int kind, const int64_t *q, size_t n, int64_t *out, hm_stream s);

/* ---- Reference dataset files and tree snapshots ------------------------- */

/* Reads a key file in the reference's text format: one signed decimal key per
 * line, as open-harmonia/script/generate-data/generate.py writes insert,
 * search and update files and open-harmonia/src/main.cpp:50-67 reads them
 * (sscanf "%lld": leading blanks skipped, text after the number ignored).
 * Call with keys == NULL to get the count in *n, then again with cap >= *n.
 * Blank lines are skipped; a line without a number gives HM_EIO. */
int hm_read_keys(const char *path, int64_t *keys, size_t cap, size_t *n);

/* Reads a range file in the reference's format: two lines per query, the
 * start key then the end key (open-harmonia/src/range.cu:349-355 reads the
 * pairs; its GPU path then ignores the end).  Count as hm_read_keys. */
int hm_read_ranges(const char *path, int64_t *start, int64_t *end, size_t cap, size_t *n);

/* Writes keys in the same text format, one per line. */
int hm_write_keys(const char *path, const int64_t *keys, size_t n);

/* One epoch of deletes: every listed key that is stored is removed (absent
 * keys and repeats are ignored); *removed (may be NULL) receives the count.
 * At most 2^31 - 1 keys per batch (HM_ETOOLARGE beyond).
 * Searches and range scans afterwards see the remaining keys only, and a later
 * upsert can store a removed key again.  Keys may be host or device memory;
 * returns when done.  No counterpart in the reference, whose
 * BPlusTree::remove is an empty stub (open-harmonia/src/bpt.cpp:771-773). */
int hm_delete_batch(hm_tree *t, const int64_t *keys, size_t n, size_t *removed, hm_stream s);

/* Writes the tree's contents (keys in order with their values) and its
 * configuration to a binary file, with a checksum.  No counterpart in the
 * reference, whose trees live only in process memory. */
int hm_snapshot_save(hm_tree *t, const char *path);

/* Bulk-loads a tree from a snapshot; cfg == NULL uses the saved
 * configuration.  HM_EIO for a missing, truncated or corrupted file. */
int hm_snapshot_load(const char *path, const hm_config *cfg, hm_tree **out);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif
