/* Test infrastructure only: plain-C restatement of the reference's batched
 * B+tree algorithms, used as the checker for the CUDA path.  Only tests, the
 * smoke check and bench.py's cpu_baseline arm may load it.
 *
 * It restates, on the product's device layout (a breadth-first key region
 * plus a prefix-sum child array, as in the reference's CFB form,
 * open-harmonia/regular_bpt/cfb.h:16-59 and traversal.cpp:36-78):
 *   - bulk build from sorted unique keys (levels bottom-up, BFS numbering,
 *     prefix[i] = index of node i's first child, prefix[0] = 1),
 *   - point search: child = number of separators <= q, found iff the leaf
 *     holds q (open-harmonia/regular_bpt/cfb.cpp:4-40,
 *     open-harmonia/src/avx.cpp:2-54, open-harmonia/src/bpt.h:252-274),
 *   - range: first L records with key >= start
 *     (open-harmonia/src/cpu-range.cpp:129-183 with end = Max_Key as in
 *     open-harmonia/src/range.cu:349-355),
 *   - batched upsert on the sorted contents, with the reference's
 *     "existing key -> key-1" rule as an option
 *     (open-harmonia/src/bpt-ppi-update-batch.cpp:47,61-67).
 */
#ifndef HM_ORACLE_H
#define HM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HMO_MAX_KEY INT64_MAX /* empty-slot sentinel, open-harmonia/src/bpt.h:26 */
#define HMO_NOT_FOUND (-1)    /* open-harmonia/src/bpt.h:272 */
#define HMO_MAX_LEVELS 32

typedef struct {
  int fanout;     /* F: key slots of an inner row (64 or 128); <= F-1 separators, <= F children */
  int leaf_cap;   /* Lc: key slots of a leaf row (8, 16, 32, 64 or 128) */
  int inner_fill; /* children per inner node at build time, 2..F */
  int leaf_fill;  /* keys per leaf at build time, 1..Lc */
} hmo_params;

typedef struct {
  hmo_params p;
  int height;       /* number of inner levels, >= 1 */
  int inner_row;    /* int64 words per inner row: F/8 index + F keys */
  int leaf_row;     /* int64 words per leaf row: (Lc>=32 ? Lc/8 : 0) index, Lc keys, Lc values */
  int leaf_index;   /* index words at the start of a leaf row */
  int64_t n_keys, n_inner, n_leaf;
  int64_t lvl_start[HMO_MAX_LEVELS + 1]; /* BFS index of each inner level; lvl_start[height] = n_inner */
  int64_t *inner;     /* n_inner * inner_row */
  int32_t *prefix;    /* n_inner; children of the last level count from n_inner */
  int64_t *leaf_rows; /* n_leaf * leaf_row; keys Max_Key and values -1 in empty slots */
  int32_t *leaf_cnt;  /* n_leaf */
  int64_t *leaf_base; /* n_leaf, exclusive scan of leaf_cnt */
} hmo_tree;

/* 0 on success; -1 bad params, -2 keys not strictly increasing (duplicate or
 * unsorted), -3 key == Max_Key, -4 out of memory. */
int hmo_build(const int64_t *sorted_keys, const int64_t *vals, int64_t n,
              const hmo_params *p, hmo_tree *out);
void hmo_free(hmo_tree *t);

/* Shape only (level sizes), no allocation: used to check the device loader. */
int hmo_shape(int64_t n, const hmo_params *p, int *height, int64_t *lvl_start,
              int64_t *n_inner, int64_t *n_leaf);

void hmo_search(const hmo_tree *t, const int64_t *q, int64_t n, int64_t *out);

/* Returns total records, or -1 if cap is too small.  offsets has n+1 entries. */
int64_t hmo_range(const hmo_tree *t, const int64_t *start, const int32_t *len,
                  int64_t n, int64_t *offsets, int64_t *okeys, int64_t *ovals,
                  int64_t cap);

/* Inclusive ranges: every record with start[i] <= key <= end[i]; returns
 * total records, or -1 if cap is too small.  offsets has n+1 entries. */
int64_t hmo_range_between(const hmo_tree *t, const int64_t *start, const int64_t *end,
                          int64_t n, int64_t *offsets, int64_t *okeys, int64_t *ovals,
                          int64_t cap);

/* Sorted contents; returns count, or -1 if cap is too small. */
int64_t hmo_export(const hmo_tree *t, int64_t *keys, int64_t *vals, int64_t cap);

#define HMO_UPSERT_SUPPLIED 0      /* existing key takes the supplied value */
#define HMO_UPSERT_REF_KEY_MINUS_1 1 /* existing key takes key-1 (reference rule) */

/* Applies one batch to sorted contents (skeys, svals, n).  Within the batch
 * the last occurrence of a key wins.  Writes the merged sorted contents to
 * (okeys, ovals) with capacity cap; returns the new count or -1 (cap), -3
 * (a batch key equals Max_Key). */
int64_t hmo_upsert(const int64_t *skeys, const int64_t *svals, int64_t n,
                   const int64_t *bkeys, const int64_t *bvals, int64_t m,
                   int flags, int64_t *okeys, int64_t *ovals, int64_t cap);

/* splitmix64 (Steele, Lea, Flood 2014): the seeded generator the synthetic
 * workloads are defined with.  Exposed so tests can check the numpy copy. */
uint64_t hmo_splitmix64(uint64_t x);

#ifdef __cplusplus
}
#endif
#endif
