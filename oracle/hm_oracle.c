/* Test infrastructure only: plain-C restatement of the reference's batched
 * B+tree algorithms (see hm_oracle.h for the list and the reference lines).
 * The product never links this file; tests compare the CUDA path with it,
 * and tests pin it against the reference library built by `make ref`. */
#include "hm_oracle.h"

#include <stdlib.h>
#include <string.h>

uint64_t hmo_splitmix64(uint64_t x) {
  uint64_t z = x + 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

static int valid_cap(int c) { return c == 8 || c == 16 || c == 32 || c == 64 || c == 128; }

static int params_ok(const hmo_params *p) {
  if (p->fanout != 64 && p->fanout != 128) return 0;
  if (!valid_cap(p->leaf_cap)) return 0;
  if (p->inner_fill < 2 || p->inner_fill > p->fanout) return 0;
  if (p->leaf_fill < 1 || p->leaf_fill > p->leaf_cap) return 0;
  return 1;
}

/* Start of part j when `total` items are split into `parts` nearly equal
 * runs, the first (total % parts) runs one longer. */
static int64_t part_start(int64_t j, int64_t total, int64_t parts) {
  int64_t q = total / parts, r = total % parts;
  return j * q + (j < r ? j : r);
}

int hmo_shape(int64_t n, const hmo_params *p, int *height, int64_t *lvl_start,
              int64_t *n_inner, int64_t *n_leaf) {
  if (!params_ok(p) || n < 0) return -1;
  int64_t nl = n == 0 ? 1 : (n + p->leaf_fill - 1) / p->leaf_fill;
  int64_t sizes[HMO_MAX_LEVELS];
  int h = 0;
  int64_t m = nl;
  do { /* at least one inner level, even over a single leaf */
    if (h >= HMO_MAX_LEVELS) return -1;
    int64_t nodes = (m + p->inner_fill - 1) / p->inner_fill;
    sizes[h++] = nodes;
    m = nodes;
  } while (m > 1);
  /* sizes[] runs bottom-up; BFS numbering runs top-down */
  int64_t acc = 0;
  for (int l = 0; l < h; l++) {
    lvl_start[l] = acc;
    acc += sizes[h - 1 - l];
  }
  lvl_start[h] = acc;
  *height = h;
  *n_inner = acc;
  *n_leaf = nl;
  return 0;
}

void hmo_free(hmo_tree *t) {
  free(t->inner);
  free(t->prefix);
  free(t->leaf_rows);
  free(t->leaf_cnt);
  free(t->leaf_base);
  memset(t, 0, sizeof(*t));
}

int hmo_build(const int64_t *keys, const int64_t *vals, int64_t n,
              const hmo_params *p, hmo_tree *t) {
  memset(t, 0, sizeof(*t));
  if (!params_ok(p) || n < 0) return -1;
  for (int64_t i = 0; i < n; i++) {
    if (keys[i] == HMO_MAX_KEY) return -3;
    if (i > 0 && keys[i] <= keys[i - 1]) return -2;
  }
  t->p = *p;
  if (hmo_shape(n, p, &t->height, t->lvl_start, &t->n_inner, &t->n_leaf)) return -1;
  const int F = p->fanout, LC = p->leaf_cap;
  t->n_keys = n;
  t->inner_row = F / 8 + F;
  t->leaf_index = LC >= 32 ? LC / 8 : 0;
  t->leaf_row = t->leaf_index + 2 * LC;
  t->inner = malloc(sizeof(int64_t) * t->n_inner * t->inner_row);
  t->prefix = malloc(sizeof(int32_t) * t->n_inner);
  t->leaf_rows = malloc(sizeof(int64_t) * t->n_leaf * t->leaf_row);
  t->leaf_cnt = malloc(sizeof(int32_t) * t->n_leaf);
  t->leaf_base = malloc(sizeof(int64_t) * t->n_leaf);
  /* first_leaf[] of the level being built: the leftmost leaf under each node,
   * whose first key is the node's subtree minimum. */
  int64_t *first_leaf = malloc(sizeof(int64_t) * t->n_leaf);
  int64_t *next_first = malloc(sizeof(int64_t) * t->n_leaf);
  if (!t->inner || !t->prefix || !t->leaf_rows || !t->leaf_cnt ||
      !t->leaf_base || !first_leaf || !next_first) {
    free(first_leaf);
    free(next_first);
    hmo_free(t);
    return -4;
  }

  /* Leaves: keys in order, evenly spread, Max_Key / -1 in empty slots; each
   * leaf row holds its keys and then their values, so a hit reads the value
   * from the record it just compared (the reference's Record_list keeps key
   * and value side by side too, open-harmonia/src/bpt.h:206-239). */
  for (int64_t j = 0; j < t->n_leaf; j++) {
    int64_t s = part_start(j, n, t->n_leaf), e = part_start(j + 1, n, t->n_leaf);
    int64_t *row = t->leaf_rows + j * t->leaf_row;
    int64_t *kr = row + t->leaf_index;
    int64_t *vr = kr + LC;
    for (int i = 0; i < LC; i++) {
      kr[i] = (s + i < e) ? keys[s + i] : HMO_MAX_KEY;
      vr[i] = (s + i < e) ? vals[s + i] : HMO_NOT_FOUND;
    }
    /* index[j] = key[8(j+1)], as inner_index in open-harmonia/src/bpt.h:78,189-191 */
    for (int x = 0; x < t->leaf_index; x++)
      row[x] = (8 * (x + 1) < LC) ? kr[8 * (x + 1)] : HMO_MAX_KEY;
    t->leaf_cnt[j] = (int32_t)(e - s);
    t->leaf_base[j] = s;
    first_leaf[j] = j;
  }

  /* Inner levels bottom-up; level l occupies BFS slots lvl_start[l]... */
  int64_t m = t->n_leaf; /* children at the level below */
  for (int l = t->height - 1; l >= 0; l--) {
    int64_t nodes = t->lvl_start[l + 1] - t->lvl_start[l];
    int64_t child_base = t->lvl_start[l + 1]; /* BFS id of the level below's first node */
    for (int64_t i = 0; i < nodes; i++) {
      int64_t c0 = part_start(i, m, nodes), c1 = part_start(i + 1, m, nodes);
      int64_t id = t->lvl_start[l] + i;
      int64_t *row = t->inner + id * t->inner_row;
      int64_t *kr = row + F / 8;
      for (int x = 0; x < F; x++) {
        int64_t c = c0 + 1 + x; /* separator x = min key of child x+1 */
        kr[x] = (c < c1) ? keys[part_start(first_leaf[c], n, t->n_leaf)] : HMO_MAX_KEY;
      }
      for (int x = 0; x < F / 8; x++)
        row[x] = (8 * (x + 1) < F) ? kr[8 * (x + 1)] : HMO_MAX_KEY;
      /* CFB prefix: prefix[i] = first child's BFS id (traversal.cpp:50-57) */
      t->prefix[id] = (int32_t)(child_base + c0);
      next_first[i] = first_leaf[c0];
    }
    int64_t *tmp = first_leaf;
    first_leaf = next_first;
    next_first = tmp;
    m = nodes;
  }
  free(first_leaf);
  free(next_first);
  return 0;
}

/* Number of keys <= q in the sorted run kr[0..len). */
static int count_le(const int64_t *kr, int len, int64_t q) {
  int c = 0;
  while (c < len && kr[c] <= q) c++;
  return c;
}

/* Child position in a row with an index of `ix` entries over `len` keys:
 * first the index (every 8th key), then the chosen 8-key slice, as in
 * Inner_node::getChildIdx_avx2_version2 (open-harmonia/src/avx.cpp:2-54)
 * and the two compare stages of full_multi_prefix_sort_8thread_kernel
 * (open-harmonia/src/full-multi-prefix-sort-8thread.cu:145-193).  Rows
 * without an index are scanned whole (open-harmonia/regular_bpt/cfb.cpp:15-19). */
static int rank_row(const int64_t *row, int ix, int len, int64_t q) {
  const int64_t *kr = row + ix;
  if (ix == 0) return count_le(kr, len, q);
  int k = count_le(row, ix, q);
  if (k > ix - 1) k = ix - 1;
  return 8 * k + count_le(kr + 8 * k, 8, q);
}

static int64_t descend(const hmo_tree *t, int64_t q) {
  int64_t node = 0;
  for (int l = 0; l < t->height; l++) {
    const int64_t *row = t->inner + node * t->inner_row;
    int c = rank_row(row, t->p.fanout / 8, t->p.fanout, q);
    node = (int64_t)t->prefix[node] + c;
  }
  return node - t->n_inner; /* leaf index, as idx - internal_node_num in cfb.cpp:32 */
}

void hmo_search(const hmo_tree *t, const int64_t *q, int64_t n, int64_t *out) {
  /* one query per iteration, like search_cpu_test's OpenMP loop
   * (open-harmonia/src/main.cpp:795-799) */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    int64_t key = q[i];
    if (key == HMO_MAX_KEY) { /* no stored key equals the sentinel */
      out[i] = HMO_NOT_FOUND;
      continue;
    }
    int64_t leaf = descend(t, key);
    const int64_t *row = t->leaf_rows + leaf * t->leaf_row;
    int r = rank_row(row, t->leaf_index, t->p.leaf_cap, key);
    const int64_t *kr = row + t->leaf_index;
    /* equality test of the matched slot, BLeaf_node::findKey (bpt.h:252-274) */
    out[i] = (r > 0 && kr[r - 1] == key) ? kr[t->p.leaf_cap + r - 1] : HMO_NOT_FOUND;
  }
}

int64_t hmo_range(const hmo_tree *t, const int64_t *start, const int32_t *len,
                  int64_t n, int64_t *offsets, int64_t *okeys, int64_t *ovals,
                  int64_t cap) {
  int64_t total = 0;
  for (int64_t i = 0; i < n; i++) {
    offsets[i] = total;
    int64_t want = len[i] > 0 ? len[i] : 0;
    if (want == 0 || start[i] == HMO_MAX_KEY) continue;
    int64_t leaf = descend(t, start[i]);
    const int64_t *kr = t->leaf_rows + leaf * t->leaf_row + t->leaf_index;
    int slot = 0; /* lower bound: first key >= start */
    while (slot < t->leaf_cnt[leaf] && kr[slot] < start[i]) slot++;
    int64_t got = 0;
    while (got < want && leaf < t->n_leaf) {
      if (slot >= t->leaf_cnt[leaf]) {
        leaf++;
        slot = 0;
        continue;
      }
      if (total >= cap) return -1;
      const int64_t *r = t->leaf_rows + leaf * t->leaf_row + t->leaf_index;
      okeys[total] = r[slot];
      ovals[total] = r[t->p.leaf_cap + slot];
      total++;
      got++;
      slot++;
    }
  }
  offsets[n] = total;
  return total;
}

/* Inclusive ranges, as BPlusTree::range_search (open-harmonia/src/bpt.cpp:695-769)
 * returns them: every record with start <= key <= end in ascending key order,
 * nothing when start > end.  The reference finds the start key's lower bound
 * (findKeyLowerBound, bpt.h:289-297) and the end key's upper bound
 * (findKeyUpperBound, bpt.h:298-306) and copies everything between them leaf
 * after leaf; here the walk from the lower bound stops at the first key > end. */
int64_t hmo_range_between(const hmo_tree *t, const int64_t *start, const int64_t *end,
                          int64_t n, int64_t *offsets, int64_t *okeys, int64_t *ovals,
                          int64_t cap) {
  int64_t total = 0;
  for (int64_t i = 0; i < n; i++) {
    offsets[i] = total;
    if (start[i] > end[i] || start[i] == HMO_MAX_KEY || t->n_keys == 0) continue;
    int64_t leaf = descend(t, start[i]);
    int slot = 0; /* lower bound: first key >= start */
    while (slot < t->leaf_cnt[leaf] && t->leaf_rows[leaf * t->leaf_row + t->leaf_index + slot] < start[i]) slot++;
    while (leaf < t->n_leaf) {
      if (slot >= t->leaf_cnt[leaf]) {
        leaf++;
        slot = 0;
        continue;
      }
      const int64_t *r = t->leaf_rows + leaf * t->leaf_row + t->leaf_index;
      if (r[slot] > end[i]) break;
      if (total >= cap) return -1;
      okeys[total] = r[slot];
      ovals[total] = r[t->p.leaf_cap + slot];
      total++;
      slot++;
    }
  }
  offsets[n] = total;
  return total;
}

int64_t hmo_export(const hmo_tree *t, int64_t *keys, int64_t *vals, int64_t cap) {
  if (cap < t->n_keys) return -1;
  int64_t o = 0;
  for (int64_t j = 0; j < t->n_leaf; j++)
    for (int s = 0; s < t->leaf_cnt[j]; s++) {
      const int64_t *r = t->leaf_rows + j * t->leaf_row + t->leaf_index;
      keys[o] = r[s];
      vals[o] = r[t->p.leaf_cap + s];
      o++;
    }
  return o;
}

typedef struct {
  int64_t key;
  int64_t idx;
} kv_idx;

static int cmp_kv_idx(const void *a, const void *b) {
  const kv_idx *x = a, *y = b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

int64_t hmo_upsert(const int64_t *skeys, const int64_t *svals, int64_t n,
                   const int64_t *bkeys, const int64_t *bvals, int64_t m,
                   int flags, int64_t *okeys, int64_t *ovals, int64_t cap) {
  for (int64_t i = 0; i < m; i++)
    if (bkeys[i] == HMO_MAX_KEY) return -3;
  kv_idx *b = malloc(sizeof(kv_idx) * (m > 0 ? m : 1));
  if (!b) return -4;
  for (int64_t i = 0; i < m; i++) {
    b[i].key = bkeys[i];
    b[i].idx = i;
  }
  qsort(b, (size_t)m, sizeof(kv_idx), cmp_kv_idx);
  int64_t u = 0; /* keep the last occurrence of each key */
  for (int64_t i = 0; i < m; i++) {
    if (i + 1 < m && b[i + 1].key == b[i].key) continue;
    b[u++] = b[i];
  }
  int64_t i = 0, j = 0, o = 0;
  while (i < n || j < u) {
    if (o >= cap) {
      free(b);
      return -1;
    }
    if (j >= u || (i < n && skeys[i] < b[j].key)) {
      okeys[o] = skeys[i];
      ovals[o++] = svals[i++];
    } else if (i >= n || b[j].key < skeys[i]) { /* new key: inserted with its value */
      okeys[o] = b[j].key;
      ovals[o++] = bvals[b[j].idx];
      j++;
    } else { /* existing key: searchAndUpdate (bpt-ppi-update-batch.cpp:47) */
      okeys[o] = skeys[i];
      ovals[o++] = (flags & HMO_UPSERT_REF_KEY_MINUS_1) ? skeys[i] - 1 : bvals[b[j].idx];
      i++;
      j++;
    }
  }
  free(b);
  return o;
}
