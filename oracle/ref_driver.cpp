// Test infrastructure only: a small C-ABI driver around the reference CPU
// B+tree (open-harmonia/src), compiled from the reference's own sources by
// oracle/Makefile into oracle/_ref/libhmref.so.  Only tests, the smoke check
// and bench.py's reference/cpu_baseline arm load it; the product library
// never does.
//
// The reference has no library API: its experiments are `main` plus one
// function per CLI option (open-harmonia/src/main.cpp:50-67,166-414).  This
// file re-hosts exactly the calls those experiments make, so that the oracle
// is the reference's own code path:
//   build   : BPlusTree::insert per key (main.cpp:56-66, bpt.cpp:357-409),
//             then BPlusTree::sort -> PPI tree (main.cpp:151-152,
//             traversal.cpp:35-129) with prefixArray (traversal.cpp:180-195)
//   search  : search_cpu_test's OpenMP loop over BPlusTree::search
//             (main.cpp:772-812, bpt.cpp:673-680, bpt-ppi.cpp:118-156);
//             after an update the Newupdate descent
//             (bpt-ppi-update.cpp:12-89), which also follows "normal" nodes
//   range   : the PPI range traversal of cpu-range.cpp:129-183 with the
//             end key forced to Max_Key (range.cu:349-355), generalised from
//             Range_Size=8 to a per-query length, and stepping to the next
//             big leaf through BLeaf_node::next (bpt.cpp:55-56) as
//             BPlusTree::range_search does (bpt.cpp:695-769), which stays
//             correct after updates append leaves out of order
//   upsert  : BPlusTree::insert_parallel_Newupdate_batch
//             (bpt-ppi-update-batch.cpp:86-200): an existing key's value
//             becomes key-1, a new key is inserted with its supplied value
//   export  : in-order walk of the big-leaf chain (bpt.h:241-337)
#include "bpt.h"

#include <omp.h>

#include <cstdint>
#include <vector>

namespace {

struct RefTree {
  BPlusTree *ppi = nullptr;
  bool updated = false;
};

BLeaf_node *leaf_for(BPlusTree *t, Inner_node *last, long long key,
                     int &relist_idx) {
  // Mirrors search_leaf_PPItree_Newupdate (bpt-ppi-update.cpp:40-59).
  if (last == nullptr) {
    relist_idx = 0;
    return static_cast<BLeaf_node *>(t->getRoot());
  }
  relist_idx = last->getChildIdx(nullptr, key);
  int idx = t->getInnerNodeIdx(last);
  if (t->isNormalInnerNode(idx))
    return static_cast<BLeaf_node *>(last->child[0]);
  return t->getBLeafNodeByIdx(idx - t->getInnerSize_wo_last_inner_node());
}

// The walk of hmref_range for one query: up to `want` records with key >=
// start, handed to emit(key, value); returns how many.
template <typename Emit>
long range_walk(BPlusTree *t, long long start, long want, Emit emit) {
  if (want <= 0 || start == Max_Key) return 0;
  Inner_node *last = t->search_last_level_inner_node_PPItree_Newupdate(start);
  int relist_idx = 0;
  BLeaf_node *node = leaf_for(t, last, start, relist_idx);
  int idx = node->findKeyLowerBound(relist_idx, start);
  if (idx < 0) {  // nothing >= start in this record list
    idx = 0;
    relist_idx++;
  }
  long got = 0;
  while (node != nullptr && got < want) {
    if (relist_idx >= node->used_relist_slot_num) {
      node = node->next;
      relist_idx = 0;
      idx = 0;
      continue;
    }
    if (idx >= node->size[relist_idx]) {
      relist_idx++;
      idx = 0;
      continue;
    }
    if (!emit(node->relist[relist_idx].r[idx].r_key, node->relist[relist_idx].r[idx].val)) return -1;
    got++;
    idx++;
  }
  return got;
}

}  // namespace

extern "C" {

int hmref_abi_version() { return 1; }

// Returns nullptr when the reference cannot represent the tree: it needs at
// least one inner node (sort() asserts the root is inner, traversal.cpp:87),
// i.e. more than 4 distinct keys.
void *hmref_build(const long long *keys, const long long *vals, long n) {
  BPlusTree *tree = new BPlusTree();
  for (long i = 0; i < n; i++) tree->insert(keys[i], vals[i]);
  if (tree->getHeight() < 2) return nullptr;
  RefTree *h = new RefTree();
  tree->sort(h->ppi);
  return h;
}

int hmref_height(void *hp) { return static_cast<RefTree *>(hp)->ppi->getHeight(); }
// The PPI tree itself, for the GPU comparison driver linked beside this file.
void *hmref_ppi_tree(void *hp) { return static_cast<RefTree *>(hp)->ppi; }
long hmref_inner_nodes(void *hp) { return static_cast<RefTree *>(hp)->ppi->getInnerSize(); }
long hmref_big_leaves(void *hp) { return static_cast<RefTree *>(hp)->ppi->getBLeafSize(); }

// Point search; out[i] is the value or -1.  threads<=0 uses OpenMP's default.
void hmref_search(void *hp, const long long *q, long n, long long *out,
                  int threads) {
  RefTree *h = static_cast<RefTree *>(hp);
  BPlusTree *t = h->ppi;
  int nt = threads > 0 ? threads : omp_get_max_threads();
  if (!h->updated) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long i = 0; i < n; i++) out[i] = t->search(q[i]);
  } else {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (long i = 0; i < n; i++) out[i] = t->search_PPItree_Newupdate(q[i]);
  }
}

// The reference's software-pipelined CPU point search, as
// search_cpu_prefetch_NTG_PPI runs it for 64-bit keys
// (cpu-search-prefetch-avxNTG.cpp:480-535; that file builds only with Boost
// and PAPI, so the loop is re-hosted here over the same tree methods): a
// group of 16 queries descends one level at a time, four at once through
// the tree's AVX2 child search (BPlusTree::getChildIdx_avx_4keys,
// avx.cpp:127-190), each inner node prefetched just before the compare that
// reads it; the last step finds the key in the big leaf's record list
// (BLeaf_node::findKey).  OpenMP over groups; a tail of fewer than 16
// queries takes BPlusTree::search.  Fresh trees only (no Newupdate nodes).
void hmref_search_prefetch(void *hp, const long long *q, long n, long long *out, int threads) {
  BPlusTree *t = static_cast<RefTree *>(hp)->ppi;
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  constexpr int kGroup = 16;
  const int height = t->getHeight();
  int *prefix = t->getPrefixArray();
  const int inner_wo_last = t->getInnerSize_wo_last_inner_node();
  const long groups = n / kGroup;
#pragma omp parallel for num_threads(nt) schedule(static)
  for (long g = 0; g < groups; g++) {
    key_t keys[kGroup];
    int node[kGroup], rel[kGroup];
    Inner_node *nodes[kGroup];
    for (int i = 0; i < kGroup; i++) {
      keys[i] = q[g * kGroup + i];
      node[i] = 0;
    }
    for (int level = 1; level < height; level++) {
      for (int b = 0; b < kGroup; b += 4) {
        for (int j = b; j < b + 4; j++) {
          nodes[j] = t->getInnerNodeByIdx(node[j]);
          __builtin_prefetch(nodes[j], 0, 3);
        }
        t->getChildIdx_avx_4keys(&nodes[b], &keys[b], &rel[b]);
        for (int j = b; j < b + 4; j++) node[j] = prefix[node[j]] + rel[j];
      }
    }
    for (int i = 0; i < kGroup; i++) {
      BLeaf_node *leaf = t->getBLeafNodeByIdx(t->getInnerNodeIdx(nodes[i]) - inner_wo_last);
      out[g * kGroup + i] = leaf->findKey(rel[i], keys[i]);
    }
  }
  for (long i = groups * kGroup; i < n; i++) out[i] = t->search(q[i]);
}

// Timing form of the range scan, as the reference's CPU range experiment
// runs it (OpenMP over blocks of SWP_P2 = 1000 queries, cpu-range.cpp:80-88):
// every query walks its records into a per-thread buffer (the reference
// fills per-query result slots); returns the record count and a checksum
// of the keys and values so the walk is not optimised away.
long hmref_range_timed(void *hp, const long long *start, const int *len, long n, int threads,
                       long long *checksum) {
  BPlusTree *t = static_cast<RefTree *>(hp)->ppi;
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  long total = 0;
  long long sum = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1000) reduction(+ : total, sum)
  for (long i = 0; i < n; i++) {
    long long acc = 0;
    const long got = range_walk(t, start[i], len[i], [&](long long k, long long v) {
      acc += k ^ v;
      return true;
    });
    total += got;
    sum += acc;
  }
  if (checksum) *checksum = sum;
  return total;
}

// Range: for query i, the first len[i] records with key >= start[i] in
// ascending key order (fewer when the key space ends).  offsets has n+1
// entries (exclusive scan of the per-query counts).  Returns the total number
// of records, or -1 if cap is too small.
long hmref_range(void *hp, const long long *start, const int *len, long n,
                 long long *offsets, long long *okeys, long long *ovals,
                 long cap) {
  BPlusTree *t = static_cast<RefTree *>(hp)->ppi;
  long total = 0;
  for (long i = 0; i < n; i++) {
    offsets[i] = total;
    const long got = range_walk(t, start[i], len[i], [&](long long k, long long v) {
      if (total >= cap) return false;
      okeys[total] = k;
      ovals[total] = v;
      total++;
      return true;
    });
    if (got < 0) return -1;
  }
  offsets[n] = total;
  return total;
}

}  // extern "C"

namespace {

// BPlusTree::range_search (bpt.cpp:695-769) from its descent on: the walk
// over big leaves and record lists between the start key's lower bound and
// the end key's upper bound, appending to v, with the leaves located by the
// Newupdate descent (leaf_for), which stays valid after updates.  The walk
// keeps the reference's steps, including the step back to the previous big
// leaf when the end key's record list holds nothing <= end.
void range_between_walk(BPlusTree *t, key_t start_key, key_t end_key, std::vector<Record> *v) {
  if (start_key > end_key) return;
  int relist_idx_start = 0, relist_idx_end = 0;
  BLeaf_node *blfnode_start =
      leaf_for(t, t->search_last_level_inner_node_PPItree_Newupdate(start_key), start_key, relist_idx_start);
  BLeaf_node *blfnode_end =
      leaf_for(t, t->search_last_level_inner_node_PPItree_Newupdate(end_key), end_key, relist_idx_end);
  int idx_start = blfnode_start->findKeyLowerBound(relist_idx_start, start_key);
  int idx_end = blfnode_end->findKeyUpperBound(relist_idx_end, end_key);
  if (idx_start == -1) {
    idx_start = 0;
    relist_idx_start++;
    if (relist_idx_start >= blfnode_start->used_relist_slot_num) {
      if (blfnode_start == blfnode_end) return;
      blfnode_start = blfnode_start->next;
      relist_idx_start = 0;
    }
  }
  if (idx_end == -1) {
    relist_idx_end--;
    if (relist_idx_end < 0) {
      if (blfnode_start == blfnode_end) return;
      BLeaf_node *temp = blfnode_start, *temp1 = blfnode_start;
      while (temp != blfnode_end) {
        temp1 = temp;
        temp = temp->next;
      }
      blfnode_end = temp1;
      relist_idx_end = -1;
    }
  }
  if (blfnode_start == blfnode_end) {
    blfnode_start->getKeyValuesRange(relist_idx_start, relist_idx_end, idx_start, idx_end, v);
    return;
  }
  blfnode_start->getKeyValuesRange(relist_idx_start, -1, idx_start, -1, v);
  for (blfnode_start = blfnode_start->next; blfnode_start != blfnode_end; blfnode_start = blfnode_start->next) {
    if (blfnode_start == nullptr) return;
    blfnode_start->getKeyValuesRange(0, -1, 0, -1, v);
  }
  blfnode_end->getKeyValuesRange(0, relist_idx_end, 0, idx_end, v);
}

}  // namespace

extern "C" {

// Inclusive ranges: for query i every record with start[i] <= key <= end[i]
// in ascending key order (nothing when start > end).  Before any update this
// calls BPlusTree::range_search itself (bpt.cpp:695-769); after an update,
// whose new nodes its pointer descent does not follow (it crashes there),
// the same walk with the Newupdate descent (range_between_walk).  walk != 0
// forces the walk (to check it against range_search).  end must not be
// Max_Key: the reference's descent asserts for that key on a PPI tree
// (mempool.h:51).  offsets has n+1 entries.  Returns the total number of
// records, or -1 if cap is too small.
long hmref_range_between(void *hp, const long long *start, const long long *end, long n,
                         long long *offsets, long long *okeys, long long *ovals, long cap, int walk) {
  RefTree *h = static_cast<RefTree *>(hp);
  BPlusTree *t = h->ppi;
  long total = 0;
  std::vector<Record> v;
  for (long i = 0; i < n; i++) {
    offsets[i] = total;
    v.clear();
    if (h->updated || walk)
      range_between_walk(t, start[i], end[i], &v);
    else
      t->range_search(start[i], end[i], &v);
    if (total + (long)v.size() > cap) return -1;
    for (const Record &r : v) {
      okeys[total] = r.r_key;
      ovals[total] = r.val;
      total++;
    }
  }
  offsets[n] = total;
  return total;
}

// One update batch through the reference's parallel update.  syn_batch and
// rebuild_batch are the reference's two batch sizes; the reference reads past
// the input unless n is a multiple of syn_batch, so other values are clamped
// to n.  Returns 0.
int hmref_upsert(void *hp, const long long *keys, const long long *vals,
                 long n, long syn_batch, long rebuild_batch) {
  RefTree *h = static_cast<RefTree *>(hp);
  if (n <= 0) return 0;
  if (syn_batch <= 0 || n % syn_batch != 0) syn_batch = n;
  if (rebuild_batch <= 0 || rebuild_batch % syn_batch != 0) rebuild_batch = syn_batch;
  std::vector<key_t> k(keys, keys + n);
  std::vector<value_t> v(vals, vals + n);
  h->ppi->insert_parallel_Newupdate_batch(k, v, (int)syn_batch, (int)rebuild_batch);
  h->updated = true;
  return 0;
}

// Sorted (key, value) contents.  Returns the record count, or -1 if cap is
// too small (the count is still walked so the caller can resize).
long hmref_export(void *hp, long long *keys, long long *vals, long cap) {
  BPlusTree *t = static_cast<RefTree *>(hp)->ppi;
  long total = 0;
  bool overflow = false;
  for (BLeaf_node *node = t->getBLeafNodeByIdx(0); node != nullptr; node = node->next) {
    for (int r = 0; r < node->used_relist_slot_num; r++) {
      for (int j = 0; j < node->size[r]; j++) {
        if (total < cap) {
          keys[total] = node->relist[r].r[j].r_key;
          vals[total] = node->relist[r].r[j].val;
        } else {
          overflow = true;
        }
        total++;
      }
    }
  }
  return overflow ? -1 : total;
}

}  // extern "C"
