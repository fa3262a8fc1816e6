// Test infrastructure only: a C-ABI driver around the reference's pointer
// B+tree (open-harmonia/regular_bpt/regular_bpt.cpp), compiled from the
// reference's own source by oracle/Makefile, with DEFAULT_ORDER 128, into
// oracle/_ref/libhmref_cfb.so.  Only bench.py's CPU figures and tests load it;
// the product library never does.
//
// The reference's fanout-128 experiments build this tree with insert()
// (regular_bpt.cpp:759-804, one key at a time, value = key in its harness)
// and its CPU point search is find() (regular_bpt.cpp:383-395): descend with
// linear scans of each node's keys, then an equality scan of the leaf.  The
// CFB re-layout (cfb.cpp, traversal.cpp) only feeds its GPU kernels.
#include "regular_bpt.h"

#include <omp.h>

extern "C" {

int hmcfb_order() { return DEFAULT_ORDER; }

// Builds the tree by inserting the keys in the given order.
void *hmcfb_build(const long long *keys, const long long *vals, long n) {
  node *root = nullptr;
  for (long i = 0; i < n; i++) root = insert(root, keys[i], vals[i]);
  return root;
}

// Point search with find(); out[i] = the value or -1.  threads <= 0 uses
// OpenMP's default.
void hmcfb_search(void *h, const long long *q, long n, long long *out, int threads) {
  node *root = static_cast<node *>(h);
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for num_threads(nt) schedule(static)
  for (long i = 0; i < n; i++) {
    record *r = find(root, q[i], false);
    out[i] = r ? r->value : -1;
  }
}

}  // extern "C"
