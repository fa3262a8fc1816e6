// GPU bulk loader: sorted (key, value) pairs -> leaves, then inner levels
// bottom-up with the breadth-first prefix-sum child array.
//
// The reference builds its tree by serial inserts and re-lays it out on the
// CPU (BPlusTree::insert + BPlusTree::sort + prepareArray,
// open-harmonia/src/bpt.cpp:357-409, open-harmonia/src/traversal.cpp:35-195),
// about four minutes at 2^26 keys.  Here every level is one kernel over
// (node, word) pairs: each thread computes one output word directly from the
// sorted keys, so the build reads the sorted arrays once and writes the tree
// once.  Keys are spread evenly: with m items over p parts, part j starts at
// j*(m/p) + min(j, m%p) (part_start), at the leaf level and at every inner
// level.
#include "hm_internal.cuh"

namespace hm {

namespace {

constexpr int kThreads = 256;

unsigned blocks_for(int64_t items) {
  int64_t b = (items + kThreads - 1) / kThreads;
  return (unsigned)(b < 1 ? 1 : b);
}

__global__ void transform_in_kernel(const int64_t *__restrict__ keys, uint64_t *__restrict__ u,
                                    int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    u[i] = (uint64_t)keys[i] ^ kSign;
}

__global__ void transform_out_kernel(const uint64_t *__restrict__ u, int64_t *__restrict__ keys,
                                     int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = (int64_t)(u[i] ^ kSign);
}

// flags bit0: duplicate key, bit1: key == Max_Key.
__global__ void check_sorted_kernel(const uint64_t *__restrict__ u, int64_t n, unsigned *flags) {
  unsigned f = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = u[i];
    if (i > 0 && u[i - 1] == k) f |= 1u;
    if ((int64_t)(k ^ kSign) == kMaxKey) f |= 2u;
  }
  if (f) atomicOr(flags, f);
}

// One thread per (leaf, word) of the leaf rows: index words, keys, values.
__global__ void leaf_kernel(const uint64_t *__restrict__ u, const int64_t *__restrict__ vals,
                            int64_t n, int64_t n_leaf, int lc, int li,
                            int64_t *__restrict__ leaf_rows, int32_t *__restrict__ leaf_cnt,
                            int64_t *__restrict__ leaf_base, int64_t *__restrict__ submin) {
  const int row = li + 2 * lc;
  const int64_t total = n_leaf * (int64_t)row;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t j = t / row;
    int w = (int)(t - j * row);
    int64_t s = part_start(j, n, n_leaf), e = part_start(j + 1, n, n_leaf);
    if (w >= li + lc) {  // value word
      int slot = w - li - lc;
      leaf_rows[t] = (s + slot < e) ? vals[s + slot] : (int64_t)HM_NOT_FOUND;
      continue;
    }
    int slot = w < li ? 8 * (w + 1) : w - li;  // index word w mirrors key slot 8(w+1)
    int64_t k = kMaxKey;
    if (slot < lc && s + slot < e) k = (int64_t)(u[s + slot] ^ kSign);
    leaf_rows[t] = k;
    if (w >= li) {
      if (slot == 0) {
        leaf_cnt[j] = (int32_t)(e - s);
        leaf_base[j] = s;
        submin[j] = (s < e) ? (int64_t)(u[s] ^ kSign) : kMaxKey;
      }
    }
  }
}

// One thread per (node, word) of one inner level.  m = nodes of the level
// below, whose subtree minima are in submin_below; child_base = BFS id of the
// level below's first node (n_inner for leaves).
__global__ void inner_kernel(int64_t nodes, int64_t m, int f, int64_t lvl_base,
                             int64_t child_base, const int64_t *__restrict__ submin_below,
                             int64_t *__restrict__ inner, int32_t *__restrict__ prefix,
                             int64_t *__restrict__ submin_here) {
  const int ix = f / 8, row = ix + f;
  const int64_t total = nodes * (int64_t)row;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    int64_t i = t / row;
    int w = (int)(t - i * row);
    int64_t c0 = part_start(i, m, nodes), c1 = part_start(i + 1, m, nodes);
    int slot = w < ix ? 8 * (w + 1) : w - ix;
    // separator `slot` = minimum key of child slot+1
    int64_t c = c0 + 1 + slot;
    int64_t k = (slot < f && c < c1) ? submin_below[c] : kMaxKey;
    inner[(lvl_base + i) * row + w] = k;
    if (w == ix) {
      prefix[lvl_base + i] = (int32_t)(child_base + c0);
      submin_here[i] = submin_below[c0];
    }
  }
}

}  // namespace

int shape(int64_t n, const hm_config &c, int *height, int64_t *lvl_start, int64_t *n_inner,
          int64_t *n_leaf) {
  if (n < 0) return HM_EINVAL;
  int64_t nl = n == 0 ? 1 : (n + c.leaf_fill - 1) / c.leaf_fill;
  int64_t sizes[kMaxLevels];
  int h = 0;
  int64_t m = nl;
  do {
    if (h >= kMaxLevels) return HM_ETOOLARGE;
    int64_t nodes = (m + c.inner_fill - 1) / c.inner_fill;
    sizes[h++] = nodes;
    m = nodes;
  } while (m > 1);
  int64_t acc = 0;
  for (int l = 0; l < h; l++) {
    lvl_start[l] = acc;
    acc += sizes[h - 1 - l];
  }
  lvl_start[h] = acc;
  if (acc > INT32_MAX / 2 || nl > INT32_MAX / 2) return HM_ETOOLARGE;
  *height = h;
  *n_inner = acc;
  *n_leaf = nl;
  return HM_OK;
}

void transform_keys_in(const int64_t *keys, uint64_t *ukeys, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  transform_in_kernel<<<min(blocks_for(n), 148u * 16), kThreads, 0, s>>>(keys, ukeys, n);
  note_launch();
}

void transform_keys_out(const uint64_t *ukeys, int64_t *keys, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  transform_out_kernel<<<min(blocks_for(n), 148u * 16), kThreads, 0, s>>>(ukeys, keys, n);
  note_launch();
}

void check_sorted_keys(const uint64_t *ukeys, int64_t n, unsigned *d_flags, cudaStream_t s) {
  if (n <= 0) return;
  check_sorted_kernel<<<min(blocks_for(n), 148u * 16), kThreads, 0, s>>>(ukeys, n, d_flags);
  note_launch();
}

int build_from_sorted(const BuildTarget &b, const uint64_t *ukeys, const int64_t *vals, int64_t n,
                      int64_t *tmp_a, int64_t *tmp_b, cudaStream_t s) {
  const BuildTarget *t = &b;
  const int lc = t->leaf_cap, f = t->fanout;
  int64_t leaf_words = t->n_leaf * (int64_t)t->leaf_row;
  leaf_kernel<<<min(blocks_for(leaf_words), 148u * 32), kThreads, 0, s>>>(
      ukeys, vals, n, t->n_leaf, lc, t->leaf_index, t->leaf_rows, t->leaf_cnt, t->leaf_base, tmp_a);
  note_launch();
  int64_t *below = tmp_a, *here = tmp_b;
  int64_t m = t->n_leaf;
  for (int l = t->height - 1; l >= 0; l--) {
    int64_t nodes = t->lvl_start[l + 1] - t->lvl_start[l];
    int64_t words = nodes * (int64_t)t->inner_row;
    inner_kernel<<<min(blocks_for(words), 148u * 32), kThreads, 0, s>>>(
        nodes, m, f, t->lvl_start[l], t->lvl_start[l + 1], below, t->inner, t->prefix, here);
    note_launch();
    int64_t *tmp = below;
    below = here;
    here = tmp;
    m = nodes;
  }
  return cuda_err(cudaGetLastError());
}

}  // namespace hm
