// Test and comparison infrastructure only: the reference's own GPU point
// search (open-harmonia/src/full-multi-prefix-sort-8thread.cu), compiled
// from the reference's source for sm_100a by oracle/Makefile into
// oracle/_ref/libhmref_gpu.so, driven on the reference's own PPI tree.  Only
// bench.py's comparison figure and tests load it; the product never does.
//
// The reference's driver (full_multi_prefix_sort_8thread, same file :329-495)
// uploads the tree with prepareGPU_v2 / prepareGPU_leaf (prepareGPU.cu:140-163),
// then per bucket of keys runs cub::DeviceRadixSort::SortPairs on bits
// [48, 64) of (key, position) (:305-309), the 8-thread kernel (:95-263), and
// copies the (leaf, list, slot) results and the positions back (:314-315),
// which its test path decodes on the host (:454-476).  This driver keeps those
// steps, with three differences, each for a reason:
//   * the upload copies the same bytes but sizes them as size_t:
//     prepareGPU_leaf's `int size = getBLeafSize() * sizeof(BLeaf_node)`
//     overflows at 2^26 64-bit keys (515,872 big leaves x 4,416 B);
//   * a launch covers exactly n / 1024 blocks of 128 threads (n a multiple of
//     1024, the keys one block takes): the kernel skips a __syncthreads for
//     keys past the count, so a partly filled block is not launched;
//   * before any launch the kernel's index arithmetic runs on the CPU over
//     the whole batch with bounds checks (node, leaf and record-list ids, and
//     the index stage finding a word above the key, without which the kernel
//     would read a slice number it never wrote); a batch that fails is
//     refused.
// CUB before the reference's headers: they #define key_t, a name CUB's
// templates use.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "bpt.h"

#include <cstdint>
#include <new>
#include <vector>

// The reference's per-query result record (full-multi-prefix-sort-8thread.cu:34-39):
// big-leaf id (or -1) and the record list (low 6 bits) and slot (high 2 bits).
struct GPU_Result {
  int blfnode;
  char idx;
};

// Defined in open-harmonia/src/full-multi-prefix-sort-8thread.cu:95.
__global__ void full_multi_prefix_sort_8thread_kernel(Inner_node *d_innode, BLeaf_node *d_bleafnode, int *d_prefix,
                                                      int inner_node_size_wo_last_inner_node, int root_idx,
                                                      key_t *d_keys, int tree_height, GPU_Result *d_gresult,
                                                      int key_count);

extern "C" void *hmref_ppi_tree(void *hp);

namespace {

constexpr int kBlock = 128;          // Block_Dim (full-multi-prefix-sort-8thread.cu:23)
constexpr int kKeysPerBlock = 1024;  // Block_Dim / Thread_Per_Query * GPU_SWP_SIZE (:97)

struct RefGpu {
  BPlusTree *t = nullptr;
  Inner_node *d_inner = nullptr;
  int *d_prefix = nullptr;
  BLeaf_node *d_leaf = nullptr;
  int n_inner = 0, n_bleaf = 0, root = 0, height = 0, inner_wo_last = 0;
};

void release(RefGpu *g) {
  if (g->d_inner) cudaFree(g->d_inner);
  if (g->d_prefix) cudaFree(g->d_prefix);
  if (g->d_leaf) cudaFree(g->d_leaf);
  delete g;
}

// The kernel's descent for one key on the host tree (the same index and
// slice rules as :126-199 and the leaf test of :214-252), with every id
// checked against the uploaded arrays; false if one would leave them.
bool check_one(const RefGpu &g, const int *prefix, key_t target) {
  int pos = g.root;
  int relist = 0;
  for (int i = 1; i < g.height; i++) {
    if (pos < 0 || pos >= g.n_inner) return false;
    const Inner_node *node = g.t->getInnerNodeByIdx(pos);
    int s = 0;  // first index word greater than the key
    for (; s < 8; s++)
      if (target < node->inner_index[s]) break;
    // none: the kernel would take a slice from shared memory it never
    // initialised for this step (inner_index_result, :119, :141-143)
    if (s == 8) return false;
    const int begin = s * 8;
    int idx = begin + 8;
    for (int k = 0; k < 8; k++)
      if (target < node->inner_key[begin + k]) {
        idx = begin + k;
        break;
      }
    if (i == g.height - 1) {
      pos = pos - g.inner_wo_last;
      relist = idx;
    } else {
      pos = prefix[pos] + idx;
    }
  }
  return pos >= 0 && pos < g.n_bleaf && relist >= 0 && relist <= BL_leafnum;
}

}  // namespace

extern "C" {

// Uploads the reference tree's inner nodes, prefix array and big leaves.
// Returns a handle, or nullptr (no device, allocation failure, a tree the
// kernel cannot search: height < 2).
void *hmrefgpu_prepare(void *hp) {
  BPlusTree *t = static_cast<BPlusTree *>(hmref_ppi_tree(hp));
  if (!t || t->getHeight() < 2 || !t->getPrefixArray()) return nullptr;
  RefGpu *g = new (std::nothrow) RefGpu();
  if (!g) return nullptr;
  g->t = t;
  g->n_inner = t->getInnerSize();
  g->n_bleaf = t->getBLeafSize();
  g->root = t->getRootIdx();
  g->height = t->getHeight();
  g->inner_wo_last = t->getInnerSize_wo_last_inner_node();
  Inner_node *h_inner = nullptr;
  unsigned int inner_bytes = 0;
  t->getInnerSegementationInfo(h_inner, inner_bytes);
  const size_t leaf_bytes = (size_t)g->n_bleaf * sizeof(BLeaf_node);
  cudaError_t e = cudaMalloc(&g->d_inner, inner_bytes);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_inner, h_inner, inner_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_prefix, (size_t)g->n_inner * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(g->d_prefix, t->getPrefixArray(), (size_t)g->n_inner * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&g->d_leaf, leaf_bytes);
  if (e == cudaSuccess) e = cudaMemcpy(g->d_leaf, t->getBLeafNodeStart(), leaf_bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess || g->root < 0) {
    cudaGetLastError();
    release(g);
    return nullptr;
  }
  return g;
}

// The CPU check alone (no device needed): how many of the n keys the kernel
// would search outside the tree's arrays (0 means the batch may be launched).
long hmrefgpu_check(void *hp, const long long *q, long n) {
  BPlusTree *t = static_cast<BPlusTree *>(hmref_ppi_tree(hp));
  if (!t || t->getHeight() < 2 || !t->getPrefixArray()) return -1;
  RefGpu g;
  g.t = t;
  g.n_inner = t->getInnerSize();
  g.n_bleaf = t->getBLeafSize();
  g.root = t->getRootIdx();
  g.height = t->getHeight();
  g.inner_wo_last = t->getInnerSize_wo_last_inner_node();
  long bad = 0;
  for (long i = 0; i < n; i++) bad += (q[i] == Max_Key || !check_one(g, t->getPrefixArray(), q[i])) ? 1 : 0;
  return bad;
}

// The kernel's whole per-key computation on the CPU (descent as check_one,
// then the leaf phase of :214-252: the first of the record list's 4 slots
// whose key is >= the query, a hit if equal), decoded as the driver decodes
// the GPU's results; out[i] = the value or -1, or -7 for a key the check
// refuses.  For finding where the GPU results depart from the CPU search.
void hmrefgpu_emulate(void *hp, const long long *q, long n, long long *out) {
  BPlusTree *t = static_cast<BPlusTree *>(hmref_ppi_tree(hp));
  RefGpu g;
  g.t = t;
  g.n_inner = t->getInnerSize();
  g.n_bleaf = t->getBLeafSize();
  g.root = t->getRootIdx();
  g.height = t->getHeight();
  g.inner_wo_last = t->getInnerSize_wo_last_inner_node();
  const int *prefix = t->getPrefixArray();
  for (long i = 0; i < n; i++) {
    const key_t target = q[i];
    if (target == Max_Key || !check_one(g, prefix, target)) {
      out[i] = -7;
      continue;
    }
    int pos = g.root, relist = 0;
    for (int lv = 1; lv < g.height; lv++) {
      const Inner_node *node = t->getInnerNodeByIdx(pos);
      int s = 0;
      while (s < 8 && !(target < node->inner_index[s])) s++;
      const int begin = s * 8;
      int idx = begin + 8;
      for (int k = 0; k < 8; k++)
        if (target < node->inner_key[begin + k]) {
          idx = begin + k;
          break;
        }
      if (lv == g.height - 1) {
        pos -= g.inner_wo_last;
        relist = idx;
      } else {
        pos = prefix[pos] + idx;
      }
    }
    const BLeaf_node *leaf = t->getBLeafNodeByIdx(pos);
    long long v = -1;
    for (int s2 = 0; s2 < 4; s2++) {
      const key_t k = leaf->relist[relist].r[s2].r_key;
      if (target <= k) {
        if (k == target) v = leaf->relist[relist].r[s2].val;
        break;
      }
    }
    out[i] = v;
  }
}

void hmrefgpu_free(void *h) {
  if (h) release(static_cast<RefGpu *>(h));
}

// Searches n keys (host memory, n a multiple of 1024 and below 2^31) as the
// reference does: copy in, SortPairs on bits [48, 64), the 8-thread kernel,
// results and positions back, decode; out[i] = the value of q[i] or -1.  The
// sort and kernel are run `reps` times on the resident keys first and their
// mean device time goes to *ms_device; the whole sequence once more with the
// copies, timed on the device, to *ms_copies.  Returns 0, -1 (bad arguments),
// -2 (the CPU check refused the batch) or -3 (a CUDA call failed).
int hmrefgpu_search(void *h, const long long *q, long n, long long *out, int reps, float *ms_device,
                    float *ms_copies) {
  RefGpu *g = static_cast<RefGpu *>(h);
  if (!g || n <= 0 || n % kKeysPerBlock != 0 || n > (1l << 30) || reps < 0) return -1;
  const int *prefix = g->t->getPrefixArray();
  for (long i = 0; i < n; i++)
    if (q[i] == Max_Key || !check_one(*g, prefix, q[i])) return -2;
  key_t *d_keys = nullptr, *d_keys_sorted = nullptr;
  int *d_pos = nullptr, *d_pos_sorted = nullptr;
  GPU_Result *d_res = nullptr;
  void *d_temp = nullptr;
  size_t temp_bytes = 0;
  std::vector<int> pos(n);
  for (long i = 0; i < n; i++) pos[i] = (int)i;
  std::vector<GPU_Result> res(n);
  std::vector<int> pos_sorted(n);
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  if (e == cudaSuccess) e = cudaMalloc(&d_keys, n * sizeof(key_t));
  if (e == cudaSuccess) e = cudaMalloc(&d_keys_sorted, n * sizeof(key_t));
  if (e == cudaSuccess) e = cudaMalloc(&d_pos, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_pos_sorted, n * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_res, n * sizeof(GPU_Result));
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, d_keys, d_keys_sorted, d_pos, d_pos_sorted, (int)n, 48,
                                        64, s);
  if (e == cudaSuccess) e = cudaMalloc(&d_temp, temp_bytes);
  auto body = [&]() {
    cudaError_t x = cub::DeviceRadixSort::SortPairs(d_temp, temp_bytes, d_keys, d_keys_sorted, d_pos, d_pos_sorted,
                                                    (int)n, 48, 64, s);
    if (x != cudaSuccess) return x;
    full_multi_prefix_sort_8thread_kernel<<<(unsigned)(n / kKeysPerBlock), kBlock, 0, s>>>(
        g->d_inner, g->d_leaf, g->d_prefix, g->inner_wo_last, g->root, d_keys_sorted, g->height, d_res, (int)n);
    return cudaGetLastError();
  };
  float msd = 0, msc = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_keys, q, n * sizeof(key_t), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_pos, pos.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = body();  // warm-up
  if (e == cudaSuccess && reps > 0) {
    cudaEventRecord(a, s);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = body();
    cudaEventRecord(b, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&msd, a, b);
    msd /= (float)reps;
  }
  if (e == cudaSuccess) e = cudaEventRecord(a, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_keys, q, n * sizeof(key_t), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_pos, pos.data(), n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = body();
  if (e == cudaSuccess) e = cudaMemcpyAsync(res.data(), d_res, n * sizeof(GPU_Result), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pos_sorted.data(), d_pos_sorted, n * sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaEventRecord(b, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&msc, a, b);
  if (d_temp) cudaFree(d_temp);
  if (d_res) cudaFree(d_res);
  if (d_pos_sorted) cudaFree(d_pos_sorted);
  if (d_pos) cudaFree(d_pos);
  if (d_keys_sorted) cudaFree(d_keys_sorted);
  if (d_keys) cudaFree(d_keys);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (s) cudaStreamDestroy(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return -3;
  }
  // decode as the reference's test path does (:460-470)
  for (long j = 0; j < n; j++) {
    const int leaf = res[j].blfnode;
    long long v = -1;
    if (leaf >= 0 && leaf < g->n_bleaf) {
      const int relist = res[j].idx & 63, slot = (res[j].idx >> 6) & 3;
      v = g->t->getLeafByIdx(leaf)->relist[relist].r[slot].val;
    }
    const int p = pos_sorted[j];
    if (p >= 0 && p < n) out[p] = v;
  }
  if (ms_device) *ms_device = msd;
  if (ms_copies) *ms_copies = msc;
  return 0;
}

}  // extern "C"
