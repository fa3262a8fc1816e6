// Many query batches of uneven size in one launch sequence, and its CUDA
// graph ("plan").
//
// The reference searches one fixed-size bucket of 41.9M queries per launch
// from a launcher pthread (launch_kernel_thread,
// open-harmonia/src/full-multi-prefix-sort-8thread.cu:276-327).  Here a set of
// batches is described once on the device (query pointer, output pointer,
// size) and searched together:
//   * small sets: one persistent search kernel whose CTAs take tiles from a
//     global counter and find their batch by binary search over the tile
//     prefix (no pre-sort);
//   * large sets: the batches are pre-sorted together as one concatenation
//     (the query pre-sort reads each batch in place and sees every batch at
//     once, so even 1K-query batches share the locality of the whole set),
//     searched, and the last inverse pass of the pre-sort writes each result
//     to its batch's output.
// Everything is enqueued on one stream with no host synchronisation and no
// allocation, so hm_plan_create can capture it in a CUDA graph that
// hm_plan_launch replays.
#include "hm_internal.cuh"

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace hm {

namespace {


// Descriptor block in device memory: batches, query prefix (nb+1),
// search-tile prefix (nb+1) and the search tile counter.
struct SetLayout {
  size_t off_batches, off_qpre, off_tpre, bytes;
};

SetLayout set_layout(int nb) {
  SetLayout l;
  l.off_batches = 0;
  l.off_qpre = align_up((int64_t)sizeof(hm_batch) * nb, 256);
  l.off_tpre = l.off_qpre + align_up(8 * (nb + 1), 256);
  l.bytes = l.off_tpre + align_up(8 * (nb + 2), 256);
  return l;
}

}  // namespace

// Work memory of a large set: the scratch of the sorted search plan.  Small
// sets need none.
size_t batches_work_bytes(const hm_tree *t, int64_t total, const SearchPlan &p) {
  if (p.bits <= 0) return 0;
  return p.scratch;
}

// Host side: fills the descriptor block image for nb batches.
int build_set(const hm_tree *t, const hm_batch *batches, int nb, std::vector<char> &img,
              int64_t *total_out, int64_t *tiles_out) {
  const SetLayout l = set_layout(nb);
  img.assign(l.bytes, 0);
  hm_batch *b = reinterpret_cast<hm_batch *>(img.data() + l.off_batches);
  int64_t *qpre = reinterpret_cast<int64_t *>(img.data() + l.off_qpre);
  int64_t *tpre = reinterpret_cast<int64_t *>(img.data() + l.off_tpre);
  const int tileq = search_tile_queries(t->cfg.group_width, t->cfg.queries_per_group);
  qpre[0] = tpre[0] = 0;
  for (int i = 0; i < nb; i++) {
    if (batches[i].n < 0 || (batches[i].n > 0 && (!batches[i].q || !batches[i].out))) return HM_EINVAL;
    b[i] = batches[i];
    qpre[i + 1] = qpre[i] + batches[i].n;
    tpre[i + 1] = tpre[i] + (batches[i].n + tileq - 1) / tileq;
  }
  tpre[nb + 1] = 0;  // tile counter, reset before every launch
  *total_out = qpre[nb];
  *tiles_out = tpre[nb];
  return HM_OK;
}

// Enqueues the whole multi-batch search on s.  d_set is the device copy of
// the descriptor block; work has batches_work_bytes(total, plan) bytes.
int enqueue_batches(hm_tree *t, char *d_set, int nb, int64_t total, int64_t tiles,
                    const SearchPlan &plan, char *work, cudaStream_t s) {
  const SetLayout l = set_layout(nb);
  const hm_batch *d_b = reinterpret_cast<const hm_batch *>(d_set + l.off_batches);
  const int64_t *qpre = reinterpret_cast<const int64_t *>(d_set + l.off_qpre);
  int64_t *tpre = reinterpret_cast<int64_t *>(d_set + l.off_tpre);
  if (total == 0) return HM_OK;
  if (plan.bits <= 0) {
    cudaMemsetAsync(tpre + nb + 1, 0, 8, s);
    return launch_search_batches(t, d_b, tpre, nb, tiles, t->cfg.group_width,
                                 t->cfg.queries_per_group, s);
  }
  // the pre-sort reads every batch's queries and the last inverse pass
  // writes every batch's results: no gathered copy of the set
  BatchView bv;
  bv.batches = d_b;
  bv.qpre = qpre;
  bv.nb = nb;
  return run_planned_search(t, plan, nullptr, total, nullptr, s, work, &bv);
}

}  // namespace hm

using namespace hm;

struct hm_plan {
  hm_tree *tree = nullptr;
  int nb = 0;
  int64_t total = 0, tiles = 0;
  SearchPlan plan;
  char *dev = nullptr;  // descriptor block + work
  size_t dev_bytes = 0;
  std::vector<hm_batch> batches;
  std::vector<char> img;
  uint64_t generation = 0;
  hm_config cfg{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int kernel_nodes = 0;
};

namespace {

void drop_graph(hm_plan *p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
}

int capture(hm_plan *p) {
  drop_graph(p);
  hm_tree *t = p->tree;
  const SetLayout l = set_layout(p->nb);
  // the tile prefix depends on the search parameters: rebuild and upload it
  int rc0 = build_set(t, p->batches.data(), p->nb, p->img, &p->total, &p->tiles);
  if (rc0) return rc0;
  p->plan = plan_search(t, p->total, p->nb);
  const size_t need = p->img.size() + batches_work_bytes(t, p->total, p->plan);
  if (need > p->dev_bytes) {  // a retune may need more work memory
    if (p->dev) cudaFree(p->dev);
    p->dev = nullptr;
    p->dev_bytes = 0;
    cudaError_t ea = cudaMalloc(&p->dev, need);
    if (ea != cudaSuccess) return cuda_err(ea);
    p->dev_bytes = need;
  }
  cudaError_t e0 = cudaMemcpy(p->dev, p->img.data(), p->img.size(), cudaMemcpyHostToDevice);
  if (e0 != cudaSuccess) return cuda_err(e0);
  // warm the kernel attribute / occupancy cache outside the capture
  int rc = launch_search_warm(t, t->cfg.group_width, t->cfg.queries_per_group);
  if (rc) return rc;
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_err(e);
  const bool prof = t->prof;
  t->prof = false;  // no timing events inside a graph
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    set_capturing(true);
    rc = enqueue_batches(t, p->dev, p->nb, p->total, p->tiles, p->plan,
                         p->dev + l.bytes, cs);
    set_capturing(false);
    cudaError_t e2 = cudaStreamEndCapture(cs, &p->graph);
    if (e == cudaSuccess) e = e2;
  }
  t->prof = prof;
  if (e == cudaSuccess && rc == HM_OK) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
  if (e == cudaSuccess && rc == HM_OK) {
    size_t nn = 0;
    cudaGraphGetNodes(p->graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(p->graph, nodes.data(), &nn);
    p->kernel_nodes = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType ty;
      if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) p->kernel_nodes++;
    }
  }
  cudaStreamDestroy(cs);
  if (rc) return rc;
  if (e != cudaSuccess) {
    drop_graph(p);
    return cuda_err(e);
  }
  p->generation = t->generation;
  p->cfg = t->cfg;
  return HM_OK;
}

}  // namespace

extern "C" {

int hm_search_batches(hm_tree *t, const hm_batch *batches, int nb, hm_stream hs) {
  if (!t || nb < 0 || (nb > 0 && !batches)) return HM_EINVAL;
  if (nb == 0) return HM_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(hs);
  std::vector<char> img;
  int64_t total = 0, tiles = 0;
  int rc = build_set(t, batches, nb, img, &total, &tiles);
  if (rc) return rc;
  const SearchPlan plan = plan_search(t, total, nb);
  const size_t set_bytes = img.size();
  ScratchLease lease(t, s);
  rc = lease.acquire(set_bytes + batches_work_bytes(t, total, plan));
  if (rc) return rc;
  char *d = static_cast<char *>(lease.ptr());
  cudaError_t e = cudaMemcpyAsync(d, img.data(), set_bytes, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_err(e);
  int tok = prof_begin(t, s);
  rc = enqueue_batches(t, d, nb, total, tiles, plan, d + set_bytes, s);
  prof_end(t, kStageBatches, tok, s);
  e = cudaStreamSynchronize(s);  // img is a host buffer the copy reads
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_err(e);
  return hm_sync(t, hs);
}

int hm_plan_create(hm_tree *t, const hm_batch *batches, int nb, hm_plan **out) {
  if (!t || !out || nb <= 0 || !batches) return HM_EINVAL;
  *out = nullptr;
  hm_plan *p = new (std::nothrow) hm_plan();
  if (!p) return HM_ENOMEM;
  p->tree = t;
  p->nb = nb;
  p->batches.assign(batches, batches + nb);
  int rc = build_set(t, batches, nb, p->img, &p->total, &p->tiles);
  if (rc) {
    delete p;
    return rc;
  }
  rc = capture(p);  // sizes and allocates the plan's device memory
  if (rc) {
    if (p->dev) cudaFree(p->dev);
    delete p;
    return rc;
  }
  *out = p;
  return HM_OK;
}

int hm_plan_launch(hm_plan *p, hm_stream hs) {
  if (!p) return HM_EINVAL;
  hm_tree *t = p->tree;
  // the graph bakes in the tree arena and search parameters: re-capture after
  // a rebuild or a retune
  if (p->generation != t->generation || std::memcmp(&p->cfg, &t->cfg, sizeof(hm_config)) != 0) {
    int rc = capture(p);
    if (rc) return rc;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(hs);
  int tok = prof_begin(t, s);
  cudaError_t e = cudaGraphLaunch(p->exec, s);
  prof_end(t, kStageBatches, tok, s);
  note_launch(p->kernel_nodes);
  return cuda_err(e);
}

int hm_plan_free(hm_plan *p) {
  if (!p) return HM_OK;
  cudaDeviceSynchronize();
  drop_graph(p);
  if (p->dev) cudaFree(p->dev);
  delete p;
  return HM_OK;
}

}  // extern "C"
