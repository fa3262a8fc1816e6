// hm_search_noalloc: the pre-sorted point search with its scratch memory in
// a fixed device array instead of the tree's allocated scratch.
//
// Some callers cannot allocate device memory at the moment they search: a
// host runtime that reserves all device memory up front and hands the library
// only its input and output buffers, a serving loop held to a fixed
// device-memory budget, or a latency-bound caller that cannot afford the
// device-wide synchronisation cudaFree implies.  For them this entry point
// takes its working space (the partitioned queries, their positions and the
// histogram counters) from one file-scope __device__ array of fixed size,
// created when the library is loaded, so a call never allocates.
//
// Rules of use:
//  * q and out must be device (or managed) memory; n <= HM_NOALLOC_MAX_QUERIES.
//  * Each GPU that loads the library holds the array (HM_NOALLOC_SCRATCH_BYTES)
//    until the process exits.
//  * The first call on a device looks the array's device address up
//    (cudaGetSymbolAddress, with that device current) and caches it; the
//    search kernels' launch shapes are resolved then too.  Both caches serve
//    the whole process, whichever thread calls next.  Make that first call
//    before any stream capture.
//  * All calls on a device share the one array, which keeps whatever the last
//    call left in it: calls whose work overlaps on the GPU (different streams,
//    or different trees searched concurrently) race and must be serialised by
//    the caller.  Every word a call reads is written earlier by the same call,
//    so nothing needs clearing between calls.
#include "hm_internal.cuh"

#include <mutex>

namespace hm {

namespace {

constexpr int64_t kMaxQueries = HM_NOALLOC_MAX_QUERIES;
constexpr int kBits = 8;  // one partition pass

// partitioned keys (8 B), positions (4 B), partition counters and scan scratch
constexpr size_t kQBytes = (size_t)kMaxQueries * 8;
constexpr size_t kPosBytes = (size_t)kMaxQueries * 4;
constexpr size_t kScratchBytes = HM_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once).
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_err(e);
  if (dev < 0 || dev >= kMaxDevices) return HM_ENODEVICE;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return e != cudaSuccess ? cuda_err(e) : HM_ECUDA;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return HM_OK;
}

bool device_accessible(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

}  // namespace hm

using namespace hm;

extern "C" int hm_search_noalloc(hm_tree *t, const int64_t *q, size_t n_, int64_t *out, hm_stream hs) {
  if (!t || (n_ > 0 && (!q || !out))) return HM_EINVAL;
  const int64_t n = (int64_t)n_;
  if (n == 0) return HM_OK;
  if (n > kMaxQueries) return HM_ETOOLARGE;
  if (!device_accessible(q) || !device_accessible(out)) return HM_EINVAL;
  static_assert(kQBytes + kPosBytes + 3 * 256 <= kScratchBytes, "scratch layout");
  if (partition_scratch_bytes(kMaxQueries, kBits, false) + kQBytes + kPosBytes + 3 * 256 > kScratchBytes)
    return HM_ETOOLARGE;
  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  char *p = static_cast<char *>(base);
  int64_t *qs = reinterpret_cast<int64_t *>(p);
  int32_t *pos = reinterpret_cast<int32_t *>(p + align_up(n * 8, 256));
  void *ps = p + align_up(n * 8, 256) + align_up(n * 4, 256);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(hs);
  rc = partition_queries(t, q, n, kBits, qs, pos, ps, s);
  if (rc) return rc;
  SearchLaunch l{qs, out, pos, n};
  return launch_search(t, l, t->cfg.group_width, t->cfg.queries_per_group, s);
}
