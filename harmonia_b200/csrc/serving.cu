// Serving loop: a request queue in front of one device-resident tree.
//
// The reference has no serving path: every experiment reads a whole file,
// runs fixed-size buckets from a launcher pthread and prints timings
// (open-harmonia/src/full-multi-prefix-sort-8thread.cu:276-495), and its
// CPU/GPU pipeline variants spin on volatile flags without a bound
// (open-harmonia/src/buffer.h:88-106).  Here:
//   * callers submit point-search, range and upsert requests with host
//     buffers and get a ticket; hm_server_wait blocks (with a timeout) until
//     the request is done; a point search whose buffers are page-locked (or
//     device memory) is copied by DMA straight from and to them, the others
//     through pinned staging filled by helper threads;
//   * a dispatcher thread admits requests in ticket order while the device
//     bytes they need fit the budget, coalesces consecutive point searches
//     (and consecutive ranges) into one launch, and keeps up to `streams`
//     launches in flight, so requests that arrive while others run on the GPU
//     are admitted as slots and memory free up (continuous batching);
//   * an upsert is an epoch barrier: it starts after the kernels of every
//     earlier request have finished (their result copies may still run) and
//     before any later request, so each read sees exactly the upserts
//     submitted before it, the same result it would get alone;
//     consecutive upserts with supplied values are applied as one epoch;
//   * every wait is bounded: the dispatcher polls launch events and the
//     caller's wait has a timeout; stop() cancels what has not started.
#include "hm_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace hm {

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  uint64_t ticket = 0;
  hm_request r{};
  int status = 1;  // 1 = pending
  Clock::time_point t_submit;
  // where a read's time goes: taken into a launch, launch enqueued (inputs
  // staged and copied), launch seen finished on the device
  Clock::time_point t_admit, t_enqueued, t_device_done;
  double latency_us = 0;
  size_t bytes = 0;  // device bytes the request needs while in flight
  // point searches: keys / out are page-locked host or device memory, which
  // the copy engines reach directly (no staging copy on the host)
  bool direct_in = false, direct_out = false;
};

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t done = nullptr;   // the launch's last copy finished
  cudaEvent_t kdone = nullptr;  // its kernels (the last reads of the tree) finished
  char *dev = nullptr;
  size_t dev_bytes = 0;
  char *pin = nullptr;
  size_t pin_bytes = 0;
  std::vector<Req *> reqs;
  // HM_REQ_SEARCH or HM_REQ_RANGE while its launch runs, -3 while the
  // completer copies its results out, -1 free, -2 retired; only the
  // dispatcher thread reads or writes it
  int kind = -1;
  int launched = -1;  // the kind of the launch being completed
  int64_t n = 0;
  size_t reserved = 0;
  bool retired = false;
  Clock::time_point t_launch;
};

// Host copies between the callers' buffers and the slots' pinned staging run
// on a few helper threads besides the dispatcher: one thread's memcpy is far
// below the host's memory bandwidth and caps the serving rate.
struct CopyJob {
  char *dst;
  const char *src;
  size_t bytes;
};

class CopyPool {
 public:
  void start(int helpers) {
    for (int i = 0; i < helpers; i++) th_.emplace_back([this] { work(); });
  }
  void stop() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      quit_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
    th_.clear();
  }
  // Runs every copy (split into kPiece pieces) on the helpers and the calling
  // thread; returns when all are done.  One caller at a time.
  void run(const std::vector<CopyJob> &jobs) {
    size_t total = 0;
    for (const CopyJob &j : jobs) total += j.bytes;
    if (th_.empty() || total < kPiece) {
      for (const CopyJob &j : jobs) std::memcpy(j.dst, j.src, j.bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      pieces_.clear();
      for (const CopyJob &j : jobs)
        for (size_t o = 0; o < j.bytes; o += kPiece)
          pieces_.push_back({j.dst + o, j.src + o, std::min(kPiece, j.bytes - o)});
      next_ = 0;
      left_ = pieces_.size();
    }
    cv_.notify_all();
    for (;;) {
      CopyJob j;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (next_ >= pieces_.size()) break;
        j = pieces_[next_++];
      }
      std::memcpy(j.dst, j.src, j.bytes);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) cv_done_.notify_all();
    }
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [this] { return left_ == 0; });
  }

 private:
  // measured on the serving mix: the dispatcher's own copies of requests
  // below a MiB (most of them) capped its rate when only larger copies were
  // shared out
  static constexpr size_t kPiece = (size_t)128 << 10;
  void work() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [this] { return quit_ || next_ < pieces_.size(); });
      if (quit_) return;
      const CopyJob j = pieces_[next_++];
      lk.unlock();
      std::memcpy(j.dst, j.src, j.bytes);
      lk.lock();
      if (--left_ == 0) cv_done_.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_, cv_done_;
  std::vector<CopyJob> pieces_;
  size_t next_ = 0, left_ = 0;
  bool quit_ = false;
  std::vector<std::thread> th_;
};

// Page-locked host memory (cudaHostAlloc, cudaHostRegister) or device
// memory: a copy engine reads or writes it without a staging copy.
bool dma_reachable(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice;
}

size_t req_device_bytes(const hm_request &r) {
  switch (r.kind) {
    case HM_REQ_SEARCH: return 16 * r.n;
    case HM_REQ_DELETE: return 8 * r.n;
    case HM_REQ_RANGE: {
      size_t recs = 0;
      for (size_t i = 0; i < r.n; i++) recs += r.lens[i] > 0 ? (size_t)r.lens[i] : 0;
      return 32 * r.n + 16 * recs;
    }
    default: return 16 * r.n;
  }
}

}  // namespace
}  // namespace hm

using namespace hm;

struct hm_server {
  hm_tree *t = nullptr;
  hm_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<Req *> queue;
  std::unordered_map<uint64_t, Req *> reqs;  // until the caller collects them
  uint64_t next_ticket = 1;
  bool stopping = false;
  std::thread th;
  std::vector<Slot> slots;
  size_t reserved = 0;
  CopyPool copies;      // the dispatcher's copies into pinned staging
  CopyPool copies_out;  // the completer's copies out to the callers' buffers
  // Launches seen finished on the device go to the completer thread, which
  // copies the results out and finishes the requests, then hands the slot
  // back (handed_back) for the dispatcher to free; both queues under mu.
  std::thread completer;
  std::deque<Slot *> to_complete, handed_back;
  std::condition_variable cv_complete;
  bool completer_quit = false;
  Slot epoch_slot;  // staging and stream of write epochs
  // stats
  std::vector<double> lat;
  std::vector<double> lat_queue, lat_stage, lat_device, lat_finish;  // reads only
  double epoch_drain_us = 0, epoch_apply_us = 0;  // summed over epochs
  uint64_t completed = 0, rejected = 0, launches = 0, epochs = 0, queries = 0, failed = 0;
  Clock::time_point t_start;
};

namespace {

double us_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::micro>(b - a).count();
}

void finish(hm_server *sv, Req *q, int status) {
  q->status = status;
  const Clock::time_point now = Clock::now();
  q->latency_us = us_between(q->t_submit, now);
  const bool read = q->r.kind == HM_REQ_SEARCH || q->r.kind == HM_REQ_RANGE;
  const bool timed = read && status == HM_OK && q->t_device_done >= q->t_enqueued && q->t_enqueued >= q->t_admit &&
                     q->t_admit >= q->t_submit;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->completed++;
  if (status != HM_OK) sv->failed++;
  sv->queries += q->r.n;
  sv->lat.push_back(q->latency_us);
  if (timed) {
    sv->lat_queue.push_back(us_between(q->t_submit, q->t_admit));
    sv->lat_stage.push_back(us_between(q->t_admit, q->t_enqueued));
    sv->lat_device.push_back(us_between(q->t_enqueued, q->t_device_done));
    sv->lat_finish.push_back(us_between(q->t_device_done, now));
  }
  sv->cv_done.notify_all();
}

// Grows a slot's buffers (only between launches of that slot).  Sizes at
// least double, and hm_server_start pre-sizes every slot for a full launch of
// point queries, so steady serving never allocates.
int slot_reserve(Slot &sl, size_t dev_need, size_t pin_need) {
  if (dev_need > sl.dev_bytes) {
    if (sl.dev) cudaFree(sl.dev);
    sl.dev = nullptr;
    size_t b = (size_t)align_up((int64_t)std::max(dev_need, 2 * sl.dev_bytes), 1 << 20);
    sl.dev_bytes = 0;
    cudaError_t e = cudaMalloc(&sl.dev, b);
    if (e != cudaSuccess) return cuda_err(e);
    sl.dev_bytes = b;
  }
  if (pin_need > sl.pin_bytes) {
    if (sl.pin) cudaFreeHost(sl.pin);
    sl.pin = nullptr;
    size_t b = (size_t)align_up((int64_t)std::max(pin_need, 2 * sl.pin_bytes), 1 << 20);
    sl.pin_bytes = 0;
    cudaError_t e = cudaMallocHost(&sl.pin, b);
    if (e != cudaSuccess) return cuda_err(e);
    sl.pin_bytes = b;
  }
  return HM_OK;
}

// Frees a slot's buffers, events and stream.
void release_slot(Slot &x) {
  if (x.dev) cudaFree(x.dev);
  if (x.pin) cudaFreeHost(x.pin);
  if (x.done) cudaEventDestroy(x.done);
  if (x.kdone) cudaEventDestroy(x.kdone);
  if (x.s) cudaStreamDestroy(x.s);
  x = Slot();
}

// Enqueues a coalesced point search of sl.reqs on the slot's stream.
int launch_points(hm_server *sv, Slot &sl) {
  hm_tree *t = sv->t;
  int64_t n = 0;
  for (Req *q : sl.reqs) n += (int64_t)q->r.n;
  const size_t qb = align_up(n * 8, 256);
  const size_t scr = run_search_scratch(t, n);
  int rc = slot_reserve(sl, 2 * qb + scr + 256, 2 * qb);
  if (rc) return rc;
  int64_t *hq = reinterpret_cast<int64_t *>(sl.pin);
  int64_t *hout = reinterpret_cast<int64_t *>(sl.pin + qb);
  int64_t o = 0;
  std::vector<CopyJob> jobs;
  for (Req *q : sl.reqs) {
    if (!q->direct_in)
      jobs.push_back({reinterpret_cast<char *>(hq + o), reinterpret_cast<const char *>(q->r.keys), q->r.n * 8});
    o += (int64_t)q->r.n;
  }
  sv->copies.run(jobs);
  int64_t *dq = reinterpret_cast<int64_t *>(sl.dev);
  int64_t *dout = reinterpret_cast<int64_t *>(sl.dev + qb);
  // Inputs: staged requests in one copy per consecutive run, the others from
  // their own buffers; results the same way back.
  cudaError_t e = cudaSuccess;
  auto copy_runs = [&](bool in) {
    int64_t at = 0, run0 = -1;
    auto flush = [&](int64_t end) {
      if (run0 >= 0 && e == cudaSuccess)
        e = in ? cudaMemcpyAsync(dq + run0, hq + run0, (end - run0) * 8, cudaMemcpyHostToDevice, sl.s)
               : cudaMemcpyAsync(hout + run0, dout + run0, (end - run0) * 8, cudaMemcpyDeviceToHost, sl.s);
      run0 = -1;
    };
    for (Req *q : sl.reqs) {
      if (in ? q->direct_in : q->direct_out) {
        flush(at);
        if (e == cudaSuccess)
          e = in ? cudaMemcpyAsync(dq + at, q->r.keys, q->r.n * 8, cudaMemcpyDefault, sl.s)
                 : cudaMemcpyAsync(q->r.out, dout + at, q->r.n * 8, cudaMemcpyDefault, sl.s);
      } else if (run0 < 0) {
        run0 = at;
      }
      at += (int64_t)q->r.n;
    }
    flush(at);
  };
  copy_runs(true);
  if (e != cudaSuccess) return cuda_err(e);
  rc = run_search(t, dq, n, dout, sl.s, sl.dev + 2 * qb, scr);
  if (rc) return rc;
  e = cudaEventRecord(sl.kdone, sl.s);
  if (e != cudaSuccess) return cuda_err(e);
  copy_runs(false);
  if (e == cudaSuccess) e = cudaEventRecord(sl.done, sl.s);
  sl.n = n;
  return cuda_err(e);
}

void complete_points(hm_server *sv, Slot &sl) {
  const size_t qb = align_up(sl.n * 8, 256);
  const int64_t *hout = reinterpret_cast<const int64_t *>(sl.pin + qb);
  int64_t o = 0;
  std::vector<CopyJob> jobs;
  for (Req *q : sl.reqs) {
    if (!q->direct_out)
      jobs.push_back({reinterpret_cast<char *>(q->r.out), reinterpret_cast<const char *>(hout + o), q->r.n * 8});
    o += (int64_t)q->r.n;
  }
  sv->copies_out.run(jobs);
  for (Req *q : sl.reqs) finish(sv, q, HM_OK);
}

// Coalesced range requests: locate + scan + copy on the slot's stream, the
// records read back when the launch completes.
int launch_ranges(hm_server *sv, Slot &sl) {
  hm_tree *t = sv->t;
  int64_t n = 0, recs = 0;
  for (Req *q : sl.reqs) {
    n += (int64_t)q->r.n;
    for (size_t i = 0; i < q->r.n; i++) recs += q->r.lens[i] > 0 ? q->r.lens[i] : 0;
  }
  const size_t b8 = align_up((n + 1) * 8, 256), b4 = align_up(n * 4 + 4, 256);
  const size_t rb = align_up(std::max<int64_t>(recs, 1) * 8, 256);
  const size_t need = b8 /*start*/ + b4 /*len*/ + 2 * b4 /*leaf, slot*/ + b8 /*count*/ + b8 /*offsets*/ +
                      2 * rb + align_up((int64_t)scan_scratch_bytes(n + 1), 256);
  int rc = slot_reserve(sl, need, b8 + b4 + b8 + 2 * rb);
  if (rc) return rc;
  char *d = sl.dev;
  int64_t *ds = reinterpret_cast<int64_t *>(d);
  int32_t *dl = reinterpret_cast<int32_t *>(d + b8);
  int32_t *fl = reinterpret_cast<int32_t *>(d + b8 + b4);
  int32_t *fs = reinterpret_cast<int32_t *>(d + b8 + 2 * b4);
  int64_t *cnt = reinterpret_cast<int64_t *>(d + b8 + 3 * b4);
  int64_t *off = reinterpret_cast<int64_t *>(d + 2 * b8 + 3 * b4);
  int64_t *ok = reinterpret_cast<int64_t *>(d + 3 * b8 + 3 * b4);
  int64_t *ov = reinterpret_cast<int64_t *>(d + 3 * b8 + 3 * b4 + rb);
  void *scan = d + 3 * b8 + 3 * b4 + 2 * rb;
  int64_t *hs = reinterpret_cast<int64_t *>(sl.pin);
  int32_t *hl = reinterpret_cast<int32_t *>(sl.pin + b8);
  int64_t o = 0;
  for (Req *q : sl.reqs) {
    std::memcpy(hs + o, q->r.keys, q->r.n * 8);
    std::memcpy(hl + o, q->r.lens, q->r.n * 4);
    o += (int64_t)q->r.n;
  }
  cudaError_t e = cudaMemcpyAsync(ds, hs, n * 8, cudaMemcpyHostToDevice, sl.s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dl, hl, n * 4, cudaMemcpyHostToDevice, sl.s);
  if (e != cudaSuccess) return cuda_err(e);
  rc = range_locate(t, ds, dl, nullptr, n, fl, fs, cnt, sl.s);
  if (rc) return rc;
  exclusive_scan_i64(cnt, off, n, scan, sl.s);
  rc = range_copy_out(t, fl, fs, off, n, ok, ov, sl.s);
  if (rc) return rc;
  e = cudaEventRecord(sl.kdone, sl.s);
  if (e != cudaSuccess) return cuda_err(e);
  char *hoff = sl.pin + b8 + b4;
  e = cudaMemcpyAsync(hoff, off, (n + 1) * 8, cudaMemcpyDeviceToHost, sl.s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hoff + b8, ok, recs * 8, cudaMemcpyDeviceToHost, sl.s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hoff + b8 + rb, ov, recs * 8, cudaMemcpyDeviceToHost, sl.s);
  if (e == cudaSuccess) e = cudaEventRecord(sl.done, sl.s);
  sl.n = n;
  return cuda_err(e);
}

void complete_ranges(hm_server *sv, Slot &sl) {
  int64_t recs = 0;
  for (Req *q : sl.reqs)
    for (size_t i = 0; i < q->r.n; i++) recs += q->r.lens[i] > 0 ? q->r.lens[i] : 0;
  const size_t b8 = align_up((sl.n + 1) * 8, 256), b4 = align_up(sl.n * 4 + 4, 256);
  const size_t rb = align_up(std::max<int64_t>(recs, 1) * 8, 256);
  const int64_t *off = reinterpret_cast<const int64_t *>(sl.pin + b8 + b4);
  const int64_t *hk = reinterpret_cast<const int64_t *>(sl.pin + b8 + b4 + b8);
  const int64_t *hv = reinterpret_cast<const int64_t *>(sl.pin + b8 + b4 + b8 + rb);
  int64_t o = 0;
  for (Req *q : sl.reqs) {
    const int64_t base = off[o], end = off[o + (int64_t)q->r.n];
    for (size_t i = 0; i <= q->r.n; i++) q->r.offsets[i] = off[o + (int64_t)i] - base;
    const int64_t cnt = end - base;
    int st = HM_OK;
    if ((size_t)cnt > q->r.out_cap) {
      st = HM_ECAPACITY;
    } else if (cnt > 0) {
      std::memcpy(q->r.out_keys, hk + base, cnt * 8);
      std::memcpy(q->r.out_vals, hv + base, cnt * 8);
    }
    o += (int64_t)q->r.n;
    finish(sv, q, st);
  }
}

// Watches the launches in flight.  A launch seen finished goes to the
// completer thread (its slot is "completing" until the completer hands it
// back); slots handed back are freed here.  With wait_us > 0, polls until at
// least one launch finished or was handed back, or the time is up.  A launch
// that has not finished within the server's device wait limit is failed with
// HM_ETIMEOUT and its slot retired (its buffers stay allocated: the stream may
// still own them).
bool poll_slots(hm_server *sv, int64_t wait_us) {
  const Clock::time_point t0 = Clock::now();
  for (;;) {
    bool any = false;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      while (!sv->handed_back.empty()) {
        Slot &sl = *sv->handed_back.front();
        sv->handed_back.pop_front();
        sv->reserved -= sl.reserved;
        sl.reserved = 0;
        sl.reqs.clear();
        sl.kind = -1;
        any = true;
      }
    }
    for (auto &sl : sv->slots) {
      if (sl.kind < 0) continue;
      cudaError_t e = cudaEventQuery(sl.done);
      if (e == cudaSuccess) {
        const Clock::time_point now = Clock::now();
        for (Req *q : sl.reqs) q->t_device_done = now;
        sl.launched = sl.kind;
        sl.kind = -3;
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          sv->to_complete.push_back(&sl);
        }
        sv->cv_complete.notify_one();
        any = true;
        continue;
      }
      if (e == cudaErrorNotReady) {
        double waited = std::chrono::duration<double, std::milli>(Clock::now() - sl.t_launch).count();
        if (waited < (double)sv->cfg.device_wait_limit_ms) continue;
        for (Req *q : sl.reqs) finish(sv, q, HM_ETIMEOUT);
        sl.retired = true;
      } else {
        for (Req *q : sl.reqs) finish(sv, q, cuda_err(e));
      }
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->reserved -= sl.reserved;
      }
      sl.reqs.clear();
      sl.kind = sl.retired ? -2 : -1;
      sl.reserved = 0;
      any = true;
    }
    if (any || wait_us <= 0) return any;
    if (std::chrono::duration<double, std::micro>(Clock::now() - t0).count() > wait_us) return false;
    std::this_thread::sleep_for(std::chrono::microseconds(5));
  }
}

// The completer thread: copies finished launches' results to the callers'
// buffers, finishes their requests, hands the slots back to the dispatcher.
void completer(hm_server *sv) {
  for (;;) {
    Slot *sl = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_complete.wait(lk, [sv] { return sv->completer_quit || !sv->to_complete.empty(); });
      if (sv->to_complete.empty()) return;  // quit, nothing left
      sl = sv->to_complete.front();
      sv->to_complete.pop_front();
    }
    if (sl->launched == HM_REQ_SEARCH)
      complete_points(sv, *sl);
    else
      complete_ranges(sv, *sl);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->handed_back.push_back(sl);
    }
    sv->cv_submit.notify_all();  // the dispatcher may be waiting for a free slot
  }
}

// A launch is running on the device, or its results are being copied out.
bool slots_busy(hm_server *sv) {
  for (auto &sl : sv->slots)
    if (sl.kind >= 0 || sl.kind == -3) return true;
  return false;
}

// A launch is running on the device (what a write epoch must wait for).
bool slots_in_flight(hm_server *sv) {
  for (auto &sl : sv->slots)
    if (sl.kind >= 0) return true;
  return false;
}

Slot *free_slot_of(hm_server *sv) {
  for (auto &sl : sv->slots)
    if (sl.kind == -1) return &sl;
  return nullptr;
}

// Applies a run of upserts as one epoch after every earlier request finished.
void run_epoch(hm_server *sv, std::vector<Req *> &ups) {
  const Clock::time_point t0 = Clock::now();
  // Every earlier read's kernels must have ended before the epoch writes the
  // tree; their result copies (device scratch to pinned staging) and the
  // completer's copies out read no tree memory and may overlap the epoch.
  // poll_slots retires a launch still unfinished after the device wait
  // limit, which ends this wait too.
  for (;;) {
    bool reading = false;
    for (auto &x : sv->slots)
      if (x.kind >= 0 && cudaEventQuery(x.kdone) == cudaErrorNotReady) reading = true;
    if (!reading) break;
    poll_slots(sv, 200);
  }
  cudaGetLastError();  // a failed query is the launch's own error, reported by poll_slots
  const Clock::time_point t1 = Clock::now();
  hm_tree *t = sv->t;
  int64_t n = 0;
  for (Req *q : ups) n += (int64_t)q->r.n;
  // A slot retired after a device timeout may still have kernels reading the
  // tree on its stream: no epoch may change the tree (in place, or by a
  // rebuild that frees the old arrays) under them, so writes fail from then on.
  bool retired = false;
  for (auto &x : sv->slots) retired |= x.kind == -2;
  if (retired) {
    for (Req *q : ups) finish(sv, q, HM_ETIMEOUT);
    return;
  }
  Slot &sl = sv->epoch_slot;
  const bool del = ups[0]->r.kind == HM_REQ_DELETE;
  const size_t b = align_up(std::max<int64_t>(n, 1) * 8, 256);
  int rc = slot_reserve(sl, 2 * b, 2 * b);
  if (rc == HM_OK && n > 0) {
    int64_t *hk = reinterpret_cast<int64_t *>(sl.pin);
    int64_t *hv = reinterpret_cast<int64_t *>(sl.pin + b);
    int64_t o = 0;
    std::vector<CopyJob> jobs;
    for (Req *q : ups) {
      jobs.push_back({reinterpret_cast<char *>(hk + o), reinterpret_cast<const char *>(q->r.keys), q->r.n * 8});
      if (!del)
        jobs.push_back({reinterpret_cast<char *>(hv + o), reinterpret_cast<const char *>(q->r.vals), q->r.n * 8});
      o += (int64_t)q->r.n;
    }
    sv->copies.run(jobs);
    int64_t *dk = reinterpret_cast<int64_t *>(sl.dev);
    int64_t *dv = reinterpret_cast<int64_t *>(sl.dev + b);
    cudaError_t e = cudaMemcpyAsync(dk, hk, n * 8, cudaMemcpyHostToDevice, sl.s);
    if (e == cudaSuccess && !del) e = cudaMemcpyAsync(dv, hv, n * 8, cudaMemcpyHostToDevice, sl.s);
    rc = cuda_err(e);
    if (rc == HM_OK)
      rc = del ? delete_epoch(t, dk, n, nullptr, sl.s) : upsert_epoch(t, dk, dv, n, ups[0]->r.flags, sl.s);
    e = cudaStreamSynchronize(sl.s);
    if (rc == HM_OK) rc = cuda_err(e);
    refresh_smem_levels(t);
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->epochs++;
    sv->epoch_drain_us += us_between(t0, t1);
    sv->epoch_apply_us += us_between(t1, Clock::now());
  }
  for (Req *q : ups) finish(sv, q, rc);
}

void dispatcher(hm_server *sv) {
  cudaSetDevice(sv->t->device);
  for (;;) {
    poll_slots(sv, 0);
    std::vector<Req *> take;
    int kind = -1;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      if (sv->queue.empty()) {
        if (sv->stopping && !slots_busy(sv)) break;
        // idle: wake for a submit, or soon to poll in-flight launches
        sv->cv_submit.wait_for(lk, std::chrono::microseconds(slots_busy(sv) ? 20 : 2000));
        continue;
      }
      Req *head = sv->queue.front();
      kind = head->r.kind;
      if (kind == HM_REQ_UPSERT || kind == HM_REQ_DELETE) {
        // one epoch: consecutive writes of the head's kind (upserts of one rule)
        while (!sv->queue.empty() && sv->queue.front()->r.kind == kind) {
          Req *q = sv->queue.front();
          if (kind == HM_REQ_UPSERT && !take.empty() &&
              (q->r.flags != HM_UPSERT_SUPPLIED || take[0]->r.flags != HM_UPSERT_SUPPLIED))
            break;
          take.push_back(q);
          sv->queue.pop_front();
        }
      } else {
        // one launch: consecutive requests of the head's kind within the budget
        Slot *free_slot = free_slot_of(sv);
        if (!free_slot) {
          if (!slots_busy(sv)) {  // every slot retired: fail what is queued
            std::vector<Req *> dead(sv->queue.begin(), sv->queue.end());
            sv->queue.clear();
            lk.unlock();
            for (Req *q : dead) finish(sv, q, HM_ETIMEOUT);
            continue;
          }
          lk.unlock();
          poll_slots(sv, 50);
          continue;
        }
        size_t bytes = 0;
        int64_t nq = 0;
        while (!sv->queue.empty()) {
          Req *q = sv->queue.front();
          if (q->r.kind != kind) break;
          if (!take.empty() && (nq + (int64_t)q->r.n > sv->cfg.max_launch_queries ||
                                sv->reserved + bytes + q->bytes > sv->cfg.device_budget_bytes))
            break;
          if (take.empty() && sv->reserved + q->bytes > sv->cfg.device_budget_bytes) break;
          take.push_back(q);
          bytes += q->bytes;
          nq += (int64_t)q->r.n;
          sv->queue.pop_front();
        }
        if (take.empty()) {  // wait for memory to free up
          lk.unlock();
          poll_slots(sv, 1000);
          continue;
        }
        sv->reserved += bytes;
        free_slot->reserved = bytes;
        free_slot->kind = kind;
        free_slot->reqs = take;
        const Clock::time_point now = Clock::now();
        for (Req *q : take) q->t_admit = now;
      }
    }
    if (kind == HM_REQ_UPSERT || kind == HM_REQ_DELETE) {
      run_epoch(sv, take);
      continue;
    }
    Slot *sl = nullptr;
    for (auto &x : sv->slots)
      if (x.kind >= 0 && !x.reqs.empty() && x.reqs[0] == take[0]) sl = &x;
    sl->t_launch = Clock::now();
    int rc = kind == HM_REQ_SEARCH ? launch_points(sv, *sl) : launch_ranges(sv, *sl);
    const Clock::time_point enq = Clock::now();
    for (Req *q : sl->reqs) q->t_enqueued = enq;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->launches++;
    }
    if (rc) {
      // nothing of this launch completes normally: wait for what it may have
      // enqueued, then fail its requests (bounded like every device wait)
      const Clock::time_point t0 = Clock::now();
      while (cudaStreamQuery(sl->s) == cudaErrorNotReady &&
             std::chrono::duration<double, std::milli>(Clock::now() - t0).count() <
                 (double)sv->cfg.device_wait_limit_ms)
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      std::vector<Req *> failed;
      failed.swap(sl->reqs);
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->reserved -= sl->reserved;
        sl->kind = -1;
        sl->reserved = 0;
      }
      for (Req *q : failed) finish(sv, q, rc);
    }
  }
}

int check_request(const hm_request *r) {
  if (!r) return HM_EINVAL;
  switch (r->kind) {
    case HM_REQ_SEARCH:
      if (r->n > 0 && (!r->keys || !r->out)) return HM_EINVAL;
      return HM_OK;
    case HM_REQ_RANGE:
      if (!r->offsets || (r->n > 0 && (!r->keys || !r->lens))) return HM_EINVAL;
      if (r->out_cap > 0 && (!r->out_keys || !r->out_vals)) return HM_EINVAL;
      return HM_OK;
    case HM_REQ_UPSERT:
      if (r->n > 0 && (!r->keys || !r->vals)) return HM_EINVAL;
      if (r->flags != HM_UPSERT_SUPPLIED && r->flags != HM_UPSERT_REF_KEY_MINUS_1) return HM_EINVAL;
      return HM_OK;
    case HM_REQ_DELETE:
      if (r->n > 0 && !r->keys) return HM_EINVAL;
      return HM_OK;
    default:
      return HM_EINVAL;
  }
}

}  // namespace

extern "C" {

int hm_server_config_default(hm_server_config *c) {
  if (!c) return HM_EINVAL;
  std::memset(c, 0, sizeof(*c));
  c->device_budget_bytes = (size_t)1 << 30;
  c->max_queue = 1 << 16;
  c->streams = 3;
  c->max_launch_queries = (int64_t)1 << 22;
  c->device_wait_limit_ms = 30000;
  return HM_OK;
}

int hm_server_start(hm_tree *t, const hm_server_config *cfg, hm_server **out) {
  if (!t || !out) return HM_EINVAL;
  *out = nullptr;
  hm_server *sv = new (std::nothrow) hm_server();
  if (!sv) return HM_ENOMEM;
  hm_server_config_default(&sv->cfg);
  if (cfg) {
    if (cfg->device_budget_bytes) sv->cfg.device_budget_bytes = cfg->device_budget_bytes;
    if (cfg->max_queue) sv->cfg.max_queue = cfg->max_queue;
    if (cfg->streams) sv->cfg.streams = cfg->streams;
    if (cfg->max_launch_queries) sv->cfg.max_launch_queries = cfg->max_launch_queries;
    if (cfg->device_wait_limit_ms) sv->cfg.device_wait_limit_ms = cfg->device_wait_limit_ms;
  }
  if (sv->cfg.streams < 1 || sv->cfg.streams > 16 || sv->cfg.max_queue < 1 || sv->cfg.max_launch_queries < 1) {
    delete sv;
    return HM_EINVAL;
  }
  sv->t = t;
  sv->slots.resize(sv->cfg.streams);
  cudaSetDevice(t->device);
  for (auto &sl : sv->slots) {
    cudaError_t e = cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.kdone, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      for (auto &x : sv->slots) release_slot(x);
      delete sv;
      return cuda_err(e);
    }
  }
  // pre-size every slot for one full launch of point queries
  {
    const int64_t n = sv->cfg.max_launch_queries;
    const size_t qb = align_up(n * 8, 256);
    const size_t dev = 2 * qb + run_search_scratch(t, n) + 256;
    for (auto &sl : sv->slots) {
      int rc = slot_reserve(sl, dev, 2 * qb);
      if (rc) {
        for (auto &x : sv->slots) release_slot(x);
        delete sv;
        return rc;
      }
    }
  }
  {
    Slot &es = sv->epoch_slot;
    cudaError_t e = cudaStreamCreateWithFlags(&es.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&es.done, cudaEventDisableTiming);
    if (e == cudaSuccess && slot_reserve(es, 2 << 20, 2 << 20) != HM_OK) e = cudaErrorMemoryAllocation;
    if (e != cudaSuccess) {
      release_slot(es);
      for (auto &x : sv->slots) release_slot(x);
      delete sv;
      return cuda_err(e);
    }
  }
  sv->t_start = Clock::now();
  const unsigned hw = std::thread::hardware_concurrency();
  sv->copies.start((int)std::min(8u, std::max(1u, hw / 4)));
  sv->copies_out.start((int)std::min(8u, std::max(1u, hw / 4)));
  sv->completer = std::thread(completer, sv);
  sv->th = std::thread(dispatcher, sv);
  *out = sv;
  return HM_OK;
}

int hm_server_submit(hm_server *sv, const hm_request *r, uint64_t *ticket) {
  if (!sv || !ticket) return HM_EINVAL;
  int rc = check_request(r);
  if (rc) return rc;
  Req *q = new (std::nothrow) Req();
  if (!q) return HM_ENOMEM;
  q->r = *r;
  q->bytes = req_device_bytes(*r);
  if (r->kind == HM_REQ_SEARCH && r->n > 0) {
    q->direct_in = dma_reachable(r->keys);
    q->direct_out = dma_reachable(r->out);
  }
  q->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->stopping) {
    delete q;
    return HM_ECANCELLED;
  }
  if ((int)sv->queue.size() >= sv->cfg.max_queue || q->bytes > sv->cfg.device_budget_bytes) {
    sv->rejected++;
    delete q;
    return HM_EBUSY;
  }
  q->ticket = sv->next_ticket++;
  sv->queue.push_back(q);
  sv->reqs[q->ticket] = q;
  *ticket = q->ticket;
  sv->cv_submit.notify_one();
  return HM_OK;
}

int hm_server_wait(hm_server *sv, uint64_t ticket, int64_t timeout_us, int *status) {
  if (!sv) return HM_EINVAL;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) return HM_EINVAL;
  Req *q = it->second;
  auto pred = [&] { return q->status != 1; };
  if (timeout_us < 0) {
    sv->cv_done.wait(lk, pred);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), pred)) {
    return HM_ETIMEOUT;
  }
  if (status) *status = q->status;
  sv->reqs.erase(it);
  delete q;
  return HM_OK;
}

int hm_server_get_stats(hm_server *sv, hm_server_stats *st) {
  if (!sv || !st) return HM_EINVAL;
  std::lock_guard<std::mutex> lk(sv->mu);
  std::memset(st, 0, sizeof(*st));
  st->completed = sv->completed;
  st->failed = sv->failed;
  st->rejected = sv->rejected;
  st->launches = sv->launches;
  st->epochs = sv->epochs;
  st->queries = sv->queries;
  st->pending = sv->queue.size();
  st->elapsed_s = std::chrono::duration<double>(Clock::now() - sv->t_start).count();
  auto pct = [](std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    size_t k = (size_t)(p * (v.size() - 1) + 0.5);
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
  };
  if (!sv->lat.empty()) {
    st->p50_us = pct(sv->lat, 0.50);
    st->p99_us = pct(sv->lat, 0.99);
    st->max_us = *std::max_element(sv->lat.begin(), sv->lat.end());
    double s = 0;
    for (double x : sv->lat) s += x;
    st->mean_us = s / sv->lat.size();
  }
  st->queue_p50_us = pct(sv->lat_queue, 0.50);
  st->queue_p99_us = pct(sv->lat_queue, 0.99);
  st->stage_p50_us = pct(sv->lat_stage, 0.50);
  st->stage_p99_us = pct(sv->lat_stage, 0.99);
  st->device_p50_us = pct(sv->lat_device, 0.50);
  st->device_p99_us = pct(sv->lat_device, 0.99);
  st->finish_p50_us = pct(sv->lat_finish, 0.50);
  st->finish_p99_us = pct(sv->lat_finish, 0.99);
  if (sv->epochs) {
    st->epoch_drain_mean_us = sv->epoch_drain_us / (double)sv->epochs;
    st->epoch_apply_mean_us = sv->epoch_apply_us / (double)sv->epochs;
  }
  return HM_OK;
}

int hm_server_reset_stats(hm_server *sv) {
  if (!sv) return HM_EINVAL;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->lat.clear();
  sv->lat_queue.clear();
  sv->lat_stage.clear();
  sv->lat_device.clear();
  sv->lat_finish.clear();
  sv->epoch_drain_us = sv->epoch_apply_us = 0;
  sv->completed = sv->failed = sv->rejected = sv->launches = sv->epochs = sv->queries = 0;
  sv->t_start = Clock::now();
  return HM_OK;
}

int hm_server_stop(hm_server *sv) {
  if (!sv) return HM_EINVAL;
  std::vector<Req *> cancelled;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stopping && !sv->th.joinable()) return HM_OK;
    sv->stopping = true;
    while (!sv->queue.empty()) {
      cancelled.push_back(sv->queue.front());
      sv->queue.pop_front();
    }
    sv->cv_submit.notify_all();
  }
  for (Req *q : cancelled) finish(sv, q, HM_ECANCELLED);
  if (sv->th.joinable()) sv->th.join();  // returns once every launch is completed
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->completer_quit = true;
  }
  sv->cv_complete.notify_all();
  if (sv->completer.joinable()) sv->completer.join();
  sv->copies.stop();
  sv->copies_out.stop();
  return HM_OK;
}

int hm_server_free(hm_server *sv) {
  if (!sv) return HM_OK;
  hm_server_stop(sv);
  for (auto &sl : sv->slots)
    if (!sl.retired) release_slot(sl);  // a retired slot's stream may still own its buffers
  release_slot(sv->epoch_slot);
  for (auto &kv : sv->reqs) delete kv.second;
  delete sv;
  return HM_OK;
}

}  // extern "C"
