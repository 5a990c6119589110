// tk_serve.cpp -- continuous-batching server for ML-KEM matrix-vector requests.
//
// A request is njobs matrix-vector jobs of one k (tk_matvec semantics) in host
// memory.  The server owns one device-memory pool of hbm_budget bytes; a
// request is admitted (FIFO) once its A, s, e and out fit in the pool, a
// request slot is free and the device job ring has room.  Admission copies the
// inputs into the pool, writes one descriptor per job into the device-resident
// ring and advances the ring's tail, all on one copy stream.  A persistent
// kernel (k_serve, tk_matvec.cu) claims published jobs as they appear: jobs of
// requests that arrive while others are on the GPU join the running loop, and
// run side by side with them.  When the last job of a request finishes, the
// kernel writes the request's generation into a flag in mapped host memory;
// the scheduler then copies the outputs back, frees the pool block and
// completes the ticket.  The device loop exits on its own after idle_exit
// seconds without work and is relaunched when work arrives.  No reference
// counterpart: the reference only times fixed batches (ntt_bench.cu:600-903).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/tk_ntt.h"
#include "tk_internal.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr uint32_t kRingCap = 1u << 16;  // job descriptors in the device ring
constexpr size_t kAlign = 256;

size_t align_up(size_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

struct Request {
  uint64_t ticket = 0;
  int k = 0;
  size_t njobs = 0;
  const int16_t *A = nullptr, *s = nullptr, *e = nullptr;
  int16_t* out = nullptr;
  size_t bytes = 0, off = 0;  // pool block
  uint32_t slot = 0, gen = 0;
  unsigned long long first = 0;  // ring index of the request's first job
  std::atomic<int> state{0};     // 0 pending, 1 published, 2 copying back, 3 done
  int status = TK_SUCCESS;
  cudaEvent_t back = nullptr;
  Clock::time_point t_submit, t_done;
};

// First-fit allocator over [0, size).
class Pool {
 public:
  void init(size_t n) {
    free_.clear();
    free_[0] = n;
  }
  bool alloc(size_t n, size_t* off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, o = it->first;
      free_.erase(it);
      if (rest) free_[o + n] = rest;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
};

}  // namespace

struct tk_server {
  int device = 0;
  tk::DeviceInfo* info = nullptr;
  size_t budget = 0;
  uint8_t* pool = nullptr;
  Pool alloc;
  tk::ServeJob* ring_dev = nullptr;
  tk::ServeJob* ring_host = nullptr;  // pinned staging
  tk::ServeCtl* ctl = nullptr;
  unsigned int* req_ctr = nullptr;    // device
  unsigned int* req_flag = nullptr;   // mapped pinned host memory
  uint32_t nslots = 0;
  std::vector<uint32_t> free_slots, slot_gen;
  cudaStream_t h2d = nullptr, d2h = nullptr, comp = nullptr;
  cudaEvent_t kernel_done = nullptr;
  bool kernel_running = false;
  unsigned long long published = 0, completed_jobs = 0;  // jobs, full width on the host
  unsigned long long idle_ns = 0;
  uint64_t launches = 0;

  std::mutex mu;
  std::condition_variable cv;        // request completions (waiters)
  std::condition_variable cv_sched;  // new requests / quit (scheduler)
  std::deque<Request*> pending;
  std::map<uint64_t, std::unique_ptr<Request>> all;
  std::vector<Request*> active;  // published or copying back
  uint64_t next_ticket = 1;
  std::atomic<bool> quit{false}, abort{false};
  int fatal = TK_SUCCESS;
  std::thread th;
};

namespace {

void fail_all(tk_server* S, int status) {
  std::lock_guard<std::mutex> lk(S->mu);
  S->fatal = status;
  for (auto& kv : S->all)
    if (kv.second->state != 3) {
      kv.second->state = 3;
      kv.second->status = status;
      kv.second->t_done = Clock::now();
    }
  S->pending.clear();
  S->active.clear();
  S->cv.notify_all();
}

// Writes a 32-bit word with a copy-engine memset: no source buffer to keep
// alive and no SM needed (the persistent kernel may hold all of them).
PFN_cuMemsetD32Async_v3020 memset32_fn() {
  static PFN_cuMemsetD32Async_v3020 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemsetD32Async", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuMemsetD32Async_v3020)p;
  });
  return fn;
}

cudaError_t set_u32(unsigned int* dst, unsigned int v, cudaStream_t st) {
  PFN_cuMemsetD32Async_v3020 f = memset32_fn();
  if (!f) return cudaErrorNotSupported;
  return f((CUdeviceptr)dst, v, 1, (CUstream)st) == CUDA_SUCCESS ? cudaSuccess
                                                                 : cudaErrorLaunchFailure;
}

cudaError_t admit(tk_server* S, Request* r) {
  if (!r->back) {
    const cudaError_t ev = cudaEventCreateWithFlags(&r->back, cudaEventDisableTiming);
    if (ev != cudaSuccess) return ev;
  }
  r->first = S->published;
  const size_t k = (size_t)r->k, vb = r->njobs * k * 512, ab = vb * k;
  uint8_t* base = S->pool + r->off;
  int16_t* A = (int16_t*)base;
  int16_t* sv = (int16_t*)(base + align_up(ab));
  int16_t* ev = r->e ? (int16_t*)(base + align_up(ab) + align_up(vb)) : nullptr;
  int16_t* out = (int16_t*)(base + align_up(ab) + align_up(vb) * (r->e ? 2 : 1));
  cudaError_t e = cudaMemcpyAsync(A, r->A, ab, cudaMemcpyHostToDevice, S->h2d);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sv, r->s, vb, cudaMemcpyHostToDevice, S->h2d);
  if (e == cudaSuccess && ev) e = cudaMemcpyAsync(ev, r->e, vb, cudaMemcpyHostToDevice, S->h2d);
  if (e != cudaSuccess) return e;
  // descriptors into the pinned staging copy of the ring (the slot's job
  // counter is zero: the device resets it when the slot's last request ends)
  for (size_t j = 0; j < r->njobs; j++) {
    tk::ServeJob& J = S->ring_host[(S->published + j) & (kRingCap - 1)];
    J.A = A + j * k * k * 256;
    J.s = sv + j * k * 256;
    J.e = ev ? ev + j * k * 256 : nullptr;
    J.out = out + j * k * 256;
    J.k = (uint32_t)r->k;
    J.req = r->slot;
    J.njobs = (uint32_t)r->njobs;
    J.gen = r->gen;
  }
  S->published += r->njobs;
  return cudaSuccess;
}

// Publishes ring entries [from, S->published): one copy per contiguous run
// (at most two), then the new tail, behind the input copies on the same stream.
cudaError_t publish(tk_server* S, unsigned long long from) {
  cudaError_t e = cudaSuccess;
  unsigned long long t = from;
  while (t < S->published && e == cudaSuccess) {
    const uint32_t pos = (uint32_t)(t & (kRingCap - 1));
    unsigned long long run = S->published - t;
    if (run > kRingCap - pos) run = kRingCap - pos;
    e = cudaMemcpyAsync(S->ring_dev + pos, S->ring_host + pos, run * sizeof(tk::ServeJob),
                        cudaMemcpyHostToDevice, S->h2d);
    t += run;
  }
  if (e != cudaSuccess) return e;
  return set_u32(&S->ctl->tail, (unsigned int)S->published, S->h2d);
}

cudaError_t ensure_kernel(tk_server* S) {
  if (S->kernel_running) return cudaSuccess;
  // the loop must see the published tail: order the launch after the copies
  cudaError_t e = cudaEventRecord(S->kernel_done, S->h2d);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(S->comp, S->kernel_done, 0);
  if (e == cudaSuccess)
    e = tk::launch_serve(S->ring_dev, kRingCap - 1, S->ctl, S->req_ctr, S->req_flag, S->idle_ns,
                         *S->info, S->comp);
  if (e == cudaSuccess) e = cudaEventRecord(S->kernel_done, S->comp);
  if (e == cudaSuccess) {
    S->kernel_running = true;
    S->launches++;
  }
  return e;
}

void scheduler(tk_server* S) {
  cudaSetDevice(S->device);
  while (true) {
    if (S->abort.load()) {
      fail_all(S, TK_ERR_TIMEOUT);
      return;
    }
    bool progress = false;
    cudaError_t err = cudaSuccess;
    // 1. admission (FIFO): pool room, a request slot, ring room; the jobs of
    // every request admitted in this pass are published together
    const unsigned long long pub0 = S->published;
    while (err == cudaSuccess) {
      Request* r = nullptr;
      // A ring entry may be overwritten only once its job has been claimed
      // and read; every job before the oldest unfinished request's first one
      // has been (the device claims in ring order and a request finishes only
      // after all of its jobs ran).
      const unsigned long long oldest = S->active.empty() ? S->published : S->active.front()->first;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->pending.empty() || S->free_slots.empty()) break;
        Request* h = S->pending.front();
        if (S->published + h->njobs - oldest > kRingCap) break;
        if (!S->alloc.alloc(h->bytes, &h->off)) break;
        S->pending.pop_front();
        h->slot = S->free_slots.back();
        S->free_slots.pop_back();
        h->gen = ++S->slot_gen[h->slot];
        r = h;
      }
      err = admit(S, r);
      r->state = 1;
      S->active.push_back(r);
      progress = true;
    }
    if (err == cudaSuccess && S->published != pub0) {
      err = publish(S, pub0);
      if (err == cudaSuccess) err = ensure_kernel(S);
    }
    // 2. completions: flag seen -> copy back; copy done -> release.  A
    // request is dropped from `active` in the same step that completes it: the
    // caller may free it (tk_server_release) as soon as the lock is released.
    std::vector<Request*> still;
    still.reserve(S->active.size());
    for (Request* r : S->active) {
      if (err != cudaSuccess) break;
      bool finished = false;
      if (r->state == 1) {
        const unsigned int f = __atomic_load_n(&S->req_flag[r->slot], __ATOMIC_ACQUIRE);
        if (f == r->gen) {
          const size_t k = (size_t)r->k, vb = r->njobs * k * 512, ab = vb * k;
          const uint8_t* out =
              S->pool + r->off + align_up(ab) + align_up(vb) * (r->e ? 2 : 1);
          err = cudaMemcpyAsync(r->out, out, vb, cudaMemcpyDeviceToHost, S->d2h);
          if (err == cudaSuccess) err = cudaEventRecord(r->back, S->d2h);
          r->state = 2;
          progress = true;
        }
      } else if (r->state == 2) {
        const cudaError_t q = cudaEventQuery(r->back);
        if (q == cudaSuccess) {
          std::lock_guard<std::mutex> lk(S->mu);
          S->alloc.release(r->off, r->bytes);
          S->free_slots.push_back(r->slot);
          S->completed_jobs += r->njobs;
          r->t_done = Clock::now();
          r->state = 3;
          S->cv.notify_all();
          progress = true;
          finished = true;
        } else if (q != cudaErrorNotReady) {
          err = q;
        }
      }
      if (!finished) still.push_back(r);
    }
    if (err != cudaSuccess) {
      fail_all(S, TK_ERR_CUDA);
      return;
    }
    S->active.swap(still);
    // 3. device loop liveness: relaunch if it went idle with work outstanding
    if (S->kernel_running) {
      const cudaError_t q = cudaEventQuery(S->kernel_done);
      if (q == cudaSuccess) {
        S->kernel_running = false;
      } else if (q != cudaErrorNotReady) {
        fail_all(S, TK_ERR_CUDA);
        return;
      }
    }
    bool waiting_for_device = false;
    for (Request* r : S->active)
      if (r->state == 1) waiting_for_device = true;
    if (waiting_for_device && !S->kernel_running) {
      if (ensure_kernel(S) != cudaSuccess) {
        fail_all(S, TK_ERR_CUDA);
        return;
      }
    }
    bool idle;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      idle = S->pending.empty() && S->active.empty();
    }
    if (idle && S->quit.load()) break;
    if (progress) continue;
    if (idle) {  // nothing admitted or pending: sleep until a submit (or 1 ms)
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_sched.wait_for(lk, std::chrono::milliseconds(1),
                           [&] { return !S->pending.empty() || S->quit.load(); });
    } else {     // work on the device: poll its completion flags
      std::this_thread::yield();
    }
  }
}

void destroy_resources(tk_server* S) {
  if (S->comp) cudaStreamSynchronize(S->comp);
  if (S->kernel_done) cudaEventDestroy(S->kernel_done);
  for (auto& kv : S->all)
    if (kv.second->back) cudaEventDestroy(kv.second->back);
  if (S->h2d) cudaStreamDestroy(S->h2d);
  if (S->d2h) cudaStreamDestroy(S->d2h);
  if (S->comp) cudaStreamDestroy(S->comp);
  if (S->pool) cudaFree(S->pool);
  if (S->ring_dev) cudaFree(S->ring_dev);
  if (S->ctl) cudaFree(S->ctl);
  if (S->req_ctr) cudaFree(S->req_ctr);
  if (S->ring_host) cudaFreeHost(S->ring_host);
  if (S->req_flag) cudaFreeHost(S->req_flag);
}

}  // namespace

extern "C" {

int tk_server_create(int device, const tk_server_config* cfg, tk_server** out) {
  if (!out) return TK_ERR_INVALID_VALUE;
  *out = nullptr;
  const size_t budget = cfg && cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : ((size_t)1 << 30);
  const int slots = cfg && cfg->max_inflight_requests > 0 ? cfg->max_inflight_requests : 1024;
  const double idle = cfg && cfg->idle_exit_seconds > 0 ? cfg->idle_exit_seconds : 0.02;
  if (slots > (1 << 20) || budget < 4096 || idle > 10.0) return TK_ERR_INVALID_VALUE;
  int rc = tk_init(device);
  if (rc) return rc;
  std::unique_ptr<tk_server> S(new tk_server);
  S->device = device;
  S->budget = budget;
  S->nslots = (uint32_t)slots;
  S->idle_ns = (unsigned long long)(idle * 1e9);
  if ((rc = tk::api_device_info(device, &S->info))) return rc;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaError_t e = cudaMalloc(&S->pool, budget);
  if (e == cudaSuccess) e = cudaMalloc(&S->ring_dev, kRingCap * sizeof(tk::ServeJob));
  if (e == cudaSuccess) e = cudaMalloc(&S->ctl, sizeof(tk::ServeCtl));
  if (e == cudaSuccess) e = cudaMemset(S->ctl, 0, sizeof(tk::ServeCtl));
  if (e == cudaSuccess) e = cudaMalloc(&S->req_ctr, slots * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(S->req_ctr, 0, slots * sizeof(unsigned int));
  if (e == cudaSuccess)
    e = cudaHostAlloc(&S->ring_host, kRingCap * sizeof(tk::ServeJob), cudaHostAllocDefault);
  if (e == cudaSuccess)
    e = cudaHostAlloc(&S->req_flag, slots * sizeof(unsigned int), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->kernel_done, cudaEventDisableTiming);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    destroy_resources(S.get());
    return e == cudaErrorMemoryAllocation ? TK_ERR_TOO_LARGE : TK_ERR_CUDA;
  }
  memset(S->req_flag, 0, slots * sizeof(unsigned int));
  S->alloc.init(budget);
  S->slot_gen.assign(slots, 0);
  for (int i = slots - 1; i >= 0; i--) S->free_slots.push_back((uint32_t)i);
  tk_server* raw = S.release();
  raw->th = std::thread(scheduler, raw);
  *out = raw;
  return TK_SUCCESS;
}

int tk_server_submit(tk_server* S, int k, size_t njobs, const int16_t* A, const int16_t* s,
                     const int16_t* e, int16_t* out, uint64_t* ticket) {
  if (!S || !ticket || !A || !s || !out || njobs == 0 || k < 2 || k > 4)
    return TK_ERR_INVALID_VALUE;
  const size_t vb = njobs * (size_t)k * 512, ab = vb * (size_t)k;
  const size_t bytes = align_up(ab) + align_up(vb) * (e ? 3 : 2);
  if (bytes > S->budget || njobs > kRingCap) return TK_ERR_TOO_LARGE;
  std::unique_ptr<Request> r(new Request);
  r->k = k;
  r->njobs = njobs;
  r->A = A;
  r->s = s;
  r->e = e;
  r->out = out;
  r->bytes = bytes;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return S->fatal;
  r->ticket = S->next_ticket++;
  *ticket = r->ticket;
  S->pending.push_back(r.get());
  S->all.emplace(r->ticket, std::move(r));
  S->cv_sched.notify_one();
  return TK_SUCCESS;
}

int tk_server_wait(tk_server* S, uint64_t ticket, double timeout_s) {
  if (!S) return TK_ERR_INVALID_VALUE;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return TK_ERR_INVALID_VALUE;
  Request* r = it->second.get();
  const auto until = Clock::now() + std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s);
  while (r->state != 3)
    if (S->cv.wait_until(lk, until) == std::cv_status::timeout && r->state != 3)
      return TK_ERR_TIMEOUT;
  return r->status;
}

int tk_server_query(tk_server* S, uint64_t ticket, int* done, double* latency_s) {
  if (!S || !done) return TK_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return TK_ERR_INVALID_VALUE;
  Request* r = it->second.get();
  *done = r->state == 3;
  if (latency_s)
    *latency_s = *done ? std::chrono::duration<double>(r->t_done - r->t_submit).count() : -1.0;
  return r->state == 3 ? r->status : TK_SUCCESS;
}

int tk_server_release(tk_server* S, uint64_t ticket) {
  if (!S) return TK_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end() || it->second->state != 3) return TK_ERR_INVALID_VALUE;
  if (it->second->back) cudaEventDestroy(it->second->back);
  S->all.erase(it);
  return TK_SUCCESS;
}

int tk_server_stats(tk_server* S, unsigned long long* jobs_done, unsigned long long* launches) {
  if (!S) return TK_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(S->mu);
  if (jobs_done) *jobs_done = S->completed_jobs;
  if (launches) *launches = S->launches;
  return S->fatal;
}

int tk_server_destroy(tk_server* S, double timeout_s) {
  if (!S) return TK_ERR_INVALID_VALUE;
  int rc = TK_SUCCESS;
  {  // let admitted and pending work finish, bounded
    std::unique_lock<std::mutex> lk(S->mu);
    const auto until = Clock::now() + std::chrono::duration<double>(timeout_s);
    auto busy = [&] {
      for (auto& kv : S->all)
        if (kv.second->state != 3) return true;
      return false;
    };
    while (busy())
      if (S->cv.wait_until(lk, until) == std::cv_status::timeout) {
        rc = TK_ERR_TIMEOUT;
        break;
      }
  }
  S->quit.store(true);
  if (rc == TK_ERR_TIMEOUT) S->abort.store(true);  // the scheduler fails what is left
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->cv_sched.notify_all();
  }
  S->th.join();
  cudaSetDevice(S->device);
  cudaStreamSynchronize(S->d2h);  // no copy into a caller's buffer after this returns
  // end the device loop (it also ends by itself after idle_exit seconds)
  unsigned int one = 1;
  cudaMemcpyAsync(&S->ctl->stop, &one, 4, cudaMemcpyHostToDevice, S->h2d);
  cudaStreamSynchronize(S->h2d);
  destroy_resources(S);
  delete S;
  return rc;
}

}  // extern "C"
