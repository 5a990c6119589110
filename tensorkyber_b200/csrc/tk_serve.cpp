// tk_serve.cpp -- continuous-batching server for ML-KEM matrix-vector requests.
//
// A request is njobs matrix-vector jobs of one k (tk_matvec semantics) in host
// memory.  Requests are admitted in arrival order.  A staged request needs a
// block of the server's device pool (hbm_budget bytes) for its A, s, e and
// out: admission copies the inputs in (one copy when the caller's A, s and e
// are contiguous; one copy for several requests admitted in the same pass
// when their inputs also lie back to back in one page-locked allocation and
// their pool blocks are consecutive, which next-fit allocation makes the
// usual case) and, after the jobs ran, the outputs are copied back.  When out
// is device-mapped page-locked host memory the device loop writes the outputs
// there itself (posted PCIe writes; no pool block for out, no copy back).
// With zero_copy, inputs in such memory are read in place too (no pool memory
// at all; uncached PCIe reads, slower than one bulk copy).  Admission writes
// one descriptor per job into the job ring, which lives in mapped page-locked
// host memory (the device reads a descriptor once, when it claims the job),
// and every admission pass then publishes its jobs with one stream write of
// the new tail, behind the input copies on the same stream.  A persistent
// kernel (k_serve, tk_matvec.cu) claims published jobs as they appear: jobs of
// requests that arrive while others are on the GPU join the running loop and
// run side by side with them.  When the last job of a request finishes, the
// kernel writes the request's generation into a flag in mapped host memory;
// the scheduler thread then completes the ticket (outputs in place) or copies
// the outputs back first (a stream write after the copy raises a second
// flag).  Per request that is up to three copy-engine operations in and one
// out, the cost that bounds the request rate (each is a few microseconds
// however small).  The device loop exits on its own after idle_exit seconds
// without work and is relaunched when work arrives.  No reference
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
#include <unordered_set>
#include <vector>

#include "../../include/tk_ntt.h"
#include "tk_internal.h"
#include "tk_pool.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr uint32_t kRingCap = 1u << 16;  // job descriptors in the device ring
constexpr size_t kAlign = 256;
// After its last piece of work the scheduler keeps polling this long before it
// sleeps on the submit condition: a request that arrives meanwhile is seen at
// once instead of after a thread wake-up.
constexpr auto kSpinAfterWork = std::chrono::microseconds(2000);
// Requests admitted and not yet finished, at most: bounds the work queued on
// the copy streams, so completions are never stuck behind a deep queue of
// input copies (further requests wait, in order, on the host).
constexpr size_t kMaxActive = 64;
// input-copy streams (the copy engine's fixed cost per operation overlaps
// across streams)
constexpr int kCopyStreams = 3;
// Under load, admission waits until this many slots under kMaxActive are free
// and then admits them in one pass, published with a single stream write:
// otherwise every freed slot would cost its own pass (copy + publish) on the
// serial copy stream.  Below this many active requests admission is immediate.
constexpr size_t kAdmitBatch = 32;
// Minimum spacing of device-loop liveness checks (an event query costs ~1 us).
constexpr auto kLivenessPeriod = std::chrono::microseconds(20);

size_t align_up(size_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

struct Request {
  uint64_t ticket = 0;
  int k = 0;
  size_t njobs = 0;
  const int16_t *A = nullptr, *s = nullptr, *e = nullptr;
  int16_t* out = nullptr;
  bool in_direct = false;   // inputs read in place (zero_copy)
  bool out_direct = false;  // outputs written in place (out is mapped pinned memory)
  bool packed = false;      // staged inputs: A, s, e go in one copy
  // packed inputs in page-locked memory: the start of that allocation (host
  // address), so that inputs of requests admitted together that lie back to
  // back in it (and in the pool) go in one copy; 0 otherwise
  uintptr_t locked_lo = 0;
  // device addresses of the caller's buffers (in place) or of the pool copies
  const int16_t *dA = nullptr, *ds = nullptr, *de = nullptr;
  int16_t* dout = nullptr;
  size_t bytes = 0, off = 0;     // pool block (staged requests)
  uint32_t slot = 0, gen = 0;
  unsigned long long first = 0;  // ring index of the request's first job
  std::atomic<int> state{0};     // 0 pending, 1 published, 2 copying back, 3 done
  int status = TK_SUCCESS;
  Clock::time_point t_submit, t_admit, t_flag, t_done;
};

}  // namespace

struct tk_server {
  int device = 0;
  tk::DeviceInfo* info = nullptr;
  size_t budget = 0;
  bool zero_copy = false;
  uint8_t* pool = nullptr;
  tk::Pool alloc;
  // end of the last pool block handed out: the next request's block is taken
  // from there (next fit), so consecutive requests get consecutive blocks and
  // their inputs can share a copy
  size_t alloc_end = 0;
  tk::ServeJob* ring = nullptr;       // job ring, mapped pinned host memory
  tk::ServeCtl* ctl = nullptr;
  unsigned int* req_ctr = nullptr;    // device
  unsigned int* req_flag = nullptr;   // mapped pinned host memory: jobs done
  unsigned int* ret_flag = nullptr;   // mapped pinned host memory: outputs back
  uint32_t nslots = 0;
  std::vector<uint32_t> free_slots, slot_gen;
  cudaStream_t h2d = nullptr, d2h = nullptr, comp = nullptr;
  // more input-copy streams: a pass's copies are dealt over h2d and these
  // (the fixed cost of each copy operation overlaps), and the pass's tail
  // write on h2d waits for all of them
  cudaStream_t h2d_more[kCopyStreams - 1] = {};
  // the admission pass's pending input copy: packed inputs of consecutive
  // requests, back to back in one page-locked allocation and in the pool
  struct {
    const uint8_t* src = nullptr;
    uint8_t* dst = nullptr;
    size_t bytes = 0;
    uintptr_t lo = 0;
  } run;
  cudaEvent_t copied[kCopyStreams - 1] = {};
  unsigned pass_streams = 0;  // bit i: h2d_more[i] took a copy in this pass
  unsigned next_stream = 0;
  cudaEvent_t kernel_done = nullptr;
  bool kernel_running = false;
  unsigned long long published = 0;  // jobs, full width on the host
  unsigned long long idle_ns = 0;
  tk_server_counters counters{};

  std::mutex mu;
  std::condition_variable cv;        // request completions (waiters)
  std::condition_variable cv_sched;  // new requests / quit (scheduler)
  std::deque<Request*> pending;
  std::map<uint64_t, std::unique_ptr<Request>> all;
  // scheduler-owned: published or copying back, in admission order; and the
  // staged requests whose copy-back was issued, in issue order
  std::vector<Request*> active;
  std::deque<Request*> copying;
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
  S->copying.clear();
  S->cv.notify_all();
}

template <class Fn>
Fn driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    return (Fn)p;
  return nullptr;
}

// Writes a 32-bit word (device memory or mapped host memory) once the work
// before it on the stream has completed: a stream memory operation, no copy
// engine, no SM (the persistent kernel may hold all of them), and it orders
// the stream's earlier writes before its own.
PFN_cuStreamWriteValue32_v11070 write_value_fn() {
  static const auto f = driver_fn<PFN_cuStreamWriteValue32_v11070>("cuStreamWriteValue32");
  return f;
}
cudaError_t set_u32(unsigned int* dst, unsigned int v, cudaStream_t st) {
  const auto f = write_value_fn();
  if (!f) return cudaErrorNotSupported;
  return f((CUstream)st, (CUdeviceptr)dst, v, CU_STREAM_WRITE_VALUE_DEFAULT) == CUDA_SUCCESS
             ? cudaSuccess
             : cudaErrorLaunchFailure;
}

// Device address of [p, p + bytes) when all of it lies in one page-locked,
// device-mapped host allocation; nullptr otherwise (the request is staged).
const void* mapped_host_range(const void* p, size_t bytes) {
  static const auto get_attr = driver_fn<PFN_cuPointerGetAttribute_v4000>("cuPointerGetAttribute");
  if (!p || !get_attr) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  CUdeviceptr start = 0;
  size_t size = 0;
  const CUdeviceptr dp = (CUdeviceptr)a.devicePointer;
  if (get_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, dp) != CUDA_SUCCESS ||
      get_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, dp) != CUDA_SUCCESS)
    return nullptr;
  if (dp < start || dp + bytes > start + size) return nullptr;
  return a.devicePointer;
}

// The host range [lo, hi) of the page-locked allocation holding p, or false
// (pageable memory, or no range query).
bool locked_allocation(const void* p, uintptr_t* lo, uintptr_t* hi) {
  static const auto get_attr = driver_fn<PFN_cuPointerGetAttribute_v4000>("cuPointerGetAttribute");
  if (!p || !get_attr) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeHost) return false;
  CUdeviceptr start = 0;
  size_t size = 0;
  const CUdeviceptr dp = (CUdeviceptr)(a.devicePointer ? a.devicePointer : p);
  if (get_attr(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, dp) != CUDA_SUCCESS ||
      get_attr(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, dp) != CUDA_SUCCESS || dp < start)
    return false;
  *lo = (uintptr_t)p - (uintptr_t)(dp - start);  // the same offset in host addresses
  *hi = *lo + size;
  return true;
}

// Issues the pass's pending input copy on the next copy stream of the
// rotation.
cudaError_t flush_run(tk_server* S) {
  if (!S->run.bytes) return cudaSuccess;
  const unsigned k_st = S->next_stream++ % kCopyStreams;
  cudaStream_t st = k_st == 0 ? S->h2d : S->h2d_more[k_st - 1];
  if (k_st) S->pass_streams |= 1u << (k_st - 1);
  const cudaError_t e =
      cudaMemcpyAsync(S->run.dst, S->run.src, S->run.bytes, cudaMemcpyHostToDevice, st);
  S->run.bytes = 0;
  std::lock_guard<std::mutex> lk(S->mu);  // counters are read under the lock
  S->counters.input_copies++;
  return e;
}

// Staged inputs: copies into the request's pool block.  Every request: its
// job descriptors into the ring.
cudaError_t admit(tk_server* S, Request* r) {
  r->first = S->published;
  const size_t k = (size_t)r->k, vb = r->njobs * k * 512, ab = vb * k;
  const size_t in_bytes = r->in_direct ? 0 : ab + vb * (r->e ? 2 : 1);
  // pool block: [A | s | e] [out], unpadded (each a whole number of 512-byte
  // polynomials), so inputs the caller keeps contiguous arrive in one copy
  uint8_t* base = S->pool + r->off;
  if (!r->out_direct) r->dout = (int16_t*)(base + in_bytes);
  if (!r->in_direct) {
    int16_t* dA = (int16_t*)base;
    int16_t* ds = (int16_t*)(base + ab);
    int16_t* de = r->e ? (int16_t*)(base + ab + vb) : nullptr;
    cudaError_t e = cudaSuccess;
    if (r->packed) {
      // joins the pending copy when it continues it in host memory (the same
      // page-locked allocation) and in the pool; else that copy goes out and
      // this one becomes the pending one.  The pass's copies all go out before
      // its tail is published.
      const uint8_t* src = (const uint8_t*)r->A;
      if (S->run.bytes && r->locked_lo && r->locked_lo == S->run.lo &&
          S->run.src + S->run.bytes == src && S->run.dst + S->run.bytes == base) {
        S->run.bytes += in_bytes;
      } else {
        e = flush_run(S);
        S->run.src = src;
        S->run.dst = base;
        S->run.bytes = in_bytes;
        S->run.lo = r->locked_lo;
      }
    } else {
      // this request's copies go to the next copy stream of the rotation
      const unsigned k_st = S->next_stream++ % kCopyStreams;
      cudaStream_t st = k_st == 0 ? S->h2d : S->h2d_more[k_st - 1];
      if (k_st) S->pass_streams |= 1u << (k_st - 1);
      e = cudaMemcpyAsync(dA, r->A, ab, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(ds, r->s, vb, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess && de) e = cudaMemcpyAsync(de, r->e, vb, cudaMemcpyHostToDevice, st);
      std::lock_guard<std::mutex> lk(S->mu);  // counters are read under the lock
      S->counters.input_copies += de ? 3 : 2;
    }
    if (e != cudaSuccess) return e;
    r->dA = dA;
    r->ds = ds;
    r->de = de;
  }
  const int16_t *A = r->dA, *sv = r->ds, *ev = r->de;
  int16_t* out = r->dout;
  // the slot's job counter is zero: the device resets it when the slot's
  // previous request ends, before that request's flag is written
  for (size_t j = 0; j < r->njobs; j++) {
    tk::ServeJob& J = S->ring[(S->published + j) & (kRingCap - 1)];
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

// Publishes the ring entries written since the last pass: the descriptors
// are already in the (host-resident) ring, so this is the new tail, written
// on the copy stream behind the input copies.
cudaError_t publish(tk_server* S) {
  std::atomic_thread_fence(std::memory_order_seq_cst);  // descriptors before the doorbell
  // the tail write waits for this pass's copies on the other copy streams
  for (int i = 0; i < kCopyStreams - 1; i++) {
    if (!(S->pass_streams & (1u << i))) continue;
    cudaError_t e = cudaEventRecord(S->copied[i], S->h2d_more[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S->h2d, S->copied[i], 0);
    if (e != cudaSuccess) return e;
  }
  S->pass_streams = 0;
  return set_u32(&S->ctl->tail, (unsigned int)S->published, S->h2d);
}

cudaError_t ensure_kernel(tk_server* S) {
  if (S->kernel_running) return cudaSuccess;
  // the previous loop (if any) has ended: clear its closing flag, then order
  // the launch after that and after the copies that published the tail
  cudaError_t e = set_u32(&S->ctl->closing, 0u, S->h2d);
  if (e == cudaSuccess) e = cudaEventRecord(S->kernel_done, S->h2d);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(S->comp, S->kernel_done, 0);
  if (e == cudaSuccess)
    e = tk::launch_serve(S->ring, kRingCap - 1, S->ctl, S->req_ctr, S->req_flag, S->idle_ns,
                         *S->info, S->comp);
  if (e == cudaSuccess) e = cudaEventRecord(S->kernel_done, S->comp);
  if (e == cudaSuccess) {
    S->kernel_running = true;
    std::lock_guard<std::mutex> lk(S->mu);  // counters are read under the lock
    S->counters.device_loop_launches++;
  }
  return e;
}

// Completes a request.  The caller may free it (tk_server_release) as soon as
// the lock is released.
void finish(tk_server* S, Request* r) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (r->bytes) S->alloc.release(r->off, r->bytes);
  S->free_slots.push_back(r->slot);
  S->counters.jobs_done += r->njobs;
  S->counters.requests_done++;
  r->t_done = Clock::now();
  auto ns = [](Clock::duration d) {
    return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(d).count();
  };
  S->counters.queue_ns += ns(r->t_admit - r->t_submit);
  S->counters.device_ns += ns(r->t_flag - r->t_admit);
  S->counters.return_ns += ns(r->t_done - r->t_flag);
  r->state = 3;
  S->cv.notify_all();
}

void scheduler(tk_server* S) {
  cudaSetDevice(S->device);
  Clock::time_point last_work = Clock::now(), last_check = last_work;
  std::unordered_set<Request*> done;
  while (true) {
    if (S->abort.load()) {
      fail_all(S, TK_ERR_TIMEOUT);
      return;
    }
    bool progress = false;
    cudaError_t err = cudaSuccess;
    // 1. admission (FIFO): a request slot, ring room and, for a staged
    // request, pool room; the jobs of every request admitted in this pass are
    // published together.  A ring entry may be overwritten only once its job
    // has been claimed and read; every job before the oldest unfinished
    // request's first one has been (the device claims in ring order and a
    // request finishes only after all of its jobs ran).
    const unsigned long long pub0 = S->published;
    const bool may_admit =
        S->active.size() < kAdmitBatch || S->active.size() + kAdmitBatch <= kMaxActive;
    while (err == cudaSuccess && may_admit) {
      const unsigned long long oldest = S->active.empty() ? S->published : S->active.front()->first;
      Request* r = nullptr;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->pending.empty() || S->free_slots.empty()) break;
        if (S->active.size() >= kMaxActive) break;  // backpressure on the copy queue
        Request* h = S->pending.front();
        if (S->published + h->njobs - oldest > kRingCap) break;
        if (h->bytes && !S->alloc.alloc_from(h->bytes, S->alloc_end, &h->off)) break;
        if (h->bytes) S->alloc_end = h->off + h->bytes;
        S->pending.pop_front();
        h->slot = S->free_slots.back();
        S->free_slots.pop_back();
        h->gen = ++S->slot_gen[h->slot];
        r = h;
      }
      r->t_admit = Clock::now();
      err = admit(S, r);
      r->state = 1;
      S->active.push_back(r);
      progress = true;
    }
    if (err == cudaSuccess) err = flush_run(S);
    if (err == cudaSuccess && S->published != pub0) {
      err = publish(S);
      if (err == cudaSuccess) err = ensure_kernel(S);
    }
    // 2. completion flags: outputs written in place are done, staged ones
    // copy back
    done.clear();
    bool waiting_for_device = false;
    for (Request* r : S->active) {
      if (err != cudaSuccess) break;
      if (r->state != 1) continue;
      const unsigned int f = __atomic_load_n(&S->req_flag[r->slot], __ATOMIC_ACQUIRE);
      if (f != r->gen) {
        waiting_for_device = true;
        continue;
      }
      progress = true;
      r->t_flag = Clock::now();
      if (r->out_direct) {
        done.insert(r);
        finish(S, r);
        continue;
      }
      const size_t vb = r->njobs * (size_t)r->k * 512;
      err = cudaMemcpyAsync(r->out, r->dout, vb, cudaMemcpyDeviceToHost, S->d2h);
      if (err == cudaSuccess) err = set_u32(&S->ret_flag[r->slot], r->gen, S->d2h);
      r->state = 2;
      S->copying.push_back(r);
    }
    // 3. copy-backs end in issue order: look at the oldest only
    while (err == cudaSuccess && !S->copying.empty()) {
      Request* r = S->copying.front();
      if (__atomic_load_n(&S->ret_flag[r->slot], __ATOMIC_ACQUIRE) != r->gen) break;
      S->copying.pop_front();
      done.insert(r);
      finish(S, r);
      progress = true;
    }
    if (err != cudaSuccess) {
      fail_all(S, TK_ERR_CUDA);
      return;
    }
    if (!done.empty())  // pointer comparisons only: these may be freed already
      S->active.erase(std::remove_if(S->active.begin(), S->active.end(),
                                     [&](Request* r) { return done.count(r) != 0; }),
                      S->active.end());
    // 4. device loop liveness: relaunch if it went idle with work outstanding
    const Clock::time_point now = Clock::now();
    if (S->kernel_running && waiting_for_device && now - last_check > kLivenessPeriod) {
      last_check = now;
      const cudaError_t q = cudaEventQuery(S->kernel_done);
      if (q == cudaSuccess) {
        S->kernel_running = false;
      } else if (q != cudaErrorNotReady) {
        fail_all(S, TK_ERR_CUDA);
        return;
      }
    }
    if (waiting_for_device && !S->kernel_running) {
      if (ensure_kernel(S) != cudaSuccess) {
        fail_all(S, TK_ERR_CUDA);
        return;
      }
    }
    if (progress || !S->active.empty()) last_work = now;
    bool idle;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      idle = S->pending.empty() && S->active.empty();
    }
    if (idle && S->quit.load()) break;
    if (progress) continue;
    if (idle && now - last_work > kSpinAfterWork) {  // sleep until a submit (or 1 ms)
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_sched.wait_for(lk, std::chrono::milliseconds(1),
                           [&] { return !S->pending.empty() || S->quit.load(); });
    } else {
      std::this_thread::yield();
    }
  }
}

void destroy_resources(tk_server* S) {
  if (S->comp) cudaStreamSynchronize(S->comp);
  for (int i = 0; i < kCopyStreams - 1; i++) {
    if (S->h2d_more[i]) {
      cudaStreamSynchronize(S->h2d_more[i]);
      cudaStreamDestroy(S->h2d_more[i]);
    }
    if (S->copied[i]) cudaEventDestroy(S->copied[i]);
  }
  if (S->kernel_done) cudaEventDestroy(S->kernel_done);
  if (S->h2d) cudaStreamDestroy(S->h2d);
  if (S->d2h) cudaStreamDestroy(S->d2h);
  if (S->comp) cudaStreamDestroy(S->comp);
  if (S->pool) cudaFree(S->pool);
  if (S->ctl) cudaFree(S->ctl);
  if (S->req_ctr) cudaFree(S->req_ctr);
  if (S->ring) cudaFreeHost(S->ring);
  if (S->req_flag) cudaFreeHost(S->req_flag);
  if (S->ret_flag) cudaFreeHost(S->ret_flag);
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
  if (!write_value_fn()) return TK_ERR_CUDA;  // stream memory operations are required
  std::unique_ptr<tk_server> S(new tk_server);
  S->device = device;
  S->budget = budget;
  S->zero_copy = cfg && cfg->zero_copy;
  S->nslots = (uint32_t)slots;
  S->idle_ns = (unsigned long long)(idle * 1e9);
  if ((rc = tk::api_device_info(device, &S->info))) return rc;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaError_t e = cudaMalloc(&S->pool, budget);
  for (int i = 0; i < kCopyStreams - 1 && e == cudaSuccess; i++) {
    e = cudaStreamCreateWithFlags(&S->h2d_more[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->copied[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaMalloc(&S->ctl, sizeof(tk::ServeCtl));
  if (e == cudaSuccess) e = cudaMemset(S->ctl, 0, sizeof(tk::ServeCtl));
  if (e == cudaSuccess) e = cudaMalloc(&S->req_ctr, slots * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(S->req_ctr, 0, slots * sizeof(unsigned int));
  if (e == cudaSuccess)
    e = cudaHostAlloc(&S->ring, kRingCap * sizeof(tk::ServeJob), cudaHostAllocMapped);
  if (e == cudaSuccess)
    e = cudaHostAlloc(&S->req_flag, slots * sizeof(unsigned int), cudaHostAllocMapped);
  if (e == cudaSuccess)
    e = cudaHostAlloc(&S->ret_flag, slots * sizeof(unsigned int), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->d2h, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->kernel_done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    destroy_resources(S.get());
    return e == cudaErrorMemoryAllocation ? TK_ERR_TOO_LARGE : TK_ERR_CUDA;
  }
  memset(S->req_flag, 0, slots * sizeof(unsigned int));
  memset(S->ret_flag, 0, slots * sizeof(unsigned int));
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
  if (njobs > kRingCap) return TK_ERR_TOO_LARGE;
  const size_t vb = njobs * (size_t)k * 512, ab = vb * (size_t)k;
  // tk_matvec's aliasing rule: out may be s itself, must not overlap A or e
  auto overlaps = [](const void* x, size_t nx, const void* y, size_t ny) {
    const uintptr_t a = (uintptr_t)x, b = (uintptr_t)y;
    return a < b + ny && b < a + nx;
  };
  if (overlaps(out, vb, A, ab) || (e && overlaps(out, vb, e, vb)) ||
      ((const void*)out != (const void*)s && overlaps(out, vb, s, vb)))
    return TK_ERR_INVALID_VALUE;
  std::unique_ptr<Request> r(new Request);
  r->k = k;
  r->njobs = njobs;
  r->A = A;
  r->s = s;
  r->e = e;
  r->out = out;
  const bool back_to_back = (const uint8_t*)s == (const uint8_t*)A + ab &&
                            (!e || (const uint8_t*)e == (const uint8_t*)s + vb);
  {
    // the driver-API range queries need a current context on this thread,
    // which a caller thread that never used CUDA does not have yet
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(S->device);
    // outputs go straight to out whenever it is device-mapped page-locked
    // memory: posted writes over PCIe, no copy back
    r->dout = (int16_t*)mapped_host_range(out, vb);
    r->out_direct = r->dout != nullptr;
    if (S->zero_copy) {
      const void* dA = mapped_host_range(A, ab);
      const void* ds = dA ? mapped_host_range(s, vb) : nullptr;
      const void* de = ds && e ? mapped_host_range(e, vb) : nullptr;
      if (ds && (de || !e)) {
        r->in_direct = true;
        r->dA = (const int16_t*)dA;
        r->ds = (const int16_t*)ds;
        r->de = (const int16_t*)de;
      }
    }
    r->packed =
        !r->in_direct && back_to_back && tk::host_span_one_copy(A, ab + vb * (e ? 2 : 1));
    uintptr_t locked_hi = 0;
    if (r->packed && !locked_allocation(A, &r->locked_lo, &locked_hi)) r->locked_lo = 0;
    if (prev != S->device) cudaSetDevice(prev);
  }
  const size_t pool_bytes =
      (r->in_direct ? 0 : ab + vb * (e ? 2 : 1)) + (r->out_direct ? 0 : vb);
  r->bytes = pool_bytes ? align_up(pool_bytes) : 0;
  if (r->bytes > S->budget) return TK_ERR_TOO_LARGE;
  r->t_submit = Clock::now();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return S->fatal;
  r->ticket = S->next_ticket++;
  *ticket = r->ticket;
  if (r->in_direct)
    S->counters.direct_requests++;
  else
    S->counters.staged_requests++;
  if (r->out_direct) S->counters.direct_outputs++;
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
  S->all.erase(it);
  return TK_SUCCESS;
}

int tk_server_stats(tk_server* S, tk_server_counters* out) {
  if (!S || !out) return TK_ERR_INVALID_VALUE;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->counters;
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
