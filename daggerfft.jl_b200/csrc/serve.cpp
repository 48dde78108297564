// Serving runtime: continuous batching of transform requests on one GPU.
//
// No counterpart in the reference (an addition beyond its API).  Requests arrive
// through dfft_server_submit from any thread.  A dispatcher thread admits
// them in arrival order while a slot (an execution stream) is free and the
// request's staging memory fits the HBM budget -- an arena carved once at
// creation, so admission never calls cudaMalloc.  Each admitted request
// runs on its own stream: optional host->device copy into the arena, the
// transform (one resident plan per shape, shared by concurrent requests;
// each request's workspace -- C2R or Bluestein scratch, fused-pass
// counters -- comes from the arena beside its staging memory), an
// optional device->host copy, and a host callback that timestamps the
// completion and wakes the dispatcher, which frees the slot and the arena
// memory and admits the next requests.  Work of different requests overlaps
// on the device; requests that arrive while others run join as soon as a
// slot and memory free up.
//
// Latency = completion time - submit time (host steady clock); the submit
// time is taken on entry to dfft_server_submit, so the build of a plan for a
// shape the server has not seen yet counts in that request's latency.  Plans
// are built outside the server mutex (one build at a time), so a cold shape
// never holds up admission or retirement of the requests already in flight.
// Every wait is bounded (DFFT_ERROR_TIMEOUT), queued requests can be
// cancelled, and a request that can never fit the budget is rejected at
// submit.
//
// Admission is in arrival order, with one bounded exception: when the
// request at the head of the queue is waiting for arena memory, up to
// `slots` later requests that fit may start before it (each of them
// finishes and frees its memory; after that many the head is served
// strictly first), so one large request does not idle the slots behind it.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <memory>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>
#include "dfft.h"
#include "dfft_plan.h"

namespace dfft {

using Clock = std::chrono::steady_clock;

// First-fit allocator over one device arena (offsets 256-byte aligned).
class Arena {
 public:
  void init(size_t bytes) {
    size_ = bytes;
    free_.clear();
    sizes_.clear();
    if (bytes) free_[0] = bytes;
    used_ = 0;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~(size_t)255;
    if (bytes == 0) bytes = 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t noff = it->first + bytes;
        free_.erase(it);
        if (rest) free_[noff] = rest;
        used_ += bytes;
        sizes_[*off] = bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off) {
    auto s = sizes_.find(off);
    if (s == sizes_.end()) return;
    const size_t bytes = s->second;
    sizes_.erase(s);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
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
  size_t used() const { return used_; }
  size_t size() const { return size_; }

 private:
  size_t size_ = 0, used_ = 0;
  std::map<size_t, size_t> free_;
  std::unordered_map<size_t, size_t> sizes_;
};

struct PlanKey {
  int transform, precision, ndim, nd, decomp;
  int64_t shape[3];
  int32_t dims[3], kinds[3];
  int64_t n;
  bool operator<(const PlanKey& o) const {
    return std::tie(transform, precision, ndim, nd, decomp, shape[0], shape[1], shape[2], dims[0], dims[1],
                    dims[2], kinds[0], kinds[1], kinds[2], n) <
           std::tie(o.transform, o.precision, o.ndim, o.nd, o.decomp, o.shape[0], o.shape[1], o.shape[2],
                    o.dims[0], o.dims[1], o.dims[2], o.kinds[0], o.kinds[1], o.kinds[2], o.n);
  }
};

struct Req {
  uint64_t id = 0;
  dfft_request r{};
  PlanKey key{};
  size_t in_bytes = 0, out_bytes = 0;
  size_t stage_bytes = 0;    // arena bytes this request needs
  Clock::time_point t_submit, t_admit, t_done;
  int state = 0;             // 0 queued, 1 running, 2 done, 3 cancelled, 4 failed
  int status = 0;
  int slot = -1;
  size_t off_in = 0, off_out = 0, off_work = 0;
  bool has_in = false, has_out = false, has_work = false;
  size_t work_bytes = 0, chirp_bytes = 0;  // the plan's workspaces, from the arena
  Plan* plan = nullptr;
};

struct Server;

// An execution slot.  The completion callback only touches the two
// atomics below and notifies the dispatcher; it never takes the server
// mutex (code holding the mutex may call CUDA functions that wait for the
// device, and with it for pending callbacks).
struct Slot {
  cudaStream_t stream = nullptr;
  Req* req = nullptr;
  Server* srv = nullptr;
  int index = 0;
  std::atomic<int> done{0};
  std::atomic<int64_t> t_done_ns{0};
};

struct Server {
  int device = 0;
  unsigned flags = 0;
  char* arena_base = nullptr;
  Arena arena;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  // dispatcher wake-up: a flag under its own mutex, which is never held
  // across a CUDA call, so the completion callback may take it (a wake-up
  // sent between the dispatcher's last check and its wait is not lost)
  std::mutex wake_mu;
  std::condition_variable wake_cv;
  bool wake = false;
  std::mutex build_mu;              // plan builds, one at a time, outside `mu`
  std::condition_variable done_cv;  // waiters
  std::deque<Req*> queue;
  std::unordered_map<uint64_t, Req*> reqs;
  std::deque<uint64_t> completed;   // finished, not yet polled
  std::vector<double> lat_ms;
  std::map<PlanKey, Plan*> shared_plans;      // one resident plan per shape
  std::vector<Plan*> all_plans;
  uint64_t next_id = 1;
  int head_bypassed = 0;            // later requests admitted past a blocked head
  bool stop = false;
  std::thread thr;
  Clock::time_point t0;
  uint64_t n_done = 0, n_rejected = 0, n_cancelled = 0, n_failed = 0;
  double bytes_done = 0;
  size_t peak_used = 0;
  int peak_running = 0;
  ~Server();
  void poke() {
    {
      std::lock_guard<std::mutex> g(wake_mu);
      wake = true;
    }
    wake_cv.notify_all();
  }
};

// Host callback at the end of a request's stream work: no CUDA calls and no
// server mutex, only the slot's atomics and a wake-up of the dispatcher.
static void CUDART_CB on_done(void* p) {
  Slot* s = static_cast<Slot*>(p);
  s->t_done_ns.store(Clock::now().time_since_epoch().count(), std::memory_order_relaxed);
  s->done.store(1, std::memory_order_release);
  s->srv->poke();
}

// Server plans own no workspace (kFlagCallerWorkspace): while it runs a
// plan only reads its tables, and each request brings its workspace (C2R
// scratch, Bluestein scratch, fused-pass counters) from the arena, so one
// resident instance serves every concurrent request of its shape.  Called
// without `mu` held: the build (device allocations, twiddle uploads, tuning
// launches) runs under build_mu only.
static Plan* get_plan(Server* S, const PlanKey& k, const dfft_request& r) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto sh = S->shared_plans.find(k);
    if (sh != S->shared_plans.end()) return sh->second;
  }
  std::lock_guard<std::mutex> bl(S->build_mu);
  {
    std::lock_guard<std::mutex> lk(S->mu);  // built by another thread meanwhile?
    auto sh = S->shared_plans.find(k);
    if (sh != S->shared_plans.end()) return sh->second;
  }
  std::unique_ptr<Plan> p(build_plan(r.ndim, r.shape, r.precision, r.transform, r.ndims, r.dims, r.r2r_kinds,
                                     r.irfft_len, r.decomp, DFFT_PLAIN,
                                     (S->flags & DFFT_FLAG_TUNE) | kFlagCallerWorkspace));
  std::lock_guard<std::mutex> lk(S->mu);
  S->all_plans.push_back(p.get());
  S->shared_plans[k] = p.get();
  return p.release();
}

static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Takes the arena memory request q needs; false (nothing taken) if it does
// not fit now.
static bool reserve(Server* S, Req* q, size_t* oin, size_t* oout, size_t* owork, bool* gin, bool* gout,
                    bool* gwork) {
  *gin = *gout = *gwork = false;
  if (q->r.in_location == DFFT_MEM_HOST) {
    if (!S->arena.alloc(q->in_bytes, oin)) return false;
    *gin = true;
  }
  if (q->r.out_location != DFFT_MEM_DEVICE) {
    if (!S->arena.alloc(q->out_bytes, oout)) {
      if (*gin) S->arena.release(*oin);
      *gin = false;
      return false;
    }
    *gout = true;
  }
  if (q->work_bytes + q->chirp_bytes) {
    if (!S->arena.alloc(round256(q->work_bytes) + q->chirp_bytes, owork)) {
      if (*gin) S->arena.release(*oin);
      if (*gout) S->arena.release(*oout);
      *gin = *gout = false;
      return false;
    }
    *gwork = true;
  }
  return true;
}

// Admit queued requests in order while a slot and arena memory are free;
// while the head waits for memory, at most `slots` later requests that fit
// go past it (head_bypassed counts them; it resets when the head starts).
static void admit(Server* S, std::unique_lock<std::mutex>& lk) {
  while (!S->queue.empty()) {
    while (!S->queue.empty() && S->queue.front()->state == 3) {  // cancelled while queued
      S->queue.pop_front();
      S->head_bypassed = 0;
    }
    if (S->queue.empty()) return;
    int free_slot = -1;
    for (auto& s : S->slots)
      if (!s->req) {
        free_slot = s->index;
        break;
      }
    if (free_slot < 0) return;
    size_t oin = 0, oout = 0, owork = 0;
    bool gin = false, gout = false, gwork = false;
    auto pick = S->queue.begin();
    if (reserve(S, *pick, &oin, &oout, &owork, &gin, &gout, &gwork)) {
      S->head_bypassed = 0;
    } else {
      if (S->head_bypassed >= (int)S->slots.size()) return;
      for (++pick; pick != S->queue.end(); ++pick)
        if ((*pick)->state != 3 && reserve(S, *pick, &oin, &oout, &owork, &gin, &gout, &gwork)) break;
      if (pick == S->queue.end()) return;
      S->head_bypassed++;
    }
    Req* q = *pick;
    S->queue.erase(pick);
    q->off_in = oin;
    q->off_out = oout;
    q->off_work = owork;
    q->has_in = gin;
    q->has_out = gout;
    q->has_work = gwork;
    q->slot = free_slot;
    q->state = 1;
    q->t_admit = Clock::now();
    Slot& sl = *S->slots[free_slot];
    sl.req = q;
    sl.done.store(0, std::memory_order_relaxed);
    S->peak_used = std::max(S->peak_used, S->arena.used());
    int running = 0;
    for (auto& s : S->slots) running += s->req ? 1 : 0;
    S->peak_running = std::max(S->peak_running, running);
    int st = DFFT_SUCCESS;  // q->plan was built (or found) at submit
    // enqueue outside the lock: the stream work does not touch server state
    lk.unlock();
    if (st == DFFT_SUCCESS) {
      try {
        const void* din = gin ? (const void*)(S->arena_base + oin) : q->r.in;
        void* dout = gout ? (void*)(S->arena_base + oout) : q->r.out;
        if (gin)
          cuda_check(cudaMemcpyAsync((void*)din, q->r.in, q->in_bytes, cudaMemcpyHostToDevice, sl.stream),
                     "cudaMemcpyAsync(H2D)");
        char* w = gwork ? S->arena_base + owork : nullptr;
        execute_plan(q->plan, din, dout, sl.stream, q->work_bytes ? w : nullptr,
                     q->chirp_bytes ? w + round256(q->work_bytes) : nullptr);
        if (q->r.out_location == DFFT_MEM_HOST)
          cuda_check(cudaMemcpyAsync(q->r.out, dout, q->out_bytes, cudaMemcpyDeviceToHost, sl.stream),
                     "cudaMemcpyAsync(D2H)");
        cuda_check(cudaLaunchHostFunc(sl.stream, on_done, &sl), "cudaLaunchHostFunc");
      } catch (const Error& e) {
        st = e.status;
        set_error(e.msg);
      }
    }
    lk.lock();
    if (st != DFFT_SUCCESS) {
      q->status = st;
      q->state = 4;
      q->t_done = Clock::now();
    }
  }
}

// Retire finished requests: free their slot (and, unless the result stays
// in the arena for the client, their memory), record the latency.
static void retire(Server* S) {
  for (auto& sp : S->slots) {
    Slot& s = *sp;
    Req* q = s.req;
    if (!q) continue;
    if (q->state == 1 && s.done.load(std::memory_order_acquire)) {
      q->t_done = Clock::time_point(Clock::duration(s.t_done_ns.load(std::memory_order_relaxed)));
      q->state = 2;
    }
    if (q->state != 2 && q->state != 4) continue;
    s.done.store(0, std::memory_order_relaxed);
    s.req = nullptr;
    if (q->has_in) {
      S->arena.release(q->off_in);
      q->has_in = false;
    }
    if (q->has_out && q->r.out_location == DFFT_MEM_HOST) {
      S->arena.release(q->off_out);
      q->has_out = false;
    }
    if (q->has_work) {
      S->arena.release(q->off_work);
      q->has_work = false;
    }
    if (q->state == 2) {
      S->n_done++;
      S->bytes_done += (double)(q->in_bytes + q->out_bytes);
      S->lat_ms.push_back(std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count());
    } else {
      S->n_failed++;
    }
    S->completed.push_back(q->id);
    S->done_cv.notify_all();
  }
}

static void dispatcher(Server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (!S->stop) {
    retire(S);
    admit(S, lk);
    retire(S);
    lk.unlock();
    {
      std::unique_lock<std::mutex> wl(S->wake_mu);
      S->wake_cv.wait_for(wl, std::chrono::milliseconds(5), [S] { return S->wake; });
      S->wake = false;
    }
    lk.lock();
  }
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
  }
  poke();
  if (thr.joinable()) thr.join();
  for (auto& s : slots)
    if (s && s->stream) {
      cudaStreamSynchronize(s->stream);
      cudaStreamDestroy(s->stream);
    }
  for (Plan* p : all_plans) delete p;
  for (auto& kv : reqs) delete kv.second;
  if (arena_base) cudaFree(arena_base);
}

}  // namespace dfft

struct dfft_server_s {
  dfft::Server* impl;
};

using dfft::Error;
using dfft::Server;

namespace {
template <class F> int guard(F&& f) {
  try {
    f();
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  } catch (...) {
    dfft::set_error("unexpected exception");
    return DFFT_ERROR_INVALID_VALUE;
  }
}
Server* srv(dfft_server s) {
  if (!s || !s->impl) throw Error{DFFT_ERROR_INVALID_VALUE, "server is NULL"};
  return s->impl;
}
}  // namespace

extern "C" {

int dfft_server_create(dfft_server* server, size_t hbm_budget_bytes, int slots, unsigned flags) {
  return guard([&] {
    if (!server) throw Error{DFFT_ERROR_INVALID_VALUE, "server is NULL"};
    if (slots < 1 || slots > 64) throw Error{DFFT_ERROR_INVALID_VALUE, "slots must be 1..64"};
    *server = nullptr;
    std::unique_ptr<Server> S(new Server());
    dfft::cuda_check(cudaGetDevice(&S->device), "cudaGetDevice");
    S->flags = flags;
    if (hbm_budget_bytes)
      dfft::cuda_check(cudaMalloc(&S->arena_base, hbm_budget_bytes), "cudaMalloc(server arena)");
    S->arena.init(hbm_budget_bytes);
    for (int i = 0; i < slots; ++i) {
      S->slots.emplace_back(new dfft::Slot());
      S->slots[i]->index = i;
      S->slots[i]->srv = S.get();
      dfft::cuda_check(cudaStreamCreateWithFlags(&S->slots[i]->stream, cudaStreamNonBlocking),
                       "cudaStreamCreate");
    }
    S->t0 = dfft::Clock::now();
    Server* raw = S.get();
    S->thr = std::thread([raw] { dfft::dispatcher(raw); });
    *server = new dfft_server_s{S.release()};
  });
}

int dfft_server_submit(dfft_server server, const dfft_request* req, uint64_t* id) {
  return guard([&] {
    Server* S = srv(server);
    if (!req || !id) throw Error{DFFT_ERROR_INVALID_VALUE, "req/id is NULL"};
    if (!req->in) throw Error{DFFT_ERROR_INVALID_VALUE, "request input is NULL"};
    if (req->out_location != DFFT_MEM_SERVER && !req->out)
      throw Error{DFFT_ERROR_INVALID_VALUE, "request output is NULL"};
    if (req->ndim < 1 || req->ndim > 3 || req->ndims < 0 || req->ndims > req->ndim)
      throw Error{DFFT_ERROR_INVALID_VALUE, "bad ndim/ndims"};
    std::unique_ptr<dfft::Req> q(new dfft::Req());
    q->r = *req;
    dfft::PlanKey k{};
    k.transform = req->transform;
    k.precision = req->precision;
    k.ndim = req->ndim;
    k.nd = req->ndims;
    k.decomp = req->decomp;
    k.n = req->irfft_len;
    for (int i = 0; i < 3; ++i) k.shape[i] = i < req->ndim ? req->shape[i] : 1;
    for (int i = 0; i < req->ndims; ++i) {
      k.dims[i] = req->dims[i];
      k.kinds[i] = req->transform == DFFT_R2R ? req->r2r_kinds[i] : 0;
    }
    q->key = k;
    q->t_submit = dfft::Clock::now();
    // the plan is built (or taken from the resident cache) at submit, so
    // admission only moves data; a build runs without the server mutex
    dfft::Plan* p = dfft::get_plan(S, k, *req);
    q->plan = p;
    std::unique_lock<std::mutex> lk(S->mu);
    q->in_bytes = p->in_bytes();
    q->out_bytes = p->out_bytes();
    q->work_bytes = p->work_bytes;
    q->chirp_bytes = p->chirp_bytes;
    q->stage_bytes = (req->in_location == DFFT_MEM_HOST ? dfft::round256(q->in_bytes) : 0) +
                     (req->out_location != DFFT_MEM_DEVICE ? dfft::round256(q->out_bytes) : 0) +
                     (q->work_bytes + q->chirp_bytes ? dfft::round256(dfft::round256(q->work_bytes) + q->chirp_bytes)
                                                      : 0);
    if (q->stage_bytes > S->arena.size()) {
      S->n_rejected++;
      throw Error{DFFT_ERROR_OUT_OF_MEMORY, "request needs " + std::to_string(q->stage_bytes) +
                                                " staging bytes, more than the server's HBM budget"};
    }
    q->id = S->next_id++;
    *id = q->id;
    dfft::Req* raw = q.release();
    S->reqs[raw->id] = raw;
    S->queue.push_back(raw);
    lk.unlock();
    S->poke();
  });
}

int dfft_server_poll(dfft_server server, uint64_t* ids, int max, int* n) {
  return guard([&] {
    Server* S = srv(server);
    if (!n || (max > 0 && !ids)) throw Error{DFFT_ERROR_INVALID_VALUE, "NULL argument"};
    std::lock_guard<std::mutex> lk(S->mu);
    int k = 0;
    while (k < max && !S->completed.empty()) {
      ids[k++] = S->completed.front();
      S->completed.pop_front();
    }
    *n = k;
  });
}

int dfft_server_wait(dfft_server server, uint64_t id, int timeout_ms, int* status) {
  return guard([&] {
    Server* S = srv(server);
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) throw Error{DFFT_ERROR_INVALID_VALUE, "unknown request id"};
    dfft::Req* q = it->second;
    const auto until = dfft::Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    auto finished = [&] {
      return q->state == 3 ||
             ((q->state == 2 || q->state == 4) && (q->slot < 0 || S->slots[q->slot]->req != q));
    };
    while (!finished()) {
      if (S->done_cv.wait_until(lk, until) == std::cv_status::timeout && !finished())
        throw Error{DFFT_ERROR_TIMEOUT, "request " + std::to_string(id) + " not finished in time"};
    }
    if (status) *status = q->state == 3 ? DFFT_ERROR_CANCELLED : q->status;
  });
}

int dfft_server_fetch(dfft_server server, uint64_t id, void* dst, int dst_location, void* stream) {
  return guard([&] {
    Server* S = srv(server);
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) throw Error{DFFT_ERROR_INVALID_VALUE, "unknown request id"};
    dfft::Req* q = it->second;
    if (!dst) throw Error{DFFT_ERROR_INVALID_VALUE, "dst is NULL"};
    if (q->state != 2 || q->r.out_location != DFFT_MEM_SERVER || !q->has_out)
      throw Error{DFFT_ERROR_NOT_READY, "no server-held result for this request"};
    dfft::cuda_check(cudaMemcpyAsync(dst, S->arena_base + q->off_out, q->out_bytes,
                                     dst_location == DFFT_MEM_HOST ? cudaMemcpyDeviceToHost
                                                                   : cudaMemcpyDeviceToDevice,
                                     reinterpret_cast<cudaStream_t>(stream)),
                     "cudaMemcpyAsync(fetch)");
  });
}

int dfft_server_result_pointer(dfft_server server, uint64_t id, void** ptr) {
  return guard([&] {
    Server* S = srv(server);
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end() || !ptr) throw Error{DFFT_ERROR_INVALID_VALUE, "unknown request id"};
    dfft::Req* q = it->second;
    if (q->state != 2 || !q->has_out) throw Error{DFFT_ERROR_NOT_READY, "no server-held result"};
    *ptr = S->arena_base + q->off_out;
  });
}

int dfft_server_release(dfft_server server, uint64_t id) {
  return guard([&] {
    Server* S = srv(server);
    {
      std::lock_guard<std::mutex> lk(S->mu);
      auto it = S->reqs.find(id);
      if (it == S->reqs.end()) throw Error{DFFT_ERROR_INVALID_VALUE, "unknown request id"};
      dfft::Req* q = it->second;
      if (q->state < 2) throw Error{DFFT_ERROR_NOT_READY, "request still queued or running"};
      if (q->slot >= 0 && S->slots[q->slot]->req == q)
        throw Error{DFFT_ERROR_NOT_READY, "request not retired yet"};
      if (q->has_out) S->arena.release(q->off_out);
      if (q->state == 3) {  // cancelled: may still sit in the admission queue
        auto qi = std::find(S->queue.begin(), S->queue.end(), q);
        if (qi != S->queue.end()) S->queue.erase(qi);
      }
      S->reqs.erase(it);
      delete q;
    }
    S->poke();
  });
}

int dfft_server_cancel(dfft_server server, uint64_t id) {
  return guard([&] {
    Server* S = srv(server);
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) throw Error{DFFT_ERROR_INVALID_VALUE, "unknown request id"};
    if (it->second->state != 0) throw Error{DFFT_ERROR_NOT_READY, "request already admitted"};
    it->second->state = 3;
    S->n_cancelled++;
    S->completed.push_back(id);
    S->done_cv.notify_all();
  });
}

int dfft_server_get_stats(dfft_server server, dfft_server_stats* st) {
  return guard([&] {
    Server* S = srv(server);
    if (!st) throw Error{DFFT_ERROR_INVALID_VALUE, "stats is NULL"};
    std::lock_guard<std::mutex> lk(S->mu);
    std::vector<double> l = S->lat_ms;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
      if (l.empty()) return 0.0;
      size_t i = (size_t)(p * (double)(l.size() - 1) + 0.5);
      return l[std::min(i, l.size() - 1)];
    };
    st->completed = S->n_done;
    st->rejected = S->n_rejected;
    st->cancelled = S->n_cancelled;
    st->failed = S->n_failed;
    st->queued = S->queue.size();
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = l.empty() ? 0.0 : l.back();
    st->bytes_moved = S->bytes_done;
    st->elapsed_s = std::chrono::duration<double>(dfft::Clock::now() - S->t0).count();
    st->arena_bytes = S->arena.size();
    st->arena_peak_bytes = S->peak_used;
    st->peak_running = S->peak_running;
    st->resident_plans = (int)S->all_plans.size();
  });
}

int dfft_server_reset_stats(dfft_server server) {
  return guard([&] {
    Server* S = srv(server);
    std::lock_guard<std::mutex> lk(S->mu);
    S->lat_ms.clear();
    S->n_done = S->n_rejected = S->n_cancelled = S->n_failed = 0;
    S->bytes_done = 0;
    S->peak_used = S->arena.used();
    S->peak_running = 0;
    S->t0 = dfft::Clock::now();
  });
}

int dfft_server_destroy(dfft_server server) {
  if (server) {
    delete server->impl;
    delete server;
  }
  return DFFT_SUCCESS;
}

}  // extern "C"
