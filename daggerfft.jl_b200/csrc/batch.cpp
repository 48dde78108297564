// Batches of independent transforms of uneven shapes.
//
// With DFFT_BATCH_PERSISTENT, complex transforms whose axis lengths the
// persistent batch kernel runs (batch_pass.cuh) execute as ONE launch of
// that kernel over a work list of every axis pass of every transform.  By
// default (and for other batches) the batch replays one CUDA graph:
//
// A batch holds N plans (any shapes, kinds and precisions).  The first
// execute with a given set of buffers captures every plan's passes into a
// graph: the plans are spread over up to kBatchStreams forked capture
// streams (fewer for large grids, see branch_count), so transforms of
// different grids become independent branches the
// GPU runs concurrently (the persistent pipelined kernels of one branch and
// the one-tile kernels of another share the SMs).  Later executes with the
// same buffers replay the instantiated graph with one cudaGraphLaunch; new
// buffers update the executable graph in place (cudaGraphExecUpdate) or,
// if the topology changed, re-instantiate it.  Capture happens on a private
// stream (capturing the legacy default stream is not allowed); the graph is
// launched on the caller's stream.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include "batch_pass.h"
#include "batch_rule.h"
#include "dfft.h"
#include "dfft_plan.h"

namespace dfft {

constexpr int kBatchStreams = 8;

struct Batch {
  int device = 0;
  std::vector<Plan*> plans;       // not owned
  std::vector<const void*> last_in;
  std::vector<void*> last_out;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t side[kBatchStreams] = {};
  cudaStream_t cap = nullptr;     // capture origin (the caller's stream may be the legacy one)
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kBatchStreams] = {};
  int launches = 0;
  std::unique_ptr<PersistentBatch> persist;  // the one-launch form, when it serves the batch
  std::mutex mu;
  ~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    for (auto& s : side)
      if (s) cudaStreamDestroy(s);
    if (cap) cudaStreamDestroy(cap);
    for (auto& e : join)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
  }
};

// Branches of the graph: batch_branch_rule (batch_rule.h) over the plans'
// input + output bytes and this device's L2 size.
static int branch_count(const Batch* B) {
  const int n = (int)B->plans.size();
  double total = 0;
  for (const Plan* p : B->plans) total += (double)(p->in_bytes() + p->out_bytes());
  int l2 = 0;
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, B->device) != cudaSuccess) {
    cudaGetLastError();
    l2 = 0;
  }
  return batch_branch_rule(n, total, l2, kBatchStreams);
}

// Records the batch into a graph on the batch's own capture stream (nothing
// runs; the graph is launched on the caller's stream afterwards).
static void capture(Batch* B, const void* const* ins, void* const* outs, cudaGraph_t* g) {
  cudaStream_t s = B->cap;
  const int n = (int)B->plans.size();
  const int k = branch_count(B);
  cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  cudaError_t err = cudaSuccess;
  try {
    cuda_check(cudaEventRecord(B->fork, s), "cudaEventRecord(fork)");
    for (int i = 0; i < k; ++i) cuda_check(cudaStreamWaitEvent(B->side[i], B->fork, 0), "cudaStreamWaitEvent");
    // a plan listed more than once whose workspace is live during a launch
    // (C2R scratch, slab-pass counters) runs its uses one after another on
    // the branch of its first use
    std::vector<int> branch(n);
    for (int i = 0; i < n; ++i) {
      branch[i] = i % k;
      if (B->plans[i]->work_bytes)
        for (int j = 0; j < i; ++j)
          if (B->plans[j] == B->plans[i]) { branch[i] = branch[j]; break; }
    }
    for (int i = 0; i < n; ++i) execute_plan(B->plans[i], ins[i], outs[i], B->side[branch[i]]);
    for (int i = 0; i < k; ++i) {
      cuda_check(cudaEventRecord(B->join[i], B->side[i]), "cudaEventRecord(join)");
      cuda_check(cudaStreamWaitEvent(s, B->join[i], 0), "cudaStreamWaitEvent(join)");
    }
  } catch (...) {
    cudaGraph_t dead = nullptr;
    cudaStreamEndCapture(s, &dead);
    if (dead) cudaGraphDestroy(dead);
    cudaGetLastError();
    throw;
  }
  err = cudaStreamEndCapture(s, g);
  cuda_check(err, "cudaStreamEndCapture");
}

Batch* build_batch(int n, const dfft_plan* plans, unsigned flags) {
  if (n < 1 || !plans) throw Error{DFFT_ERROR_INVALID_VALUE, "a batch needs at least one plan"};
  std::unique_ptr<Batch> B(new Batch());
  cuda_check(cudaGetDevice(&B->device), "cudaGetDevice");
  for (int i = 0; i < n; ++i) {
    if (!plans[i] || !plans[i]->impl) throw Error{DFFT_ERROR_INVALID_VALUE, "NULL plan in batch"};
    if (plans[i]->impl->device != B->device)
      throw Error{DFFT_ERROR_INVALID_VALUE, "every plan of a batch must live on the current device"};
    B->plans.push_back(plans[i]->impl);
    B->launches += (int)plans[i]->impl->passes.size();
  }
  if ((flags & DFFT_BATCH_PERSISTENT) && !(flags & DFFT_BATCH_GRAPH)) {
    // a pass is claimed about `lag` transforms after the one it depends on:
    // the caller's (flag bits 8-15), else the graph's branch count
    // (transforms whose buffers fit L2 at once), at least 4 (64 uneven
    // ComplexF32 grids: lag 1 3.85 ms, 2 3.23, 4 2.91, 16 2.91, 64 2.92)
    const int user_lag = (int)((flags >> 8) & 0xFFu);
    double total = 0;
    for (const Plan* p : B->plans) total += (double)(p->in_bytes() + p->out_bytes());
    int l2 = 0;
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, B->device) != cudaSuccess) {
      cudaGetLastError();
      l2 = 0;
    }
    const int lag = user_lag > 0 ? user_lag : std::max(4, batch_branch_rule(n, total, l2, kBatchStreams));
    B->persist = make_persistent_batch(B->plans, lag < 1 ? 1 : lag);
    if (B->persist) B->launches = 1;
  }
  for (auto& s : B->side) cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking), "cudaStreamCreate");
  for (auto& e : B->join) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming), "cudaEventCreate");
  return B.release();
}

void execute_batch(Batch* B, const void* const* ins, void* const* outs, cudaStream_t s) {
  if (!ins || !outs) throw Error{DFFT_ERROR_INVALID_VALUE, "ins/outs is NULL"};
  std::lock_guard<std::mutex> lk(B->mu);
  const int n = (int)B->plans.size();
  for (int i = 0; i < n; ++i)
    if (!ins[i] || !outs[i]) throw Error{DFFT_ERROR_INVALID_VALUE, "NULL buffer in batch"};
  int cur = -1;
  cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
  if (cur != B->device) cuda_check(cudaSetDevice(B->device), "cudaSetDevice");
  if (B->persist) {
    try {
      launch_persistent_batch(B->persist.get(), ins, outs, s);
    } catch (...) {
      if (cur != B->device) cudaSetDevice(cur);
      throw;
    }
    if (cur != B->device) cudaSetDevice(cur);
    return;
  }
  bool same = B->exec && (int)B->last_in.size() == n;
  for (int i = 0; same && i < n; ++i) same = B->last_in[i] == ins[i] && B->last_out[i] == outs[i];
  if (!same) {
    cudaGraph_t g = nullptr;
    capture(B, ins, outs, &g);
    bool updated = false;
    if (B->exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(B->exec, g, &info) == cudaSuccess) updated = true;
      else cudaGetLastError();
    }
    if (!updated) {
      if (B->exec) cudaGraphExecDestroy(B->exec);
      B->exec = nullptr;
      cudaError_t e = cudaGraphInstantiate(&B->exec, g, 0);
      cudaGraphDestroy(g);
      cuda_check(e, "cudaGraphInstantiate");
    } else {
      cudaGraphDestroy(g);
    }
    B->last_in.assign(ins, ins + n);
    B->last_out.assign(outs, outs + n);
  }
  cudaError_t e = cudaGraphLaunch(B->exec, s);
  if (cur != B->device) cudaSetDevice(cur);
  cuda_check(e, "cudaGraphLaunch");
}

}  // namespace dfft

struct dfft_batch_s {
  dfft::Batch* impl;
};

using dfft::Error;

extern "C" {

int dfft_batch_create(dfft_batch* batch, int nplans, const dfft_plan* plans) {
  return dfft_batch_create_ex(batch, nplans, plans, 0u);
}

int dfft_batch_create_ex(dfft_batch* batch, int nplans, const dfft_plan* plans, unsigned flags) {
  try {
    if (!batch) throw Error{DFFT_ERROR_INVALID_VALUE, "batch is NULL"};
    *batch = nullptr;
    *batch = new dfft_batch_s{dfft::build_batch(nplans, plans, flags)};
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  } catch (...) {
    dfft::set_error("unexpected exception");
    return DFFT_ERROR_INVALID_VALUE;
  }
}

int dfft_batch_execute(dfft_batch batch, const void* const* ins, void* const* outs, void* stream) {
  try {
    if (!batch || !batch->impl) throw Error{DFFT_ERROR_INVALID_VALUE, "batch is NULL"};
    dfft::execute_batch(batch->impl, ins, outs, reinterpret_cast<cudaStream_t>(stream));
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  }
}

int dfft_batch_launches(dfft_batch batch, int* launches) {
  if (!batch || !batch->impl || !launches) {
    dfft::set_error("NULL argument");
    return DFFT_ERROR_INVALID_VALUE;
  }
  *launches = batch->impl->launches;
  return DFFT_SUCCESS;
}

int dfft_batch_destroy(dfft_batch batch) {
  if (batch) {
    delete batch->impl;
    delete batch;
  }
  return DFFT_SUCCESS;
}

}  // extern "C"
