// Host side of the persistent batch kernel (batch_pass.cuh): which batches it
// serves, their work list, and the launch.
#include <algorithm>
#include <cstring>
#include "batch_pass.h"
#include "batch_pass.cuh"
#include "dfft.h"
#include "dfft_plan.h"

namespace dfft {

template __global__ void batch_persistent<float>(const BatchGeom);
template __global__ void batch_persistent<double>(const BatchGeom);

namespace {

// threads per column of the lengths the kernel runs (0: not run)
int batch_threads_per_column(int L) {
  switch (L) {
#define DFFT_BATCH_P(L_, P_, ...) \
  case L_: return P_;
    DFFT_BATCH_LENGTHS(DFFT_BATCH_P)
#undef DFFT_BATCH_P
    default: return 0;
  }
}

bool is_c2c(int t) { return t == DFFT_FFT || t == DFFT_IFFT || t == DFFT_FFT_INPLACE || t == DFFT_IFFT_INPLACE; }
bool is_inv(int t) { return t == DFFT_IFFT || t == DFFT_IFFT_INPLACE; }

}  // namespace

PersistentBatch::~PersistentBatch() {
  if (d_phases) cudaFree(d_phases);
  if (d_ctr) cudaFree(d_ctr);
}

std::unique_ptr<PersistentBatch> make_persistent_batch(const std::vector<Plan*>& plans, int lag) {
  if (plans.empty()) return nullptr;
  const int prec = plans[0]->precision;
  for (const Plan* p : plans) {
    if (!is_c2c(p->transform) || p->precision != prec || p->chirp_bytes || p->dims.empty()) return nullptr;
    for (int a : p->dims) {
      const int64_t L = p->in_shape[a];
      if (L > 4096 || batch_threads_per_column((int)L) == 0) return nullptr;
    }
  }
  std::unique_ptr<PersistentBatch> B(new PersistentBatch());
  B->dbl = prec == DFFT_F64 ? 1 : 0;
  const int esz = B->dbl ? 16 : 8;
  // one phase per axis pass, in each transform's stage order (inverse:
  // dims in reverse, src/fft.jl:650-776)
  struct Raw {
    int plan, pass;
    Pass p;
  };
  std::vector<std::vector<Raw>> per(plans.size());
  size_t smem = 0;
  for (size_t i = 0; i < plans.size(); ++i) {
    const Plan* pl = plans[i];
    std::vector<int> order = pl->dims;
    if (is_inv(pl->transform)) std::reverse(order.begin(), order.end());
    const int64_t* S = pl->in_shape;
    for (size_t k = 0; k < order.size(); ++k) {
      const int a = order[k];
      PassSpec s;
      s.dbl = B->dbl;
      s.L = (int)S[a];
      long long I = 1, O = 1;
      for (int j = 0; j < a; ++j) I *= S[j];
      for (int j = a + 1; j < 3; ++j) O *= S[j];
      s.I = I;
      s.O = O;
      s.inverse = is_inv(pl->transform) ? 1 : 0;
      s.scale = s.inverse ? 1.0 / (double)s.L : 1.0;
      s.in.kind = s.out.kind = IO_CPLX;
      s.in.si = s.out.si = 1;
      s.in.so = s.out.so = I * s.L;
      s.in.sk = s.out.sk = I;
      s.fast_io = true;
      s.variant = VARIANT_DIRECT;
      Pass p = make_pass(s);
      const int P = batch_threads_per_column(s.L);
      if (p.d.P != P) return nullptr;  // the plan table and the kernel disagree: keep the graph
      const int C = kBatchThreads / P;
      smem = std::max(smem, (size_t)(C + 1) * (size_t)p.d.ld * esz);
      per[i].push_back(Raw{(int)i, (int)k, std::move(p)});
    }
  }
  if (smem > 200 * 1024) return nullptr;
  // staggered work list: pass k of transform i at slot i + k * lag, older
  // transforms' later passes first within a slot
  if (lag < 1) lag = 1;
  int maxk = 0;
  for (auto& v : per) maxk = std::max(maxk, (int)v.size());
  const int n = (int)plans.size();
  std::vector<std::pair<int, int>> seq;  // (plan, pass)
  for (int slot = 0; slot < n + (maxk - 1) * lag; ++slot)
    for (int k = maxk - 1; k >= 0; --k) {
      const int i = slot - k * lag;
      if (i >= 0 && i < n && k < (int)per[i].size()) seq.push_back({i, k});
    }
  std::vector<std::vector<int>> index(plans.size());
  for (size_t i = 0; i < plans.size(); ++i) index[i].assign(per[i].size(), -1);
  long long start = 0;
  for (auto [i, k] : seq) {
    Raw& r = per[i][k];
    BatchPhase ph{};
    ph.d = r.p.d;
    const long long C = kBatchThreads / r.p.d.P, per_item = C * kBatchTilesPerItem;
    ph.tiles = (int)((r.p.d.Q + per_item - 1) / per_item);
    ph.start = start;
    ph.dep = k > 0 ? index[i][k - 1] : -1;
    index[i][k] = (int)B->phases.size();
    B->phase_plan.push_back(i);
    B->phase_first.push_back(k == 0);
    start += ph.tiles;
    B->phases.push_back(ph);
    for (auto& t : r.p.tables) B->tables.push_back(t);
  }
  B->total = start;
  B->smem = smem;
  const void* fn = B->dbl ? reinterpret_cast<const void*>(&batch_persistent<double>)
                          : reinterpret_cast<const void*>(&batch_persistent<float>);
  B->fn = fn;
  cuda_check(ensure_smem_attr(fn, smem), "cudaFuncSetAttribute(batch)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBatchThreads, smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) return nullptr;
  int dev = 0, sms = 148;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  long long grid = (long long)sms * occ;
  if (grid > B->total) grid = B->total;
  B->grid = (unsigned)(grid > 0 ? grid : 1);
  cuda_check(cudaMalloc(&B->d_phases, sizeof(BatchPhase) * B->phases.size()), "cudaMalloc(batch phases)");
  B->ctr_bytes = 8 + 4 * B->phases.size();
  cuda_check(cudaMalloc(&B->d_ctr, B->ctr_bytes), "cudaMalloc(batch counters)");
  B->err = device_error_word();
  return B;
}

void launch_persistent_batch(PersistentBatch* B, const void* const* ins, void* const* outs, cudaStream_t s) {
  // buffers go into the phase descriptors (uploaded again when they change)
  bool same = (int)B->last_in.size() == (int)B->phase_plan.size();
  for (size_t j = 0; same && j < B->phase_plan.size(); ++j) {
    const int i = B->phase_plan[j];
    same = B->last_in[j] == ins[i] && B->last_out[j] == outs[i];
  }
  if (!same) {
    B->last_in.resize(B->phases.size());
    B->last_out.resize(B->phases.size());
    for (size_t j = 0; j < B->phases.size(); ++j) {
      const int i = B->phase_plan[j];
      B->phases[j].d.in.p = B->phase_first[j] ? const_cast<void*>(ins[i]) : outs[i];
      B->phases[j].d.out.p = outs[i];
      B->last_in[j] = ins[i];
      B->last_out[j] = outs[i];
    }
    cuda_check(cudaMemcpyAsync(B->d_phases, B->phases.data(), sizeof(BatchPhase) * B->phases.size(),
                               cudaMemcpyHostToDevice, s),
               "cudaMemcpyAsync(batch phases)");
  }
  cuda_check(cudaMemsetAsync(B->d_ctr, 0, B->ctr_bytes, s), "cudaMemsetAsync(batch counters)");
  BatchGeom g{};
  g.phases = static_cast<const BatchPhase*>(B->d_phases);
  g.nphases = (int)B->phases.size();
  g.total = B->total;
  g.next = static_cast<unsigned long long*>(B->d_ctr);
  g.done = reinterpret_cast<unsigned*>(static_cast<char*>(B->d_ctr) + 8);
  g.err = B->err;
  void* args[] = {&g};
  cuda_check(cudaLaunchKernel(B->fn, dim3(B->grid), dim3(kBatchThreads), args, B->smem, s),
             "cudaLaunchKernel(batch)");
}

}  // namespace dfft
