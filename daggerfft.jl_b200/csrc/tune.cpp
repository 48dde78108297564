// Autotuner and wisdom cache (the analogue of FFTW wisdom, which the
// reference imports at load and exports after every new plan:
// src/fft.jl:113-124,162).
//
// A pass is identified by (device, precision, L, I, O, in/out kinds, r2r
// kinds, R2C post-pass, complex fast path).  With DFFT_FLAG_TUNE the planner
// times every launch candidate of an unseen pass -- kernel variant (direct
// one-tile-per-CTA, persistent TMA-pipelined, dynamic) x columns per CTA --
// on scratch buffers with CUDA events and keeps the fastest.  Results live in
// a process-wide table that dfft_wisdom_export/import write to and read from
// a text file.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include "dfft.h"
#include "dfft_internal.h"

namespace dfft {

namespace {

struct Choice {
  int variant;
  int C;
  float ms;
};

std::mutex g_w_mu;
std::map<std::string, Choice> g_wisdom;

std::string device_tag() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
  std::string n(prop.name);
  for (char& c : n)
    if (c == ' ' || c == '|') c = '_';
  return n + "_sm" + std::to_string(prop.multiProcessorCount);
}

std::string key_of(const PassSpec& s) {
  std::ostringstream o;
  o << device_tag() << "|" << s.dbl << "|" << s.L << "|" << s.I << "|" << s.O << "|" << s.in.kind << ","
    << s.out.kind << "," << s.in.r2r << "," << s.out.r2r << "|" << (int)s.epi << (int)s.fast_io << s.inverse;
  return o.str();
}

// Bytes of one side of a pass (for the scratch buffers the tuner times on).
size_t side_bytes(const PassSpec& s, const IoAny& io, bool out) {
  const size_t rsz = s.dbl ? 8 : 4, csz = 2 * rsz;
  // extent of the side along the axis = so / I
  const long long ext = s.I > 0 ? io.so / s.I : 1;
  const bool cplx = io.kind == IO_CPLX || io.kind == IO_TRUNC || io.kind == IO_HERM_PAIR ||
                    io.kind == IO_HERM_FULL;
  (void)out;
  return (size_t)(s.I * s.O) * (size_t)ext * (cplx ? csz : rsz);
}

}  // namespace

bool wisdom_lookup(const PassSpec& s, int* variant, int* C) {
  std::lock_guard<std::mutex> lk(g_w_mu);
  auto it = g_wisdom.find(key_of(s));
  if (it == g_wisdom.end()) return false;
  *variant = it->second.variant;
  *C = it->second.C;
  return true;
}

Pass tune_pass(const PassSpec& s) {
  // candidate list
  std::vector<std::pair<int, int>> cands;
  for (int v : {VARIANT_PIPE, VARIANT_DIRECT, VARIANT_DYNAMIC}) {
    PassSpec t = s;
    t.variant = v;
    t.C = 0;
    Pass base;
    try {
      base = make_pass(t);
    } catch (const Error&) {
      continue;
    }
    const int C0 = (int)base.d.C;
    for (int C : {C0 / 4, C0 / 2, C0, C0 * 2, C0 * 4}) {
      if (C < 1) continue;
      if (std::find(cands.begin(), cands.end(), std::make_pair(v, C)) == cands.end())
        cands.push_back({v, C});
    }
  }
  // producer-fed strided kernels: one candidate per launch shape
  for (int i = 0; find_strided_kernel(s.dbl, s.L, i); ++i) {
    PassSpec t = s;
    t.variant = VARIANT_FEED;
    t.C = i;
    try {
      make_pass(t);
      cands.push_back({VARIANT_FEED, i});
    } catch (const Error&) {
    }
  }
  // cp.async strided kernels (rows TMA cannot address): one per launch shape
  for (int i = 0; find_async_kernel(s.dbl, s.L, i); ++i) {
    PassSpec t = s;
    t.variant = VARIANT_ASYNC;
    t.C = i;
    try {
      make_pass(t);
      cands.push_back({VARIANT_ASYNC, i});
    } catch (const Error&) {
    }
  }
  if (cands.empty()) return make_pass(s);
  const size_t ib = side_bytes(s, s.in, false), ob = side_bytes(s, s.out, true);
  void *in = nullptr, *out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&] {
    if (in) cudaFree(in);
    if (out) cudaFree(out);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
  };
  if (cudaMalloc(&in, ib + 256) != cudaSuccess || cudaMalloc(&out, ob + 256) != cudaSuccess) {
    cleanup();
    cudaGetLastError();
    return make_pass(s);  // no room to tune: heuristic choice
  }
  cudaMemset(in, 0, ib + 256);
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bv = VARIANT_AUTO, bc = 0;
  // DFFT_TUNE_VERBOSE=1 prints every candidate's time to stderr
  const char* ev = std::getenv("DFFT_TUNE_VERBOSE");
  const bool verbose = ev && ev[0] && ev[0] != '0';
  for (auto& vc : cands) {
    PassSpec t = s;
    t.variant = vc.first;
    t.C = vc.second;
    Pass p;
    try {
      p = make_pass(t);
    } catch (const Error&) {
      continue;
    }
    if (vc.first != VARIANT_FEED && vc.first != VARIANT_ASYNC && (int)p.d.C != vc.second)
      continue;  // clamped to another candidate
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) ok = launch_pass(p, in, out, st) == cudaSuccess;
    if (!ok) { cudaGetLastError(); continue; }
    cudaEventRecord(e0, st);
    const int reps = 5;
    for (int i = 0; i < reps && ok; ++i) ok = launch_pass(p, in, out, st) == cudaSuccess;
    cudaEventRecord(e1, st);
    if (!ok || cudaEventSynchronize(e1) != cudaSuccess) { cudaGetLastError(); continue; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= reps;
    if (verbose)
      std::fprintf(stderr, "dfft tune: L=%d I=%lld O=%lld variant=%d C=%d threads=%u grid=%u smem=%zu %.4f ms\n",
                   s.L, s.I, s.O, vc.first, vc.second, p.block.x, p.grid.x, p.smem, ms);
    if (ms < best) { best = ms; bv = vc.first; bc = vc.second; }
  }
  cleanup();
  if (bv == VARIANT_AUTO) return make_pass(s);
  {
    std::lock_guard<std::mutex> lk(g_w_mu);
    g_wisdom[key_of(s)] = Choice{bv, bc, best};
  }
  PassSpec t = s;
  t.variant = bv;
  t.C = bc;
  return make_pass(t);
}

int choose_slab(int dbl, int L, long long O, int inverse, const std::vector<Pass>& split,
                unsigned flags) {
  std::ostringstream ko;
  ko << device_tag() << "|slab|" << dbl << "|" << L << "|" << O << "|" << inverse;
  const std::string key = ko.str();
  if (!(flags & DFFT_FLAG_NO_WISDOM)) {
    std::lock_guard<std::mutex> lk(g_w_mu);
    auto it = g_wisdom.find(key);
    if (it != g_wisdom.end()) return it->second.variant;
  }
  std::vector<Pass> cands;
  std::vector<int> idx;
  const bool tune = (flags & DFFT_FLAG_TUNE) != 0;
  for (int v = 0; const SlabKernel* k = find_slab_kernel(dbl, L, v); ++v) {
    if (!tune && !k->dflt && !(flags & DFFT_FLAG_FUSE)) continue;
    try {
      cands.push_back(make_slab_pass(dbl, L, O, inverse, v));
      idx.push_back(v);
    } catch (const Error& e) {
      if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
    }
    if (!tune && !cands.empty()) return idx[0];
  }
  if (cands.empty()) return -1;
  // time every fused variant and the per-axis pair on scratch arrays
  const size_t bytes = (size_t)L * L * (size_t)O * (dbl ? 16 : 8);
  void *in = nullptr, *out = nullptr, *ctr = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&] {
    if (in) cudaFree(in);
    if (out) cudaFree(out);
    if (ctr) cudaFree(ctr);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
  };
  if (cudaMalloc(&in, bytes) != cudaSuccess || cudaMalloc(&out, bytes) != cudaSuccess ||
      cudaMalloc(&ctr, cands[0].ctr_bytes) != cudaSuccess) {
    cleanup();
    cudaGetLastError();
    return idx[0];
  }
  cudaMemset(in, 0, bytes);
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const char* ev = std::getenv("DFFT_TUNE_VERBOSE");
  const bool verbose = ev && ev[0] && ev[0] != '0';
  auto time_it = [&](const std::vector<const Pass*>& ps) -> float {
    auto run = [&] {
      bool ok = true;
      for (const Pass* p : ps) {
        void* bufs[2] = {in, out};
        ok = ok && launch_pass(*p, bufs[p->src == BUF_IN ? 0 : 1], out, st, ctr) == cudaSuccess;
      }
      return ok;
    };
    for (int i = 0; i < 2; ++i)
      if (!run()) { cudaGetLastError(); return 1e30f; }
    const int reps = 5;
    cudaEventRecord(e0, st);
    for (int i = 0; i < reps; ++i)
      if (!run()) { cudaGetLastError(); return 1e30f; }
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) { cudaGetLastError(); return 1e30f; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  int best = -1;
  float best_ms = 1e30f;
  if (!split.empty()) {
    std::vector<const Pass*> ps;
    for (const Pass& p : split) ps.push_back(&p);
    best_ms = time_it(ps);
    if (verbose) std::fprintf(stderr, "dfft tune: slab L=%d O=%lld per-axis passes %.4f ms\n", L, O, best_ms);
  }
  for (size_t i = 0; i < cands.size(); ++i) {
    Pass& p = cands[i];
    p.src = BUF_IN;
    p.dst = BUF_OUT;
    const float ms = time_it({&p});
    if (verbose)
      std::fprintf(stderr, "dfft tune: slab L=%d O=%lld variant=%d threads=%u tile=%d lag=%d grid=%u smem=%zu %.4f ms\n",
                   L, O, idx[i], p.block.x, p.geom.C, p.sgeom.lag, p.grid.x, p.smem, ms);
    if (ms < best_ms) { best_ms = ms; best = idx[i]; }
  }
  cleanup();
  {
    std::lock_guard<std::mutex> lk(g_w_mu);
    g_wisdom[key] = Choice{best, 0, best_ms};
  }
  return best;
}

Pass plan_pass(const PassSpec& s, unsigned flags) {
  if (!(flags & DFFT_FLAG_NO_WISDOM)) {
    int v = 0, C = 0;
    if (wisdom_lookup(s, &v, &C)) {
      PassSpec t = s;
      t.variant = v;
      t.C = C;
      try {
        return make_pass(t);
      } catch (const Error&) {
      }
    }
  }
  // only plain complex passes are timed: the other side kinds read twiddle
  // tables that the planner attaches after the pass is built
  if ((flags & DFFT_FLAG_TUNE) && s.fast_io) return tune_pass(s);
  return make_pass(s);
}

int wisdom_export(const char* path) {
  std::lock_guard<std::mutex> lk(g_w_mu);
  std::ofstream f(path);
  if (!f) return DFFT_ERROR_INVALID_VALUE;
  f << "# dfft wisdom v1: key variant C ms\n";
  for (auto& kv : g_wisdom) f << kv.first << " " << kv.second.variant << " " << kv.second.C << " " << kv.second.ms << "\n";
  return f ? DFFT_SUCCESS : DFFT_ERROR_INVALID_VALUE;
}

int wisdom_import(const char* path) {
  std::ifstream f(path);
  if (!f) return DFFT_ERROR_INVALID_VALUE;
  std::string line;
  std::lock_guard<std::mutex> lk(g_w_mu);
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string key;
    Choice c{0, 0, 0};
    if (is >> key >> c.variant >> c.C >> c.ms) g_wisdom[key] = c;
  }
  return DFFT_SUCCESS;
}

void wisdom_forget() {
  std::lock_guard<std::mutex> lk(g_w_mu);
  g_wisdom.clear();
}

int wisdom_size() {
  std::lock_guard<std::mutex> lk(g_w_mu);
  return (int)g_wisdom.size();
}

}  // namespace dfft
