// The plan object behind the opaque dfft_plan handle.
#pragma once
#include <vector>
#include "dfft_internal.h"

namespace dfft {

struct Plan {
  int device = 0;
  int ndim = 3;
  int precision = 0;
  int transform = 0;
  int decomp = 0;
  int method = 0;
  unsigned flags = 0;
  std::vector<int> dims;          // 0-based transformed axes
  int64_t in_shape[3] = {1, 1, 1};
  int64_t out_shape[3] = {1, 1, 1};
  size_t in_elem = 0, out_elem = 0;
  std::vector<Pass> passes;
  void* work = nullptr;           // plan-owned workspace (C2R over several dims, slab-pass counters)
  size_t work_bytes = 0;
  void* chirp = nullptr;          // Bluestein scratch (Q*M complex per axis, max over axes)
  size_t chirp_bytes = 0;
  ~Plan();
  size_t in_bytes() const;
  size_t out_bytes() const;
};

Plan* build_plan(int ndim, const int64_t* shape, int precision, int transform, int ndims,
                 const int32_t* dims, const int32_t* r2r_kinds, int64_t irfft_len, int decomp,
                 int method, unsigned flags);

// The fused 2-D slab pass of a distributed Slab transform with the output
// (forward) or input (inverse) in the rank-split layout (dfft_slab_split_create).
Plan* build_slab_split_plan(int precision, int inverse, int64_t L, int64_t nslab, int64_t zr, int nranks,
                            int split_dim, unsigned flags);

// work / chirp: workspaces supplied by the caller for this execution (null:
// the plan's own); a plan built with kFlagCallerWorkspace owns none.
void execute_plan(const Plan* p, const void* in, void* out, cudaStream_t stream, void* work = nullptr,
                  void* chirp = nullptr);

// Internal plan flag (above the public DFFT_FLAG_* bits): allocate no
// workspace; every execution brings its own (the serving runtime's arena).
constexpr unsigned kFlagCallerWorkspace = 1u << 30;

}  // namespace dfft

struct dfft_plan_s {
  dfft::Plan* impl;
};
