// Redistribution between two blockings of a 3-D array: the GPU side of
// create_gpu_workspace / gpu_coalesced_redistribute! (src/fftgpu.jl:126-415)
// and of its copy kernels pack_kernel!, unpack_kernel!, local_copy_kernel!
// (src/fftgpu.jl:452-495).
//
// The reference launches one kernel per copy pattern with one thread per
// element and a div/mod per element.  Here a whole pattern list (every local
// copy of a redistribution, or every block packed for all peers) is one
// launch: the list lives on the device with a prefix sum of its x-rows, each
// warp copies whole x-rows (contiguous in both the source and the
// destination block, column-major), 16 bytes per lane when both rows are
// 16-byte aligned.  A flat send/receive buffer is just a block whose extents
// equal the copied counts, so pack and unpack are the same kernel.
#include <cstring>
#include <mutex>
#include <vector>
#include "dfft.h"
#include "dfft_internal.h"

namespace dfft {

struct DevBlock {
  const char* src;
  char* dst;
  long long src_off;   // byte offset of the first element (src_start)
  long long dst_off;
  long long sy, sz;    // source strides of dims 2 and 3 (bytes)
  long long dy, dz;    // destination strides (bytes)
  long long nx_bytes;  // bytes per x-row
  long long ny;        // rows per z-plane
  long long row0;      // first global row of this block (prefix sum)
};

__device__ __forceinline__ int find_block(const DevBlock* b, int n, long long row) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b[mid].row0 <= row) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One warp per x-row, grid-stride over all rows of all blocks.
__global__ void __launch_bounds__(256) copy_blocks_kernel(const DevBlock* __restrict__ blocks, int nblocks,
                                                          long long nrows) {
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long row = warp; row < nrows; row += nwarps) {
    const int bi = find_block(blocks, nblocks, row);
    const DevBlock& B = blocks[bi];
    const long long r = row - B.row0;
    const long long y = r % B.ny, z = r / B.ny;
    const char* s = B.src + B.src_off + y * B.sy + z * B.sz;
    char* d = B.dst + B.dst_off + y * B.dy + z * B.dz;
    const long long nb = B.nx_bytes;
    if ((((uintptr_t)s | (uintptr_t)d) & 15) == 0) {
      const long long n16 = nb >> 4;
      for (long long i = lane; i < n16; i += 32)
        reinterpret_cast<uint4*>(d)[i] = __ldg(reinterpret_cast<const uint4*>(s) + i);
      for (long long i = (n16 << 4) + lane * 4; i < nb; i += 128)
        *reinterpret_cast<uint32_t*>(d + i) = *reinterpret_cast<const uint32_t*>(s + i);
    } else if ((((uintptr_t)s | (uintptr_t)d | (uintptr_t)nb) & 7) == 0) {
      const long long n8 = nb >> 3;
      for (long long i = lane; i < n8; i += 32)
        reinterpret_cast<uint2*>(d)[i] = __ldg(reinterpret_cast<const uint2*>(s) + i);
    } else {
      const long long n4 = nb >> 2;
      for (long long i = lane; i < n4; i += 32)
        reinterpret_cast<uint32_t*>(d)[i] = reinterpret_cast<const uint32_t*>(s)[i];
    }
  }
}

struct CopyPlan {
  int device = 0;
  DevBlock* dev = nullptr;
  int nblocks = 0;
  long long nrows = 0;
  long long bytes = 0;
  ~CopyPlan() {
    if (dev) {
      int cur = -1;
      cudaGetDevice(&cur);
      if (cur != device) cudaSetDevice(device);
      cudaFree(dev);
      if (cur != device && cur >= 0) cudaSetDevice(cur);
    }
  }
};

static int sm_count_dev() {
  int dev = 0, v = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 148;
}

CopyPlan* build_copy_plan(const dfft_block_copy* blocks, int n, int elem_bytes) {
  if (n < 0 || (n > 0 && !blocks)) throw Error{DFFT_ERROR_INVALID_VALUE, "blocks is NULL"};
  if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16)
    throw Error{DFFT_ERROR_INVALID_VALUE, "elem_bytes must be 4, 8 or 16"};
  std::vector<DevBlock> hb;
  hb.reserve(n);
  long long rows = 0, bytes = 0;
  for (int i = 0; i < n; ++i) {
    const dfft_block_copy& b = blocks[i];
    for (int k = 0; k < 3; ++k) {
      if (b.count[k] < 0 || b.src_start[k] < 0 || b.dst_start[k] < 0 ||
          b.src_start[k] + b.count[k] > b.src_dims[k] || b.dst_start[k] + b.count[k] > b.dst_dims[k])
        throw Error{DFFT_ERROR_INVALID_VALUE,
                    "block " + std::to_string(i) + " reaches outside its source or destination"};
    }
    if (b.count[0] == 0 || b.count[1] == 0 || b.count[2] == 0) continue;
    if (!b.src || !b.dst) throw Error{DFFT_ERROR_INVALID_VALUE, "block with NULL pointer"};
    DevBlock d;
    d.src = reinterpret_cast<const char*>(b.src);
    d.dst = reinterpret_cast<char*>(b.dst);
    const long long e = elem_bytes;
    d.sy = b.src_dims[0] * e;
    d.sz = b.src_dims[0] * b.src_dims[1] * e;
    d.dy = b.dst_dims[0] * e;
    d.dz = b.dst_dims[0] * b.dst_dims[1] * e;
    d.src_off = b.src_start[0] * e + b.src_start[1] * d.sy + b.src_start[2] * d.sz;
    d.dst_off = b.dst_start[0] * e + b.dst_start[1] * d.dy + b.dst_start[2] * d.dz;
    d.nx_bytes = b.count[0] * e;
    d.ny = b.count[1];
    d.row0 = rows;
    rows += b.count[1] * b.count[2];
    bytes += b.count[0] * b.count[1] * b.count[2] * e;
    hb.push_back(d);
  }
  std::unique_ptr<CopyPlan> P(new CopyPlan());
  cuda_check(cudaGetDevice(&P->device), "cudaGetDevice");
  P->nblocks = (int)hb.size();
  P->nrows = rows;
  P->bytes = bytes;
  if (!hb.empty()) {
    cuda_check(cudaMalloc(&P->dev, hb.size() * sizeof(DevBlock)), "cudaMalloc(copy plan)");
    cuda_check(cudaMemcpy(P->dev, hb.data(), hb.size() * sizeof(DevBlock), cudaMemcpyHostToDevice),
               "cudaMemcpy(copy plan)");
  }
  return P.release();
}

void execute_copy_plan(const CopyPlan* P, cudaStream_t s) {
  if (P->nrows == 0) return;
  int cur = -1;
  cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
  if (cur != P->device) cuda_check(cudaSetDevice(P->device), "cudaSetDevice");
  const long long warps_needed = P->nrows;
  long long blocks = (warps_needed + 7) / 8;
  const long long cap = (long long)sm_count_dev() * 8;
  if (blocks > cap) blocks = cap;
  copy_blocks_kernel<<<(unsigned)blocks, 256, 0, s>>>(P->dev, P->nblocks, P->nrows);
  cudaError_t e = cudaGetLastError();
  if (cur != P->device) cudaSetDevice(cur);
  cuda_check(e, "copy_blocks_kernel");
}

}  // namespace dfft

struct dfft_copy_plan_s {
  dfft::CopyPlan* impl;
};

using dfft::Error;

extern "C" {

int dfft_copy_plan_create(dfft_copy_plan* plan, const dfft_block_copy* blocks, int nblocks,
                          int elem_bytes) {
  try {
    if (!plan) throw Error{DFFT_ERROR_INVALID_VALUE, "plan is NULL"};
    *plan = nullptr;
    *plan = new dfft_copy_plan_s{dfft::build_copy_plan(blocks, nblocks, elem_bytes)};
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  } catch (...) {
    dfft::set_error("unexpected exception");
    return DFFT_ERROR_INVALID_VALUE;
  }
}

int dfft_copy_plan_execute(dfft_copy_plan plan, void* stream) {
  try {
    if (!plan || !plan->impl) throw Error{DFFT_ERROR_INVALID_VALUE, "plan is NULL"};
    dfft::execute_copy_plan(plan->impl, reinterpret_cast<cudaStream_t>(stream));
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  }
}

int dfft_copy_plan_bytes(dfft_copy_plan plan, int64_t* bytes) {
  if (!plan || !plan->impl || !bytes) {
    dfft::set_error("NULL argument");
    return DFFT_ERROR_INVALID_VALUE;
  }
  *bytes = plan->impl->bytes;
  return DFFT_SUCCESS;
}

int dfft_copy_plan_destroy(dfft_copy_plan plan) {
  if (plan) {
    delete plan->impl;
    delete plan;
  }
  return DFFT_SUCCESS;
}

}  // extern "C"
