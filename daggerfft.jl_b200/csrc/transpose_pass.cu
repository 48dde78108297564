// The last pass of a four-step axis: the L1-point transforms leave element
// (i, k1, k2, o) at i + k1 I + k2 I L1 + o I L; the output wants it at
// i + k2 I + k1 I L2 + o I L (index k2 + L2 k1 along the axis).  This pass
// swaps the two middle axes.  With I = 1 it is a 32 x 32 tiled transpose
// through shared memory (both sides coalesced); with I > 1 each warp moves
// whole rows of I contiguous elements.
#include "dfft_internal.h"

namespace dfft {

template <typename V>
__global__ void __launch_bounds__(256) swap_axes_tiled(const V* __restrict__ in, V* __restrict__ out,
                                                       const SwapGeom g) {
  __shared__ V tile[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const long long ta = (g.A + 31) / 32, tb = (g.B + 31) / 32;
  const long long per = ta * tb;
  for (long long t = blockIdx.x; t < per * g.O; t += gridDim.x) {
    const long long o = t / per, r = t % per;
    const long long a0 = (r % ta) * 32, b0 = (r / ta) * 32;
    const long long base = o * g.A * g.B;
    // read rows of a (contiguous), 8 b-rows per pass
    for (int j = ty; j < 32; j += 8) {
      const long long a = a0 + tx, b = b0 + j;
      if (a < g.A && b < g.B) tile[j][tx] = in[base + a + b * g.A];
    }
    __syncthreads();
    // write rows of b (contiguous)
    for (int j = ty; j < 32; j += 8) {
      const long long b = b0 + tx, a = a0 + j;
      if (a < g.A && b < g.B) out[base + b + a * g.B] = tile[tx][j];
    }
    __syncthreads();
  }
}

template <typename V>
__global__ void __launch_bounds__(256) swap_axes_rows(const V* __restrict__ in, V* __restrict__ out,
                                                      const SwapGeom g) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  const long long rows = g.A * g.B * g.O;
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows; r += warps) {
    const long long a = r % g.A, b = (r / g.A) % g.B, o = r / (g.A * g.B);
    const V* src = in + g.I * (a + g.A * (b + g.B * o));
    V* dst = out + g.I * (b + g.B * (a + g.A * o));
    for (long long i = lane; i < g.I; i += 32) dst[i] = src[i];
  }
}

template __global__ void swap_axes_tiled<float2>(const float2*, float2*, const SwapGeom);
template __global__ void swap_axes_tiled<double2>(const double2*, double2*, const SwapGeom);
template __global__ void swap_axes_rows<float2>(const float2*, float2*, const SwapGeom);
template __global__ void swap_axes_rows<double2>(const double2*, double2*, const SwapGeom);

const void* swap_axes_kernel(int dbl, bool tiled) {
  if (tiled) return dbl ? (const void*)&swap_axes_tiled<double2> : (const void*)&swap_axes_tiled<float2>;
  return dbl ? (const void*)&swap_axes_rows<double2> : (const void*)&swap_axes_rows<float2>;
}

}  // namespace dfft
