// Instantiations of the pipelined real passes (real_pass): R2C (first pass
// of rfft) and C2R (last pass of irfft) for half lengths M = 32..256, with
// the radices of the static plans for M.  threads = C*P stage threads + one
// producer warp; 2 tile buffers.
#include "dfft_internal.h"

namespace dfft {

#define DFFT_REAL_INST1(T, LB, MINB, DIR, M, P, C, ...)                                   \
  template __global__ void real_pass<T, LB, MINB, 2, DIR, M, P, C, __VA_ARGS__>(const PassDesc, \
                                                                                const RealGeom);
#define DFFT_REAL_INST(T, LB, MINB, M, P, C, ...)        \
  DFFT_REAL_INST1(T, LB, MINB, 1, M, P, C, __VA_ARGS__)  \
  DFFT_REAL_INST1(T, LB, MINB, 2, M, P, C, __VA_ARGS__)
// R2C and C2R kernels of one launch shape
#define K(T, LB, MINB, M, P, C, ...)                                  \
  (const void*)&real_pass<T, LB, MINB, 2, 1, M, P, C, __VA_ARGS__>, \
      (const void*)&real_pass<T, LB, MINB, 2, 2, M, P, C, __VA_ARGS__>

DFFT_REAL_INST(float, 160, 4, 32, 4, 32, 8, 4)
DFFT_REAL_INST(float, 128, 4, 48, 6, 16, 6, 8)
DFFT_REAL_INST(float, 160, 4, 64, 8, 16, 8, 8)
DFFT_REAL_INST(float, 160, 4, 96, 8, 16, 12, 8)
DFFT_REAL_INST(float, 160, 4, 128, 8, 16, 16, 8)
DFFT_REAL_INST(float, 128, 4, 192, 12, 8, 12, 16)
DFFT_REAL_INST(float, 160, 4, 256, 16, 8, 16, 16)
DFFT_REAL_INST(double, 96, 4, 32, 4, 16, 8, 4)
DFFT_REAL_INST(double, 128, 3, 48, 6, 16, 6, 8)
DFFT_REAL_INST(double, 96, 4, 64, 8, 8, 8, 8)
DFFT_REAL_INST(double, 96, 4, 96, 8, 8, 12, 8)
DFFT_REAL_INST(double, 96, 4, 128, 8, 8, 16, 8)
DFFT_REAL_INST(double, 128, 2, 192, 12, 8, 12, 16)
DFFT_REAL_INST(double, 96, 4, 256, 16, 4, 16, 16)

static const SlabKernel kRealKernels[] = {
    // dbl, M, P, nst, radices, threads, C, NB, dflt, R2C and C2R kernels
    {0, 32, 4, 2, {8, 4}, 160, 32, 2, 1, K(float, 160, 4, 32, 4, 32, 8, 4)},
    {0, 48, 6, 2, {6, 8}, 128, 16, 2, 1, K(float, 128, 4, 48, 6, 16, 6, 8)},
    {0, 64, 8, 2, {8, 8}, 160, 16, 2, 1, K(float, 160, 4, 64, 8, 16, 8, 8)},
    {0, 96, 8, 2, {12, 8}, 160, 16, 2, 1, K(float, 160, 4, 96, 8, 16, 12, 8)},
    {0, 128, 8, 2, {16, 8}, 160, 16, 2, 1, K(float, 160, 4, 128, 8, 16, 16, 8)},
    {0, 192, 12, 2, {12, 16}, 128, 8, 2, 1, K(float, 128, 4, 192, 12, 8, 12, 16)},
    {0, 256, 16, 2, {16, 16}, 160, 8, 2, 1, K(float, 160, 4, 256, 16, 8, 16, 16)},
    {1, 32, 4, 2, {8, 4}, 96, 16, 2, 1, K(double, 96, 4, 32, 4, 16, 8, 4)},
    {1, 48, 6, 2, {6, 8}, 128, 16, 2, 1, K(double, 128, 3, 48, 6, 16, 6, 8)},
    {1, 64, 8, 2, {8, 8}, 96, 8, 2, 1, K(double, 96, 4, 64, 8, 8, 8, 8)},
    {1, 96, 8, 2, {12, 8}, 96, 8, 2, 1, K(double, 96, 4, 96, 8, 8, 12, 8)},
    {1, 128, 8, 2, {16, 8}, 96, 8, 2, 1, K(double, 96, 4, 128, 8, 8, 16, 8)},
    {1, 192, 12, 2, {12, 16}, 128, 8, 2, 1, K(double, 128, 2, 192, 12, 8, 12, 16)},
    {1, 256, 16, 2, {16, 16}, 96, 4, 2, 1, K(double, 96, 4, 256, 16, 4, 16, 16)},
};

#undef K

const SlabKernel* find_real_kernel(int dbl, int M) {
  for (const SlabKernel& k : kRealKernels)
    if (k.dbl == dbl && k.L == M) return &k;
  return nullptr;
}

}  // namespace dfft
