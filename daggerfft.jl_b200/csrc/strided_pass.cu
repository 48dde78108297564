// Instantiations of the producer-warp strided axis pass (axis_pass_strided)
// and its launch shapes, fastest first (B200, 512^3 / 256^3 / 128^3 arrays).
// threads = CS*P stage threads + one producer warp; MINB = CTAs per SM that
// NB tile buffers of CS*L elements leave room for.
// the producer-fed strided pass: packed FP32 adds for its butterflies
#define DFFT_PACKED_F32 1
#include "dfft_internal.h"

namespace dfft {

#define DFFT_STRIDED_INST1(T, LB, MINB, NB, DIR, L, P, CS, ...)                                       \
  template __global__ void axis_pass_strided<T, LB, MINB, NB, DIR, L, P, CS, __VA_ARGS__>(           \
      const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap,       \
      const StridedGeom);
#define DFFT_STRIDED_INST(T, LB, MINB, NB, L, P, CS, ...)          \
  DFFT_STRIDED_INST1(T, LB, MINB, NB, 1, L, P, CS, __VA_ARGS__)     \
  DFFT_STRIDED_INST1(T, LB, MINB, NB, 2, L, P, CS, __VA_ARGS__)
// forward and inverse kernels of one launch shape
#define K(T, LB, MINB, NB, L, P, CS, ...)                                          \
  (const void*)&axis_pass_strided<T, LB, MINB, NB, 1, L, P, CS, __VA_ARGS__>,     \
      (const void*)&axis_pass_strided<T, LB, MINB, NB, 2, L, P, CS, __VA_ARGS__>

// ComplexF32, L = 512 (8 x 8 x 8)
DFFT_STRIDED_INST(float, 288, 3, 2, 512, 32, 8, 8, 8, 8)
DFFT_STRIDED_INST(float, 288, 2, 3, 512, 32, 8, 8, 8, 8)
DFFT_STRIDED_INST(float, 160, 6, 2, 512, 32, 4, 8, 8, 8)
DFFT_STRIDED_INST(float, 544, 1, 2, 512, 32, 16, 8, 8, 8)
// ComplexF32, L = 512 (32 x 16): one exchange, 32 elements per thread
DFFT_STRIDED_INST(float, 288, 1, 2, 512, 16, 16, 32, 16)
DFFT_STRIDED_INST(float, 288, 1, 3, 512, 16, 16, 32, 16)
DFFT_STRIDED_INST(float, 160, 3, 2, 512, 16, 8, 32, 16)
// ComplexF32, L = 256 (16 x 16) and 128 (16 x 8)
DFFT_STRIDED_INST(float, 288, 3, 2, 256, 16, 16, 16, 16)
DFFT_STRIDED_INST(float, 288, 2, 3, 256, 16, 16, 16, 16)
DFFT_STRIDED_INST(float, 160, 6, 2, 256, 16, 8, 16, 16)
DFFT_STRIDED_INST(float, 160, 6, 2, 128, 8, 16, 16, 8)
DFFT_STRIDED_INST(float, 160, 4, 3, 128, 8, 16, 16, 8)
// ComplexF64, L = 512 and 256
DFFT_STRIDED_INST(double, 288, 3, 2, 512, 64, 4, 8, 8, 8)
DFFT_STRIDED_INST(double, 160, 4, 2, 512, 32, 4, 8, 8, 8)
DFFT_STRIDED_INST(double, 160, 3, 2, 256, 16, 8, 16, 16)
DFFT_STRIDED_INST(double, 96, 5, 2, 256, 16, 4, 16, 16)
// lengths of the batched and serving configurations (16 float / 8 double
// columns: rows of 128 bytes)
DFFT_STRIDED_INST(float, 128, 8, 2, 48, 6, 16, 6, 8)
DFFT_STRIDED_INST(float, 160, 6, 2, 64, 8, 16, 8, 8)
DFFT_STRIDED_INST(float, 160, 6, 2, 80, 8, 16, 10, 8)
DFFT_STRIDED_INST(float, 160, 6, 2, 96, 8, 16, 12, 8)
DFFT_STRIDED_INST(float, 192, 5, 2, 120, 10, 16, 12, 10)
DFFT_STRIDED_INST(float, 192, 4, 2, 160, 10, 16, 10, 16)
DFFT_STRIDED_INST(float, 224, 4, 2, 192, 12, 16, 12, 16)
DFFT_STRIDED_INST(float, 416, 2, 2, 384, 48, 8, 6, 8, 8)
DFFT_STRIDED_INST(double, 96, 6, 2, 64, 8, 8, 8, 8)
DFFT_STRIDED_INST(double, 96, 5, 2, 96, 8, 8, 12, 8)
DFFT_STRIDED_INST(double, 96, 6, 2, 128, 8, 8, 16, 8)
DFFT_STRIDED_INST(double, 128, 3, 2, 192, 12, 8, 12, 16)
DFFT_STRIDED_INST(double, 416, 1, 2, 384, 48, 8, 6, 8, 8)

static const SlabKernel kStridedKernels[] = {
    // dbl, L, P, nst, radices, threads, CS, NB, dflt, forward and inverse kernels
    {0, 512, 16, 2, {32, 16}, 288, 16, 2, 1, K(float, 288, 1, 2, 512, 16, 16, 32, 16)},
    {0, 512, 32, 3, {8, 8, 8}, 288, 8, 3, 1, K(float, 288, 2, 3, 512, 32, 8, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 288, 8, 2, 1, K(float, 288, 3, 2, 512, 32, 8, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 160, 4, 2, 1, K(float, 160, 6, 2, 512, 32, 4, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 544, 16, 2, 1, K(float, 544, 1, 2, 512, 32, 16, 8, 8, 8)},
    {0, 512, 16, 2, {32, 16}, 288, 16, 3, 1, K(float, 288, 1, 3, 512, 16, 16, 32, 16)},
    {0, 512, 16, 2, {32, 16}, 160, 8, 2, 1, K(float, 160, 3, 2, 512, 16, 8, 32, 16)},
    {0, 256, 16, 2, {16, 16}, 288, 16, 2, 1, K(float, 288, 3, 2, 256, 16, 16, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 288, 16, 3, 1, K(float, 288, 2, 3, 256, 16, 16, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 160, 8, 2, 1, K(float, 160, 6, 2, 256, 16, 8, 16, 16)},
    {0, 128, 8, 2, {16, 8}, 160, 16, 2, 1, K(float, 160, 6, 2, 128, 8, 16, 16, 8)},
    {0, 128, 8, 2, {16, 8}, 160, 16, 3, 1, K(float, 160, 4, 3, 128, 8, 16, 16, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 288, 4, 2, 1, K(double, 288, 3, 2, 512, 64, 4, 8, 8, 8)},
    {1, 512, 32, 3, {8, 8, 8}, 160, 4, 2, 1, K(double, 160, 4, 2, 512, 32, 4, 8, 8, 8)},
    {1, 256, 16, 2, {16, 16}, 160, 8, 2, 1, K(double, 160, 3, 2, 256, 16, 8, 16, 16)},
    {1, 256, 16, 2, {16, 16}, 96, 4, 2, 1, K(double, 96, 5, 2, 256, 16, 4, 16, 16)},
    {0, 48, 6, 2, {6, 8}, 128, 16, 2, 1, K(float, 128, 8, 2, 48, 6, 16, 6, 8)},
    {0, 64, 8, 2, {8, 8}, 160, 16, 2, 1, K(float, 160, 6, 2, 64, 8, 16, 8, 8)},
    {0, 80, 8, 2, {10, 8}, 160, 16, 2, 1, K(float, 160, 6, 2, 80, 8, 16, 10, 8)},
    {0, 96, 8, 2, {12, 8}, 160, 16, 2, 1, K(float, 160, 6, 2, 96, 8, 16, 12, 8)},
    {0, 120, 10, 2, {12, 10}, 192, 16, 2, 1, K(float, 192, 5, 2, 120, 10, 16, 12, 10)},
    {0, 160, 10, 2, {10, 16}, 192, 16, 2, 1, K(float, 192, 4, 2, 160, 10, 16, 10, 16)},
    {0, 192, 12, 2, {12, 16}, 224, 16, 2, 1, K(float, 224, 4, 2, 192, 12, 16, 12, 16)},
    {0, 384, 48, 3, {6, 8, 8}, 416, 8, 2, 1, K(float, 416, 2, 2, 384, 48, 8, 6, 8, 8)},
    {1, 64, 8, 2, {8, 8}, 96, 8, 2, 1, K(double, 96, 6, 2, 64, 8, 8, 8, 8)},
    {1, 96, 8, 2, {12, 8}, 96, 8, 2, 1, K(double, 96, 5, 2, 96, 8, 8, 12, 8)},
    {1, 128, 8, 2, {16, 8}, 96, 8, 2, 1, K(double, 96, 6, 2, 128, 8, 8, 16, 8)},
    {1, 192, 12, 2, {12, 16}, 128, 8, 2, 1, K(double, 128, 3, 2, 192, 12, 8, 12, 16)},
    {1, 384, 48, 3, {6, 8, 8}, 416, 8, 2, 1, K(double, 416, 1, 2, 384, 48, 8, 6, 8, 8)},
};

#undef K

const SlabKernel* find_strided_kernel(int dbl, int L, int v) {
  int i = 0;
  for (const SlabKernel& k : kStridedKernels)
    if (k.dbl == dbl && k.L == L && i++ == v) return &k;
  return nullptr;
}

}  // namespace dfft
