// Instantiations of the fused 2-D slab pass and the launch variants the
// planner chooses from.  The radices are those of the static plan for the
// same length (the stage twiddle table is built from them); the planner
// checks that they agree.
// the fused slab pass is issue-bound: packed FP32 adds for its butterflies
#define DFFT_PACKED_F32 1
#include "dfft_internal.h"

namespace dfft {

#define DFFT_SLAB_INST1(T, LB, MINB, NB, DIR, MODE, L, P, CS, ...)                                    \
  template __global__ void slab_xy_pass<T, LB, MINB, NB, DIR, MODE, L, P, CS, __VA_ARGS__>(          \
      const PassDesc, const PassDesc, const __grid_constant__ CUtensorMap,                           \
      const __grid_constant__ CUtensorMap, const SlabGeom);
#define DFFT_SLAB_INST(T, LB, MINB, NB, L, P, CS, ...)              \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 1, 0, L, P, CS, __VA_ARGS__)      \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 2, 0, L, P, CS, __VA_ARGS__)      \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 1, 1, L, P, CS, __VA_ARGS__)      \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 2, 1, L, P, CS, __VA_ARGS__)      \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 1, 2, L, P, CS, __VA_ARGS__)      \
  DFFT_SLAB_INST1(T, LB, MINB, NB, 2, 2, L, P, CS, __VA_ARGS__)
// forward and inverse kernels of one launch shape: plain, rows split by
// rank, columns split by rank (y-phase first)
#define K(T, LB, MINB, NB, L, P, CS, ...)                                        \
  (const void*)&slab_xy_pass<T, LB, MINB, NB, 1, 0, L, P, CS, __VA_ARGS__>,     \
      (const void*)&slab_xy_pass<T, LB, MINB, NB, 2, 0, L, P, CS, __VA_ARGS__>, \
      (const void*)&slab_xy_pass<T, LB, MINB, NB, 1, 1, L, P, CS, __VA_ARGS__>, \
      (const void*)&slab_xy_pass<T, LB, MINB, NB, 2, 1, L, P, CS, __VA_ARGS__>, \
      (const void*)&slab_xy_pass<T, LB, MINB, NB, 1, 2, L, P, CS, __VA_ARGS__>, \
      (const void*)&slab_xy_pass<T, LB, MINB, NB, 2, 2, L, P, CS, __VA_ARGS__>

// threads = CS*P stage threads + one producer warp; MINB = CTAs per SM that
// the NB tile buffers of CS*L elements leave room for
// ComplexF32, L = 512 (8 x 8 x 8)
DFFT_SLAB_INST(float, 160, 5, 2, 512, 32, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 160, 6, 2, 512, 32, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 288, 4, 2, 512, 64, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 160, 4, 3, 512, 32, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 288, 2, 3, 512, 32, 8, 8, 8, 8)
// ComplexF32, L = 512 (32 x 16): one exchange per axis, 32 elements per thread
DFFT_SLAB_INST(float, 160, 3, 2, 512, 16, 8, 32, 16)
// ComplexF32, L = 256 (16 x 16) and 128 (16 x 8)
DFFT_SLAB_INST(float, 160, 5, 2, 256, 16, 8, 16, 16)
DFFT_SLAB_INST(float, 160, 6, 2, 256, 16, 8, 16, 16)
DFFT_SLAB_INST(float, 160, 4, 3, 256, 16, 8, 16, 16)
DFFT_SLAB_INST(float, 288, 2, 3, 256, 16, 16, 16, 16)
DFFT_SLAB_INST(float, 160, 6, 2, 128, 8, 16, 16, 8)
DFFT_SLAB_INST(float, 160, 4, 3, 128, 8, 16, 16, 8)
// ComplexF64, L = 512 and 256
DFFT_SLAB_INST(double, 160, 4, 2, 512, 64, 2, 8, 8, 8)
DFFT_SLAB_INST(double, 160, 5, 2, 512, 64, 2, 8, 8, 8)
DFFT_SLAB_INST(double, 160, 3, 3, 512, 64, 2, 8, 8, 8)
DFFT_SLAB_INST(double, 96, 5, 2, 256, 16, 4, 16, 16)
DFFT_SLAB_INST(double, 96, 6, 2, 256, 16, 4, 16, 16)
DFFT_SLAB_INST(double, 96, 3, 3, 256, 16, 4, 16, 16)

// Variants of one (precision, L) are listed fastest first (B200, 512^3 /
// 256^3 / 128^3 arrays); `dflt` marks the ones an untuned plan may use (at
// L = 128 the per-axis passes are faster, so only DFFT_FLAG_TUNE or
// DFFT_FLAG_FUSE selects the fused kernel there).
static const SlabKernel kSlabKernels[] = {
    // dbl, L, P, nst, radices, threads, CS, NB, dflt, forward and inverse kernels
    {0, 512, 16, 2, {32, 16}, 160, 8, 2, 1, K(float, 160, 3, 2, 512, 16, 8, 32, 16)},
    {0, 512, 32, 3, {8, 8, 8}, 160, 4, 2, 1, K(float, 160, 6, 2, 512, 32, 4, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 160, 4, 2, 1, K(float, 160, 5, 2, 512, 32, 4, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 160, 4, 3, 1, K(float, 160, 4, 3, 512, 32, 4, 8, 8, 8)},
    {0, 512, 64, 3, {8, 8, 8}, 288, 4, 2, 1, K(float, 288, 4, 2, 512, 64, 4, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 288, 8, 3, 1, K(float, 288, 2, 3, 512, 32, 8, 8, 8, 8)},
    {0, 256, 16, 2, {16, 16}, 160, 8, 2, 1, K(float, 160, 6, 2, 256, 16, 8, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 160, 8, 2, 1, K(float, 160, 5, 2, 256, 16, 8, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 160, 8, 3, 1, K(float, 160, 4, 3, 256, 16, 8, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 288, 16, 3, 1, K(float, 288, 2, 3, 256, 16, 16, 16, 16)},
    {0, 128, 8, 2, {16, 8}, 160, 16, 2, 0, K(float, 160, 6, 2, 128, 8, 16, 16, 8)},
    {0, 128, 8, 2, {16, 8}, 160, 16, 3, 0, K(float, 160, 4, 3, 128, 8, 16, 16, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 160, 2, 2, 1, K(double, 160, 5, 2, 512, 64, 2, 8, 8, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 160, 2, 2, 1, K(double, 160, 4, 2, 512, 64, 2, 8, 8, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 160, 2, 3, 1, K(double, 160, 3, 3, 512, 64, 2, 8, 8, 8)},
    {1, 256, 16, 2, {16, 16}, 96, 4, 2, 1, K(double, 96, 6, 2, 256, 16, 4, 16, 16)},
    {1, 256, 16, 2, {16, 16}, 96, 4, 2, 1, K(double, 96, 5, 2, 256, 16, 4, 16, 16)},
    {1, 256, 16, 2, {16, 16}, 96, 4, 3, 1, K(double, 96, 3, 3, 256, 16, 4, 16, 16)},
};

#undef K

const SlabKernel* find_slab_kernel(int dbl, int L, int v) {
  int i = 0;
  for (const SlabKernel& k : kSlabKernels)
    if (k.dbl == dbl && k.L == L && i++ == v) return &k;
  return nullptr;
}

}  // namespace dfft
