// Instantiations of the fused 2-D slab pass and the launch variants the
// planner chooses from.  The radices are those of the static plan for the
// same length (the stage twiddle table is built from them); the planner
// checks that they agree.
#include "dfft_internal.h"

namespace dfft {

#define DFFT_SLAB_INST(T, LB, MINB, L, P, CS, ...)                                                     \
  template __global__ void slab_xy_pass<T, LB, MINB, L, P, CS, __VA_ARGS__>(                         \
      const PassDesc, const PassDesc, const __grid_constant__ CUtensorMap, const SlabGeom);

// ComplexF32, L = 512 (8 x 8 x 8): tiles of 2-8 pencils, one or two radix-8
// butterflies per thread and stage
DFFT_SLAB_INST(float, 160, 4, 512, 32, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 288, 2, 512, 32, 8, 8, 8, 8)
DFFT_SLAB_INST(float, 96, 4, 512, 16, 4, 8, 8, 8)
DFFT_SLAB_INST(float, 160, 2, 512, 16, 8, 8, 8, 8)
DFFT_SLAB_INST(float, 544, 2, 512, 64, 8, 8, 8, 8)
DFFT_SLAB_INST(float, 288, 4, 512, 64, 4, 8, 8, 8)
// ComplexF32, L = 256 (16 x 16) and 128 (16 x 8)
DFFT_SLAB_INST(float, 160, 4, 256, 16, 8, 16, 16)
DFFT_SLAB_INST(float, 288, 2, 256, 16, 16, 16, 16)
DFFT_SLAB_INST(float, 96, 8, 256, 16, 4, 16, 16)
DFFT_SLAB_INST(float, 160, 4, 128, 8, 16, 16, 8)
DFFT_SLAB_INST(float, 96, 8, 128, 8, 8, 16, 8)
// ComplexF64, L = 512 and 256
DFFT_SLAB_INST(double, 288, 1, 512, 64, 4, 8, 8, 8)
DFFT_SLAB_INST(double, 160, 3, 512, 64, 2, 8, 8, 8)
DFFT_SLAB_INST(double, 96, 3, 256, 16, 4, 16, 16)
DFFT_SLAB_INST(double, 160, 1, 256, 16, 8, 16, 16)

#define K(T, LB, MINB, L, P, CS, ...) (const void*)&slab_xy_pass<T, LB, MINB, L, P, CS, __VA_ARGS__>

static const SlabKernel kSlabKernels[] = {
    // dbl, L, P, nst, radices, threads (stage threads + producer warp), CS, kernel
    {0, 512, 32, 3, {8, 8, 8}, 160, 4, K(float, 160, 4, 512, 32, 4, 8, 8, 8)},
    {0, 512, 32, 3, {8, 8, 8}, 288, 8, K(float, 288, 2, 512, 32, 8, 8, 8, 8)},
    {0, 512, 16, 3, {8, 8, 8}, 96, 4, K(float, 96, 4, 512, 16, 4, 8, 8, 8)},
    {0, 512, 16, 3, {8, 8, 8}, 160, 8, K(float, 160, 2, 512, 16, 8, 8, 8, 8)},
    {0, 512, 64, 3, {8, 8, 8}, 544, 8, K(float, 544, 2, 512, 64, 8, 8, 8, 8)},
    {0, 512, 64, 3, {8, 8, 8}, 288, 4, K(float, 288, 4, 512, 64, 4, 8, 8, 8)},
    {0, 256, 16, 2, {16, 16}, 160, 8, K(float, 160, 4, 256, 16, 8, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 288, 16, K(float, 288, 2, 256, 16, 16, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 96, 4, K(float, 96, 8, 256, 16, 4, 16, 16)},
    {0, 128, 8, 2, {16, 8}, 160, 16, K(float, 160, 4, 128, 8, 16, 16, 8)},
    {0, 128, 8, 2, {16, 8}, 96, 8, K(float, 96, 8, 128, 8, 8, 16, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 160, 2, K(double, 160, 3, 512, 64, 2, 8, 8, 8)},
    {1, 512, 64, 3, {8, 8, 8}, 288, 4, K(double, 288, 1, 512, 64, 4, 8, 8, 8)},
    {1, 256, 16, 2, {16, 16}, 96, 4, K(double, 96, 3, 256, 16, 4, 16, 16)},
    {1, 256, 16, 2, {16, 16}, 160, 8, K(double, 160, 1, 256, 16, 8, 16, 16)},
};

#undef K

const SlabKernel* find_slab_kernel(int dbl, int L, int v) {
  int i = 0;
  for (const SlabKernel& k : kSlabKernels)
    if (k.dbl == dbl && k.L == L && i++ == v) return &k;
  return nullptr;
}

}  // namespace dfft
