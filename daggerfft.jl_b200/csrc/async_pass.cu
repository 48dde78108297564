// Instantiations of the cp.async strided axis pass (axis_pass_async) and its
// launch shapes, fastest first.  threads = CS*P (all run the stages); MINB =
// CTAs per SM that the NB tile buffers of CS*L elements leave room for.
// ComplexF32 only: a ComplexF64 row is a 16-byte multiple, which TMA
// addresses (axis_pass_strided).
#include "dfft_internal.h"

namespace dfft {

#define DFFT_ASYNC_INST1(T, LB, MINB, NB, DIR, L, P, CS, ...)                                         \
  template __global__ void axis_pass_async<T, LB, MINB, NB, DIR, L, P, CS, __VA_ARGS__>(const PassDesc, \
                                                                                       const AsyncGeom);
#define DFFT_ASYNC_INST(T, LB, MINB, NB, L, P, CS, ...)        \
  DFFT_ASYNC_INST1(T, LB, MINB, NB, 1, L, P, CS, __VA_ARGS__)   \
  DFFT_ASYNC_INST1(T, LB, MINB, NB, 2, L, P, CS, __VA_ARGS__)
#define K(T, LB, MINB, NB, L, P, CS, ...)                                        \
  (const void*)&axis_pass_async<T, LB, MINB, NB, 1, L, P, CS, __VA_ARGS__>,     \
      (const void*)&axis_pass_async<T, LB, MINB, NB, 2, L, P, CS, __VA_ARGS__>

DFFT_ASYNC_INST(float, 128, 3, 2, 512, 16, 8, 32, 16)
DFFT_ASYNC_INST(float, 256, 1, 2, 512, 16, 16, 32, 16)
DFFT_ASYNC_INST(float, 256, 3, 2, 256, 16, 16, 16, 16)
DFFT_ASYNC_INST(float, 128, 6, 2, 256, 16, 8, 16, 16)
DFFT_ASYNC_INST(float, 128, 6, 2, 128, 8, 16, 16, 8)
DFFT_ASYNC_INST(float, 128, 6, 2, 64, 8, 16, 8, 8)
DFFT_ASYNC_INST(float, 128, 6, 2, 96, 8, 16, 12, 8)
DFFT_ASYNC_INST(float, 192, 4, 2, 192, 12, 16, 12, 16)
DFFT_ASYNC_INST(float, 384, 2, 2, 384, 48, 8, 6, 8, 8)

// `dflt`: an untuned plan uses the shape.  Measured (B200, dim-2 pass of a
// Float32 rfft's half spectrum): 257 x 512 x 512 0.272 ms against 0.367 for
// the one-tile direct kernel; 129 x 256 x 256 0.047 against 0.035 (there the
// direct kernel's six CTAs per SM hide the load latency better), so the
// other lengths are tuner candidates only.  Three buffers of the first
// shape (200 KB, leaving little L1 for the 8-byte copies) measured 0.364 ms.
static const SlabKernel kAsyncKernels[] = {
    // dbl, L, P, nst, radices, threads, CS, NB, dflt, forward and inverse kernels
    {0, 512, 16, 2, {32, 16}, 256, 16, 2, 1, K(float, 256, 1, 2, 512, 16, 16, 32, 16)},
    {0, 512, 16, 2, {32, 16}, 128, 8, 2, 0, K(float, 128, 3, 2, 512, 16, 8, 32, 16)},
    {0, 256, 16, 2, {16, 16}, 256, 16, 2, 0, K(float, 256, 3, 2, 256, 16, 16, 16, 16)},
    {0, 256, 16, 2, {16, 16}, 128, 8, 2, 0, K(float, 128, 6, 2, 256, 16, 8, 16, 16)},
    {0, 128, 8, 2, {16, 8}, 128, 16, 2, 0, K(float, 128, 6, 2, 128, 8, 16, 16, 8)},
    {0, 64, 8, 2, {8, 8}, 128, 16, 2, 0, K(float, 128, 6, 2, 64, 8, 16, 8, 8)},
    {0, 96, 8, 2, {12, 8}, 128, 16, 2, 0, K(float, 128, 6, 2, 96, 8, 16, 12, 8)},
    {0, 192, 12, 2, {12, 16}, 192, 16, 2, 0, K(float, 192, 4, 2, 192, 12, 16, 12, 16)},
    {0, 384, 48, 3, {6, 8, 8}, 384, 8, 2, 0, K(float, 384, 2, 2, 384, 48, 8, 6, 8, 8)},
};

const SlabKernel* find_async_kernel(int dbl, int L, int v) {
  int seen = 0;
  for (const SlabKernel& k : kAsyncKernels)
    if (k.dbl == dbl && k.L == L && seen++ == v) return &k;
  return nullptr;
}

}  // namespace dfft
