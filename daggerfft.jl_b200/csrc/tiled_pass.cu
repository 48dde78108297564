// Instantiations of the tile-staged R2R pass (tiled_pass) for DCT-II and
// DCT-III: FFT lengths 128, 256, 512, contiguous (whole pencils) and strided
// (column tiles) axes.  threads = C*P stage threads + one producer warp;
// two tile buffers.
#include "dfft_internal.h"

namespace dfft {

#define DFFT_TILED_INST(T, LB, MINB, S, K, L, P, C, ...)                                              \
  template __global__ void tiled_pass<T, LB, MINB, 2, S, K, L, P, C, __VA_ARGS__>(                   \
      const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap,       \
      const TiledGeom);
#define DFFT_TILED_BOTH(T, LB, MINB, S, L, P, C, ...)        \
  DFFT_TILED_INST(T, LB, MINB, S, 5, L, P, C, __VA_ARGS__)   \
  DFFT_TILED_INST(T, LB, MINB, S, 4, L, P, C, __VA_ARGS__)
#define K(T, LB, MINB, S, KIND, L, P, C, ...) (const void*)&tiled_pass<T, LB, MINB, 2, S, KIND, L, P, C, __VA_ARGS__>

// kinds 5 = REDFT10 (DCT-II), 4 = REDFT01 (DCT-III)
DFFT_TILED_BOTH(double, 160, 3, 0, 128, 8, 16, 16, 8)
DFFT_TILED_BOTH(double, 160, 3, 1, 128, 8, 16, 16, 8)
DFFT_TILED_BOTH(double, 160, 3, 0, 256, 16, 8, 16, 16)
DFFT_TILED_BOTH(double, 160, 3, 1, 256, 16, 8, 16, 16)
DFFT_TILED_BOTH(double, 160, 3, 0, 512, 64, 2, 8, 8, 8)
DFFT_TILED_BOTH(double, 288, 2, 1, 512, 64, 4, 8, 8, 8)
DFFT_TILED_BOTH(float, 160, 3, 0, 128, 8, 16, 16, 8)
DFFT_TILED_BOTH(float, 160, 3, 1, 128, 8, 16, 16, 8)
DFFT_TILED_BOTH(float, 160, 3, 0, 256, 16, 8, 16, 16)
DFFT_TILED_BOTH(float, 288, 2, 1, 256, 16, 16, 16, 16)
DFFT_TILED_BOTH(float, 160, 3, 0, 512, 64, 2, 8, 8, 8)
DFFT_TILED_BOTH(float, 288, 2, 1, 512, 64, 4, 8, 8, 8)

#define E(DBL, T, LB, MINB, S, L, P, NST, RAD, C, ...)                                             \
  {DBL, L, P, NST, RAD, LB, C, S, 5, K(T, LB, MINB, S, 5, L, P, C, __VA_ARGS__)},                 \
      {DBL, L, P, NST, RAD, LB, C, S, 4, K(T, LB, MINB, S, 4, L, P, C, __VA_ARGS__)}
#define R2(a, b) {a, b}
#define R3(a, b, c) {a, b, c}

static const TiledKernel kTiledKernels[] = {
    // dbl, L, P, nst, radices, threads, C, strided, kind, kernel
    E(1, double, 160, 3, 0, 128, 8, 2, R2(16, 8), 16, 16, 8),
    E(1, double, 160, 3, 1, 128, 8, 2, R2(16, 8), 16, 16, 8),
    E(1, double, 160, 3, 0, 256, 16, 2, R2(16, 16), 8, 16, 16),
    E(1, double, 160, 3, 1, 256, 16, 2, R2(16, 16), 8, 16, 16),
    E(1, double, 160, 3, 0, 512, 64, 3, R3(8, 8, 8), 2, 8, 8, 8),
    E(1, double, 288, 2, 1, 512, 64, 3, R3(8, 8, 8), 4, 8, 8, 8),
    E(0, float, 160, 3, 0, 128, 8, 2, R2(16, 8), 16, 16, 8),
    E(0, float, 160, 3, 1, 128, 8, 2, R2(16, 8), 16, 16, 8),
    E(0, float, 160, 3, 0, 256, 16, 2, R2(16, 16), 8, 16, 16),
    E(0, float, 288, 2, 1, 256, 16, 2, R2(16, 16), 16, 16, 16),
    E(0, float, 160, 3, 0, 512, 64, 3, R3(8, 8, 8), 2, 8, 8, 8),
    E(0, float, 288, 2, 1, 512, 64, 3, R3(8, 8, 8), 4, 8, 8, 8),
};

#undef E
#undef K

const TiledKernel* find_tiled_kernel(int dbl, int L, int strided, int kind) {
  for (const TiledKernel& k : kTiledKernels)
    if (k.dbl == dbl && k.L == L && k.strided == strided && k.kind == kind) return &k;
  return nullptr;
}

}  // namespace dfft
