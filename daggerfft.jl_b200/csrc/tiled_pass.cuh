// Tile-staged R2R passes for DCT-II / DCT-III (FFTW REDFT10 / REDFT01, the
// R2R(...) kinds of src/fft.jl:1-11 the README's 2-D DCT uses): a producer
// warp moves whole input tiles into NB shared-memory buffers -- C whole
// pencils by one 1-D bulk copy along the contiguous axis (STRIDED = 0), C
// columns x n rows by TMA boxes of the real tensor {I, n, O} along a strided
// axis (STRIDED = 1) -- and the stage threads run the stages with the kind's
// load map (first stage) and store map (last stage) applied while reading
// and writing the tile, compiled in for the kind (r2r_load / r2r_store);
// every read of a tile precedes the first stage's barrier, so the output
// overwrites the input in place, and the tile leaves by the same kind of
// copy, which the producer issues when the buffer is handed back.  The FFT runs in a padded complex work buffer, one column per C.
// Bounded waits as in the other pipelined passes.
#pragma once
#include "real_pass.cuh"

namespace dfft {

// The tile of one column / pencil seen through a kind's maps (stride S
// between its elements: C in a strided tile, 1 in a contiguous one).
template <typename T, int KIND, int S> struct R2RLoadView {
  typedef typename cvec<T>::type V;
  const T* p;
  int N;
  const V* w;
  __device__ __forceinline__ V ld(int b, int off) const { return r2r_load<T, KIND>(p, 0, S, N, w, b + off); }
};
template <typename T, int KIND, int S> struct R2RStoreView {
  typedef typename cvec<T>::type V;
  T* p;
  int N;
  const V* w;
  __device__ __forceinline__ void st(int b, int off, V v) const {
    r2r_store<T, KIND>(p, 0, S, N, w, b + off, v, (T)1);
  }
};

struct TiledGeom {
  long long ntiles;  // contiguous: pencils / C; strided: tiles_i * O
  int tiles_i;       // strided: tiles along I
  int n_in, n_out;   // elements per pencil / rows per column (side type T)
  int lb, nlb;       // strided: rows per TMA box, boxes per tile
  int ld;            // padded complex work elements per column
  int bstride;       // bytes between tile buffers (128-byte multiple)
  const void* src;   // global input
  void* dst;         // global output
  int* err;
};

template <typename T, int LB, int MINB, int NB, int STRIDED, int KIND, int L, int P, int C, int... Rs>
__global__ void __launch_bounds__(LB, MINB)
    tiled_pass(const PassDesc d, const __grid_constant__ CUtensorMap tin,
               const __grid_constant__ CUtensorMap tout, const TiledGeom g) {
  typedef typename cvec<T>::type V;
  constexpr int NC = C * P;
  static_assert(NC % 32 == 0 && NC + 32 == LB, "whole warps of stage threads plus one producer warp");
  static_assert(NB >= 2 && NB <= 4, "tile buffers");
  extern __shared__ __align__(128) unsigned char smem_tiled[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_tiled);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem_tiled + 32);
  int& s_cabort = *reinterpret_cast<int*>(smem_tiled + 64);
  long long* s_tile = reinterpret_cast<long long*>(smem_tiled + 80);  // NB entries
  unsigned char* bufs = smem_tiled + kSlabHeader;
  const size_t bst = (size_t)g.bstride;
  V* work = reinterpret_cast<V*>(bufs + NB * bst);
  const int tid = threadIdx.x;
  volatile int* verr = g.err;

  if (tid == 0) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_fence_init();
    s_cabort = 0;
    if ((smem_u32(bufs) & 127u) || (bst & 127u) ||
        (STRIDED && g.nlb > 1 && (((size_t)g.lb * C * sizeof(T)) & 127u))) {
      atomicExch(g.err, DFFT_DEVERR_TMA_ALIGN);
      s_cabort = 1;
    }
  }
  __syncthreads();

  if (tid >= NC) {
    if (tid == NC) {
      // ---------------- producer ----------------
      const uint32_t in_bytes = (uint32_t)((size_t)C * g.n_in * sizeof(T));
      const uint32_t out_bytes = (uint32_t)((size_t)C * g.n_out * sizeof(T));
      int fills[NB] = {};
      long long pend[NB];  // transformed tile in buffer b still to be stored, or -1
      for (int bb = 0; bb < NB; ++bb) pend[bb] = -1;
      bool failed = false;
      // waits until the stage threads hand buffer b back, then stores its
      // tile and waits until the store has read the buffer
      auto drain = [&](int b) -> bool {
        if (pend[b] < 0) return true;
        if (!mbar_wait_bounded(&empty[b], (uint32_t)((fills[b] - 1) & 1))) return false;
        unsigned char* buf = bufs + b * bst;
        if (STRIDED) {
          const int ti = (int)(pend[b] % g.tiles_i);
          const int o = (int)(pend[b] / g.tiles_i);
          for (int kb = 0; kb < g.nlb; ++kb)
            tma_store_3d(&tout, buf + (size_t)kb * g.lb * C * sizeof(T), ti * C, kb * g.lb, o);
        } else {
          bulk_store_1d(reinterpret_cast<T*>(g.dst) + pend[b] * C * g.n_out, buf, out_bytes);
        }
        bulk_commit();
        bulk_wait_read_all();
        pend[b] = -1;
        return true;
      };
      long long tile = blockIdx.x;
      for (int it = 0;; ++it) {
        const int b = it % NB;
        if (!drain(b)) {
          failed = true;
          break;
        }
        const bool more = tile < g.ntiles && *verr == 0 && !s_cabort;
        s_tile[b] = more ? tile : -1;
        ++fills[b];
        if (!more) {
          mbar_arrive(&full[b]);
          break;
        }
        unsigned char* buf = bufs + b * bst;
        mbar_expect_tx(&full[b], in_bytes);
        if (STRIDED) {
          const int ti = (int)(tile % g.tiles_i);
          const int o = (int)(tile / g.tiles_i);
          for (int kb = 0; kb < g.nlb; ++kb)
            tma_load_3d(buf + (size_t)kb * g.lb * C * sizeof(T), &tin, &full[b], ti * C, kb * g.lb, o);
        } else {
          bulk_load_1d(buf, reinterpret_cast<const T*>(g.src) + tile * C * g.n_in, in_bytes, &full[b]);
        }
        pend[b] = tile;
        tile += gridDim.x;
      }
      for (int bb = 0; bb < NB && !failed; ++bb)
        if (!drain(bb)) failed = true;
      if (failed && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
      bulk_wait_all();
      for (int bb = 0; bb < NB; ++bb)
        if (fills[bb] > 0) mbar_wait_bounded(&full[bb], (uint32_t)((fills[bb] - 1) & 1));
    }
  } else {
    // ---------------- stage threads ----------------
    const int c = STRIDED ? tid % C : tid / P;
    const int t = STRIDED ? tid / C : tid % P;
    const PadCol<V> col{work + (size_t)c * g.ld};
    const GlobalTw<V> tw{reinterpret_cast<const V*>(d.tw)};
    constexpr int S = STRIDED ? C : 1;
    constexpr int DIR = KIND == K_REDFT01 ? 2 : 1;  // REDFT01 runs as an inverse FFT
    typedef R2RLoadView<T, KIND, S> In;
    typedef R2RStoreView<T, KIND, S> Out;
    // the tile's element (column c, row / element k) sits at c + k*C
    // (strided) or c*n + k (contiguous)
    const size_t ib = STRIDED ? c : (size_t)c * g.n_in;
    const size_t ob = STRIDED ? c : (size_t)c * g.n_out;
    const V* w_in = reinterpret_cast<const V*>(d.in.w);
    const V* w_out = reinterpret_cast<const V*>(d.out.w);
    for (int it = 0;; ++it) {
      const int b = it % NB;
      if (!mbar_wait_bounded(&full[b], (uint32_t)((it / NB) & 1))) s_cabort = 1;
      stage_sync<NC>();
      if (s_cabort) break;
      const long long tile = s_tile[b];
      if (tile < 0) break;
      unsigned char* buf = bufs + b * bst;
      const In in{reinterpret_cast<const T*>(buf) + ib, d.in.n, w_in};
      const Out out{reinterpret_cast<T*>(buf) + ob, d.out.n, w_out};
      static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, In, PadCol<V>, Out, GlobalTw<V>, Rs...>(d, t, in, col, out,
                                                                                            tw, 0, 0, true);
      fence_proxy_async_smem();  // the producer's store reads the tile next
      stage_sync<NC>();
      if (tid == 0) mbar_arrive(&empty[b]);  // hand the transformed tile to the producer
    }
    if (tid == 0 && s_cabort && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
  }
  __syncthreads();
}

}  // namespace dfft
