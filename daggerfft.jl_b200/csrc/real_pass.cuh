// Pipelined real passes along the contiguous axis: the R2C first pass of
// rfft and the C2R last pass of irfft (apply_fft! with the RFFT/IRFFT tags,
// src/fft.jl:146-174, src/fftgpu.jl:85-124), as one half-length complex FFT
// between a pack step and a twiddle step.
//
//   R2C, real length 2M:  z_m = x_{2m} + i x_{2m+1}  (the real pencil read
//   as M complex pairs), Z = FFT_M(z), and for k = 0..M
//     X_k = E_k + w^k O_k,  E_k = (Z_k + conj Z_{M-k})/2,
//                           O_k = -i (Z_k - conj Z_{M-k})/2,  w = e^{-2 pi i/2M}.
//   C2R: Z'_k = (A + B) + i conj(w^k) (A - B) with A = X_k,
//   B = conj X_{M-k} (Im X_0 and Im X_M ignored), z = IFFT_M(Z') / (2M),
//   x_{2m} = Re z_m, x_{2m+1} = Im z_m.
//
// Persistent CTAs of C*P stage threads plus one producer warp.  A tile is C
// consecutive pencils: its input and its output are each one contiguous run
// in global memory (C*M or C*(M+1) complex elements), moved into / out of an
// NB-deep ring of tile buffers by 1-D bulk copies that the producer issues
// (the store when the stage threads hand the buffer back, before refilling
// it).  The side of M elements per pencil sits in the buffer with the
// pencils PS = M + 64 bytes apart (one bulk copy per pencil; M complex
// elements are a 16-byte multiple), so the pencils a warp reads or writes
// at once alternate between the two halves of the banks instead of all
// mapping onto the same ones; the side of M+1 elements stays dense (one
// bulk copy) and the pack / unpack step walks it in the flattened
// [pencil][k] order, 32 consecutive elements per warp.  R2C: the stages read
// the padded tile and run in a padded work buffer; the post-pass writes the
// M+1 outputs of each pencil back into the (consumed) tile buffer.  C2R: the
// pre-pass reads the dense tile and writes the work buffer; the stages end
// in the padded tile.
// The stage twiddles and the M+1 entries of w^k sit in shared memory.
// Waits are bounded as in the other pipelined passes.
#pragma once
#include "slab_pass.cuh"

namespace dfft {

struct RealGeom {
  long long ntiles;  // pencils / C
  int ntw;           // stage-twiddle entries
  int ld;            // padded work-buffer elements per pencil
  int bstride;       // elements between tile buffers (128-byte multiple)
  int* err;
};

// DIR: 1 = R2C (forward), 2 = C2R (inverse).  d.L = M; d.tw: stage
// twiddles; d.tw2: w^k = exp(-2 pi i k / 2M), k = 0..M.
template <typename T, int LB, int MINB, int NB, int DIR, int M, int P, int C, int... Rs>
__global__ void __launch_bounds__(LB, MINB) real_pass(const PassDesc d, const RealGeom g) {
  typedef typename cvec<T>::type V;
  constexpr int NC = C * P;
  static_assert(NC % 32 == 0 && NC + 32 == LB, "whole warps of stage threads plus one producer warp");
  static_assert(NB >= 2 && NB <= 4, "tile buffers");
  constexpr int IN_E = DIR == 1 ? M : M + 1;   // complex elements per input pencil
  constexpr int OUT_E = DIR == 1 ? M + 1 : M;  // and per output pencil
  constexpr int PS = M + 64 / (int)sizeof(V);  // pencil stride of the M-element side in a buffer
  extern __shared__ __align__(128) unsigned char smem_real[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_real);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem_real + 32);
  int& s_cabort = *reinterpret_cast<int*>(smem_real + 64);
  long long* s_tile = reinterpret_cast<long long*>(smem_real + 80);  // NB entries
  V* stw = reinterpret_cast<V*>(smem_real + kSlabHeader);
  V* sw = stw + g.ntw;  // M+1 entries of w^k
  const size_t tw_bytes = ((size_t)(g.ntw + M + 1) * sizeof(V) + 127) & ~(size_t)127;
  V* bufs = reinterpret_cast<V*>(smem_real + kSlabHeader + tw_bytes);
  const size_t bst = (size_t)g.bstride;
  V* work = bufs + NB * bst;
  const int tid = threadIdx.x;
  volatile int* verr = g.err;

  if (tid == 0) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_fence_init();
    s_cabort = 0;
    if ((smem_u32(bufs) & 127u) || ((bst * sizeof(V)) & 127u)) {
      atomicExch(g.err, DFFT_DEVERR_TMA_ALIGN);
      s_cabort = 1;
    }
  }
  {
    const V* gt = reinterpret_cast<const V*>(d.tw);
    for (int i = tid; i < g.ntw; i += blockDim.x) stw[i] = gt[i];
    const V* gw = reinterpret_cast<const V*>(d.tw2);
    for (int i = tid; i <= M; i += blockDim.x) sw[i] = gw[i];
  }
  __syncthreads();

  if (tid >= NC) {
    if (tid == NC) {
      // ---------------- producer ----------------
      const uint32_t in_bytes = (uint32_t)((size_t)C * IN_E * sizeof(V));
      const uint32_t out_bytes = (uint32_t)((size_t)C * OUT_E * sizeof(V));
      const V* src = reinterpret_cast<const V*>(d.in.p);
      V* dst = reinterpret_cast<V*>(d.out.p);
      int fills[NB] = {};
      long long pend[NB];  // transformed tile in buffer b still to be stored, or -1
      for (int bb = 0; bb < NB; ++bb) pend[bb] = -1;
      bool failed = false;
      // waits until the stage threads hand buffer b back, then stores its
      // tile and waits until the store has read the buffer
      auto drain = [&](int b) -> bool {
        if (pend[b] < 0) return true;
        if (!mbar_wait_bounded(&empty[b], (uint32_t)((fills[b] - 1) & 1))) return false;
        if constexpr (DIR == 1) {
          bulk_store_1d(dst + pend[b] * C * OUT_E, bufs + b * bst, out_bytes);
        } else {
          for (int cc = 0; cc < C; ++cc)
            bulk_store_1d(dst + (pend[b] * C + cc) * M, bufs + b * bst + cc * PS, (uint32_t)(M * sizeof(V)));
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
        mbar_expect_tx(&full[b], in_bytes);
        if constexpr (DIR == 1) {
          for (int cc = 0; cc < C; ++cc)
            bulk_load_1d(bufs + b * bst + cc * PS, src + (tile * C + cc) * M, (uint32_t)(M * sizeof(V)), &full[b]);
        } else {
          bulk_load_1d(bufs + b * bst, src + tile * C * IN_E, in_bytes, &full[b]);
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
    const StageTw<V> tw{stw};
    const int t = tid % P, c = tid / P;
    const PadCol<V> pad{work + (size_t)c * g.ld};
    for (int it = 0;; ++it) {
      const int b = it % NB;
      if (!mbar_wait_bounded(&full[b], (uint32_t)((it / NB) & 1))) s_cabort = 1;
      stage_sync<NC>();
      if (s_cabort) break;
      const long long tile = s_tile[b];
      if (tile < 0) break;
      V* buf = bufs + b * bst;
      if constexpr (DIR == 1) {
        const StrideCol<V> padded{buf + (size_t)c * PS, 1};
        static_stages<T, M, P, true, 1, NC, 1, 1, 1, 0, StrideCol<V>, PadCol<V>, PadCol<V>, StageTw<V>, Rs...>(
            d, t, padded, pad, pad, tw, 0, 0, true);
        // post-pass: X_k of pencil cc, k = 0..M, into the consumed tile
        // buffer, dense: element e = cc*(M+1) + k
        for (int e = tid; e < C * (M + 1); e += NC) {
          const int cc = e / (M + 1), k = e - cc * (M + 1);
          const PadCol<V> z{work + (size_t)cc * g.ld};
          const V zk = z.ld(k == M ? 0 : k, 0);
          const V zm = cconj(z.ld(k == 0 ? 0 : M - k, 0));
          const V ev = cscale(cadd(zk, zm), (T)0.5);
          const V od = cscale(cmul_mi(csub(zk, zm)), (T)0.5);
          buf[e] = cscale(cadd(ev, cmul(sw[k], od)), (T)d.scale);
        }
      } else {
        // pre-pass: Z'_k of pencil cc, k = 0..M-1, from the dense tile
        // (element cc*(M+1) + k) into the work buffer
        for (int e = tid; e < C * M; e += NC) {
          const int cc = e / M, k = e - cc * M;
          const V* x = buf + (size_t)cc * (M + 1);
          V A = x[k];
          V B = cconj(x[M - k]);
          if (k == 0) {
            A.y = (T)0;
            B.y = (T)0;
          }
          const PadCol<V> z{work + (size_t)cc * g.ld};
          z.st(k, 0, cadd(cadd(A, B), cmul_pi(cmul(cconj(sw[k]), csub(A, B)))));
        }
        stage_sync<NC>();
        const StrideCol<V> padded{buf + (size_t)c * PS, 1};
        static_stages<T, M, P, true, 1, NC, 2, 1, 1, 0, PadCol<V>, PadCol<V>, StrideCol<V>, StageTw<V>, Rs...>(
            d, t, pad, pad, padded, tw, 0, 0, true);
      }
      fence_proxy_async_smem();  // the producer's bulk store reads the tile next
      stage_sync<NC>();
      if (tid == 0) mbar_arrive(&empty[b]);  // hand the transformed tile to the producer
    }
    if (tid == 0 && s_cabort && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
  }
  __syncthreads();
}

}  // namespace dfft
