// Mixed-precision tensor-core axis pass for ComplexF32 length 512 (the
// "mixed" arithmetic form): the 512-point DFT of every pencil runs as two
// dense complex matrix products on the 5th-generation tensor cores,
//
//   n = 16*n1 + n2, k = k1 + 32*k2   (n1, k1 < 32; n2, k2 < 16)
//   stage A: Y[n2, k1] = sum_n1 x[16 n1 + n2] W32^(n1 k1)       (radix 32)
//   twiddle: Y'[n2, k1] = Y[n2, k1] W512^(n2 k1)                 (FP32, CUDA cores)
//   stage B: X[k1 + 32 k2] = sum_n2 Y'[n2, k1] W16^(n2 k2)       (radix 16)
//
// Each product is a real GEMM over interleaved-free (re block, im block)
// vectors: D[M = pencil rows][N = 2 x outputs] = A[M][K = 2 x inputs] B[K][N]
// with B the real form [[Wr, Wi], [-Wi, Wr]] of the DFT matrix (K-major in
// shared memory, FP64-generated).  Operands are FP16 hi + lo splits of FP32
// values: D = A_hi B_hi + A_lo B_hi + A_hi B_lo, accumulated in FP32 in
// tensor memory (the dropped A_lo B_lo term and the split residuals are
// about 2^-22 of each value).  Per-pencil scaling: stage A's operands are
// scaled by a power of two sA that puts the pencil's largest |re|, |im| in
// [2^14, 2^15); stage B's by sA / 32 (|Y| <= 32 max|x|, so the bound holds
// without a second reduction, and the 1/32 rides on the twiddle table);
// the epilogue multiplies by 32 / sA (and 1/512 for the inverse), all exact
// powers of two.  The tensor cores round each MMA's FP32
// accumulation toward zero, so a long chain of K-steps into one accumulator
// shrinks every result by a few ulps (a bias that adds up over passes: a
// 12-step chain measured 1.75e-6 over a 4-pass round trip).  The products
// therefore go to separate accumulators -- the hi x hi part in chains of at
// most two K-steps, the two cross terms (about 2^-11 of it) in their own --
// which the epilogue adds in FP32 with round-to-nearest.  (An n-step chain
// shrinks the result, projected on itself, by about delta*(n+1)/2 with
// delta = 0.36 * 2^-23 per rounding: 6.5 + 3.5 delta per pass for one chain
// per stage, 1.5 + 1 delta with these splits.)  Before each split the values of one pencil
// are scaled by a power of two so that the pencil's largest |re|, |im|
// lies in [2^14, 2^15) (per-pencil scaling: FP16's range and the lo parts'
// precision follow each pencil's own magnitude); the scale is undone
// exactly after the product.  Twiddles and the inverse's 1/512 stay FP32 /
// exact.
//
// (Each value's FP16 hi + lo split keeps about 22 bits relative to the value
// itself, so a scale set by a bound rather than the exact maximum only
// matters for values far below the pencil's norm.)
//
// Tile: 16 pencils (columns of a strided axis, or whole contiguous pencils)
// x 512 points, 64 KB of ComplexF32, worked on by two groups of 8 pencils.
// Per group, stage A is M = 128 rows (pencil, n2) x N = 64 x K = 64, one
// M = 128 MMA per K-step; stage B is M = 256 rows (pencil, k1) x N = 32 x
// K = 32, two M = 128 MMAs per K-step.  TMEM (512 columns, 256 per group):
// stage A at +0 (hi x hi K-steps 0-1), +64 (K-steps 2-3), +128 (cross
// terms); stage B block j at 96 j (hi x hi K-step 0 at +0, K-step 1 at +32,
// cross terms at +64), reusing stage A's columns once its epilogue has read
// them.
//
// Warp roles (320 threads, one CTA per SM, persistent over tiles):
//   warps 0-7  convert / epilogue threads in two independent groups of four
//              warps, group gr owning pencils 8gr..8gr+7 of every tile with
//              its own operand buffer (32 KB), 256 TMEM columns and
//              barriers, so that one group's conversions overlap the other
//              group's products.  Thread tl of a group owns stage-A row tl =
//              (pencil tl/16, n2 = tl%16) -- its prep (FP32 tile -> scaled
//              FP16 hi/lo, K-major 128B-swizzled rows), its TMEM row in the
//              stage-A epilogue (unscale, twiddle, rescale, split into the
//              stage-B operand, MN-major 128B-swizzled) -- and two stage-B
//              rows (pencil, k1) in the final epilogue (unscale, store FP32).
//   warp 8     producer: TMA / bulk loads into two tile buffers, TMA / bulk
//              stores of finished tiles.
//   warp 9     TMEM allocation; lane 0 issues the tcgen05.mma products and
//              commits them to mbarriers.
// Every mbarrier wait is bounded (~2 s) and also gives up when another role
// has set the CTA's abort flag; on expiry the kernel records
// DFFT_DEVERR_TMA_TIMEOUT, waits (bounded) for its copies and products in
// flight, frees its tensor memory and returns.
#pragma once
#include <cuda_fp16.h>
#include "tma_pass.cuh"

namespace dfft {

struct MixedGeom {
  long long ntiles;   // tiles of 16 pencils
  long long ncols;    // contiguous: pencils (the last tile may be partial)
  int tiles_i;        // strided: tiles along the inner extent I
  int lb, nlb;        // strided: rows per TMA box, boxes per tile
  float out_scale;    // 1 (forward) or 1/512 (inverse), exact
  const unsigned char* consts;  // operand images of the DFT matrices + twiddles (kMixConstBytes)
  int* err;
};

// Shared-memory map (bytes from a 1024-byte aligned base).
constexpr int kMixTile = 16 * 512 * 8;          // one FP32 complex tile (64 KB)
constexpr int kMixOpA = 2 * kMixTile;           // operand hi (32 KB), lo at +32 KB
constexpr int kMixOpBytes = 32768;
constexpr int kMixB32 = kMixOpA + 2 * kMixOpBytes;  // DFT32 operand hi (8 KB), lo (8 KB)
constexpr int kMixB16 = kMixB32 + 16384;            // DFT16 operand hi (4 KB), lo (4 KB)
constexpr int kMixTw = kMixB16 + 8192;              // twiddles [n2][k1], rows of 33 (4224 B)
constexpr int kMixConstBytes = kMixTw + 16 * 33 * 8 - kMixB32;
constexpr int kMixMisc = kMixTw + 16 * 33 * 8;      // barriers, TMEM address, scales
constexpr int kMixSmem = kMixMisc + 256 + 1024;     // + alignment slack
constexpr int kMixThreads = 320;
constexpr int kMixTmemCols = 512;

// ---- tcgen05 wrappers -----------------------------------------------------

// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets, descriptor version 1, 128-byte swizzle.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  const uint32_t lo = ((saddr & 0x3FFFFu) >> 4) | ((lbo >> 4) << 16);
  const uint32_t hi = (sbo >> 4) | (1u << 14) | (2u << 29);
  return ((uint64_t)hi << 32) | lo;
}
// Instruction descriptor of kind::f16 with FP16 A and B, FP32 D.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N, int a_mn_major, int b_mn_major) {
  return (1u << 4) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// The same with the A operand in tensor memory (row m in lane m, K packed
// two FP16 values per 32-bit column).
__device__ __forceinline__ void umma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

#define DFFT_R8(i) "=r"(r[i]), "=r"(r[i + 1]), "=r"(r[i + 2]), "=r"(r[i + 3]), "=r"(r[i + 4]), \
                   "=r"(r[i + 5]), "=r"(r[i + 6]), "=r"(r[i + 7])
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : DFFT_R8(0), DFFT_R8(8), DFFT_R8(16), DFFT_R8(24)
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,"
      "%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
      : DFFT_R8(0), DFFT_R8(8), DFFT_R8(16), DFFT_R8(24), DFFT_R8(32), DFFT_R8(40), DFFT_R8(48), DFFT_R8(56)
      : "r"(taddr));
}
#define DFFT_W8(i) "r"(r[i]), "r"(r[i + 1]), "r"(r[i + 2]), "r"(r[i + 3]), "r"(r[i + 4]), \
                   "r"(r[i + 5]), "r"(r[i + 6]), "r"(r[i + 7])
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t* r) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      DFFT_W8(0), DFFT_W8(8), DFFT_W8(16), DFFT_W8(24)
      : "memory");
}
#undef DFFT_W8
#undef DFFT_R8

// Power-of-two scale that puts a pencil maximum m in [2^14, 2^15) (clamped
// so that the scale and its reciprocal are normal; m = 0 gives a harmless
// large scale).
__device__ __forceinline__ float mix_scale(float m) {
  int e = (int)((__float_as_uint(m) >> 23) & 0xFF);
  int b = 268 - e;
  b = b < 1 ? 1 : (b > 253 ? 253 : b);
  return __uint_as_float((uint32_t)b << 23);
}
// The reciprocal of a scale from mix_scale (exact: a power of two).
__device__ __forceinline__ float mix_inv(float s) {
  return __uint_as_float((254u - (__float_as_uint(s) >> 23)) << 23);
}
// x rounded to 11 significant bits (ties away from zero) with integer
// operations: the result is exactly representable in FP16 in its normal
// range, so its FP16 conversion is exact and the residual x - r11(x) is
// exact in FP32.  (Converting the FP16 hi part back to FP32 instead would
// run two more conversions per pair on the quarter-rate conversion pipe,
// which the FP16 packs already load.)
__device__ __forceinline__ float r11(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
// FP16 hi / lo split of a pair of FP32 values (already scaled).
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const float ha = r11(a), hb = r11(b);
  const __half2 h = __floats2half2_rn(ha, hb);
  const __half2 l = __floats2half2_rn(a - ha, b - hb);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}
__device__ __forceinline__ void sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
               : "memory");
}
__device__ __forceinline__ float2 lds64(uint32_t addr) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void sts64(uint32_t addr, float x, float y) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(x), "f"(y) : "memory");
}
// Bounded mbarrier wait that also leaves when the CTA's abort flag is set.
__device__ __forceinline__ bool mix_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned i = 1; i < kWaitLimit; ++i) {
    __nanosleep(32);  // leave the issue slots and the shared-memory pipe to the working warps
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > kWaitNs) return false;
    }
  }
  return false;
}
// Non-blocking test of a phase (try_wait may park the thread for a while,
// which a poller of several barriers cannot afford).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// The same wait with a warp-uniform result (every lane waits; the warp
// proceeds only if all lanes saw the phase complete), so that the
// .sync.aligned tensor-memory loads after it run converged.
__device__ __forceinline__ bool mix_wait_warp(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  const bool ok = mix_wait(bar, parity, abort_flag);
  return __all_sync(0xffffffffu, ok) != 0;
}

// Stage-B row blocks: M = pos(cl) * 32 + k1 for pencil cl (0..7) of a
// group: pencils 2q and 2q + 1 land in row blocks 0 and 1 of warp quarter
// q, the warp whose stage-A rows they were (so their scales are in its
// lanes), and a strided tile's final epilogue holds both columns of a
// 16-byte chunk of the 128-byte swizzled tile row.
__device__ __forceinline__ int mix_pos(int cl) { return 4 * (cl & 1) + (cl >> 1); }

// Byte offset of element (k, c) of a tile: strided tiles are [k][c] rows of
// 16 complex (128 bytes) in TMA's 128-byte swizzle; contiguous tiles are
// [c][k] pencils of 4 KB.
template <bool STRIDED> __device__ __forceinline__ uint32_t tile_off(int k, int c) {
  if constexpr (STRIDED) return (uint32_t)(k * 128 + ((((c >> 1) ^ (k & 7)) << 4) | ((c & 1) << 3)));
  else return (uint32_t)(c * 4096 + k * 8);
}

// STRIDED: the axis has element stride I > 1 (tile = 16 adjacent columns,
// TMA boxes {16, lb, 1} of the tensor {I, 512, O}); otherwise the axis is
// contiguous (tile = 16 whole pencils, one bulk copy).  The direction is in
// `consts` (DFT matrices and twiddles) and g.out_scale.
template <bool STRIDED>
__global__ void __launch_bounds__(kMixThreads, 1)
    mixed_pass(const void* in, void* out, const __grid_constant__ CUtensorMap tin,
               const __grid_constant__ CUtensorMap tout, const MixedGeom g) {
  extern __shared__ __align__(1024) unsigned char smem_mix_raw[];
  const uint32_t raw = smem_u32(smem_mix_raw);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  unsigned char* sm = smem_mix_raw + pad;
  const uint32_t sb = raw + pad;  // aligned base (shared address)
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kMixMisc);
  uint64_t* full = bars;        // [2] tile loaded
  uint64_t* outrdy = bars + 2;  // [2] tile transformed (both groups)
  uint64_t* opA = bars + 4;     // [2] per group: stage-A operands written
  uint64_t* opB = bars + 6;     // [2] stage-B operands written
  uint64_t* accA = bars + 8;    // [2] stage-A products done
  uint64_t* accB = bars + 10;   // [2] stage-B products done
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kMixMisc + 112);
  volatile int* s_abort = reinterpret_cast<volatile int*>(sm + kMixMisc + 116);
  volatile int* s_g0 = reinterpret_cast<volatile int*>(sm + kMixMisc + 120);  // group 0's last prepped tile
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  volatile int* verr = g.err;

  if (tid == 0) {
    // full, accA, accB: one arrival (expect_tx / tcgen05.commit); outrdy:
    // one per convert warp; opA, opB: one per warp of the group
    for (int i = 0; i < 12; ++i) mbar_init(&bars[i], (i < 2 || i >= 8) ? 1 : (i < 4 ? 8 : 4));
    mbar_fence_init();
    *s_abort = 0;
    *s_g0 = -1;
  }
  // constants: DFT operand images and the twiddle table
  {
    const uint4* src = reinterpret_cast<const uint4*>(g.consts);
    uint4* dst = reinterpret_cast<uint4*>(sm + kMixB32);
    for (int i = tid; i < kMixConstBytes / 16; i += kMixThreads) dst[i] = src[i];
  }
  if (warp == 9) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(kMixTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();  // constants (generic writes) are read by the tensor cores
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;

  const long long first = blockIdx.x, step = gridDim.x;

  if (warp < 8) {
    // ---------------- convert / epilogue threads ----------------
    // group gr = warps 4gr..4gr+3: pencils 8gr..8gr+7 of every tile, its own
    // operand buffer, tensor memory (256 columns) and barriers
    const int gr = warp >> 2, q = warp & 3;
    const int tl = tid & 127;                  // stage-A row of the group
    const int cl = tl >> 4, n2 = tl & 15;      // pencil within the group, n2
    const int c = 8 * gr + cl;                 // pencil within the tile
    const uint32_t opHi = sb + kMixOpA + (uint32_t)gr * 32768u, opLo = opHi + 16384u;
    const uint32_t twb = sb + kMixTw;
    const uint32_t tg = tmem + (uint32_t)gr * 256u + ((uint32_t)(q * 32) << 16);
    int it = 0;
    for (long long tile = first; tile < g.ntiles; tile += step, ++it) {
      const int b = it & 1;
      const uint32_t par = (uint32_t)(it & 1);
      if (!mix_wait_warp(&full[b], (uint32_t)((it >> 1) & 1), s_abort)) { *s_abort = 1; break; }
      // group 1 runs half a step behind group 0 (its prep starts once group
      // 0's stage-A products are queued), so that each group's conversions
      // overlap the other group's products instead of competing with them
      if (gr == 1) {
        // a monotonic counter, not a barrier phase: group 0 may be more than
        // one phase ahead
        bool ok = true;
        if (*s_g0 < it) {
          const uint64_t t0 = global_ns();
          while (*s_g0 < it) {
            __nanosleep(32);
            if (*s_abort || global_ns() - t0 > kWaitNs) { ok = false; break; }
          }
        }
        if (!__all_sync(0xffffffffu, ok)) { *s_abort = 1; break; }
      }
      const uint32_t tb = sb + (uint32_t)b * kMixTile;
      // ---- stage-A operands: row tl = (cl, n2), K = [re n1 0..31 | im n1 0..31]
      float2 v[32];
#pragma unroll
      for (int n1 = 0; n1 < 32; ++n1) v[n1] = lds64(tb + tile_off<STRIDED>(16 * n1 + n2, c));
      float m = 0.f;
#pragma unroll
      for (int n1 = 0; n1 < 32; ++n1) m = fmaxf(m, fmaxf(fabsf(v[n1].x), fabsf(v[n1].y)));
#pragma unroll
      for (int o = 8; o >= 1; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      const float sA = mix_scale(m);
      {
        // the row goes to tensor memory (lane tl of the group's columns
        // 192-223 hi, 224-255 lo): word w holds K = 2w, 2w + 1
        uint32_t hw[32], lw[32];
#pragma unroll
        for (int w = 0; w < 32; ++w) {
          const int n1 = (2 * w) & 31;
          const float a0 = (w < 16 ? v[n1].x : v[n1].y) * sA;
          const float a1 = (w < 16 ? v[n1 + 1].x : v[n1 + 1].y) * sA;
          split2(a0, a1, hw[w], lw[w]);
        }
        tmem_st32(tg + 192u, hw);
        tmem_st32(tg + 224u, lw);
        tmem_wait_st();
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&opA[gr]);
      if (gr == 0 && q == 0 && lane == 0) *s_g0 = it;
      // ---- stage-A epilogue: TMEM row tl -> twiddle (and 1/32), split
      if (!mix_wait_warp(&accA[gr], par, s_abort)) { *s_abort = 1; break; }
      tc_fence_after();
      uint32_t r[64];
#pragma unroll
      for (int part = 0; part < 2; ++part) {  // real parts (columns 0-31), then imaginary
        uint32_t t0[32], t1[32];
        tmem_ld32(tg + (uint32_t)(32 * part), t0);
        tmem_ld32(tg + 64u + (uint32_t)(32 * part), t1);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; ++i) r[32 * part + i] = __float_as_uint(__uint_as_float(t0[i]) + __uint_as_float(t1[i]));
        tmem_ld32(tg + 128u + (uint32_t)(32 * part), t0);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 32; ++i) r[32 * part + i] = __float_as_uint(__uint_as_float(r[32 * part + i]) + __uint_as_float(t0[i]));
      }
      // the values carry the stage-A scale sA; the twiddles carry 1/32, so
      // the stage-B operands come out scaled by sA / 32
#pragma unroll
      for (int k1 = 0; k1 < 32; ++k1) {
        const float2 w = lds64(twb + (uint32_t)((n2 * 33 + k1) * 8));
        const float yr = __uint_as_float(r[k1]), yi = __uint_as_float(r[32 + k1]);
        r[k1] = __float_as_uint(yr * w.x - yi * w.y);
        r[32 + k1] = __float_as_uint(yr * w.y + yi * w.x);
      }
      tc_fence_before();
      {
        // stage-B operand, MN-major: M = pos*32 + k1 (atoms of 64 rows, 4 KB
        // apart), K = [re n2 0..15 | im n2 0..15] (groups of 8 rows, 1 KB apart)
        const int kr = n2 & 7;
        const int pos = mix_pos(cl);
#pragma unroll
        for (int part = 0; part < 2; ++part) {
          const uint32_t kbase = (uint32_t)((pos >> 1) * 4096 + (2 * part + (n2 >> 3)) * 1024 + kr * 128);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj) {
            uint32_t h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int k1 = 8 * jj + 2 * e;
              split2(__uint_as_float(r[32 * part + k1]), __uint_as_float(r[32 * part + k1 + 1]), h[e], l[e]);
            }
            const uint32_t off = kbase + (uint32_t)(((((pos & 1) * 4 + jj) ^ kr) << 4));
            sts128(opHi + off, h[0], h[1], h[2], h[3]);
            sts128(opLo + off, l[0], l[1], l[2], l[3]);
          }
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&opB[gr]);
      // ---- stage-B epilogue: rows (pencil of position 4j + q, k1 = lane) of
      // blocks j = 0, 1
      if (!mix_wait_warp(&accB[gr], par, s_abort)) { *s_abort = 1; break; }
      tc_fence_after();
      {
        uint32_t rr[2][32];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          uint32_t rc[32];
          const uint32_t tb_ = tg + (uint32_t)(j * 96);
          tmem_ld32(tb_, rr[j]);
          tmem_ld32(tb_ + 32u, rc);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) rr[j][i] = __float_as_uint(__uint_as_float(rr[j][i]) + __uint_as_float(rc[i]));
          tmem_ld32(tb_ + 64u, rc);
          tmem_wait_ld();
#pragma unroll
          for (int i = 0; i < 32; ++i) rr[j][i] = __float_as_uint(__uint_as_float(rr[j][i]) + __uint_as_float(rc[i]));
        }
        // pencils 2q (block 0) and 2q + 1 (block 1): stage-A rows of this
        // warp's lanes 0-15 and 16-31, whose scale undoes sA / 32 exactly
        const int cc = 8 * gr + 2 * q;
        const float f0 = g.out_scale * 32.0f * mix_inv(__shfl_sync(0xffffffffu, sA, 0));
        const float f1 = g.out_scale * 32.0f * mix_inv(__shfl_sync(0xffffffffu, sA, 16));
        if constexpr (STRIDED) {
          // one 16-byte chunk (both columns) per row
#pragma unroll
          for (int k2 = 0; k2 < 16; ++k2)
            sts128(tb + tile_off<STRIDED>(lane + 32 * k2, cc), __float_as_uint(__uint_as_float(rr[0][k2]) * f0),
                   __float_as_uint(__uint_as_float(rr[0][16 + k2]) * f0),
                   __float_as_uint(__uint_as_float(rr[1][k2]) * f1),
                   __float_as_uint(__uint_as_float(rr[1][16 + k2]) * f1));
        } else {
#pragma unroll
          for (int k2 = 0; k2 < 16; ++k2) {
            sts64(tb + tile_off<STRIDED>(lane + 32 * k2, cc), __uint_as_float(rr[0][k2]) * f0,
                  __uint_as_float(rr[0][16 + k2]) * f0);
            sts64(tb + tile_off<STRIDED>(lane + 32 * k2, cc + 1), __uint_as_float(rr[1][k2]) * f1,
                  __uint_as_float(rr[1][16 + k2]) * f1);
          }
        }
      }
      tc_fence_before();
      fence_proxy_async_smem();  // the tile is next read by the store
      __syncwarp();
      if (lane == 0) mbar_arrive(&outrdy[b]);
    }
  } else if (warp == 8) {
    // ---------------- producer ----------------
    if (lane == 0) {
      int loads[2] = {0, 0};
      bool failed = false;
      auto issue_load = [&](int b, long long tile) {
        void* dst = sm + (size_t)b * kMixTile;
        if constexpr (STRIDED) {
          const int ti = (int)(tile % g.tiles_i);
          const int o = (int)(tile / g.tiles_i);
          mbar_expect_tx(&full[b], (uint32_t)kMixTile);
          for (int kb = 0; kb < g.nlb; ++kb)
            tma_load_3d(static_cast<unsigned char*>(dst) + (size_t)kb * g.lb * 128, &tin, &full[b], ti * 16,
                        kb * g.lb, o);
        } else {
          const long long q0 = tile * 16;
          const long long nv = (g.ncols - q0) < 16 ? (g.ncols - q0) : 16;
          const uint32_t bytes = (uint32_t)(nv * 4096);
          mbar_expect_tx(&full[b], bytes);
          bulk_load_1d(dst, static_cast<const unsigned char*>(in) + q0 * 4096, bytes, &full[b]);
        }
        ++loads[b];
      };
      auto issue_store = [&](int b, long long tile) {
        const void* src = sm + (size_t)b * kMixTile;
        if constexpr (STRIDED) {
          const int ti = (int)(tile % g.tiles_i);
          const int o = (int)(tile / g.tiles_i);
          for (int kb = 0; kb < g.nlb; ++kb)
            tma_store_3d(&tout, static_cast<const unsigned char*>(src) + (size_t)kb * g.lb * 128, ti * 16,
                         kb * g.lb, o);
        } else {
          const long long q0 = tile * 16;
          const long long nv = (g.ncols - q0) < 16 ? (g.ncols - q0) : 16;
          bulk_store_1d(static_cast<unsigned char*>(out) + q0 * 4096, src, (uint32_t)(nv * 4096));
        }
        bulk_commit();
      };
      int it = 0;
      long long tile = first;
      // prime both buffers
      for (; it < 2 && tile < g.ntiles; ++it, tile += step) issue_load(it, tile);
      // then: store tile dit once transformed, refill its buffer with the next tile
      long long done_tile = first;
      int dit = 0;
      for (; done_tile < g.ntiles; done_tile += step, ++dit) {
        const int b = dit & 1;
        if (!mix_wait(&outrdy[b], (uint32_t)((dit >> 1) & 1), s_abort)) { failed = true; break; }
        issue_store(b, done_tile);
        if (tile < g.ntiles) {
          bulk_wait_read_all();  // the store has read the buffer
          issue_load(b, tile);
          tile += step;
          ++it;
        }
      }
      bulk_wait_all();
      if (failed) {
        *s_abort = 1;
        // loads still in flight land in shared memory: wait for them
        for (int b = 0; b < 2; ++b)
          if (loads[b] > 0) mbar_wait_bounded(&full[b], (uint32_t)((loads[b] - 1) & 1));
      }
    }
  } else {
    // ---------------- MMA issuer (warp 9, lane 0) ----------------
    // serves the two groups in the order their operands become ready
    if (lane == 0) {
      // descriptors for K-step 0; a K-step adds its byte offset / 16 to the
      // start-address field (no carry: every operand lies below 256 KB)
      const uint64_t dB32h = umma_desc_sw128(sb + kMixB32, 16, 1024), dB32l = umma_desc_sw128(sb + kMixB32 + 8192, 16, 1024);
      const uint64_t dB16h = umma_desc_sw128(sb + kMixB16, 16, 1024), dB16l = umma_desc_sw128(sb + kMixB16 + 4096, 16, 1024);
      uint64_t dBh[2], dBl[2];
      for (int gq = 0; gq < 2; ++gq) {
        const uint32_t hi = sb + kMixOpA + (uint32_t)gq * 32768u;
        dBh[gq] = umma_desc_sw128(hi, 4096, 1024);
        dBl[gq] = umma_desc_sw128(hi + 16384u, 4096, 1024);
      }
      constexpr uint32_t idA = umma_idesc_f16(128, 64, 0, 0);
      constexpr uint32_t idB = umma_idesc_f16(128, 32, 1, 0);
      const long long ntile = g.ntiles > first ? (g.ntiles - first + step - 1) / step : 0;
      long long done[2] = {0, 0};  // tiles each group has had both stages issued for
      int stage[2] = {0, 0};       // next request: 0 stage A, 1 stage B
      uint64_t* last_bar[2] = {nullptr, nullptr};  // last commit per group, and its phase parity
      uint32_t last_par[2] = {0, 0};
      const uint64_t t0 = global_ns();
      uint64_t t_last = t0;
      unsigned spins = 0;
      while ((done[0] < ntile || done[1] < ntile) && !*s_abort) {
        bool progressed = false;
#pragma unroll
        for (int gq = 0; gq < 2; ++gq) {
          if (done[gq] >= ntile) continue;
          const uint32_t par = (uint32_t)(done[gq] & 1);
          const uint32_t d = tmem + (uint32_t)gq * 256u;
          if (stage[gq] == 0) {
            if (!mbar_test(&opA[gq], par)) continue;
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              const uint64_t o = (uint64_t)(2 * s);                // 32 bytes of B
              const uint32_t ah = d + 192u + (uint32_t)(8 * s);    // 8 columns of A (16 FP16 of K)
              const uint32_t al = d + 224u + (uint32_t)(8 * s);
              umma_f16_ts(d + (uint32_t)((s >> 1) * 64), ah, dB32h + o, idA, s & 1);  // hi x hi, chains of two
              umma_f16_ts(d + 128u, al, dB32h + o, idA, s > 0);                        // cross terms
              umma_f16_ts(d + 128u, ah, dB32l + o, idA, 1);
            }
            umma_commit(&accA[gq]);
            last_bar[gq] = &accA[gq];
            last_par[gq] = par;
            stage[gq] = 1;
          } else {
            if (!mbar_test(&opB[gq], par)) continue;
            tc_fence_after();
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              const uint32_t dj = d + (uint32_t)(j * 96);
#pragma unroll
              for (int s = 0; s < 2; ++s) {
                const uint64_t oa = (uint64_t)(j * 512 + s * 128);  // (j * 8192 + s * 2048) bytes
                const uint64_t ob = (uint64_t)(2 * s);
                umma_f16(dj + (uint32_t)(32 * s), dBh[gq] + oa, dB16h + ob, idB, 0);  // hi x hi, one K-step each
                umma_f16(dj + 64u, dBl[gq] + oa, dB16h + ob, idB, s > 0);            // cross terms
                umma_f16(dj + 64u, dBh[gq] + oa, dB16l + ob, idB, 1);
              }
            }
            umma_commit(&accB[gq]);
            last_bar[gq] = &accB[gq];
            last_par[gq] = par;
            stage[gq] = 0;
            ++done[gq];
          }
          progressed = true;
        }
        if (progressed) {
          t_last = global_ns();
          spins = 0;
          continue;
        }
        __nanosleep(20);
        if ((++spins & 255) == 0 && global_ns() - t_last > kWaitNs) {
          *s_abort = 1;  // neither group handed over operands in time
          break;
        } else if (spins > kWaitLimit) {
          *s_abort = 1;
          break;
        }
      }
      (void)t0;
      // products still running read shared memory and write tensor memory:
      // wait (bounded) for each group's last commit before the CTA frees either
      for (int gq = 0; gq < 2; ++gq)
        if (last_bar[gq]) mbar_wait_bounded(last_bar[gq], last_par[gq]);
    }
  }
  if (*s_abort && tid == 0 && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 9) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMixTmemCols)
                 : "memory");
  }
}

}  // namespace dfft
