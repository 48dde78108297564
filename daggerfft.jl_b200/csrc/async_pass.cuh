// Strided C2C axis pass for layouts TMA cannot address: rows whose byte
// stride is not a multiple of 16 (the half-spectrum of a ComplexF32 rfft of
// even length n has n/2+1 elements per row: 65, 129, 257 -> 520, 1032, 2056
// bytes).  This is the second pass of rfft and the second-to-last of irfft
// over dims (1, 2, ...) (apply_fft! per axis, src/fft.jl:168-174,
// src/fftgpu.jl:118-124, on the layout the R2C pass leaves).
//
// Persistent CTAs of CS*P threads, all of which run the stages.  A tile is
// CS consecutive columns of the flattened column index q = qi + I*qo (so no
// tile is left partly empty at the end of each run of I columns) x L rows;
// every thread copies its share of tile i+NB-1 into a ring of NB shared
// buffers with 8- or 16-byte cp.async (zero-filled past the last column)
// before it transforms tile i, so the copies of the next NB-1 tiles overlap
// the stages of the current one.  The first stage reads the dense [row][column]
// tile, the middle stages run in the row-swizzled layout with the stage
// twiddles in shared memory, and the last stage stores straight to global
// memory, CS consecutive elements per row (coalesced, 8-byte aligned).
// No waits on other CTAs or on flags: nothing to bound beyond cp.async
// completion.
#pragma once
#include "tiled_pass.cuh"

namespace dfft {

struct AsyncGeom {
  long long ntiles;  // ceil(Q / CS)
  long long Q;       // columns: I * O
  long long I;       // columns along the contiguous axes
  int ntw;           // stage-twiddle entries
  int bstride;       // elements between the tile buffers (128-byte multiple)
};

// cp.async of one element (8 or 16 bytes); src_bytes 0 fills zeros
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, bool valid) {
  const uint32_t d = smem_u32(dst);
  const int n = valid ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename T, int LB, int MINB, int NB, int DIR, int L, int P, int CS, int... Rs>
__global__ void __launch_bounds__(LB, MINB) axis_pass_async(const PassDesc d, const AsyncGeom g) {
  typedef typename cvec<T>::type V;
  static_assert(CS * P == LB, "every thread runs the stages");
  static_assert(NB >= 2 && NB <= 4, "tile buffers");
  static_assert((CS * L) % LB == 0, "whole copy rounds");
  constexpr int R0 = first_radix<Rs...>::value;
  constexpr bool kPow2 = (L & (L - 1)) == 0 && (((Rs & (Rs - 1)) == 0) && ...);
  extern __shared__ __align__(128) unsigned char smem_async[];
  V* stw = reinterpret_cast<V*>(smem_async);
  const size_t tw_bytes = ((size_t)g.ntw * sizeof(V) + 127) & ~(size_t)127;
  V* bufs = reinterpret_cast<V*>(smem_async + tw_bytes);
  const int tid = threadIdx.x;
  {
    const V* gtw = reinterpret_cast<const V*>(d.tw);
    for (int i = tid; i < g.ntw; i += LB) stw[i] = gtw[i];
  }
  const V* src = reinterpret_cast<const V*>(d.in.p);
  // thread tid copies column c = tid % CS, rows t, t + LB/CS, ... of a tile
  // (LB is a multiple of CS): element e = tid + i*LB of the [row][column]
  // tile is row t + i*LB/CS of column c
  const StageTw<V> tw{stw};
  const int c = tid % CS, t = tid / CS;
  auto issue = [&](long long tile, V* buf) {
    const long long q = tile * CS + c;
    const bool ok = q < g.Q;
    const V* s = ok ? src + (q % g.I) * d.in.si + (q / g.I) * d.in.so + (long long)t * d.in.sk : src;
    const long long rstep = ok ? (long long)(LB / CS) * d.in.sk : 0;
#pragma unroll 4
    for (int i = 0; i < CS * L / LB; ++i) cp_async_elem<sizeof(V)>(buf + tid + i * LB, s + i * rstep, ok);
  };
  const long long first = blockIdx.x, step = gridDim.x;
  // prologue: tiles 0 .. NB-2 of this CTA, one commit group each
#pragma unroll
  for (int i = 0; i < NB - 1; ++i) {
    if (first + i * step < g.ntiles) issue(first + i * step, bufs + (size_t)i * g.bstride);
    cp_async_commit();
  }
  int it = 0;
  for (long long tile = first; tile < g.ntiles; tile += step, ++it) {
    V* buf = bufs + (size_t)(it % NB) * g.bstride;
    const long long ahead = tile + (long long)(NB - 1) * step;
    if (ahead < g.ntiles) issue(ahead, bufs + (size_t)((it + NB - 1) % NB) * g.bstride);
    cp_async_commit();
    cp_async_wait<NB - 1>();  // this thread's copies of the current tile have landed
    __syncthreads();          // and everyone else's (and, first time, the twiddles)
    const long long q = tile * CS + c;
    const bool cv = q < g.Q;
    const long long ob = cv ? (q % g.I) * d.out.si + (q / g.I) * d.out.so : 0;
    const StrideColC<V, CS> dense{buf + c};
    if constexpr (kPow2) {
      const YSwzCol<V, CS, R0> sw{buf + c};
      static_stages<T, L, P, true, 3, 0, DIR, 1, 1, 0, StrideColC<V, CS>, YSwzCol<V, CS, R0>, StrideColC<V, CS>,
                    StageTw<V>, Rs...>(d, t, dense, sw, dense, tw, 0, ob, cv);
    } else {
      static_stages<T, L, P, true, 3, 0, DIR, 1, 1, 0, StrideColC<V, CS>, StrideColC<V, CS>, StrideColC<V, CS>,
                    StageTw<V>, Rs...>(d, t, dense, dense, dense, tw, 0, ob, cv);
    }
    __syncthreads();  // the next iteration's copies refill the buffer of tile i-1
  }
  cp_async_wait<0>();
}

}  // namespace dfft
