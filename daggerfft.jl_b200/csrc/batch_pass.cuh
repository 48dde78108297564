// Persistent kernel for a batch of complex transforms of uneven shapes: ONE
// launch walks a work list of (transform, axis pass, tile) items.
//
// Work list.  Every axis pass of every transform is a "phase" of tiles of C
// columns (C = kBatchThreads / P for its length).  Phases are laid out in a
// staggered order -- axis a of transform i at slot i + a * lag -- so that a
// pass is claimed about `lag` transforms after the pass it depends on,
// which is then normally finished: the transforms in flight at a time are
// few, and their buffers stay in L2 between their passes (each pass reads
// what the previous one wrote).
//
// Each CTA claims items one at a time from a global counter (so items are
// claimed in list order), waits -- bounded -- until the phase its item
// depends on (the previous axis of the same transform) has finished all its
// tiles, runs the tile (the static-plan stage body: first stage from global
// memory, stages through shared memory, last stage to global memory), and
// publishes the tile in its phase's counter with release semantics.
// Progress does not need co-residency: an item depends only on items earlier
// in the list, every claimed item is held by a running CTA, so the earliest
// unfinished item can always proceed.  A wait that expires (~2 s) records
// DFFT_DEVERR_TMA_TIMEOUT in the device error word; every CTA then stops
// claiming items.
#pragma once
#include "tma_pass.cuh"

namespace dfft {

constexpr int kBatchThreads = 256;
constexpr int kBatchTilesPerItem = 8;  // tiles per work item (a tile is ~256 x radix elements)

struct BatchPhase {
  PassDesc d;        // one axis pass (in / out pointers filled at execute)
  long long start;   // first item of the phase in the work list
  int tiles;         // items of the phase (kBatchTilesPerItem tiles each)
  int dep;           // phase that must be complete first, or -1
};

struct BatchGeom {
  const BatchPhase* phases;
  int nphases;
  long long total;              // items in the work list
  unsigned long long* next;     // next item to claim (zeroed before each launch)
  unsigned* done;               // finished tiles per phase (zeroed before each launch)
  int* err;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Work item `item` of a direct static pass of length L with P threads per
// column and compile-time radices: kBatchTilesPerItem tiles of C columns,
// each the body of axis_pass_static with the tile in place of the block
// index.  Threads beyond the C * P that a tile uses run the stages on a
// scratch column (C) with no global access.  (Consecutive tiles need no
// barrier between them: the last stage of a tile reads the shared buffer
// before a barrier, then writes only global memory.)
template <typename T, int L, int P, int... Rs>
__device__ __noinline__ void batch_tile(const PassDesc& d, long long item, unsigned char* smem) {
  typedef typename cvec<T>::type V;
  constexpr int C = kBatchThreads / P;
  const int tid = threadIdx.x;
  int c, t;
  if (d.cfast) { c = tid % C; t = tid / C; }
  else { t = tid % P; c = tid / P; }
  const bool active = tid < C * P;
  if (!active) { c = C; t = 0; }
  V* sm = reinterpret_cast<V*>(smem);
  const PadCol<V> col{sm + (size_t)c * d.ld};
  const GlobalTw<V> tw{reinterpret_cast<const V*>(d.tw)};
  for (int u = 0; u < kBatchTilesPerItem; ++u) {
    const long long q = (item * kBatchTilesPerItem + u) * C + c;
    const bool cv = active && q < d.Q;
    const long long qi = cv ? q % d.I : 0;
    const long long qo = cv ? q / d.I : 0;
    const long long ib = qi * d.in.si + io_outer(d.in, qo);
    const long long ob = qi * d.out.si + io_outer(d.out, qo);
    static_stages<T, L, P, true, 0, 0, 0, 1, 1, 0, PadCol<V>, PadCol<V>, PadCol<V>, GlobalTw<V>, Rs...>(
        d, t, col, col, col, tw, ib, ob, cv);
  }
}

// The lengths the persistent kernel runs (radices and threads per column as
// in the static-plan table); other lengths keep the graph of per-plan passes.
#define DFFT_BATCH_LENGTHS(X)                       \
  X(16, 1, 16) X(24, 4, 6, 4) X(32, 4, 8, 4)        \
  X(40, 5, 5, 8) X(48, 6, 6, 8) X(60, 6, 10, 6)     \
  X(64, 8, 8, 8) X(72, 6, 12, 6) X(80, 8, 10, 8)    \
  X(96, 8, 12, 8) X(100, 10, 10, 10)                \
  X(120, 10, 12, 10) X(128, 8, 16, 8)               \
  X(144, 12, 12, 12) X(160, 10, 10, 16)             \
  X(192, 12, 12, 16) X(256, 16, 16, 16)

template <typename T>
__global__ void __launch_bounds__(kBatchThreads, 2) batch_persistent(const BatchGeom g) {
  extern __shared__ __align__(16) unsigned char smem_batch[];
  __shared__ long long s_item;
  __shared__ int s_phase, s_stop;
  __shared__ __align__(16) PassDesc s_d;
  const int tid = threadIdx.x;
  volatile int* verr = g.err;
  int ph = 0;  // thread 0: phase of the last claimed item (claims only increase)
  for (;;) {
    if (tid == 0) {
      long long n = *verr != 0 ? g.total : (long long)atomicAdd(g.next, 1ull);
      int stop = n >= g.total;
      if (!stop) {
        while (ph + 1 < g.nphases && g.phases[ph + 1].start <= n) ++ph;
        const int dep = g.phases[ph].dep;
        if (dep >= 0) {
          const unsigned need = (unsigned)g.phases[dep].tiles;
          if (ld_acquire_u32(g.done + dep) < need) {
            const uint64_t t0 = global_ns();
            for (unsigned i = 0;; ++i) {
              __nanosleep(64);
              if (ld_acquire_u32(g.done + dep) >= need) break;
              if (*verr != 0 || i >= kWaitLimit || ((i & 63) == 0 && global_ns() - t0 > kWaitNs)) {
                if (*verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
                stop = 1;
                break;
              }
            }
          }
        }
      }
      s_item = n;
      s_phase = ph;
      s_stop = stop;
    }
    __syncthreads();
    if (s_stop) break;
    const BatchPhase& P = g.phases[s_phase];
    // every thread acquires what the dependency's CTAs released
    if (P.dep >= 0) (void)ld_acquire_u32(g.done + P.dep);
    {
      const unsigned* src = reinterpret_cast<const unsigned*>(&P.d);
      unsigned* dst = reinterpret_cast<unsigned*>(&s_d);
      for (int i = tid; i < (int)(sizeof(PassDesc) / 4); i += kBatchThreads) dst[i] = src[i];
    }
    __syncthreads();
    const long long tile = s_item - P.start;
    switch (s_d.L) {
#define DFFT_BATCH_CASE(L, P_, ...) \
  case L: batch_tile<T, L, P_, __VA_ARGS__>(s_d, tile, smem_batch); break;
      DFFT_BATCH_LENGTHS(DFFT_BATCH_CASE)
#undef DFFT_BATCH_CASE
      default:
        if (tid == 0 && *verr == 0) atomicExch(g.err, DFFT_DEVERR_BATCH_ITEM);
        break;
    }
    // every thread's stores happen before the barrier, and thread 0's
    // gpu-scope release after it publishes them (cumulativity); the shared
    // buffer is then free for the next item
    __syncthreads();
    if (tid == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.done + s_phase) : "memory");
  }
}

}  // namespace dfft
