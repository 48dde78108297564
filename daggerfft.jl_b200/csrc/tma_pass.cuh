// Persistent, TMA-pipelined pass for the strided axes of a C2C transform.
//
// A tile is C adjacent columns x L rows (row k of the tile is C contiguous
// complex elements at i0 + k*I + o*I*L).  It is moved by the Tensor Memory
// Accelerator as a 3-D box {C, Lb, 1} of the tensor {I, L, O}: the box lands
// in shared memory as [k][c] (c fastest), which the cfast thread mapping
// reads and writes without bank conflicts in every Stockham stage, and the
// finished tile leaves the same buffer through a bulk-tensor store.
//
// Each CTA owns NBUF tile buffers and walks tiles blockIdx.x, +gridDim.x, ...
// While it computes tile i, the loads of tiles i+1 .. i+NBUF-1 are in flight
// and the store of tile i-1 drains, so HBM traffic overlaps the shared-memory
// FFT.  Ordering: threads write the tile, fence.proxy.async, barrier, then one
// thread issues the store; a buffer is reloaded only after
// cp.async.bulk.wait_group.read confirms its previous store has read it.
//
// Every mbarrier wait is bounded; on expiry the kernel records
// DFFT_DEVERR_TMA_TIMEOUT in the device error word, drains its own copies
// (bounded) and returns.
#pragma once
#include <cuda.h>
#include "axis_pass.cuh"

namespace dfft {

constexpr int kTmaBufs = 3;
constexpr unsigned kWaitLimit = 1u << 26;   // try_wait rounds before giving up
constexpr uint64_t kWaitNs = 2000000000ull;  // and at most ~2 s of wall time
enum : int { DFFT_DEVERR_TMA_TIMEOUT = 1 };

struct TmaGeom {
  int C;              // columns per tile
  int tiles_i;        // tiles along the inner extent I
  long long ntiles;   // tiles_i * O
  int lb;             // rows per TMA box (<= 256)
  int nlb;            // boxes per tile (L / lb)
  int xscale;         // TMA x units per column: 1 (complex float), 2 (complex double)
  unsigned tile_bytes;
  int* err;           // device error word
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the phase of `parity` to complete; gives up after ~2 s.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned i = 1; i < kWaitLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 0 && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x,
                                            int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y,
                                             int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <typename V>
__device__ __forceinline__ void tma_issue_tile_load(const CUtensorMap* map, V* buf, uint64_t* bar,
                                                    const TmaGeom& g, long long tile, int C) {
  const int ti = (int)(tile % g.tiles_i);
  const int o = (int)(tile / g.tiles_i);
  mbar_expect_tx(bar, g.tile_bytes);
  for (int b = 0; b < g.nlb; ++b)
    tma_load_3d(buf + (size_t)b * g.lb * C, map, bar, ti * C * g.xscale, b * g.lb, o);
}

template <typename V>
__device__ __forceinline__ void tma_issue_tile_store(const CUtensorMap* map, const V* buf,
                                                     const TmaGeom& g, long long tile, int C) {
  const int ti = (int)(tile % g.tiles_i);
  const int o = (int)(tile / g.tiles_i);
  for (int b = 0; b < g.nlb; ++b)
    tma_store_3d(map, buf + (size_t)b * g.lb * C, ti * C * g.xscale, b * g.lb, o);
}

template <typename T, int LB, int L, int P, int... Rs>
__global__ void __launch_bounds__(LB) axis_pass_tma(const PassDesc d,
                                                    const __grid_constant__ CUtensorMap tin,
                                                    const __grid_constant__ CUtensorMap tout,
                                                    const TmaGeom g) {
  typedef typename cvec<T>::type V;
  extern __shared__ __align__(128) unsigned char smem_tma[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_tma);
  __shared__ int s_abort;
  V* bufs = reinterpret_cast<V*>(smem_tma + 128);
  const int C = g.C;
  const size_t buf_elems = (size_t)C * L;
  const int tid = threadIdx.x;
  const int c = tid % C;
  const int t = tid / C;
  const V* tw = reinterpret_cast<const V*>(d.tw);
  if (tid == 0) {
    for (int b = 0; b < kTmaBufs; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();
  const long long first = blockIdx.x;
  const long long step = gridDim.x;
  int issued[kTmaBufs] = {0, 0, 0};   // loads issued per buffer (thread 0)
  if (tid == 0) {
    for (int b = 0; b < kTmaBufs - 1; ++b) {
      const long long tile = first + b * step;
      if (tile < g.ntiles) {
        tma_issue_tile_load(&tin, bufs + b * buf_elems, &bars[b], g, tile, C);
        ++issued[b];
      }
    }
  }
  int it = 0;
  for (long long tile = first; tile < g.ntiles; tile += step, ++it) {
    const int buf = it % kTmaBufs;
    const uint32_t parity = (uint32_t)((it / kTmaBufs) & 1);
    if (!mbar_wait_bounded(&bars[buf], parity)) s_abort = 1;
    __syncthreads();
    if (s_abort) break;
    V* sb = bufs + buf * buf_elems;
    const StrideCol<V> col{sb + c, C};
    static_stages<T, L, P, true, true, 1, 0, StrideCol<V>, Rs...>(d, t, col, tw, 0, 0, true);
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      // the buffer of tile it-1 is free once its store has read shared memory
      bulk_wait_read_all();
      const long long next = tile + (long long)(kTmaBufs - 1) * step;
      if (next < g.ntiles) {
        const int nb = (it + kTmaBufs - 1) % kTmaBufs;
        tma_issue_tile_load(&tin, bufs + nb * buf_elems, &bars[nb], g, next, C);
        ++issued[nb];
      }
      tma_issue_tile_store(&tout, sb, g, tile, C);
      bulk_commit();
    }
  }
  if (tid == 0) {
    bulk_wait_all();
    if (s_abort) {
      atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
      // loads still in flight land in this CTA's shared memory: wait for
      // the last load issued into each buffer (bounded) before the CTA
      // releases it
      for (int b = 0; b < kTmaBufs; ++b)
        if (issued[b] > 0) mbar_wait_bounded(&bars[b], (uint32_t)((issued[b] - 1) & 1));
    }
  }
  __syncthreads();
}

}  // namespace dfft
