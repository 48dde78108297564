// Persistent, TMA-pipelined passes.
//
// Strided axes (CONTIG = false).  A tile is C adjacent columns x L rows (row
// k of the tile is C contiguous complex elements at i0 + k*I + o*I*L).  The
// Tensor Memory Accelerator moves it as 3-D boxes {C, Lb, 1} of the tensor
// {I, L, O}: the boxes land in shared memory as [k][c] (c fastest), which the
// cfast thread mapping reads and writes without bank conflicts in every
// Stockham stage, and the finished tile leaves the same buffer through a
// bulk-tensor store.
//
// Contiguous axis (CONTIG = true).  A tile is C whole pencils, one contiguous
// run of C*L elements moved by a 1-D bulk copy.  It lands dense ([c][k]);
// the first stage reads it there and writes a padded work buffer (the
// stride-R writes of the early stages would conflict in the dense layout),
// the middle stages stay in the work buffer, and the last stage (whose writes
// are unit-stride) puts the result back into the dense buffer for the bulk
// store.
//
// Each CTA owns kTmaBufs tile buffers and walks tiles blockIdx.x, +gridDim.x,
// ...  While it computes tile i, the loads of tiles i+1 .. i+kTmaBufs-1 are in
// flight and the store of tile i-1 drains, so HBM traffic overlaps the
// shared-memory FFT.  Ordering: threads write the tile, fence.proxy.async,
// barrier, then one thread issues the store; a buffer is reloaded only after
// cp.async.bulk.wait_group.read confirms its previous store has read it.
// The contiguous variant copies the stage twiddles once per CTA into shared
// memory (StageTw layout); the strided variant reads the L-entry table
// through L1 (in its cfast mapping a warp needs only two twiddles per
// element), which keeps its shared-memory footprint (three 64 KB tiles for
// L = 512) small enough that L1 keeps its share of the SRAM.
//
// Every mbarrier wait is bounded (~2 s); on expiry the kernel records
// DFFT_DEVERR_TMA_TIMEOUT in the device error word, waits (bounded) for the
// copies it issued and returns.
#pragma once
#include <cuda.h>
#include "axis_pass.cuh"

namespace dfft {

constexpr int kTmaBufs = 3;
constexpr unsigned kWaitLimit = 1u << 26;    // try_wait rounds before giving up
constexpr uint64_t kWaitNs = 2000000000ull;  // and at most ~2 s of wall time
enum : int { DFFT_DEVERR_TMA_TIMEOUT = 1, DFFT_DEVERR_TMA_ALIGN = 2, DFFT_DEVERR_BATCH_ITEM = 3 };

struct TmaGeom {
  int C;              // columns (strided) or pencils (contiguous) per tile
  int tiles_i;        // strided: tiles along the inner extent I
  long long ntiles;   // number of tiles
  long long ncols;    // contiguous: number of pencils
  int lb;             // strided: rows per TMA box (<= 256)
  int nlb;            // strided: boxes per tile (L / lb)
  int xscale;         // TMA x units per column: 1 (complex float), 2 (complex double)
  int ld;             // contiguous: padded work-buffer elements per pencil
  int ntw;            // stage-twiddle entries to stage in shared memory
  int bstride;        // elements between tile buffers (a multiple of 128 bytes)
  unsigned tile_bytes;
  int* err;           // device error word
  // strided variant, first pass of a four-step axis (null otherwise): row k
  // of column q leaves times W_lf^((q / tw_div) * k), read from the two
  // tables W_lf^(m mod tw_b) (tw_lo) and W_lf^(tw_b * (m / tw_b)) (tw_hi)
  const void* tw_lo;
  const void* tw_hi;
  long long tw_div, tw_lf;
  int tw_b;
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
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_store_1d(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
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

template <typename V, bool CONTIG, int L>
__device__ __forceinline__ void pipe_issue_load(const PassDesc& d, const CUtensorMap* map, V* buf,
                                                uint64_t* bar, const TmaGeom& g, long long tile) {
  if (CONTIG) {
    const long long q0 = tile * g.C;
    const long long nv = (g.ncols - q0) < g.C ? (g.ncols - q0) : g.C;
    const uint32_t bytes = (uint32_t)(nv * L * (long long)sizeof(V));
    mbar_expect_tx(bar, bytes);
    bulk_load_1d(buf, reinterpret_cast<const V*>(d.in.p) + q0 * L, bytes, bar);
  } else {
    const int ti = (int)(tile % g.tiles_i);
    const int o = (int)(tile / g.tiles_i);
    mbar_expect_tx(bar, g.tile_bytes);
    for (int b = 0; b < g.nlb; ++b)
      tma_load_3d(buf + (size_t)b * g.lb * g.C, map, bar, ti * g.C * g.xscale, b * g.lb, o);
  }
}

template <typename V, bool CONTIG, int L>
__device__ __forceinline__ void pipe_issue_store(const PassDesc& d, const CUtensorMap* map,
                                                 const V* buf, const TmaGeom& g, long long tile) {
  if (CONTIG) {
    const long long q0 = tile * g.C;
    const long long nv = (g.ncols - q0) < g.C ? (g.ncols - q0) : g.C;
    bulk_store_1d(reinterpret_cast<V*>(d.out.p) + q0 * L, buf, (uint32_t)(nv * L * (long long)sizeof(V)));
  } else {
    const int ti = (int)(tile % g.tiles_i);
    const int o = (int)(tile / g.tiles_i);
    for (int b = 0; b < g.nlb; ++b)
      tma_store_3d(map, buf + (size_t)b * g.lb * g.C, ti * g.C * g.xscale, b * g.lb, o);
  }
}

// Shared-memory layout of the pipelined kernels (bytes):
//   [0, 128)                  kTmaBufs mbarriers; abort flag at byte 64
//   [128, 128 + tw)           stage twiddles (ntw entries, padded to 128 bytes)
//   then kTmaBufs tile buffers of C*L elements, bstride apart
//   then (CONTIG) one padded work buffer of C*ld elements
// Bulk-tensor copies need 128-byte aligned shared addresses: the twiddle
// region, the buffer stride and (host-checked) every box offset inside a
// buffer are multiples of 128 bytes; the kernel re-checks and reports
// DFFT_DEVERR_TMA_ALIGN instead of issuing a misaligned copy.
// CS: columns per tile fixed at compile time (strided variant; 0 = runtime,
// contiguous variant).
template <typename T, int LB, bool CONTIG, int CS, int L, int P, int... Rs>
__global__ void __launch_bounds__(LB) axis_pass_pipe(const PassDesc d,
                                                     const __grid_constant__ CUtensorMap tin,
                                                     const __grid_constant__ CUtensorMap tout,
                                                     const TmaGeom g) {
  typedef typename cvec<T>::type V;
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_pipe);
  int& s_abort = *reinterpret_cast<int*>(smem_pipe + 64);  // inside the barrier block
  V* stw = reinterpret_cast<V*>(smem_pipe + 128);
  const size_t tw_bytes = ((size_t)g.ntw * sizeof(V) + 127) & ~(size_t)127;
  V* bufs = reinterpret_cast<V*>(smem_pipe + 128 + tw_bytes);
  const size_t buf_elems = (size_t)g.bstride;
  V* work = bufs + kTmaBufs * buf_elems;
  const int tid = threadIdx.x;
  int c, t;
  if constexpr (CONTIG) { t = tid % P; c = tid / P; }
  else if constexpr (CS > 0) { c = tid % CS; t = tid / CS; }
  else { c = tid % g.C; t = tid / g.C; }
  if (tid == 0) {
    for (int b = 0; b < kTmaBufs; ++b) mbar_init(&bars[b], 1);
    mbar_fence_init();
    s_abort = 0;
    const uint32_t a0 = smem_u32(bufs);
    const uint32_t bs = (uint32_t)(buf_elems * sizeof(V));
    const uint32_t box = CONTIG ? 0u : (uint32_t)((size_t)g.lb * g.C * sizeof(V));
    const uint32_t need = CONTIG ? 15u : 127u;
    if ((a0 & need) || (bs & need) || (g.nlb > 1 && (box & 127u))) {
      atomicExch(g.err, DFFT_DEVERR_TMA_ALIGN);
      s_abort = 1;
    }
  }
  const V* gtw = reinterpret_cast<const V*>(d.tw);
  for (int i = tid; i < g.ntw; i += blockDim.x) stw[i] = gtw[i];
  __syncthreads();
  if (s_abort) return;  // misaligned layout: nothing was issued
  const int C = g.C;
  const StageTw<V> tw{stw};
  const GlobalTw<V> twl{reinterpret_cast<const V*>(d.tw2)};
  const long long first = blockIdx.x;
  const long long step = gridDim.x;
  int issued[kTmaBufs] = {0, 0, 0};  // loads issued per buffer (thread 0)
  if (tid == 0) {
    for (int b = 0; b < kTmaBufs - 1; ++b) {
      const long long tile = first + b * step;
      if (tile < g.ntiles) {
        pipe_issue_load<V, CONTIG, L>(d, &tin, bufs + b * buf_elems, &bars[b], g, tile);
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
    if (CONTIG) {
      const StrideCol<V> dense{sb + (size_t)c * L, 1};
      const PadCol<V> pad{work + (size_t)c * g.ld};
      static_stages<T, L, P, true, 1, 0, 0, 1, 1, 0, StrideCol<V>, PadCol<V>, StrideCol<V>, StageTw<V>,
                    Rs...>(d, t, dense, pad, dense, tw, 0, 0, true);
    } else {
      if constexpr (CS > 0) {
        const StrideColC<V, CS> col{sb + c};
        static_stages<T, L, P, true, 1, 0, 0, 1, 1, 0, StrideColC<V, CS>, StrideColC<V, CS>,
                      StrideColC<V, CS>, GlobalTw<V>, Rs...>(d, t, col, col, col, twl, 0, 0, true);
      } else {
        const StrideCol<V> col{sb + c, C};
        static_stages<T, L, P, true, 1, 0, 0, 1, 1, 0, StrideCol<V>, StrideCol<V>, StrideCol<V>,
                      GlobalTw<V>, Rs...>(d, t, col, col, col, twl, 0, 0, true);
      }
      if (g.tw_lo) {
        // the four-step twiddle on the transformed tile (row k at k * C + c;
        // the stages ended with a barrier), then a barrier before the store
        const V* lo = reinterpret_cast<const V*>(g.tw_lo);
        const V* hi = reinterpret_cast<const V*>(g.tw_hi);
        const long long q0 = (tile % g.tiles_i) * (long long)C;
        for (int e = tid; e < C * L; e += blockDim.x) {
          const int k = e / C;
          const long long q = q0 + (e - k * C);
          const long long m = ((q / g.tw_div) * (long long)k) % g.tw_lf;
          const V w = cmul(ldg_c(lo + m % g.tw_b), ldg_c(hi + m / g.tw_b));
          sb[e] = cmul(sb[e], w);
        }
        __syncthreads();
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      // the buffer of tile it-1 is free once its store has read shared memory
      bulk_wait_read_all();
      const long long next = tile + (long long)(kTmaBufs - 1) * step;
      if (next < g.ntiles) {
        const int nb = (it + kTmaBufs - 1) % kTmaBufs;
        pipe_issue_load<V, CONTIG, L>(d, &tin, bufs + nb * buf_elems, &bars[nb], g, next);
        ++issued[nb];
      }
      pipe_issue_store<V, CONTIG, L>(d, &tout, sb, g, tile);
      bulk_commit();
    }
  }
  if (tid == 0) {
    bulk_wait_all();
    if (s_abort) {
      atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
      // loads still in flight land in this CTA's shared memory: wait for the
      // last load issued into each buffer (bounded) before the CTA exits
      for (int b = 0; b < kTmaBufs; ++b)
        if (issued[b] > 0) mbar_wait_bounded(&bars[b], (uint32_t)((issued[b] - 1) & 1));
    }
  }
  __syncthreads();
}

}  // namespace dfft
