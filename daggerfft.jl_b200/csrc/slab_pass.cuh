// Fused 2-D (dim 1, dim 2) pass over the L x L slabs of an L x L x O array:
// the Slab decomposition's first stage (a 2-D FFT per slab, src/fft.jl:735,
// src/fftgpu.jl:541) in ONE sweep of HBM instead of two.
//
// Work is a global sequence of jobs.  An x-job transforms CS whole pencils
// of a slab (one 1-D bulk copy in, stage 1 from the dense tile, the other
// stages in a swizzled layout in the same buffer, the last stage stored
// straight to the output with coalesced writes).  A y-job transforms CS
// columns x L rows of a slab: TMA 3-D boxes of the output, which the slab's
// x-jobs wrote a moment earlier and which is still in L2, the middle stages
// in a row-swizzled layout, and a TMA store of the dense result.  The sequence is round-major: round r holds the T = L/CS
// x-jobs of slab r followed by the T y-jobs of slab r - lag, so a y-job is
// claimed `lag` rounds after its slab's x-jobs and normally finds them
// finished; only a few slabs (a few MB) are resident in L2 between the two
// phases, so every element is read from and written to DRAM once for both
// axes.
//
// Each persistent CTA has CS*P stage threads and one producer warp.  The
// producer (lane 0) claims runs of consecutive jobs through an atomic
// counter, works through them in order, waits
// until a y-job's slab has all its x-tiles, issues the tile loads into
// NB buffers (full barriers), and, when the stage threads hand a buffer
// back (empty barriers), publishes a finished x-tile in the slab's counter
// or issues the TMA store of a finished y-tile (and waits until the store
// has read the buffer before refilling it).  The stage threads synchronise
// on named barrier 1 only, so no global atomic, counter wait or store wait
// sits on their path.
//
// Progress: x-jobs never wait on other jobs, a CTA works through its claimed
// jobs in claim order, and a producer publishes its own finished x-tiles
// before it waits on a slab counter, so the unfinished job with the smallest
// sequence number can always proceed: the sequence completes whether or not
// all CTAs are resident.  Every wait (mbarrier, slab counter) is bounded;
// after a timeout the CTA records DFFT_DEVERR_TMA_TIMEOUT, and every CTA
// stops claiming jobs once the device error word is set.  The counters (one
// 64-bit job counter, then one 32-bit counter per slab) are zeroed by the
// host before each launch.
#pragma once
#include "tma_pass.cuh"

namespace dfft {

struct SlabGeom {
  long long nslab;   // O: slabs in the array (batch included)
  int tiles;         // T = L / CS tiles per phase per slab
  int lag;           // rounds between a slab's x-jobs and its y-jobs
  int xscale;        // TMA x units per complex element (1 float, 2 double)
  int lb, nlb;       // rows per TMA box, boxes per y tile
  int ntw;           // stage-twiddle entries staged in shared memory
  int bstride;       // elements between tile buffers (128-byte multiple)
  // Rank-split layouts (distributed Slab exchange).  A side with R rows per
  // rank holds row y of slab z (a pencil of L elements) at row
  //   (y mod R) + R * (z + zr * (y / R)),
  // so the rows every rank owns (R of them per slab) form one contiguous
  // block per rank.  R = L is the plain layout.  The x-phase reads the
  // input with rin and writes the output with rout; the y-phase reads and
  // writes the output (tensor map {L, rout, ...}) with rout.
  int rin, rout;
  long long zr;
  unsigned long long* jobs;  // next job in the sequence
  unsigned* done;            // x-tiles finished, per slab
  int* err;
};

constexpr int kSlabClaim = 1;     // jobs per claim of the slab pass
constexpr int kSlabHeader = 256;  // shared-memory bytes before the stage twiddles

struct SlabJob {
  int kind;    // 0 none, 1 x-job, 2 y-job
  int slab;
  int tile;
  int pad;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Shared-memory layouts of the tiles between the first and the last stage.
// Both are XOR permutations inside aligned 128-byte groups (no padding),
// chosen so that every stage's 32-lane accesses of 8-byte (16-byte) elements
// fill each 128-byte wavefront: the first stage's radix-R0 writes land
// R0 elements (x-phase) or R0 rows (y-phase) apart, which the plain layout
// maps onto the same banks.
//   x-phase, pencil c, element k:  c*L + xswz(c, k)
//   y-phase, row k, column c:      yswz(k)*CS + c
template <int ESZ, int L, int R0> __device__ __forceinline__ int xswz(int c, int k) {
  if constexpr (ESZ == 8 && L == 512 && R0 == 8) return k ^ (((k >> 4) & 7) | (((k >> 6) & 1) << 3));
  else if constexpr (ESZ == 8 && L == 512 && R0 == 32) return k ^ ((k >> 5) & 15);
  else if constexpr (ESZ == 8 && L >= 256 && R0 == 16) return k ^ ((k >> 4) & 15);
  else if constexpr (ESZ == 8 && L == 128) return k ^ (((k >> 4) & 7) | ((c & 1) << 3));
  else if constexpr (ESZ == 16 && L == 512 && R0 == 8) return k ^ ((k >> 3) & 7);
  else if constexpr (ESZ == 16 && L >= 256 && R0 == 16) return k ^ ((k >> 4) & 7);
  else return k;
}
template <int ESZ, int CS, int R0> __device__ __forceinline__ int yswz(int k) {
  constexpr int slots = 128 / ESZ;                 // elements per 128 bytes
  constexpr int mask = (slots > CS ? slots / CS : 1) - 1;
  return k ^ ((k / R0) & mask);
}
// Both swizzles are linear over GF(2) in the bits of k (each XORed bit is
// one bit of k or of c), and a stage's index splits into a per-butterfly
// base and an offset r * stride with disjoint bits (L and the radices are
// powers of two), so swz(base | off) = swz(base) ^ swz(off): one swizzle per
// butterfly and one XOR with a constant per access.
template <typename V, int L, int R0> struct XSwzCol {
  static_assert((L & (L - 1)) == 0, "bit-split addressing needs a power-of-two length");
  V* p;  // the pencil's dense start
  int c;
  __device__ __forceinline__ int at(int b, int off) const {
    return xswz<sizeof(V), L, R0>(c, b) ^ xswz<sizeof(V), L, R0>(0, off);
  }
  __device__ __forceinline__ V ld(int b, int off) const { return p[at(b, off)]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[at(b, off)] = v; }
};
template <typename V, int CS, int R0> struct YSwzCol {
  static_assert((R0 & (R0 - 1)) == 0, "bit-split addressing needs power-of-two radices");
  V* p;  // the tile buffer + column
  __device__ __forceinline__ int at(int b, int off) const {
    return (yswz<sizeof(V), CS, R0>(b) ^ yswz<sizeof(V), CS, R0>(off)) * CS;
  }
  __device__ __forceinline__ V ld(int b, int off) const { return p[at(b, off)]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[at(b, off)] = v; }
};
template <int R, int... Rest> struct first_radix { static constexpr int value = R; };

// Tile buffer of CS pencils written in pieces of 2^rsh elements: element k
// of pencil c at ((k >> rsh) * CS + c) * 2^rsh + (k mod 2^rsh), so piece s of
// all CS pencils is one contiguous run (one bulk store per rank block).
template <typename V> struct PieceCol {
  V* p;  // the tile buffer
  int c, cs, rsh;
  __device__ __forceinline__ int at(int b, int off) const {
    const int k = b + off;
    return ((((k >> rsh) * cs) + c) << rsh) | (k & ((1 << rsh) - 1));
  }
  __device__ __forceinline__ V ld(int b, int off) const { return p[at(b, off)]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[at(b, off)] = v; }
};

// Row index (in units of L elements) of row y of slab z in a side with R
// rows per rank (see SlabGeom).
__device__ __forceinline__ long long split_row(int R, long long zr, long long z, int y) {
  return (long long)(y % R) + (long long)R * (z + zr * (long long)(y / R));
}
// The same for the kernel's two forms: SPLIT = false is the plain layout
// (row z * L + y, no run-time division), SPLIT = true reads R from g.
template <bool SPLIT, int L>
__device__ __forceinline__ long long slab_row(int R, long long zr, long long z, int y) {
  if constexpr (SPLIT) return split_row(R, zr, z, y);
  else return z * L + y;
}

// dx: x-phase descriptor (in -> out, contiguous pencils, FAST_IO global
// stores); dy: y-phase descriptor (scale / inverse of the second axis).
// tout: tensor map {L*xscale, L, O} over the output (y-phase loads/stores).
// Shared memory: [0, kSlabHeader) full barriers (byte 0), empty barriers
// (byte 32), the stage threads' abort flag (byte 64) and the buffers' job
// records (byte 80); stage twiddles; NB tile buffers.
// MINB: CTAs per SM the tile buffers allow (register budget per thread).
// DIR: 1 forward, 2 inverse (compiled in: no per-element direction tests).
// MODE 0: x-phase then y-phase, plain layouts (the rin / rout / zr fields
// unused; tin unused).  MODE 1: the same order, rows split by rank
// (SlabGeom; the x-phase reads dx.in.p with rin and writes dx.out.p with
// rout, the y-phase reads and writes through tout = the rout layout).
// MODE 2: y-phase first, columns split by rank: the y-phase reads through
// tin (the input; its x columns in blocks of rin per rank: column x of row
// y of slab z at (x mod rin) + rin * (y + L * (z + zr * (x / rin)))) and
// writes the plain intermediate through tout; the x-phase reads the
// intermediate (dx.in.p) and writes dx.out.p in the same column-split
// layout with rout (pieces of rout elements of each pencil, one block per
// rank).  rin / rout = L is the plain layout.
template <typename T, int LB, int MINB, int NB, int DIR, int MODE, int L, int P, int CS, int... Rs>
__global__ void __launch_bounds__(LB, MINB)
    slab_xy_pass(const PassDesc dx, const PassDesc dy, const __grid_constant__ CUtensorMap tin,
                 const __grid_constant__ CUtensorMap tout, const SlabGeom g) {
  typedef typename cvec<T>::type V;
  constexpr bool SPLIT = MODE == 1;     // rows split by rank (x-phase first)
  constexpr bool YX = MODE == 2;        // y-phase first, columns split by rank
  constexpr int K1 = YX ? 2 : 1;        // job kind of the first phase
  constexpr int K2 = YX ? 1 : 2;        // and of the second
  constexpr int NC = CS * P;  // stage threads
  static_assert(NC % 32 == 0 && NC + 32 == LB, "whole warps of stage threads plus one producer warp");
  static_assert(NB >= 2 && NB <= 4, "tile buffers");
  extern __shared__ __align__(128) unsigned char smem_slab[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_slab);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem_slab + 32);
  int& s_cabort = *reinterpret_cast<int*>(smem_slab + 64);
  SlabJob* s_job = reinterpret_cast<SlabJob*>(smem_slab + 80);
  V* stw = reinterpret_cast<V*>(smem_slab + kSlabHeader);
  const size_t tw_bytes = ((size_t)g.ntw * sizeof(V) + 127) & ~(size_t)127;
  V* bufs = reinterpret_cast<V*>(smem_slab + kSlabHeader + tw_bytes);
  const size_t bst = (size_t)g.bstride;
  const int tid = threadIdx.x;
  const long long Tt = g.tiles;
  volatile int* verr = g.err;

  if (tid == 0) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_fence_init();
    s_cabort = 0;
    const uint32_t a0 = smem_u32(bufs);
    if ((a0 & 127u) || ((bst * sizeof(V)) & 127u) || (g.nlb > 1 && (((size_t)g.lb * CS * sizeof(V)) & 127u))) {
      atomicExch(g.err, DFFT_DEVERR_TMA_ALIGN);
      s_cabort = 1;
    }
  }
  const V* gtw = reinterpret_cast<const V*>(dx.tw);
  for (int i = tid; i < g.ntw; i += blockDim.x) stw[i] = gtw[i];
  __syncthreads();

  if (tid >= NC) {
    if (tid == NC) {
      // ---------------- producer ----------------
      const unsigned long long total =
          (unsigned long long)(g.nslab + g.lag) * 2ull * (unsigned long long)Tt;
      const uint32_t tile_bytes = (uint32_t)((size_t)CS * L * sizeof(V));
      int fills[NB] = {};  // arrivals on full[b]
      int kindb[NB] = {};  // job in buffer b not yet handed back
      int slabb[NB] = {};
      int tileb[NB] = {};
      bool failed = false;
      // waits until the stage threads hand buffer b back; publishes an
      // x-tile, or stores a y-tile and waits until the store has read it
      auto settle = [&](int b) -> bool {
        if (kindb[b] == 0) return true;
        if (!mbar_wait_bounded(&empty[b], (uint32_t)((fills[b] - 1) & 1))) return false;
        const V* buf = bufs + b * bst;
        if (kindb[b] == 1 && !YX) {
          // the transformed pencils, contiguous in the output (CS divides
          // rout): one bulk store
          V* dst = reinterpret_cast<V*>(dx.out.p) + slab_row<SPLIT, L>(g.rout, g.zr, slabb[b], tileb[b] * CS) * L;
          bulk_store_1d(dst, buf, tile_bytes);
        } else if (kindb[b] == 1) {
          // pieces of rout elements of the CS pencils, one block per rank
          // (the stage threads left piece s of every pencil together)
          const int y0 = tileb[b] * CS;
          const uint32_t piece = (uint32_t)((size_t)CS * g.rout * sizeof(V));
          for (int s = 0; s * g.rout < L; ++s)
            bulk_store_1d(reinterpret_cast<V*>(dx.out.p) +
                              (long long)g.rout * (y0 + (long long)L * (slabb[b] + g.zr * s)),
                          buf + (size_t)s * CS * g.rout, piece);
        } else {
          for (int kb = 0; kb < g.nlb; ++kb) {
            const int y = kb * g.lb;  // boxes never straddle a rank's rows (lb divides rout)
            if constexpr (SPLIT)
              tma_store_3d(&tout, buf + (size_t)kb * g.lb * CS, tileb[b] * CS * g.xscale, y % g.rout,
                           (int)(slabb[b] + g.zr * (y / g.rout)));
            else
              tma_store_3d(&tout, buf + (size_t)kb * g.lb * CS, tileb[b] * CS * g.xscale, y, slabb[b]);
          }
        }
        bulk_commit();
        if (kindb[b] == K1) {
          // a first-phase tile: complete before it is published (async-proxy
          // writes, made visible to the generic release by the proxy fence;
          // readers fence again before their bulk / tensor loads)
          bulk_wait_all();
          fence_proxy_async_global();
          asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.done + slabb[b]) : "memory");
        } else {
          bulk_wait_read_all();  // the buffer is free once the store has read it
        }
        kindb[b] = 0;
        return true;
      };
      auto wait_slab = [&](int slab) -> bool {
        const uint64_t t0 = global_ns();
        for (unsigned i = 0; i < kWaitLimit; ++i) {
          if (ld_acquire_gpu(g.done + slab) >= (unsigned)Tt) return true;
          if (*verr != 0) return false;
          if ((i & 63) == 0 && global_ns() - t0 > kWaitNs) return false;
          __nanosleep(64);
        }
        return false;
      };
      // jobs are claimed kSlabClaim at a time (consecutive sequence numbers)
      unsigned long long next = 0, chunk_end = 0;
      for (int it = 0;; ++it) {
        const int b = it % NB;
        if (!settle(b)) { failed = true; break; }
        SlabJob J{0, 0, 0, 0};
        while (*verr == 0) {
          if (next == chunk_end) {
            next = atomicAdd(g.jobs, (unsigned long long)kSlabClaim);
            chunk_end = next + kSlabClaim;
          }
          const unsigned long long n = next++;
          if (n >= total) break;
          const long long r = (long long)(n / (2ull * Tt));
          const long long i = (long long)(n % (2ull * Tt));
          if (i < Tt) {
            if (r >= g.nslab) continue;
            J = SlabJob{K1, (int)r, (int)i, 0};
          } else {
            const long long sl = r - g.lag;
            if (sl < 0 || sl >= g.nslab) continue;
            J = SlabJob{K2, (int)sl, (int)(i - Tt), 0};
          }
          break;
        }
        if (J.kind == K2 && ld_acquire_gpu(g.done + J.slab) < (unsigned)Tt) {
          // first-phase tiles of that slab may sit in this CTA's other
          // buffers: publish them first
          bool ok = true;
          for (int bb = 0; bb < NB; ++bb)
            if (kindb[bb] == K1) ok = settle(bb) && ok;
          if (!ok || !wait_slab(J.slab)) { failed = true; J.kind = 0; }
        }
        s_job[b] = J;
        ++fills[b];
        if (J.kind == 0) {
          mbar_arrive(&full[b]);  // no more work: the stage threads leave
          break;
        }
        V* buf = bufs + b * bst;
        mbar_expect_tx(&full[b], tile_bytes);
        if (J.kind == 1) {
          // CS divides rin: the tile's CS pencils are contiguous in both
          // layouts (MODE 2: the plain intermediate the y-phase wrote)
          if constexpr (YX) fence_proxy_async_global();  // after the acquire, before these async reads
          bulk_load_1d(buf, reinterpret_cast<const V*>(dx.in.p) +
                                (YX ? ((long long)J.slab * L + (long long)J.tile * CS)
                                    : slab_row<SPLIT, L>(g.rin, g.zr, J.slab, J.tile * CS)) * L,
                       tile_bytes, &full[b]);
        } else if constexpr (YX) {
          // columns x0.. of the input, in the rank block holding them
          const int x0 = J.tile * CS;
          for (int kb = 0; kb < g.nlb; ++kb)
            tma_load_3d(buf + (size_t)kb * g.lb * CS, &tin, &full[b], (x0 % g.rin) * g.xscale, kb * g.lb,
                        (int)(J.slab + g.zr * (x0 / g.rin)));
        } else {
          fence_proxy_async_global();  // after the acquire, before these async-proxy reads
          for (int kb = 0; kb < g.nlb; ++kb) {
            const int y = kb * g.lb;
            if constexpr (SPLIT)
              tma_load_3d(buf + (size_t)kb * g.lb * CS, &tout, &full[b], J.tile * CS * g.xscale, y % g.rout,
                          (int)(J.slab + g.zr * (y / g.rout)));
            else
              tma_load_3d(buf + (size_t)kb * g.lb * CS, &tout, &full[b], J.tile * CS * g.xscale, y, J.slab);
          }
        }
        kindb[b] = J.kind;
        slabb[b] = J.slab;
        tileb[b] = J.tile;
      }
      // publish the first-phase tiles and store the others still held by
      // this CTA (on the error path too: other CTAs may wait for them)
      for (int bb = 0; bb < NB; ++bb)
        if (!settle(bb)) failed = true;
      if (failed && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
      bulk_wait_all();
      // no bulk copy may still be landing in shared memory when the CTA exits
      for (int bb = 0; bb < NB; ++bb)
        if (fills[bb] > 0) mbar_wait_bounded(&full[bb], (uint32_t)((fills[bb] - 1) & 1));
    }
  } else {
    // ---------------- stage threads ----------------
    // both phases have the same length and radices: one stage-twiddle table
    // (for the inverse, with 1/L folded into the last stage's entries; both
    // phases scale by 1/L)
    typedef typename std::conditional<DIR == 2, StageTwScaledLast<V>, StageTw<V>>::type TWT;
    const TWT tw{stw};
    constexpr int R0 = first_radix<Rs...>::value;
    for (int it = 0;; ++it) {
      const int b = it % NB;
      if (!mbar_wait_bounded(&full[b], (uint32_t)((it / NB) & 1))) s_cabort = 1;
      stage_sync<NC>();
      if (s_cabort) break;
      const SlabJob J = s_job[b];
      if (J.kind == 0) break;
      V* buf = bufs + b * bst;
      if (J.kind == 1) {
        // pencils in place: dense in, swizzled between stages, dense out
        // (the producer bulk-stores the tile)
        const int t = tid % P, c = tid / P;
        const StrideCol<V> dense{buf + (size_t)c * L, 1};
        const XSwzCol<V, L, R0> sw{buf + (size_t)c * L, c};
        if constexpr (YX) {
          // out in pieces of rout elements, piece s of every pencil together
          const PieceCol<V> pc{buf, c, CS, __ffs(g.rout) - 1};
          static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, StrideCol<V>, XSwzCol<V, L, R0>, PieceCol<V>,
                        TWT, Rs...>(dx, t, dense, sw, pc, tw, 0, 0, true);
        } else {
          static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, StrideCol<V>, XSwzCol<V, L, R0>, StrideCol<V>,
                        TWT, Rs...>(dx, t, dense, sw, dense, tw, 0, 0, true);
        }
      } else {
        const int c = tid % CS, t = tid / CS;
        const StrideColC<V, CS> dense{buf + c};
        const YSwzCol<V, CS, R0> sw{buf + c};
        static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, StrideColC<V, CS>, YSwzCol<V, CS, R0>, StrideColC<V, CS>,
                      TWT, Rs...>(dy, t, dense, sw, dense, tw, 0, 0, true);
      }
      fence_proxy_async_smem();  // the buffer is next read (store) or written (load) by TMA
      stage_sync<NC>();
      if (tid == 0) mbar_arrive(&empty[b]);  // the producer publishes (x) or stores (y) the tile
    }
    if (tid == 0 && s_cabort && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
  }
  __syncthreads();
}

}  // namespace dfft

namespace dfft {

// ---------------------------------------------------------------------------
// Strided-axis pass with a producer warp (the y-phase machinery of the slab
// pass without the slab dependency): tile t of the tensor {I*xscale, L, O}
// is CS columns x L rows (x = (t % tiles_i)*CS, z = t / tiles_i), loaded
// and stored by TMA boxes {CS*xscale, lb, 1}; CTA b takes tiles b, b+grid, ...
// The producer (lane 0 of the last warp) fills NB buffers as the stage
// threads hand them back, storing each transformed tile (TMA) before it
// refills the buffer; the stage threads run the stages in the
// row-swizzled layout with the stage twiddles in shared memory and sync on
// named barrier 1.  Bounded waits as in the slab pass.
// ---------------------------------------------------------------------------

struct StridedGeom {
  long long ntiles;  // tiles_i * O
  int tiles_i;       // tiles along I
  int xscale, lb, nlb;
  int ntw, bstride;
  int* err;
};

template <typename T, int LB, int MINB, int NB, int DIR, int L, int P, int CS, int... Rs>
__global__ void __launch_bounds__(LB, MINB)
    axis_pass_strided(const PassDesc d, const __grid_constant__ CUtensorMap tin,
                      const __grid_constant__ CUtensorMap tout, const StridedGeom g) {
  typedef typename cvec<T>::type V;
  constexpr int NC = CS * P;
  static_assert(NC % 32 == 0 && NC + 32 == LB, "whole warps of stage threads plus one producer warp");
  static_assert(NB >= 2 && NB <= 4, "tile buffers");
  constexpr int R0 = first_radix<Rs...>::value;
  constexpr bool kPow2 = (L & (L - 1)) == 0 && (((Rs & (Rs - 1)) == 0) && ...);
  extern __shared__ __align__(128) unsigned char smem_str[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_str);
  uint64_t* empty = reinterpret_cast<uint64_t*>(smem_str + 32);
  int& s_cabort = *reinterpret_cast<int*>(smem_str + 64);
  long long* s_tile = reinterpret_cast<long long*>(smem_str + 80);  // NB entries
  V* stw = reinterpret_cast<V*>(smem_str + kSlabHeader);
  const size_t tw_bytes = ((size_t)g.ntw * sizeof(V) + 127) & ~(size_t)127;
  V* bufs = reinterpret_cast<V*>(smem_str + kSlabHeader + tw_bytes);
  const size_t bst = (size_t)g.bstride;
  const int tid = threadIdx.x;
  volatile int* verr = g.err;

  if (tid == 0) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_fence_init();
    s_cabort = 0;
    const uint32_t a0 = smem_u32(bufs);
    if ((a0 & 127u) || ((bst * sizeof(V)) & 127u) || (g.nlb > 1 && (((size_t)g.lb * CS * sizeof(V)) & 127u))) {
      atomicExch(g.err, DFFT_DEVERR_TMA_ALIGN);
      s_cabort = 1;
    }
  }
  const V* gtw = reinterpret_cast<const V*>(d.tw);
  for (int i = tid; i < g.ntw; i += blockDim.x) stw[i] = gtw[i];
  __syncthreads();

  if (tid >= NC) {
    if (tid == NC) {
      // ---------------- producer ----------------
      const uint32_t tile_bytes = (uint32_t)((size_t)CS * L * sizeof(V));
      int fills[NB] = {};
      long long pend[NB];  // transformed tile in buffer b still to be stored, or -1
      for (int bb = 0; bb < NB; ++bb) pend[bb] = -1;
      bool failed = false;
      // waits until the stage threads hand buffer b back, then stores its
      // tile and waits until the store has read the buffer
      auto drain = [&](int b) -> bool {
        if (pend[b] < 0) return true;
        if (!mbar_wait_bounded(&empty[b], (uint32_t)((fills[b] - 1) & 1))) return false;
        const int ti = (int)(pend[b] % g.tiles_i);
        const int o = (int)(pend[b] / g.tiles_i);
        const V* buf = bufs + b * bst;
        for (int kb = 0; kb < g.nlb; ++kb)
          tma_store_3d(&tout, buf + (size_t)kb * g.lb * CS, ti * CS * g.xscale, kb * g.lb, o);
        bulk_commit();
        bulk_wait_read_all();
        pend[b] = -1;
        return true;
      };
      long long tile = blockIdx.x;
      for (int it = 0;; ++it) {
        const int b = it % NB;
        // the buffer's previous tile must be handed back and stored first
        if (!drain(b)) {
          failed = true;
          break;
        }
        const bool more = tile < g.ntiles && *verr == 0 && !s_cabort;
        s_tile[b] = more ? tile : -1;
        ++fills[b];
        if (!more) {
          mbar_arrive(&full[b]);  // no more tiles: the stage threads leave
          break;
        }
        const int ti = (int)(tile % g.tiles_i);
        const int o = (int)(tile / g.tiles_i);
        V* buf = bufs + b * bst;
        mbar_expect_tx(&full[b], tile_bytes);
        for (int kb = 0; kb < g.nlb; ++kb)
          tma_load_3d(buf + (size_t)kb * g.lb * CS, &tin, &full[b], ti * CS * g.xscale, kb * g.lb, o);
        pend[b] = tile;
        tile += gridDim.x;
      }
      // the tiles the stage threads still hold
      for (int bb = 0; bb < NB && !failed; ++bb)
        if (!drain(bb)) failed = true;
      if (failed && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
      bulk_wait_all();
      // no bulk copy may still be landing in shared memory when the CTA exits
      for (int bb = 0; bb < NB; ++bb)
        if (fills[bb] > 0) mbar_wait_bounded(&full[bb], (uint32_t)((fills[bb] - 1) & 1));
    }
  } else {
    // ---------------- stage threads ----------------
    const StageTw<V> tw{stw};
    const int c = tid % CS, t = tid / CS;
    for (int it = 0;; ++it) {
      const int b = it % NB;
      if (!mbar_wait_bounded(&full[b], (uint32_t)((it / NB) & 1))) s_cabort = 1;
      stage_sync<NC>();
      if (s_cabort) break;
      const long long tile = s_tile[b];
      if (tile < 0) break;
      V* buf = bufs + b * bst;
      const StrideColC<V, CS> dense{buf + c};
      if constexpr (kPow2) {
        // row-swizzled middle stages (bit-split addressing)
        const YSwzCol<V, CS, R0> sw{buf + c};
        static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, StrideColC<V, CS>, YSwzCol<V, CS, R0>,
                      StrideColC<V, CS>, StageTw<V>, Rs...>(d, t, dense, sw, dense, tw, 0, 0, true);
      } else {
        // other lengths: the plain [row][column] tile (rows of 128 bytes)
        static_stages<T, L, P, true, 1, NC, DIR, 1, 1, 0, StrideColC<V, CS>, StrideColC<V, CS>,
                      StrideColC<V, CS>, StageTw<V>, Rs...>(d, t, dense, dense, dense, tw, 0, 0, true);
      }
      fence_proxy_async_smem();  // the producer's TMA store reads the tile next
      stage_sync<NC>();
      if (tid == 0) mbar_arrive(&empty[b]);  // hand the transformed tile to the producer
    }
    if (tid == 0 && s_cabort && *verr == 0) atomicExch(g.err, DFFT_DEVERR_TMA_TIMEOUT);
  }
  __syncthreads();
}

}  // namespace dfft
