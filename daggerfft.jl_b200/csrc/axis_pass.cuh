// One batched 1-D transform pass along one axis of a column-major array.
//
// Data model.  A pass transforms Q independent "columns" of FFT length L.
// Column q is split as (qi, qo) = (q % I, q / I); element k of column q of a
// side (input or output) sits at  p[qi*si + qo*so + k*sk]  of that side.  One
// kernel therefore serves the contiguous axis (I = 1: a column is a whole
// pencil) and the strided axes (I = product of the faster dims: consecutive
// columns are adjacent in memory, so the strided loads coalesce).
//
// Work split.  A CTA owns C consecutive columns and runs P threads per column.
// With cfast the column index sits in the fastest thread bits (strided axes:
// a warp reads adjacent elements of one row of the tile); otherwise the
// butterfly index does (contiguous axis: a warp reads one pencil).
//
// Algorithm.  Stockham autosort FFT, stages s = 0..nst-1 with radix R_s and
// Ns = R_0*...*R_{s-1}.  Butterfly j of stage s reads k = j + r*(L/R_s),
// multiplies by w_{Ns*R}^{(j mod Ns)*r}, runs a radix-R_s codelet and writes
// k' = (j - j mod Ns)*R_s + j mod Ns + r*Ns.  The first stage reads straight
// from global memory and the last stage writes straight to global memory (both
// index patterns are unit-stride in j), so a pass costs one read and one write
// of HBM; the nst-1 intermediate exchanges go through shared memory.
//
// The inverse transform runs the forward kernel on conjugated data
// (IDFT(x) = conj(DFT(conj(x)))), with the 1/L scale folded into the store.
//
// Two kernels share the stage body:
//   * axis_pass_static<T, FAST_IO, LB, L, P, R...>: radices known at compile
//     time, every stage inlined and constant-folded (the hot path);
//   * axis_pass_dynamic<T, EMAX>: radices read from the descriptor, one
//     out-of-line function per radix (any 13-smooth length).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>
#include "codelets.cuh"

namespace dfft {

constexpr int kMaxStages = 16;

// How a side of a pass maps FFT elements to memory.
enum IoKind : int {
  IO_CPLX = 0,       // complex elements
  IO_REAL_PAIR = 1,  // real pairs: z_m <-> (x_{2m}, x_{2m+1})
  IO_REAL = 2,       // load (x_k, 0) / store Re z_k
  IO_HERM_PAIR = 3,  // load only: even-length C2R pre-pass (real length 2n)
  IO_HERM_FULL = 4,  // load only: odd-length C2R, Hermitian mirror
  IO_TRUNC = 5,      // store only: complex, keep k <= n
  IO_R2R = 6,        // FFTW r2r kind `r2r` on real data of extent n
  IO_CPLX_TW = 7     // store only: complex times w[(j * k) mod n], j = (b mod t_ia) / t_i
                     // (the twiddle between the two passes of a four-step axis)
};

// FFTW r2r kind numbers (fftw_r2r_kind).
enum : int { K_DHT = 2, K_REDFT00 = 3, K_REDFT01 = 4, K_REDFT10 = 5, K_REDFT11 = 6,
             K_RODFT00 = 7, K_RODFT01 = 8, K_RODFT10 = 9, K_RODFT11 = 10 };

struct IoAny {
  void* p;
  long long si, so, sk;
  int kind;          // IoKind
  int r2r;           // FFTW kind for IO_R2R
  int n;             // logical extent (see the kinds)
  const void* w;     // twiddle table for the kinds that need one
  // Bluestein wrapping (chirp-z) of any kind: element k < chirp_n is
  // multiplied by chirp[k] after loading / before storing, elements
  // k >= chirp_n load as zero and are not stored; mul[k] multiplies a load.
  const void* chirp;
  const void* mul;
  int chirp_n;
  // Two-level column split of the outer index (four-step output): with
  // o1 > 0 the column base is (qo mod o1) * so + (qo / o1) * so2.
  long long o1, so2;
  // Sub-axis of a four-step pair: the column at base b holds elements
  // j + t_m * k of the whole axis, j = (b mod t_ia) / t_i.  IO_CPLX_TW
  // multiplies by w[(j * k) mod n]; with t_m > 0 the chirp and mul tables
  // are indexed by j + t_m * k (Bluestein around a four-step pair).
  long long t_i, t_ia;
  int t_m;
};

// Column base of side `io` for the outer column index qo.
__host__ __device__ __forceinline__ long long io_outer(const IoAny& io, long long qo) {
  return io.o1 > 0 ? (qo % io.o1) * io.so + (qo / io.o1) * io.so2 : qo * io.so;
}

struct PassDesc {
  int L;                    // transform length of this pass
  int nst;                  // number of Stockham stages (dynamic kernel only)
  int radix[kMaxStages];
  int ns[kMaxStages];
  int tws[kMaxStages];
  int P;                    // threads per column
  int C;                    // columns per CTA
  int ld;                   // shared-memory elements reserved per column
  int inverse;              // 1: conjugate on load and on store
  int cfast;                // thread -> (column, butterfly) mapping
  int epi;                  // 1: R2C half-length post-pass on the way out
  long long Q;              // number of columns
  long long I;              // column split q -> (q % I, q / I)
  double scale;             // multiplier applied at the store
  const void* tw;           // L entries exp(-2 pi i m / L)
  const void* tw2;          // epi: L+1 entries exp(-2 pi i m / (2L))
  IoAny in, out;
};

// Bank-conflict swizzle for the shared-memory exchange: one pad element per
// 128 bytes of complex data.
template <typename V> __device__ __forceinline__ int swz(int k) {
  return sizeof(V) == 8 ? k + (k >> 4) : k + (k >> 3);
}

template <typename V> __device__ __forceinline__ V ldg_c(const V* p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Element access for every side kind.  The r2r maps (FFTW kinds, all
// unnormalised) express each kind as one complex FFT:
//   kind      FFT length  input map                            output
//   REDFT10   N           v_k = x_{2k} | x_{2N-2k-1}            Y_k = 2 Re(e^{-i pi k/2N} V_k)
//   RODFT10   N           as REDFT10 on (-1)^n x_n              Y_{N-1-k} = that value
//   REDFT01   N, inverse  V_n = e^{i pi n/2N}(x_n - i x_{N-n})  y_{2m} | y_{2N-2m-1} = Re v_m
//   RODFT01   N, inverse  as REDFT01 on x reversed              times (-1)^k
//   REDFT11   2N          x_n e^{-i pi n/2N}, zero-padded       Y_k = 2 Re(e^{-i pi (2k+1)/4N} X_k)
//   RODFT11   2N          as REDFT11 on x reversed              times (-1)^k
//   REDFT00   2(N-1)      even extension                        Y_k = Re X_k
//   RODFT00   2(N+1)      odd extension [0, x, 0, -rev(x)]      Y_k = -Im X_{k+1}
//   DHT       N           x_n                                   Y_k = Re X_k - Im X_k
// ---------------------------------------------------------------------------

// One FFTW r2r kind's load map (element k of the FFT input, from real data
// of extent N at p[b + n*sk]) and store map (FFT output element k, scaled
// by s, into the real result); w is the kind's twiddle table.
template <typename T, int KIND>
__device__ __forceinline__ typename cvec<T>::type r2r_load(const T* p, long long b, long long sk, int N,
                                                         const typename cvec<T>::type* w, int k) {
  typedef typename cvec<T>::type V;
  const T z = (T)0;
  if constexpr (KIND == K_REDFT10 || KIND == K_RODFT10) {
    const int n = (2 * k < N) ? 2 * k : 2 * N - 2 * k - 1;
    T v = p[b + n * sk];
    if (KIND == K_RODFT10 && (n & 1)) v = -v;
    return mk<V>(v, z);
  } else if constexpr (KIND == K_REDFT01 || KIND == K_RODFT01) {
    const bool rev = (KIND == K_RODFT01);
    const T a = p[b + (rev ? N - 1 - k : k) * sk];
    const T c = (k == 0) ? z : p[b + (rev ? k - 1 : N - k) * sk];
    return cmul(ldg_c(w + k), mk<V>(a, -c));
  } else if constexpr (KIND == K_REDFT11 || KIND == K_RODFT11) {
    if (k >= N) return mk<V>(z, z);
    const T a = p[b + (KIND == K_RODFT11 ? N - 1 - k : k) * sk];
    const V t = ldg_c(w + k);
    return mk<V>(a * t.x, a * t.y);
  } else if constexpr (KIND == K_REDFT00) {
    const int n = (k < N) ? k : 2 * (N - 1) - k;
    return mk<V>(p[b + n * sk], z);
  } else if constexpr (KIND == K_RODFT00) {
    if (k == 0 || k == N + 1) return mk<V>(z, z);
    if (k <= N) return mk<V>(p[b + (k - 1) * sk], z);
    return mk<V>(-p[b + (2 * N + 1 - k) * sk], z);
  } else {  // K_DHT
    return mk<V>(p[b + k * sk], z);
  }
}

template <typename T, int KIND>
__device__ __forceinline__ void r2r_store(T* p, long long b, long long sk, int N, const typename cvec<T>::type* w,
                                          int k, typename cvec<T>::type v, T s) {
  typedef typename cvec<T>::type V;
  if constexpr (KIND == K_REDFT10 || KIND == K_RODFT10) {
    const V t = ldg_c(w + k);
    p[b + (KIND == K_RODFT10 ? N - 1 - k : k) * sk] = (T)2 * (v.x * t.x - v.y * t.y) * s;
  } else if constexpr (KIND == K_REDFT01 || KIND == K_RODFT01) {
    const int n = (2 * k < N) ? 2 * k : 2 * N - 2 * k - 1;
    T y = v.x * s;
    if (KIND == K_RODFT01 && (n & 1)) y = -y;
    p[b + n * sk] = y;
  } else if constexpr (KIND == K_REDFT11 || KIND == K_RODFT11) {
    if (k >= N) return;
    const V t = ldg_c(w + k);
    T y = (T)2 * (v.x * t.x - v.y * t.y) * s;
    if (KIND == K_RODFT11 && (k & 1)) y = -y;
    p[b + k * sk] = y;
  } else if constexpr (KIND == K_REDFT00) {
    if (k < N) p[b + k * sk] = v.x * s;
  } else if constexpr (KIND == K_RODFT00) {
    if (k >= 1 && k <= N) p[b + (k - 1) * sk] = -v.y * s;
  } else {  // K_DHT
    p[b + k * sk] = (v.x - v.y) * s;
  }
}

template <typename T>
__device__ __forceinline__ typename cvec<T>::type load_raw(const IoAny& io, long long b, int k) {
  typedef typename cvec<T>::type V;
  const T z = (T)0;
  switch (io.kind) {
    case IO_CPLX:
      return reinterpret_cast<const V*>(io.p)[b + k * io.sk];
    case IO_REAL_PAIR: {
      const T* p = reinterpret_cast<const T*>(io.p);
      if (io.sk == 1) return *reinterpret_cast<const V*>(p + b + 2 * (long long)k);
      return mk<V>(p[b + (2 * k) * io.sk], p[b + (2 * k + 1) * io.sk]);
    }
    case IO_REAL:
      return mk<V>(reinterpret_cast<const T*>(io.p)[b + k * io.sk], z);
    case IO_HERM_PAIR: {
      // Z'_k = (A + B) + i conj(w^k) (A - B), A = X_k, B = conj(X_{n-k});
      // the inverse FFT of Z' (length n) interleaves to 2n * x.
      const V* p = reinterpret_cast<const V*>(io.p);
      V A = p[b + k * io.sk];
      V B = cconj(p[b + (io.n - k) * io.sk]);
      if (k == 0) { A.y = (T)0; B.y = (T)0; }  // c2r ignores Im X_0 and Im X_{n}
      V wk;
      if (io.w) {
        wk = cconj(ldg_c(reinterpret_cast<const V*>(io.w) + k));
      } else {  // exp(+2 pi i k / (2n)), computed in the kernel
        double sn, cs;
        sincospi((double)k / (double)io.n, &sn, &cs);
        wk = mk<V>((T)cs, (T)sn);
      }
      return cadd(cadd(A, B), cmul_pi(cmul(wk, csub(A, B))));
    }
    case IO_HERM_FULL: {
      const V* p = reinterpret_cast<const V*>(io.p);
      if (io.t_m > 0) {
        // sub-axis of a four-step pair: element kf of the whole axis, whose
        // column starts j rows before b, rows t_i apart
        const long long j = (b % io.t_ia) / io.t_i;
        const long long kf = j + (long long)io.t_m * k;
        const long long b0 = b - j * io.t_i;
        if (kf == 0) return mk<V>(p[b0].x, z);
        if (2 * kf <= io.n) return p[b0 + kf * io.t_i];
        return cconj(p[b0 + (io.n - kf) * io.t_i]);
      }
      if (k == 0) return mk<V>(p[b].x, z);  // c2r ignores Im X_0
      if (2 * k <= io.n) return p[b + k * io.sk];
      return cconj(p[b + (io.n - k) * io.sk]);
    }
    default: {  // IO_R2R
      const T* p = reinterpret_cast<const T*>(io.p);
      const V* w = reinterpret_cast<const V*>(io.w);
      // a four-step sub-axis reads element kf of the whole axis (column
      // base moved back by j rows, rows t_i apart)
      long long bb = b, ss = io.sk;
      int kk = k;
      if (io.t_m > 0) {
        const long long j = (b % io.t_ia) / io.t_i;
        bb = b - j * io.t_i;
        ss = io.t_i;
        kk = (int)(j + (long long)io.t_m * k);
      }
      switch (io.r2r) {
        case K_REDFT10: return r2r_load<T, K_REDFT10>(p, bb, ss, io.n, w, kk);
        case K_RODFT10: return r2r_load<T, K_RODFT10>(p, bb, ss, io.n, w, kk);
        case K_REDFT01: return r2r_load<T, K_REDFT01>(p, bb, ss, io.n, w, kk);
        case K_RODFT01: return r2r_load<T, K_RODFT01>(p, bb, ss, io.n, w, kk);
        case K_REDFT11: return r2r_load<T, K_REDFT11>(p, bb, ss, io.n, w, kk);
        case K_RODFT11: return r2r_load<T, K_RODFT11>(p, bb, ss, io.n, w, kk);
        case K_REDFT00: return r2r_load<T, K_REDFT00>(p, bb, ss, io.n, w, kk);
        case K_RODFT00: return r2r_load<T, K_RODFT00>(p, bb, ss, io.n, w, kk);
        default: return r2r_load<T, K_DHT>(p, bb, ss, io.n, w, kk);
      }
    }
  }
}

template <typename T>
__device__ __forceinline__ void store_raw(const IoAny& io, long long b, int k,
                                          typename cvec<T>::type v, T s) {
  typedef typename cvec<T>::type V;
  switch (io.kind) {
    case IO_CPLX:
      reinterpret_cast<V*>(io.p)[b + k * io.sk] = cscale(v, s);
      return;
    case IO_TRUNC: {
      // (a four-step sub-axis keeps the outputs whose whole-axis index fits)
      const long long kf = io.t_m > 0 ? (b % io.t_ia) / io.t_i + (long long)io.t_m * k : (long long)k;
      if (kf <= io.n) reinterpret_cast<V*>(io.p)[b + k * io.sk] = cscale(v, s);
      return;
    }
    case IO_CPLX_TW: {
      const long long j = (b % io.t_ia) / io.t_i;
      const V w = ldg_c(reinterpret_cast<const V*>(io.w) +
                        (long long)(((unsigned long long)j * (unsigned long long)k) % (unsigned long long)io.n));
      reinterpret_cast<V*>(io.p)[b + k * io.sk] = cscale(cmul(v, w), s);
      return;
    }
    case IO_REAL_PAIR: {
      T* p = reinterpret_cast<T*>(io.p);
      if (io.sk == 1) { *reinterpret_cast<V*>(p + b + 2 * (long long)k) = cscale(v, s); return; }
      p[b + (2 * k) * io.sk] = v.x * s;
      p[b + (2 * k + 1) * io.sk] = v.y * s;
      return;
    }
    case IO_REAL:
      reinterpret_cast<T*>(io.p)[b + k * io.sk] = v.x * s;
      return;
    default: {  // IO_R2R
      T* p = reinterpret_cast<T*>(io.p);
      const V* w = reinterpret_cast<const V*>(io.w);
      long long bb = b, ss = io.sk;  // the whole axis, as for the load
      int kk = k;
      if (io.t_m > 0) {
        const long long j = (b % io.t_ia) / io.t_i;
        bb = b - j * io.t_i;
        ss = io.t_i;
        kk = (int)(j + (long long)io.t_m * k);
      }
      switch (io.r2r) {
        case K_REDFT10: r2r_store<T, K_REDFT10>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_RODFT10: r2r_store<T, K_RODFT10>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_REDFT01: r2r_store<T, K_REDFT01>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_RODFT01: r2r_store<T, K_RODFT01>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_REDFT11: r2r_store<T, K_REDFT11>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_RODFT11: r2r_store<T, K_RODFT11>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_REDFT00: r2r_store<T, K_REDFT00>(p, bb, ss, io.n, w, kk, v, s); return;
        case K_RODFT00: r2r_store<T, K_RODFT00>(p, bb, ss, io.n, w, kk, v, s); return;
        default: r2r_store<T, K_DHT>(p, bb, ss, io.n, w, kk, v, s); return;
      }
    }
  }
}

// Index along the whole axis of element k of the column at base b.
__device__ __forceinline__ long long axis_index(const IoAny& io, long long b, int k) {
  return io.t_m > 0 ? (b % io.t_ia) / io.t_i + (long long)io.t_m * k : (long long)k;
}

// Element access with the optional Bluestein chirp / filter multiply.
template <typename T>
__device__ __forceinline__ typename cvec<T>::type load_elem(const IoAny& io, long long b, int k) {
  typedef typename cvec<T>::type V;
  if (io.chirp) {
    const long long n = axis_index(io, b, k);
    if (n >= io.chirp_n) return mk<V>((T)0, (T)0);
    return cmul(load_raw<T>(io, b, k), ldg_c(reinterpret_cast<const V*>(io.chirp) + n));
  }
  V v = load_raw<T>(io, b, k);
  if (io.mul) v = cmul(v, ldg_c(reinterpret_cast<const V*>(io.mul) + axis_index(io, b, k)));
  return v;
}

template <typename T>
__device__ __forceinline__ void store_elem(const IoAny& io, long long b, int k,
                                           typename cvec<T>::type v, T s) {
  typedef typename cvec<T>::type V;
  if (io.chirp) {
    const long long n = axis_index(io, b, k);
    if (n >= io.chirp_n) return;
    v = cmul(v, ldg_c(reinterpret_cast<const V*>(io.chirp) + n));
  }
  store_raw<T>(io, b, k, v, s);
}

// ---------------------------------------------------------------------------
// Stage body.
// ---------------------------------------------------------------------------

// Shared-memory view of one column.  PadCol: column-major with one pad
// element per 128 bytes (direct-load kernels); StrideCol: the [k][c] layout a
// TMA tile box lands in (c fastest), conflict-free for the cfast mapping.
// Every view is addressed as (base, off): element base + off, where the
// stage passes its per-butterfly index as base and r * stride (a constant
// once the radix loop is unrolled) as off.  Views whose layout is a bitwise
// map use it to split the address into a per-butterfly part and a constant.
template <typename V> struct PadCol {
  V* p;
  __device__ __forceinline__ V ld(int b, int off) const { return p[swz<V>(b + off)]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[swz<V>(b + off)] = v; }
};
template <typename V> struct StrideCol {
  V* p;
  int s;
  __device__ __forceinline__ V ld(int b, int off) const { return p[(b + off) * s]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[(b + off) * s] = v; }
};
// StrideCol with a compile-time stride: every tile offset becomes an
// immediate of the shared-memory instruction instead of a live register.
template <typename V, int S> struct StrideColC {
  V* p;
  __device__ __forceinline__ V ld(int b, int off) const { return p[(b + off) * S]; }
  __device__ __forceinline__ void st(int b, int off, V v) const { p[(b + off) * S] = v; }
};

// Twiddle sources.  GlobalTw reads w_L^{jm*r*ts} from the L-entry table;
// StageTw reads a stage-major table laid out [stage][jm][r-1] (entry
// Ns - R_0 + jm*(R-1) + r-1 holds exp(-2 pi i jm r / (Ns R))), which the
// persistent kernels keep in shared memory: lanes with consecutive jm read
// consecutive (R-1)-strided entries, conflict-free.
template <typename V> struct GlobalTw {
  const V* p;
  __device__ __forceinline__ V w(int off, int jm, int r, int R, int ts) const {
    return ldg_c(p + jm * r * ts);
  }
};
template <typename V> struct StageTw {
  const V* p;
  __device__ __forceinline__ V w(int off, int jm, int r, int R, int ts) const {
    return p[off + jm * (R - 1) + r - 1];
  }
};
// The same table with the last stage's entries pre-multiplied by the
// inverse's 1/L (exact for power-of-two L): the last stage of an inverse
// then scales only its r = 0 inputs, and the DFT carries the scale to every
// output (linearity), instead of scaling every output.
template <typename V> struct StageTwScaledLast : StageTw<V> {};
template <class TW> struct scaled_last_tw { static constexpr bool value = false; };
template <typename V> struct scaled_last_tw<StageTwScaledLast<V>> { static constexpr bool value = true; };
// Twiddles computed in the kernel (no table in memory): exp(-2 pi i jm r ts / L)
// with the CUDA math library's sincospi in double precision.
template <typename V> struct ComputedTw {
  int L;
  __device__ __forceinline__ V w(int off, int jm, int r, int R, int ts) const {
    typedef typename scalar_of<V>::type S;
    const long long m = ((long long)jm * r * ts) % L;
    double sn, cs;
    sincospi(2.0 * (double)m / (double)L, &sn, &cs);
    return mk<V>((S)cs, (S)-sn);
  }
};

// The same stage-major table read from global memory through L1.
template <typename V> struct StageTwG {
  const V* p;
  __device__ __forceinline__ V w(int off, int jm, int r, int R, int ts) const {
    return ldg_c(p + off + jm * (R - 1) + r - 1);
  }
};

// Barrier between the stages: the whole CTA (BAR = 0) or named barrier 1
// over the BAR threads that run the stages (the other warps of the CTA do
// something else, e.g. feed the tile pipeline).
template <int BAR> __device__ __forceinline__ void stage_sync() {
  if constexpr (BAR == 0) __syncthreads();
  else asm volatile("bar.sync 1, %0;" ::"n"(BAR) : "memory");
}

// BMAX: upper bound on butterflies per thread; in the static kernels it is
// exactly ceil((L/R)/P), in the dynamic kernel EMAX/R.
// SMEM_IO: 0 = the first stage reads and the last stage writes global
// memory; 1 = both go through shared memory (pipelined kernels); 2 = the
// first stage reads shared memory, the last stage writes whole pencils to
// global memory (unit stride); 3 = the same with the output's row stride.
// CIN/COUT: the shared-memory views the stage reads and writes (they differ
// when a stage moves a tile between a dense TMA buffer and a padded one).
// toff: offset of this stage in a StageTw table (Ns - R_0).
template <typename T, int R, int BMAX, bool FAST_IO, int SMEM_IO, int BAR, int DIR, class CIN, class COUT, class TW>
__device__ __forceinline__ void stage_body(const PassDesc& d, int L, int P, int Ns, int ts, int toff,
                                           bool first, bool last, int t, const CIN& cin,
                                           const COUT& cout, const TW& tw, long long ib,
                                           long long ob, bool cv) {
  typedef typename cvec<T>::type V;
  const int Lr = L / R;
  // direction: at run time (DIR 0), or compiled in (1 forward: no
  // conjugation, unit scale; 2 inverse)
  const bool inv = DIR == 0 ? d.inverse != 0 : DIR == 2;
  // scale folded into the last stage's twiddles (inverse kernels whose
  // table says so): only the r = 0 inputs are scaled here
  const bool fold = scaled_last_tw<TW>::value && DIR == 2 && last && !first;
  const T scale = DIR == 1 || fold ? (T)1 : (T)d.scale;
  const bool to_global = SMEM_IO != 1 && last && !d.epi;
  const bool from_global = SMEM_IO == 0 && first;
  V v[BMAX][R];
#pragma unroll
  for (int b = 0; b < BMAX; ++b) {
    const int j = t + b * P;
    if (j < Lr) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k = j + r * Lr;
        if (from_global) {
          V x;
          if (!cv) x = mk<V>((T)0, (T)0);
          else if (FAST_IO) x = reinterpret_cast<const V*>(d.in.p)[ib + k * d.in.sk];
          else x = load_elem<T>(d.in, ib, k);
          if (inv) x.y = -x.y;
          v[b][r] = x;
        } else {
          V x = cin.ld(j, r * Lr);
          if (SMEM_IO != 0 && first && inv) x.y = -x.y;
          v[b][r] = x;
        }
      }
    }
  }
  if (!from_global) stage_sync<BAR>();
#pragma unroll
  for (int b = 0; b < BMAX; ++b) {
    const int j = t + b * P;
    if (j < Lr) {
      const int jm = j % Ns;
      if (!first) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b][r] = cmul(v[b][r], tw.w(toff, jm, r, R, ts));
        if (fold) v[b][0] = cscale(v[b][0], (T)d.scale);
      }
      Dft<R>::run(v[b]);
      const int o0 = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k = o0 + r * Ns;
        if (to_global) {
          if (cv) {
            V y = v[b][r];
            if (inv) y.y = -y.y;
            // SMEM_IO 2 (the fused slab pass) stores whole pencils: unit stride;
            // SMEM_IO 3 (the cp.async strided pass) rows d.out.sk apart
            if (FAST_IO) reinterpret_cast<V*>(d.out.p)[ob + (SMEM_IO == 2 ? k : k * d.out.sk)] = cscale(y, scale);
            else store_elem<T>(d.out, ob, k, y, scale);
          }
        } else if (SMEM_IO == 1 && last) {
          V y = v[b][r];
          if (inv) y.y = -y.y;
          cout.st(o0, r * Ns, cscale(y, scale));
        } else {
          cout.st(o0, r * Ns, v[b][r]);
        }
      }
    }
  }
  if (!to_global) stage_sync<BAR>();
}

// Shared prologue: thread -> (column, butterfly lane), column base offsets.
struct ColCtx {
  int c, t;
  bool cv;
  long long ib, ob;
};

__device__ __forceinline__ ColCtx col_ctx(const PassDesc& d, int P) {
  ColCtx x;
  const int tid = threadIdx.x;
  if (d.cfast) { x.c = tid % d.C; x.t = tid / d.C; }
  else { x.t = tid % P; x.c = tid / P; }
  const long long q = (long long)blockIdx.x * d.C + x.c;
  x.cv = q < d.Q;
  const long long qi = x.cv ? q % d.I : 0;
  const long long qo = x.cv ? q / d.I : 0;
  x.ib = qi * d.in.si + io_outer(d.in, qo);
  x.ob = qi * d.out.si + io_outer(d.out, qo);
  return x;
}

// R2C post-pass over the half-length spectrum Z (length M) in shared memory:
// X_k = E_k + w^k O_k, E = (Z_k + conj Z_{M-k})/2, O = -i (Z_k - conj Z_{M-k})/2.
template <typename T>
__device__ __forceinline__ void r2c_epilogue(const PassDesc& d, int P, const ColCtx& x,
                                             const typename cvec<T>::type* col) {
  typedef typename cvec<T>::type V;
  const int M = d.L;
  const V* w2 = reinterpret_cast<const V*>(d.tw2);
  if (!x.cv) return;
  for (int k = x.t; k <= M; k += P) {
    V zk = col[swz<V>(k == M ? 0 : k)];
    V zm = cconj(col[swz<V>(k == 0 ? 0 : M - k)]);
    V e = cscale(cadd(zk, zm), (T)0.5);
    V o = cscale(cmul_mi(csub(zk, zm)), (T)0.5);
    store_elem<T>(d.out, x.ob, k, cadd(e, cmul(ldg_c(w2 + k), o)), (T)d.scale);
  }
}

// ---------------------------------------------------------------------------
// Static-plan kernel.
// ---------------------------------------------------------------------------

// Compile-time stage sequence.  The first stage reads CFIRST, the last
// stage writes CLAST, every other access goes through CMID.
template <typename T, int L, int P, bool FAST_IO, int SMEM_IO, int BAR, int DIR, int NS, int R0, int S, class CFIRST,
          class CMID, class CLAST, class TW, int R, int... Rest>
__device__ __forceinline__ void static_stages(const PassDesc& d, int t, const CFIRST& cf,
                                              const CMID& cm, const CLAST& cl, const TW& tw,
                                              long long ib, long long ob, bool cv) {
  constexpr int Lr = L / R;
  constexpr int BM = (Lr + P - 1) / P;
  constexpr int TS = L / (NS * R);
  constexpr bool FIRST = (S == 0);
  constexpr bool LAST = (sizeof...(Rest) == 0);
  constexpr int R0_ = FIRST ? R : R0;
  if constexpr (FIRST && LAST) {
    stage_body<T, R, BM, FAST_IO, SMEM_IO, BAR, DIR>(d, L, P, NS, TS, NS - R0_, true, true, t, cf, cl, tw, ib, ob, cv);
  } else if constexpr (FIRST) {
    stage_body<T, R, BM, FAST_IO, SMEM_IO, BAR, DIR>(d, L, P, NS, TS, NS - R0_, true, false, t, cf, cm, tw, ib, ob, cv);
  } else if constexpr (LAST) {
    stage_body<T, R, BM, FAST_IO, SMEM_IO, BAR, DIR>(d, L, P, NS, TS, NS - R0_, false, true, t, cm, cl, tw, ib, ob, cv);
  } else {
    stage_body<T, R, BM, FAST_IO, SMEM_IO, BAR, DIR>(d, L, P, NS, TS, NS - R0_, false, false, t, cm, cm, tw, ib, ob, cv);
  }
  if constexpr (sizeof...(Rest) > 0)
    static_stages<T, L, P, FAST_IO, SMEM_IO, BAR, DIR, NS * R, R0_, S + 1, CFIRST, CMID, CLAST, TW, Rest...>(
        d, t, cf, cm, cl, tw, ib, ob, cv);
}

template <typename T, bool FAST_IO, int LB, int L, int P, int... Rs>
__global__ void __launch_bounds__(LB) axis_pass_static(const PassDesc d) {
  typedef typename cvec<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sm = reinterpret_cast<V*>(smem_raw);
  const ColCtx x = col_ctx(d, P);
  const PadCol<V> col{sm + x.c * d.ld};
  const GlobalTw<V> tw{reinterpret_cast<const V*>(d.tw)};
  static_stages<T, L, P, FAST_IO, 0, 0, 0, 1, 1, 0, PadCol<V>, PadCol<V>, PadCol<V>, GlobalTw<V>, Rs...>(
      d, x.t, col, col, col, tw, x.ib, x.ob, x.cv);
  if (!FAST_IO && d.epi) r2c_epilogue<T>(d, P, x, col.p);
}

// ---------------------------------------------------------------------------
// Dynamic-plan kernel (fallback for lengths without a static plan).
// ---------------------------------------------------------------------------

template <typename T, int R, int EMAX, bool CTW>
__device__ __noinline__ void dyn_stage(const PassDesc& d, int s, int t, typename cvec<T>::type* col,
                                       const typename cvec<T>::type* tw, long long ib, long long ob,
                                       bool cv) {
  typedef typename cvec<T>::type V;
  const PadCol<V> c{col};
  if constexpr (CTW) {
    const ComputedTw<V> g{d.L};
    stage_body<T, R, EMAX / R, false, 0, 0, 0>(d, d.L, d.P, d.ns[s], d.tws[s], 0, s == 0,
                                             s == d.nst - 1, t, c, c, g, ib, ob, cv);
  } else {
    const GlobalTw<V> g{tw};
    stage_body<T, R, EMAX / R, false, 0, 0, 0>(d, d.L, d.P, d.ns[s], d.tws[s], 0, s == 0,
                                             s == d.nst - 1, t, c, c, g, ib, ob, cv);
  }
}

// CTW: twiddles computed in the kernel instead of read from d.tw (no table).
template <typename T, int EMAX, bool CTW = false>
__global__ void __launch_bounds__(1024) axis_pass_dynamic(const PassDesc d) {
  typedef typename cvec<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* sm = reinterpret_cast<V*>(smem_raw);
  const ColCtx x = col_ctx(d, d.P);
  V* col = sm + x.c * d.ld;
  const V* tw = reinterpret_cast<const V*>(d.tw);
  for (int s = 0; s < d.nst; ++s) {
    switch (d.radix[s]) {
      case 1: dyn_stage<T, 1, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 2: dyn_stage<T, 2, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 3: dyn_stage<T, 3, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 4: dyn_stage<T, 4, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 5: dyn_stage<T, 5, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 7: dyn_stage<T, 7, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 8: dyn_stage<T, 8, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 11: dyn_stage<T, 11, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 13: dyn_stage<T, 13, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      case 16: dyn_stage<T, 16, EMAX, CTW>(d, s, x.t, col, tw, x.ib, x.ob, x.cv); break;
      default: break;
    }
  }
  if (d.epi) r2c_epilogue<T>(d, d.P, x, col);
}

}  // namespace dfft
