// In-register complex arithmetic and small forward DFT codelets.
//
// Every codelet computes the unnormalised forward DFT
//     X_k = sum_n x_n * exp(-2*pi*i*n*k/R)
// in place on an array of R complex values held in registers.  Inverse
// transforms are obtained by the caller through conjugation
// (IDFT(x) = conj(DFT(conj(x)))), so only the forward sign is compiled.
//
// Radices: 2, 4 (butterflies), odd primes 3/5/7/11/13 (symmetric-pair form,
// O(R^2/2) multiply-adds), composites 8 = 2x4, 16 = 4x4, 32 = 4x8,
// 6 = 2x3, 10 = 2x5, 12 = 4x3, 15 = 3x5 (one Cooley-Tukey split in registers
// with compile-time twiddles from roots.cuh).
#pragma once
#include <cuda_runtime.h>
#include "roots.cuh"

namespace dfft {

template <typename T> struct cvec;
template <> struct cvec<float> { typedef float2 type; };
template <> struct cvec<double> { typedef double2 type; };

template <typename V> struct scalar_of;
template <> struct scalar_of<float2> { typedef float type; };
template <> struct scalar_of<double2> { typedef double type; };

template <typename V> __device__ __forceinline__ V mk(typename scalar_of<V>::type a,
                                                      typename scalar_of<V>::type b) {
  V r; r.x = a; r.y = b; return r;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mk<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cconj(V a) { return mk<V>(a.x, -a.y); }
template <typename V, typename S> __device__ __forceinline__ V cscale(V a, S s) { return mk<V>(a.x * s, a.y * s); }
// ComplexF32 adds and subtracts as packed two-lane FP32 instructions
// (add / sub.rn.f32x2, sm_100; the same round-to-nearest sums as the scalar
// form).  Half the issue slots for the butterflies: the fused slab pass,
// bound by instruction issue, runs 9 % faster with them and the
// producer-fed strided pass 3 % faster (512^3, B200); the 1024-thread
// pipelined strided pass, bound by its barriers, runs 15 % slower.  A
// translation unit opts in by defining DFFT_PACKED_F32 before including
// this header.
#ifdef DFFT_PACKED_F32
__device__ __forceinline__ unsigned long long f2bits(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 bitsf2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2bits(a)), "l"(f2bits(b)));
  return bitsf2(r);
}
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2bits(a)), "l"(f2bits(b)));
  return bitsf2(r);
}
#endif

// multiply by -i and +i
template <typename V> __device__ __forceinline__ V cmul_mi(V a) { return mk<V>(a.y, -a.x); }
template <typename V> __device__ __forceinline__ V cmul_pi(V a) { return mk<V>(-a.y, a.x); }

// Multiply by w_R^e = exp(-2*pi*i*e/R) with e a compile-time constant after
// unrolling; the trivial angles are strength-reduced.
template <int R, typename V> __device__ __forceinline__ V twiddle_const(V a, int e) {
  typedef typename scalar_of<V>::type S;
  e %= R;
  if (e == 0) return a;
  if (4 * e == R) return cmul_mi(a);
  if (2 * e == R) return mk<V>(-a.x, -a.y);
  if (4 * e == 3 * R) return cmul_pi(a);
  const S c = (S)root_cos<R>(e);
  const S s = (S)root_sin<R>(e);
  if (8 * e == R) return mk<V>(c * (a.x + a.y), c * (a.y - a.x));           // (1-i)/sqrt2
  if (8 * e == 3 * R) return mk<V>(c * (a.x - a.y), c * (a.x + a.y));       // (-1-i)/sqrt2
  // (a.x + i a.y)(c - i s)
  return mk<V>(a.x * c + a.y * s, a.y * c - a.x * s);
}

template <int R> struct Dft;

template <> struct Dft<1> {
  template <typename V> __device__ __forceinline__ static void run(V (&)[1]) {}
};

template <> struct Dft<2> {
  template <typename V> __device__ __forceinline__ static void run(V (&x)[2]) {
    V t = x[0];
    x[0] = cadd(t, x[1]);
    x[1] = csub(t, x[1]);
  }
};

template <> struct Dft<4> {
  template <typename V> __device__ __forceinline__ static void run(V (&x)[4]) {
    V t0 = cadd(x[0], x[2]);
    V t1 = csub(x[0], x[2]);
    V t2 = cadd(x[1], x[3]);
    V t3 = cmul_mi(csub(x[1], x[3]));
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    x[1] = cadd(t1, t3);
    x[3] = csub(t1, t3);
  }
};

// Odd prime P: X_k = x0 + sum_m [cos(2 pi k m/P) a_m - i sin(2 pi k m/P) b_m],
// a_m = x_m + x_{P-m}, b_m = x_m - x_{P-m}; X_{P-k} takes +i.
template <int P> struct DftOdd {
  template <typename V> __device__ __forceinline__ static void run(V (&x)[P]) {
    typedef typename scalar_of<V>::type S;
    constexpr int H = (P - 1) / 2;
    V a[H], b[H];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      a[m - 1] = cadd(x[m], x[P - m]);
      b[m - 1] = csub(x[m], x[P - m]);
    }
    V x0 = x[0];
    V sum = x0;
#pragma unroll
    for (int m = 0; m < H; ++m) sum = cadd(sum, a[m]);
    V out[P];
    out[0] = sum;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      V re = x0;
      V im = mk<V>((S)0, (S)0);
#pragma unroll
      for (int m = 1; m <= H; ++m) {
        const int e = (k * m) % P;
        const S c = (S)root_cos<P>(e);
        const S s = (S)root_sin<P>(e);
        re.x += c * a[m - 1].x; re.y += c * a[m - 1].y;
        im.x += s * b[m - 1].x; im.y += s * b[m - 1].y;
      }
      // X_k = re - i*im, X_{P-k} = re + i*im
      out[k] = mk<V>(re.x + im.y, re.y - im.x);
      out[P - k] = mk<V>(re.x - im.y, re.y + im.x);
    }
#pragma unroll
    for (int k = 0; k < P; ++k) x[k] = out[k];
  }
};
template <> struct Dft<3> : DftOdd<3> {};
template <> struct Dft<5> : DftOdd<5> {};
template <> struct Dft<7> : DftOdd<7> {};
template <> struct Dft<11> : DftOdd<11> {};
template <> struct Dft<13> : DftOdd<13> {};

// R = R1*R2 in registers: n = R2*n1 + n2, k = k1 + R1*k2.
template <int R1, int R2> struct DftComposite {
  template <typename V> __device__ __forceinline__ static void run(V (&x)[R1 * R2]) {
    constexpr int R = R1 * R2;
    V y[R2][R1];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
      V t[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n1] = x[R2 * n1 + n2];
      Dft<R1>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) y[n2][k1] = twiddle_const<R>(t[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      V t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = y[n2][k1];
      Dft<R2>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) x[k1 + R1 * k2] = t[k2];
    }
  }
};
template <> struct Dft<8> : DftComposite<2, 4> {};
template <> struct Dft<16> : DftComposite<4, 4> {};
template <> struct Dft<32> : DftComposite<4, 8> {};
template <> struct Dft<6> : DftComposite<2, 3> {};
template <> struct Dft<10> : DftComposite<2, 5> {};
template <> struct Dft<12> : DftComposite<4, 3> {};
template <> struct Dft<15> : DftComposite<3, 5> {};

}  // namespace dfft
