// Host side of the mixed-precision tensor-core pass (mixed_pass.cuh):
// kernel instances, the operand images of the DFT matrices (generated in
// long double, split into FP16 hi + lo, laid out in the 128-byte swizzled
// K-major order the tensor cores read) and pass construction.
#include <cmath>
#include <cstring>
#include <mutex>
#include "dfft.h"
#include "dfft_internal.h"
#include "mixed_pass.cuh"

namespace dfft {

template __global__ void mixed_pass<true>(const void*, void*, const __grid_constant__ CUtensorMap,
                                          const __grid_constant__ CUtensorMap, const MixedGeom);
template __global__ void mixed_pass<false>(const void*, void*, const __grid_constant__ CUtensorMap,
                                           const __grid_constant__ CUtensorMap, const MixedGeom);

namespace {

// IEEE binary16 bits of v, round to nearest even (normal and subnormal
// range; |v| stays far below the largest finite value here).
uint16_t half_bits(long double v) {
  uint16_t sign = 0;
  if (v < 0) {
    sign = 0x8000;
    v = -v;
  }
  if (v == 0) return sign;
  int e = 0;
  frexpl(v, &e);  // v = f * 2^e, f in [0.5, 1)
  e -= 1;         // v = g * 2^e, g in [1, 2)
  if (e < -14) {  // subnormal: multiples of 2^-24
    const long double m = nearbyintl(ldexpl(v, 24));
    return (uint16_t)(sign | (uint16_t)m);  // m == 1024 is the smallest normal, encoded alike
  }
  long double m = nearbyintl(ldexpl(v, 10 - e));  // in [1024, 2048]
  if (m >= 2048) {
    m = 1024;
    ++e;
  }
  return (uint16_t)(sign | (uint16_t)((e + 15) << 10) | (uint16_t)(m - 1024));
}

long double half_value(uint16_t h) {
  const int e = (h >> 10) & 31, m = h & 1023;
  long double v = e == 0 ? ldexpl((long double)m, -24) : ldexpl((long double)(1024 + m), e - 25);
  return (h & 0x8000) ? -v : v;
}

const long double kPi = 3.141592653589793238462643383279502884L;

// Real form of the complex DFT matrix W_R^(n k) (sign -1 forward, +1
// inverse) as the K-major B operand: row n (output; n < R real part of
// output n, else imaginary part of output n - R), column k (input; k < R
// real part, else imaginary part), FP16 hi and lo images, 128-byte rows,
// 16-byte chunks swizzled by row % 8.
void dft_operand(int R, int sign, unsigned char* hi, unsigned char* lo) {
  for (int n = 0; n < 2 * R; ++n)
    for (int k = 0; k < 2 * R; ++k) {
      const int ko = n % R, ki = k % R;
      const long double ang = 2 * kPi * (long double)((ko * ki) % R) / (long double)R;
      const long double wr = cosl(ang), wi = sign * sinl(ang);
      long double v;
      if (n < R) v = (k < R) ? wr : -wi;
      else v = (k < R) ? wi : wr;
      const uint16_t h = half_bits(v);
      const uint16_t l = half_bits(v - half_value(h));
      const size_t off = (size_t)n * 128 + (size_t)((((k >> 3) ^ (n & 7)) << 4) + (k & 7) * 2);
      std::memcpy(hi + off, &h, 2);
      std::memcpy(lo + off, &l, 2);
    }
}

std::mutex g_mix_mu;
std::shared_ptr<DevTable> g_mix_consts[64][2];

}  // namespace

// The constants image of one direction on the current device (cached).
std::shared_ptr<DevTable> mixed_consts(int inverse) {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64) throw Error{DFFT_ERROR_INVALID_VALUE, "device index out of range"};
  std::lock_guard<std::mutex> lk(g_mix_mu);
  auto& slot = g_mix_consts[dev][inverse ? 1 : 0];
  if (slot) return slot;
  std::vector<unsigned char> img(kMixConstBytes, 0);
  const int sign = inverse ? 1 : -1;
  unsigned char* b32 = img.data();                    // kMixB32 - kMixB32
  unsigned char* b16 = img.data() + (kMixB16 - kMixB32);
  float* tw = reinterpret_cast<float*>(img.data() + (kMixTw - kMixB32));
  dft_operand(32, sign, b32, b32 + 8192);
  dft_operand(16, sign, b16, b16 + 4096);
  for (int n2 = 0; n2 < 16; ++n2)
    for (int k1 = 0; k1 < 32; ++k1) {
      const long double ang = 2 * kPi * (long double)((n2 * k1) % 512) / 512.0L;
      // W512^(n2 k1) / 32: the stage-B operands carry the stage-A scale / 32
      tw[2 * (n2 * 33 + k1)] = (float)(cosl(ang) / 32);
      tw[2 * (n2 * 33 + k1) + 1] = (float)(sign * sinl(ang) / 32);
    }
  auto t = std::make_shared<DevTable>();
  t->device = dev;
  t->bytes = img.size();
  cuda_check(cudaMalloc(&t->p, t->bytes), "cudaMalloc(mixed constants)");
  cuda_check(cudaMemcpy(t->p, img.data(), t->bytes, cudaMemcpyHostToDevice), "cudaMemcpy(mixed constants)");
  slot = t;
  return t;
}

bool mixed_supported(int dbl, int L, long long I) {
  // length 512 ComplexF32; strided axes need rows TMA can address
  return !dbl && L == 512 && (I == 1 || (I % 2 == 0 && I >= 16));
}

Pass make_mixed_pass(long long I, long long O, int inverse) {
  if (!mixed_supported(0, 512, I))
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "the mixed form covers ComplexF32 axes of length 512"};
  Pass p;
  p.mixed = true;
  p.mstrided = I > 1;
  p.fn = p.mstrided ? reinterpret_cast<const void*>(&mixed_pass<true>)
                    : reinterpret_cast<const void*>(&mixed_pass<false>);
  auto consts = mixed_consts(inverse);
  p.tables.push_back(consts);
  MixedGeom& g = p.mgeom;
  g.consts = static_cast<const unsigned char*>(consts->p);
  g.out_scale = inverse ? 1.0f / 512.0f : 1.0f;
  g.err = device_error_word();
  if (p.mstrided) {
    g.tiles_i = (int)((I + 15) / 16);
    g.ntiles = (long long)g.tiles_i * O;
    g.lb = 256;
    g.nlb = 2;
    p.tI = I;
    p.tL = 512;
    p.tO = O;
  } else {
    g.ncols = O;
    g.ntiles = (O + 15) / 16;
  }
  p.d.L = 512;
  p.d.inverse = inverse;
  p.d.Q = I * O;
  p.d.I = I;
  p.smem = (size_t)kMixSmem;
  p.block = dim3(kMixThreads);
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(mixed)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "mixed kernel cannot be resident"};
  int dev = 0, sms = 148;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
  long long nb = (long long)sms;
  if (nb > g.ntiles) nb = g.ntiles;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 0));
  return p;
}

}  // namespace dfft
