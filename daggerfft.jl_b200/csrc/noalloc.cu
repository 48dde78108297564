// dfft_irfft_noalloc_f32: a ComplexF32 -> Float32 irfft that allocates no
// device memory.
//
// Who needs it.  Some callers cannot call cudaMalloc at the moment they
// transform: code running inside another framework's memory pool (an XLA or
// PyTorch custom op, CUDA.jl's pooled allocator), where a raw allocation
// bypasses the pool's accounting and can fail when the pool already holds
// nearly all of HBM, or serving code held to a fixed memory budget, where an
// allocation on the request path may synchronise the device.  The regular
// plan API allocates twiddle tables and, for an irfft over several dims, a
// workspace for the intermediate half-spectrum.  This entry point needs
// neither: twiddles are computed in the kernel, and the intermediate lives in
// the file-scope device array below, which every GPU that loads the library
// holds until the process exits.
//
// Limits and behaviour.
//  * The intermediate (d/2+1)*n2*n3 complex values must fit the array:
//    at most kNoAllocElems = 2^21 ComplexF32 (16 MiB); larger sizes are
//    rejected with DFFT_ERROR_INVALID_VALUE.
//  * The array is shared by every call on a device and keeps the last
//    call's contents; the first pass overwrites every element it later
//    reads, so nothing needs clearing.  Calls whose kernels overlap on the
//    GPU (two streams, two threads) race on it: serialise them.
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current).  With CUDA's lazy
//    module loading that lookup is also when the library's device code is
//    loaded on that device and the 16 MiB array is reserved, so the first
//    call itself does allocate: make it once at start-up (a tiny ndim = 1
//    call will do), before the caller's memory pool has grown to fill the
//    GPU and before any stream capture.
//  * Every length is checked (13-smooth, stage count, one CTA, shared
//    memory) before anything is launched, so a rejected call leaves the
//    stream and the array untouched.
#include <mutex>
#include "dfft.h"
#include "dfft_internal.h"

namespace dfft {

constexpr long long kNoAllocElems = 1LL << 21;  // ComplexF32 elements (16 MiB)

static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocElems];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_na_mu;
float2* g_na_ptr[kMaxDevices] = {};
bool g_na_attr[kMaxDevices] = {};

// Device address of the scratch array for the current device (looked up
// once per device; host code must not use the symbol itself as a pointer).
cudaError_t noalloc_setup(int dev, float2** out) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_na_ptr[dev] = reinterpret_cast<float2*>(p);
  }
  if (!g_na_attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&axis_pass_dynamic<float, 16, true>),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) return e;
    g_na_attr[dev] = true;
  }
  *out = g_na_ptr[dev];
  return cudaSuccess;
}

// Radices of the dynamic kernel, without allocating (16/8/4/2, 13/11/7/5/3),
// at most kMaxStages of them.  Returns the stage count, 0 when L has a prime
// factor above 13, -1 when it needs more than kMaxStages stages.
int radices(int L, int* r) {
  int n = L, k = 0;
  auto put = [&](int x) {
    if (k >= kMaxStages) return false;
    r[k++] = x;
    return true;
  };
  const int odd[] = {13, 11, 7, 5, 3};
  for (int p : odd)
    while (n % p == 0) {
      if (!put(p)) return -1;
      n /= p;
    }
  int e = 0;
  while (n % 2 == 0) { ++e; n /= 2; }
  if (n != 1) return 0;
  for (; e >= 4; e -= 4)
    if (!put(16)) return -1;
  if (e == 3 && !put(8)) return -1;
  if (e == 2 && !put(4)) return -1;
  if (e == 1 && !put(2)) return -1;
  if (k == 0) put(1);
  return k;
}

IoAny side(int kind, long long I, long long extent) {
  IoAny x{};
  x.kind = kind;
  x.si = 1;
  x.so = I * extent;
  x.sk = I;
  return x;
}

// One pass of the computed-twiddle dynamic kernel: descriptor, CTA shape and
// shared memory, or an error for a length it cannot run (nothing launched).
struct NaPass {
  PassDesc d;
  int C;
  size_t col;
};

int prepare(int L, long long I, long long O, double scale, NaPass* np) {
  PassDesc& d = np->d;
  d = PassDesc{};
  int rad[kMaxStages];
  const int nst = radices(L, rad);
  if (nst == 0) {
    set_error("irfft_noalloc: length " + std::to_string(L) + " has a prime factor above 13");
    return DFFT_ERROR_UNSUPPORTED_SIZE;
  }
  if (nst < 0) {
    set_error("irfft_noalloc: length " + std::to_string(L) + " needs more than " +
              std::to_string(kMaxStages) + " radix stages");
    return DFFT_ERROR_UNSUPPORTED_SIZE;
  }
  d.L = L;
  d.nst = nst;
  int ns = 1, P = 1;
  for (int i = 0; i < nst; ++i) {
    d.radix[i] = rad[i];
    d.ns[i] = ns;
    d.tws[i] = L / (ns * rad[i]);
    ns *= rad[i];
    const int B = 16 / rad[i];
    const int need = (L / rad[i] + B - 1) / B;
    if (need > P) P = need;
  }
  if (P > 1024) {
    set_error("irfft_noalloc: length " + std::to_string(L) + " exceeds one CTA");
    return DFFT_ERROR_UNSUPPORTED_SIZE;
  }
  d.P = P;
  int ld = (L - 1) + ((L - 1) >> 4) + 1;
  if ((ld & 1) == 0) ld += 1;
  d.ld = ld;
  d.cfast = I > 1 ? 1 : 0;
  d.inverse = 1;
  d.scale = scale;
  d.Q = I * O;
  d.I = I;
  const size_t col = (size_t)ld * sizeof(float2);
  if (col > 200 * 1024) {
    set_error("irfft_noalloc: length " + std::to_string(L) + " does not fit shared memory");
    return DFFT_ERROR_UNSUPPORTED_SIZE;
  }
  int C;
  if (d.cfast) {
    C = 16;
    while (C * P < 256 && C < 64) C *= 2;
  } else {
    C = 1;
    while (C * 2 * P <= 256) C *= 2;
  }
  while (C > 1 && (C * P > 1024 || (size_t)C * col > 200 * 1024)) C /= 2;
  d.C = C;
  np->C = C;
  np->col = col;
  return DFFT_SUCCESS;
}

int launch(NaPass& np, IoAny in, IoAny out, cudaStream_t st) {
  np.d.in = in;
  np.d.out = out;
  const long long nblk = (np.d.Q + np.C - 1) / np.C;
  void* args[] = {&np.d};
  cudaError_t e = cudaLaunchKernel(reinterpret_cast<const void*>(&axis_pass_dynamic<float, 16, true>),
                                   dim3((unsigned)nblk), dim3((unsigned)(np.C * np.d.P)), args,
                                   (size_t)np.C * np.col, st);
  if (e != cudaSuccess) {
    set_error(std::string("irfft_noalloc: launch failed: ") + cudaGetErrorString(e));
    return DFFT_ERROR_CUDA;
  }
  return DFFT_SUCCESS;
}

}  // namespace
}  // namespace dfft

extern "C" int dfft_irfft_noalloc_f32(const void* in, void* out, int ndim, const int64_t* shape,
                                      void* stream) {
  using namespace dfft;
  if (!in || !out || !shape || ndim < 1 || ndim > 3) {
    set_error("irfft_noalloc: NULL argument or ndim outside 1..3");
    return DFFT_ERROR_INVALID_VALUE;
  }
  long long R[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) {
    if (shape[i] < 1 || shape[i] > 0x7fffffffLL) {
      set_error("irfft_noalloc: shape entries must be in 1..2^31-1");
      return DFFT_ERROR_INVALID_VALUE;
    }
    R[i] = shape[i];
  }
  const long long d = R[0];
  const long long H[3] = {d / 2 + 1, R[1], R[2]};
  const long long n_mid = H[0] * H[1] * H[2];
  if (ndim > 1 && n_mid > kNoAllocElems) {
    set_error("irfft_noalloc: the intermediate needs " + std::to_string(n_mid) +
              " complex elements; the static workspace holds at most " + std::to_string(kNoAllocElems));
    return DFFT_ERROR_INVALID_VALUE;
  }
  // every pass is checked before the device is touched or anything launched
  const long long O1 = H[1] * H[2];
  const bool even = d % 2 == 0;
  const int L1 = even ? (int)(d / 2) : (int)d;
  NaPass passes[3];
  for (int a = ndim - 1; a >= 1; --a) {
    long long I = 1, O = 1;
    for (int k = 0; k < a; ++k) I *= H[k];
    for (int k = a + 1; k < 3; ++k) O *= H[k];
    const int stt = prepare((int)H[a], I, O, 1.0 / (double)H[a], &passes[a]);
    if (stt) return stt;
  }
  {
    const int stt = prepare(L1, 1, O1, 1.0 / (double)d, &passes[0]);
    if (stt) return stt;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("irfft_noalloc: no usable current device");
    return DFFT_ERROR_CUDA;
  }
  float2* scratch = nullptr;
  cudaError_t e = noalloc_setup(dev, &scratch);
  if (e != cudaSuccess) {
    set_error(std::string("irfft_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return DFFT_ERROR_CUDA;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // inverse C2C along dims ndim..2 (the reference's inverse stage order),
  // the first into the static workspace, the rest in place there
  const void* src = in;
  for (int a = ndim - 1; a >= 1; --a) {
    long long I = 1;
    for (int k = 0; k < a; ++k) I *= H[k];
    IoAny i = side(IO_CPLX, I, H[a]);
    IoAny o = side(IO_CPLX, I, H[a]);
    i.p = const_cast<void*>(src);
    o.p = scratch;
    const int stt = launch(passes[a], i, o, st);
    if (stt) return stt;
    src = scratch;
  }
  // C2R along dim 1
  IoAny i, o;
  if (even) {
    i = side(IO_HERM_PAIR, 1, H[0]);
    i.n = L1;
    o = side(IO_REAL_PAIR, 1, d);
  } else {
    i = side(IO_HERM_FULL, 1, H[0]);
    i.n = (int)d;
    o = side(IO_REAL, 1, d);
  }
  i.p = const_cast<void*>(src);
  i.w = nullptr;  // twiddles computed in the kernel
  o.p = out;
  return launch(passes[0], i, o, st);
}
