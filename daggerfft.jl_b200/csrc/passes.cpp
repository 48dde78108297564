// Pass construction: radix plan lookup, launch shape, twiddle tables.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>
#include <cuda.h>
#include "dfft.h"
#include "dfft_internal.h"
#include "static_plans.h"

namespace dfft {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    throw Error{e == cudaErrorMemoryAllocation ? DFFT_ERROR_OUT_OF_MEMORY : DFFT_ERROR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

// ---------------------------------------------------------------------------
// twiddle tables
// ---------------------------------------------------------------------------

DevTable::~DevTable() {
  if (p) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(p);
    if (cur != device && cur >= 0) cudaSetDevice(cur);
  }
}

namespace {
std::mutex g_tab_mu;
std::map<std::tuple<int, int, long long, long long, long long, int, bool>, std::weak_ptr<DevTable>>
    g_tabs;
}  // namespace

std::shared_ptr<DevTable> twiddle_table(int dbl, long long D, long long a, long long b, int count,
                                        bool conj) {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  auto key = std::make_tuple(dev, dbl, D, a, b, count, conj);
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto it = g_tabs.find(key);
  if (it != g_tabs.end()) {
    if (auto sp = it->second.lock()) return sp;
  }
  const long double two_pi = 2.0L * acosl(-1.0L);
  const size_t esz = dbl ? 16 : 8;
  std::vector<unsigned char> host(esz * (size_t)(count > 0 ? count : 1));
  for (int k = 0; k < count; ++k) {
    // exact integer reduction of the phase keeps the angle in [0, 2 pi)
    long long m = ((a * (long long)k + b) % D + D) % D;
    long double ang = two_pi * (long double)m / (long double)D;
    long double c = cosl(ang), s = -sinl(ang);
    if (conj) s = -s;
    if (dbl) {
      double v[2] = {(double)c, (double)s};
      std::memcpy(host.data() + esz * k, v, esz);
    } else {
      float v[2] = {(float)c, (float)s};
      std::memcpy(host.data() + esz * k, v, esz);
    }
  }
  auto t = std::make_shared<DevTable>();
  t->device = dev;
  t->bytes = host.size();
  cuda_check(cudaMalloc(&t->p, t->bytes), "cudaMalloc(twiddles)");
  cuda_check(cudaMemcpy(t->p, host.data(), t->bytes, cudaMemcpyHostToDevice), "cudaMemcpy(twiddles)");
  g_tabs[key] = t;
  return t;
}

// ---------------------------------------------------------------------------
// static plan lookup
// ---------------------------------------------------------------------------

namespace {
std::once_flag g_static_once;
std::unordered_map<int, const StaticPlan*> g_static[2];

void build_static_index() {
  for (int dbl = 0; dbl < 2; ++dbl) {
    const StaticPlanTable* t = dbl ? kTable_f64 : kTable_f32;
    for (int part = 0; part < kTableParts; ++part) {
      for (int i = 0; i < *t[part].count; ++i) g_static[dbl][t[part].plans[i].L] = &t[part].plans[i];
    }
  }
}

const StaticPlan* find_static(int dbl, int L) {
  std::call_once(g_static_once, build_static_index);
  auto it = g_static[dbl].find(L);
  return it == g_static[dbl].end() ? nullptr : it->second;
}

// Radix list for the dynamic kernel: 16/8/4/2 for the power of two, then
// the odd primes 3, 5, 7, 11, 13.  Empty if L has another prime factor.
std::vector<int> dynamic_radices(int L) {
  std::vector<int> r;
  int n = L;
  const int odd[] = {13, 11, 7, 5, 3};
  for (int p : odd) {
    while (n % p == 0) { r.push_back(p); n /= p; }
  }
  int e = 0;
  while (n % 2 == 0) { ++e; n /= 2; }
  if (n != 1) return {};
  while (e >= 4) { r.push_back(16); e -= 4; }
  if (e == 3) r.push_back(8);
  if (e == 2) r.push_back(4);
  if (e == 1) r.push_back(2);
  if (r.empty()) r.push_back(1);
  return r;
}

std::mutex g_attr_mu;
std::map<std::pair<int, const void*>, size_t> g_attr;
}  // namespace

cudaError_t ensure_smem_attr(const void* fn, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_attr_mu);
  auto key = std::make_pair(dev, fn);
  auto it = g_attr.find(key);
  if (it != g_attr.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) g_attr[key] = bytes;
  return e;
}

// ---------------------------------------------------------------------------
// device error word and TMA descriptors
// ---------------------------------------------------------------------------

namespace {
std::mutex g_err_mu;
std::map<int, int*> g_err_words;

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;
std::once_flag g_encode_once;

void load_encode() {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_encode = reinterpret_cast<EncodeTiledFn>(fn);
}
}  // namespace

int* device_error_word() {
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_err_mu);
  auto it = g_err_words.find(dev);
  if (it != g_err_words.end()) return it->second;
  int* w = nullptr;
  cuda_check(cudaMalloc(&w, sizeof(int)), "cudaMalloc(error word)");
  cuda_check(cudaMemset(w, 0, sizeof(int)), "cudaMemset(error word)");
  g_err_words[dev] = w;
  return w;
}

// Tensor map over the real tensor {I, n, O} of a strided tiled pass.
static cudaError_t encode_real_map(CUtensorMap* m, void* base, const Pass& p, int dbl) {
  std::call_once(g_encode_once, load_encode);
  if (!g_encode) return cudaErrorNotSupported;
  const cuuint64_t esz = dbl ? 8 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)p.tI, (cuuint64_t)p.tL, (cuuint64_t)p.tO};
  cuuint64_t strides[2] = {(cuuint64_t)p.tI * esz, (cuuint64_t)p.tI * esz * (cuuint64_t)p.tL};
  cuuint32_t box[3] = {(cuuint32_t)p.geom.C, (cuuint32_t)p.geom.lb, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(m, dbl ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

static cudaError_t encode_map_dims(CUtensorMap* m, void* base, const Pass& p, long long tI, long long tL,
                                   long long tO) {
  std::call_once(g_encode_once, load_encode);
  if (!g_encode) return cudaErrorNotSupported;
  const cuuint64_t esz = 8;
  const cuuint64_t xs = (cuuint64_t)p.geom.xscale;
  cuuint64_t dims[3] = {(cuuint64_t)tI * xs, (cuuint64_t)tL, (cuuint64_t)tO};
  cuuint64_t strides[2] = {(cuuint64_t)tI * xs * esz, (cuuint64_t)tI * xs * esz * (cuuint64_t)tL};
  cuuint32_t box[3] = {(cuuint32_t)(p.geom.C * p.geom.xscale), (cuuint32_t)p.geom.lb, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

static cudaError_t encode_map(CUtensorMap* m, void* base, const Pass& p) {
  return encode_map_dims(m, base, p, p.tI, p.tL, p.tO);
}

// Tensor map over {I, L, O} ComplexF32 (8-byte elements) with boxes of 16
// columns x 256 rows in the 128-byte swizzle the mixed pass reads and writes.
static cudaError_t encode_map_sw128(CUtensorMap* m, void* base, const Pass& p) {
  std::call_once(g_encode_once, load_encode);
  if (!g_encode) return cudaErrorNotSupported;
  cuuint64_t dims[3] = {(cuuint64_t)p.tI, (cuuint64_t)p.tL, (cuuint64_t)p.tO};
  cuuint64_t strides[2] = {(cuuint64_t)p.tI * 8, (cuuint64_t)p.tI * 8 * (cuuint64_t)p.tL};
  cuuint32_t box[3] = {16, (cuuint32_t)p.mgeom.lb, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

static int sm_count() {
  static int v = 0;
  if (!v) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
  }
  return v;
}

// Rows per TMA box: the largest divisor of L not above 256.
static int box_rows(int L) {
  for (int r = L < 256 ? L : 256; r >= 1; --r)
    if (L % r == 0) return r;
  return 1;
}

static int swz_host(int k, int esz) { return esz == 8 ? k + (k >> 4) : k + (k >> 3); }

static size_t max_smem_per_block() {
  static size_t v = 0;
  if (!v) {
    int dev = 0, bytes = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        bytes <= 0)
      bytes = 227 * 1024;
    v = (size_t)bytes;
  }
  return v;
}

// Stage-major twiddle table for a radix sequence (StageTw layout): entry
// Ns - R_0 + jm*(R-1) + r-1 of stage s >= 1 is exp(-2 pi i jm r / (Ns R)),
// times last_scale in the last stage (StageTwScaledLast: the inverse's 1/L
// folded into the table).
static std::shared_ptr<DevTable> stage_twiddles(int dbl, int L, const std::vector<int>& rad,
                                                double last_scale = 1.0) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, std::vector<int>, double>, std::weak_ptr<DevTable>> cache;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  auto key = std::make_tuple(dev * 2 + dbl, L, rad, last_scale);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end())
    if (auto sp = it->second.lock()) return sp;
  const int R0 = rad.empty() ? 1 : rad[0];
  const int n = L - R0 > 0 ? L - R0 : 1;
  const size_t esz = dbl ? 16 : 8;
  std::vector<unsigned char> host(esz * (size_t)n, 0);
  const long double two_pi = 2.0L * acosl(-1.0L);
  int Ns = R0;
  for (size_t st = 1; st < rad.size(); ++st) {
    const int R = rad[st];
    for (int jm = 0; jm < Ns; ++jm)
      for (int r = 1; r < R; ++r) {
        const long long D = (long long)Ns * R;
        const long long m = ((long long)jm * r) % D;
        const long double ang = two_pi * (long double)m / (long double)D;
        const long double f = st + 1 == rad.size() ? (long double)last_scale : 1.0L;
        const long double c = f * cosl(ang), sn = -f * sinl(ang);
        const size_t e = (size_t)(Ns - R0 + jm * (R - 1) + r - 1);
        if (dbl) { double v[2] = {(double)c, (double)sn}; std::memcpy(&host[esz * e], v, esz); }
        else { float v[2] = {(float)c, (float)sn}; std::memcpy(&host[esz * e], v, esz); }
      }
    Ns *= R;
  }
  auto t = std::make_shared<DevTable>();
  t->device = dev;
  t->bytes = host.size();
  cuda_check(cudaMalloc(&t->p, t->bytes), "cudaMalloc(stage twiddles)");
  cuda_check(cudaMemcpy(t->p, host.data(), t->bytes, cudaMemcpyHostToDevice), "cudaMemcpy(stage twiddles)");
  cache[key] = t;
  return t;
}

// Which kernel a pass may use.
static bool pipe_strided_ok(const PassSpec& s, const StaticPlan* sp, size_t esz) {
  return sp && sp->pipe_s && s.fast_io && !s.epi && s.I > 1 && (s.I * (long long)esz) % 16 == 0 &&
         s.I < (1LL << 31) && s.O < (1LL << 31);
}
static bool pipe_contig_ok(const PassSpec& s, const StaticPlan* sp, size_t esz) {
  return sp && sp->pipe_c && s.fast_io && !s.epi && s.I == 1 && ((long long)s.L * (long long)esz) % 16 == 0;
}

static bool feed_ok(const PassSpec& s, size_t esz) {
  return s.fast_io && !s.epi && s.I > 1 && (s.I * (long long)esz) % 16 == 0 && s.I < (1LL << 31) &&
         s.O < (1LL << 31) && find_strided_kernel(s.dbl, s.L, 0) != nullptr;
}

// Strided C2C pass fed by a producer warp (axis_pass_strided); s.C selects
// the launch shape.
static Pass make_feed_pass(const PassSpec& s) {
  const int L = s.L;
  const int esz = s.dbl ? 16 : 8;
  if (!feed_ok(s, esz)) throw Error{DFFT_ERROR_INVALID_VALUE, "producer-fed strided variant not available"};
  const SlabKernel* k = find_strided_kernel(s.dbl, L, s.C < 0 ? 0 : s.C);
  if (!k) throw Error{DFFT_ERROR_INVALID_VALUE, "no such strided launch shape"};
  if (s.I < k->cs) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "fewer columns than one tile"};
  // the forward kernels have conjugation off and unit scale compiled in
  if (!s.inverse && s.scale != 1.0) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "scaled forward strided pass"};
  const std::vector<int> rad(k->radix, k->radix + k->nst);
  Pass p;
  p.feed = true;
  p.is_static = true;
  p.fn = s.inverse ? k->fn_inv : k->fn;
  PassDesc& d = p.d;
  d.L = L;
  d.nst = k->nst;
  int ns = 1;
  for (int i = 0; i < d.nst; ++i) {
    d.radix[i] = rad[i];
    d.ns[i] = ns;
    d.tws[i] = L / (ns * rad[i]);
    ns *= rad[i];
  }
  d.P = k->P;
  d.C = k->cs;
  d.ld = L;
  d.inverse = s.inverse;
  d.cfast = 1;
  d.Q = s.I * s.O;
  d.I = s.I;
  d.scale = s.scale;
  d.in = s.in;
  d.out = s.out;
  for (auto& t : s.keep) p.tables.push_back(t);
  auto stw = stage_twiddles(s.dbl, L, rad);
  p.tables.push_back(stw);
  d.tw = stw->p;
  StridedGeom& g = p.fgeom;
  g.xscale = s.dbl ? 2 : 1;
  g.lb = box_rows(L);
  g.nlb = L / g.lb;
  g.tiles_i = (int)((s.I + k->cs - 1) / k->cs);
  g.ntiles = (long long)g.tiles_i * s.O;
  g.ntw = k->nst > 1 ? L - rad[0] : 0;
  const size_t bstride = ((size_t)k->cs * L * esz + 127) & ~(size_t)127;
  g.bstride = (int)(bstride / esz);
  g.err = device_error_word();
  if (g.nlb > 1 && ((size_t)g.lb * k->cs * esz) % 128 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "TMA box offsets would not be 128-byte aligned"};
  if (((size_t)k->cs * g.xscale * 8) % 16 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "TMA rows would not be 16-byte multiples"};
  p.geom.C = k->cs;
  p.geom.xscale = g.xscale;
  p.geom.lb = g.lb;
  p.tI = s.I;
  p.tL = L;
  p.tO = s.O;
  const size_t tw_bytes = ((size_t)g.ntw * esz + 127) & ~(size_t)127;
  p.smem = kSlabHeader + tw_bytes + (size_t)k->nb * bstride;
  p.block = dim3((unsigned)k->lb);
  if (p.smem > max_smem_per_block()) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "strided tiles do not fit"};
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(strided)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "strided kernel cannot be resident"};
  long long nb = (long long)sm_count() * occ;
  if (nb > g.ntiles) nb = g.ntiles;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
  return p;
}

// Strided C2C pass whose rows TMA cannot address (a row stride that is not
// a multiple of 16 bytes): tiles copied by cp.async (axis_pass_async);
// s.C selects the launch shape.
static bool async_ok(const PassSpec& s, size_t esz) {
  (void)esz;
  return s.fast_io && !s.epi && s.I > 1 && s.I < (1LL << 31) && s.O < (1LL << 31) &&
         find_async_kernel(s.dbl, s.L, 0) != nullptr && s.in.si == 1 && s.out.si == 1;
}

static Pass make_async_pass(const PassSpec& s) {
  const int L = s.L;
  const int esz = s.dbl ? 16 : 8;
  if (!async_ok(s, esz)) throw Error{DFFT_ERROR_INVALID_VALUE, "cp.async strided variant not available"};
  const SlabKernel* k = find_async_kernel(s.dbl, L, s.C < 0 ? 0 : s.C);
  if (!k) throw Error{DFFT_ERROR_INVALID_VALUE, "no such cp.async launch shape"};
  if (!s.inverse && s.scale != 1.0) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "scaled forward strided pass"};
  const std::vector<int> rad(k->radix, k->radix + k->nst);
  Pass p;
  p.async_ = true;
  p.is_static = true;
  p.fn = s.inverse ? k->fn_inv : k->fn;
  PassDesc& d = p.d;
  d.L = L;
  d.nst = k->nst;
  int ns = 1;
  for (int i = 0; i < d.nst; ++i) {
    d.radix[i] = rad[i];
    d.ns[i] = ns;
    d.tws[i] = L / (ns * rad[i]);
    ns *= rad[i];
  }
  d.P = k->P;
  d.C = k->cs;
  d.ld = L;
  d.inverse = s.inverse;
  d.cfast = 1;
  d.Q = s.I * s.O;
  d.I = s.I;
  d.scale = s.scale;
  d.in = s.in;
  d.out = s.out;
  for (auto& t : s.keep) p.tables.push_back(t);
  auto stw = stage_twiddles(s.dbl, L, rad);
  p.tables.push_back(stw);
  d.tw = stw->p;
  AsyncGeom& g = p.ageom;
  g.I = s.I;
  g.Q = s.I * s.O;
  g.ntiles = (g.Q + k->cs - 1) / k->cs;
  g.ntw = k->nst > 1 ? L - rad[0] : 0;
  const size_t bstride = ((size_t)k->cs * L * esz + 127) & ~(size_t)127;
  g.bstride = (int)(bstride / esz);
  const size_t tw_bytes = ((size_t)g.ntw * esz + 127) & ~(size_t)127;
  p.smem = tw_bytes + (size_t)k->nb * bstride;
  p.block = dim3((unsigned)k->lb);
  if (p.smem > max_smem_per_block()) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "strided tiles do not fit"};
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(async)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "cp.async kernel cannot be resident"};
  long long nb = (long long)sm_count() * occ;
  if (nb > g.ntiles) nb = g.ntiles;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
  return p;
}

// R2C first pass / C2R last pass over whole contiguous pencils (I = 1):
// real_pass when a kernel exists for the half length and the pencils split
// into whole tiles.
static int real_kind(const PassSpec& s) {
  const long long L = s.L;
  if (s.I != 1 || s.in.sk != 1 || s.out.sk != 1 || s.in.chirp || s.out.chirp || s.in.mul || s.out.mul) return 0;
  if (s.epi && !s.inverse && s.in.kind == IO_REAL_PAIR && s.out.kind == IO_CPLX && s.in.so == 2 * L &&
      s.out.so == L + 1)
    return 1;
  if (!s.epi && s.inverse && s.in.kind == IO_HERM_PAIR && s.out.kind == IO_REAL_PAIR && s.in.so == L + 1 &&
      s.in.n == L && s.out.so == 2 * L)
    return 2;
  return 0;
}

static Pass make_real_pass(const PassSpec& s) {
  const int kind = real_kind(s);
  const int M = s.L;
  const int esz = s.dbl ? 16 : 8;
  const SlabKernel* k = kind ? find_real_kernel(s.dbl, M) : nullptr;
  if (!k) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "no pipelined real kernel for this pass"};
  if (s.O % k->cs != 0) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "pencils do not split into whole tiles"};
  const std::vector<int> rad(k->radix, k->radix + k->nst);
  Pass p;
  p.real = true;
  p.is_static = true;
  p.fn = kind == 1 ? k->fn : k->fn_inv;
  PassDesc& d = p.d;
  d.L = M;
  d.nst = k->nst;
  int ns = 1;
  for (int i = 0; i < d.nst; ++i) {
    d.radix[i] = rad[i];
    d.ns[i] = ns;
    d.tws[i] = M / (ns * rad[i]);
    ns *= rad[i];
  }
  // work-buffer column stride: the P lanes of a pencil touch P consecutive
  // 8-byte slots of a bank row, so pencils P slots apart (mod 16) fill the
  // row evenly (ComplexF64: P lanes of 16 bytes fill whole rows anyway)
  int ld = swz_host(M - 1, esz) + 1;
  if (esz == 8) {
    while (ld % 16 != k->P % 16) ++ld;
  } else if ((ld & 1) == 0) {
    ld += 1;
  }
  d.P = k->P;
  d.C = k->cs;
  d.ld = ld;
  d.inverse = kind == 2 ? 1 : 0;
  d.cfast = 0;
  d.epi = 0;
  d.Q = s.O;
  d.I = 1;
  d.scale = s.scale;
  d.in = s.in;
  d.out = s.out;
  for (auto& t : s.keep) p.tables.push_back(t);
  auto stw = stage_twiddles(s.dbl, M, rad);
  p.tables.push_back(stw);
  d.tw = stw->p;
  auto w = twiddle_table(s.dbl, 2LL * M, 1, 0, M + 1, false);
  p.tables.push_back(w);
  d.tw2 = w->p;
  RealGeom& g = p.rgeom;
  g.ntiles = s.O / k->cs;
  g.ntw = k->nst > 1 ? M - rad[0] : 0;
  g.ld = ld;
  // a buffer holds the C pencils of M elements PS = M + 64 bytes apart
  // (bank spread), or C*(M+1) dense elements
  const size_t ps = (size_t)M + 64 / esz;
  const size_t bstride = ((size_t)k->cs * ps * esz + 127) & ~(size_t)127;
  g.bstride = (int)(bstride / esz);
  g.err = device_error_word();
  const size_t tw_bytes = ((size_t)(g.ntw + M + 1) * esz + 127) & ~(size_t)127;
  p.smem = kSlabHeader + tw_bytes + (size_t)k->nb * bstride + (size_t)k->cs * ld * esz;
  p.block = dim3((unsigned)k->lb);
  if (p.smem > max_smem_per_block()) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "real tiles do not fit"};
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(real)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "real kernel cannot be resident"};
  long long nb = (long long)sm_count() * occ;
  if (nb > g.ntiles) nb = g.ntiles;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
  return p;
}

// R2R passes whose tiles are whole contiguous pencils (1) or strided
// columns (2) of the real data: tiled_pass.
static int tiled_kind(const PassSpec& s) {
  if (s.in.kind != IO_R2R || s.out.kind != IO_R2R || s.epi || s.in.chirp || s.out.chirp || s.in.mul ||
      s.out.mul || s.in.n != s.out.n || s.in.r2r != s.out.r2r ||
      (s.in.r2r != K_REDFT10 && s.in.r2r != K_REDFT01))
    return 0;
  const long long n = s.in.n;
  if (s.I == 1 && s.in.sk == 1 && s.out.sk == 1 && s.in.so == n && s.out.so == n) return 1;
  if (s.I > 1 && s.in.sk == s.I && s.out.sk == s.I && s.in.so == s.I * n && s.out.so == s.I * n) return 2;
  return 0;
}

static Pass make_tiled_pass(const PassSpec& s) {
  const int kind = tiled_kind(s);
  const int L = s.L;
  const int rsz = s.dbl ? 8 : 4, csz = 2 * rsz;
  const TiledKernel* k = kind ? find_tiled_kernel(s.dbl, L, kind == 2 ? 1 : 0, s.in.r2r) : nullptr;
  if (!k) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "no tiled kernel for this pass"};
  const int n = s.in.n;
  const int C = k->cs;
  Pass p;
  p.tiled = kind;
  p.tdbl = s.dbl;
  p.is_static = true;
  p.fn = k->fn;
  TiledGeom& g = p.tgeom;
  g.n_in = g.n_out = n;
  if (kind == 1) {
    if (s.O % C != 0 || ((size_t)C * n * rsz) % 16 != 0)
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "pencils do not split into whole tiles"};
    g.ntiles = s.O / C;
    g.tiles_i = 1;
    g.lb = n;
    g.nlb = 1;
  } else {
    if (s.I < C || (s.I * rsz) % 16 != 0 || ((size_t)C * rsz) % 16 != 0 || s.I >= (1LL << 31) ||
        s.O >= (1LL << 31))
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "columns cannot be tiled by TMA"};
    g.tiles_i = (int)((s.I + C - 1) / C);
    g.ntiles = (long long)g.tiles_i * s.O;
    g.lb = box_rows(n);
    g.nlb = n / g.lb;
    if (g.nlb > 16 || (g.nlb > 1 && ((size_t)g.lb * C * rsz) % 128 != 0))
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "rows cannot be split into TMA boxes"};
    p.geom.C = C;
    p.geom.lb = g.lb;
    p.tI = s.I;
    p.tL = n;
    p.tO = s.O;
  }
  PassDesc& d = p.d;
  d.L = L;
  d.nst = k->nst;
  int ns = 1;
  for (int i = 0; i < d.nst; ++i) {
    d.radix[i] = k->radix[i];
    d.ns[i] = ns;
    d.tws[i] = L / (ns * k->radix[i]);
    ns *= k->radix[i];
  }
  int ld = swz_host(L - 1, csz) + 1;
  if ((ld & 1) == 0) ld += 1;
  d.P = k->P;
  d.C = C;
  d.ld = ld;
  d.inverse = s.inverse;
  d.cfast = kind == 2 ? 1 : 0;
  d.epi = 0;
  d.Q = s.I * s.O;
  d.I = s.I;
  d.scale = s.scale;
  d.in = s.in;
  d.out = s.out;
  for (auto& t : s.keep) p.tables.push_back(t);
  auto tw = twiddle_table(s.dbl, L, 1, 0, L, false);
  p.tables.push_back(tw);
  d.tw = tw->p;
  g.ld = ld;
  g.bstride = (int)(((size_t)C * n * rsz + 127) & ~(size_t)127);
  g.err = device_error_word();
  p.smem = kSlabHeader + 2 * (size_t)g.bstride + (size_t)C * ld * csz;
  p.block = dim3((unsigned)k->lb);
  if (p.smem > max_smem_per_block()) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "tiles do not fit"};
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(tiled)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "tiled kernel cannot be resident"};
  long long nb = (long long)sm_count() * occ;
  if (nb > g.ntiles) nb = g.ntiles;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
  return p;
}

Pass make_pass(const PassSpec& s) {
  if (s.variant == VARIANT_FEED) return make_feed_pass(s);
  if (s.variant == VARIANT_ASYNC) return make_async_pass(s);
  if (s.variant == VARIANT_AUTO && tiled_kind(s)) {
    try {
      return make_tiled_pass(s);
    } catch (const Error& e) {
      if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
    }
  }
  if (s.variant == VARIANT_AUTO && real_kind(s)) {
    try {
      return make_real_pass(s);
    } catch (const Error& e) {
      if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
    }
  }
  Pass p;
  PassDesc& d = p.d;
  const int L = s.L;
  if (L < 1) throw Error{DFFT_ERROR_INVALID_VALUE, "transform length must be >= 1"};
  const int esz = s.dbl ? 16 : 8;
  const size_t smax = max_smem_per_block();
  const StaticPlan* sp = find_static(s.dbl, L);
  if (sp && sp->P > sp->lb) sp = nullptr;
  int variant = s.variant;
  if (variant == VARIANT_AUTO) {
    // strided axes: the producer-fed kernel for passes of 16 MiB and more
    // (below that its persistent grid is not filled and the one-tile kernels
    // are as fast), unless rows lie 1 MiB or more apart (each tile then
    // touches L pages, and the narrower tile rows of that kernel pay the
    // address translation twice as often)
    if (feed_ok(s, esz) && s.I * (long long)esz < (1LL << 20) &&
        (double)s.I * (double)s.O * (double)L * esz >= (double)(16 << 20)) {
      // the first (fastest) default launch shape whose tile width fits I
      for (int v = 0; const SlabKernel* k = find_strided_kernel(s.dbl, L, v); ++v) {
        if (!k->dflt || k->cs > s.I) continue;
        PassSpec t = s;
        t.variant = VARIANT_FEED;
        t.C = v;
        try {
          return make_pass(t);
        } catch (const Error&) {
        }
        break;
      }
    }
    // the same passes with rows TMA cannot address: cp.async tiles
    if (!feed_ok(s, esz) && (s.I * (long long)esz) % 16 != 0 && async_ok(s, esz) &&
        (double)s.I * (double)s.O * (double)L * esz >= (double)(16 << 20)) {
      for (int v = 0; const SlabKernel* k = find_async_kernel(s.dbl, L, v); ++v) {
        if (!k->dflt || k->cs > s.I) continue;
        PassSpec t = s;
        t.variant = VARIANT_ASYNC;
        t.C = v;
        try {
          return make_pass(t);
        } catch (const Error&) {
        }
        break;
      }
    }
    if (pipe_strided_ok(s, sp, esz) || pipe_contig_ok(s, sp, esz)) {
      PassSpec t = s;
      t.variant = VARIANT_PIPE;
      try {
        return make_pass(t);
      } catch (const Error&) {
      }
    }
    variant = sp ? VARIANT_DIRECT : VARIANT_DYNAMIC;
  }
  if (variant == VARIANT_PIPE && !(pipe_strided_ok(s, sp, esz) || pipe_contig_ok(s, sp, esz)))
    throw Error{DFFT_ERROR_INVALID_VALUE, "pipelined variant not available for this pass"};
  if (variant == VARIANT_DIRECT && !sp)
    throw Error{DFFT_ERROR_INVALID_VALUE, "no static plan for this length"};

  std::vector<int> rad;
  int P = 0, lb = 1024;
  if (variant == VARIANT_DYNAMIC) {
    rad = dynamic_radices(L);
    if (rad.empty())
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE,
                  "length " + std::to_string(L) + " has a prime factor above 13"};
    const int EMAX = 16;
    P = 1;
    for (int R : rad) {
      int B = EMAX / R;
      int need = (L / R + B - 1) / B;
      if (need > P) P = need;
    }
    lb = 1024;
    p.fn = dynamic_kernel(s.dbl);
  } else {
    rad.assign(sp->radix, sp->radix + sp->nst);
    P = sp->P;
    lb = variant == VARIANT_PIPE ? sp->pipe_lb : sp->lb;
    p.is_static = true;
    if (variant == VARIANT_DIRECT) p.fn = s.fast_io ? sp->fast : sp->any;
  }
  if ((int)rad.size() > kMaxStages)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "too many stages for length " + std::to_string(L)};
  if (P > lb)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "length " + std::to_string(L) + " exceeds one CTA"};
  d.L = L;
  d.nst = (int)rad.size();
  int ns = 1;
  for (int i = 0; i < d.nst; ++i) {
    d.radix[i] = rad[i];
    d.ns[i] = ns;
    d.tws[i] = L / (ns * rad[i]);
    ns *= rad[i];
  }
  d.P = P;
  int ld = swz_host(L - 1, esz) + 1;
  if ((ld & 1) == 0) ld += 1;
  d.ld = ld;
  d.cfast = s.I > 1 ? 1 : 0;
  d.inverse = s.inverse;
  d.epi = s.epi ? 1 : 0;
  const long long Q = s.I * s.O;
  d.Q = Q;
  d.I = s.I;
  d.scale = s.scale;
  d.in = s.in;
  d.out = s.out;
  for (auto& t : s.keep) p.tables.push_back(t);
  const size_t col_bytes = (size_t)ld * esz;

  if (variant == VARIANT_PIPE) {
    const bool contig = s.I == 1;
    p.fn = contig ? sp->pipe_c : sp->pipe_s;
    p.tma = !contig;
    p.pipe = true;
    auto stw = stage_twiddles(s.dbl, L, rad);
    p.tables.push_back(stw);
    d.tw = stw->p;
    auto twl = twiddle_table(s.dbl, L, 1, 0, L, false);
    p.tables.push_back(twl);
    d.tw2 = twl->p;
    TmaGeom& g = p.geom;
    g.ntw = (contig && d.nst > 1) ? L - rad[0] : 0;
    const size_t tw_bytes = ((size_t)g.ntw * esz + 127) & ~(size_t)127;
    auto bstride_bytes = [&](int C) { return ((size_t)C * L * esz + 127) & ~(size_t)127; };
    auto smem_for = [&](int C) {
      return 128 + tw_bytes + (size_t)kTmaBufs * bstride_bytes(C) + (contig ? (size_t)C * ld * esz : 0);
    };
    int C = s.C;
    if (!contig) {
      // the strided kernel has its tile width compiled in
      if (C > 0 && C != sp->pipe_cs)
        throw Error{DFFT_ERROR_INVALID_VALUE, "strided pipelined kernel has a fixed tile width"};
      C = sp->pipe_cs;
    } else if (C <= 0) {
      C = 1;
      while (C * 2 * P <= 256 && smem_for(C * 2) <= smax) C *= 2;
    }
    while (C > 1 && (C * P > lb || smem_for(C) > smax)) C /= 2;
    if (!contig && C % 2) C = 2;  // 16-byte TMA rows for complex float
    if (C * P > lb || smem_for(C) > smax)
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "pipelined tile does not fit"};
    if (!contig) {
      // every TMA box must start 128 bytes apart inside the tile buffer
      const int lbr = box_rows(L);
      if (L / lbr > 1 && ((size_t)lbr * C * esz) % 128 != 0)
        throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "TMA box offsets would not be 128-byte aligned"};
    }
    d.C = C;
    g.C = C;
    g.xscale = s.dbl ? 2 : 1;
    g.ld = ld;
    g.bstride = (int)(bstride_bytes(C) / esz);
    g.err = device_error_word();
    if (contig) {
      g.ncols = Q;
      g.ntiles = (Q + C - 1) / C;
      g.tiles_i = 1;
      g.lb = L;
      g.nlb = 1;
      g.tile_bytes = (unsigned)((size_t)C * L * esz);
    } else {
      p.tI = s.I;
      p.tL = L;
      p.tO = s.O;
      g.tiles_i = (int)((s.I + C - 1) / C);
      g.ntiles = (long long)g.tiles_i * s.O;
      g.ncols = Q;
      g.lb = box_rows(L);
      g.nlb = L / g.lb;
      g.tile_bytes = (unsigned)((size_t)C * L * esz);
    }
    p.block = dim3((unsigned)(C * P));
    p.smem = smem_for(C);
    cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(pipe)");
    int occ = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
               "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "pipelined kernel cannot be resident"};
    long long nb = (long long)sm_count() * occ;
    if (nb > g.ntiles) nb = g.ntiles;
    p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
    return p;
  }

  if (col_bytes > smax)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE,
                "length " + std::to_string(L) + " does not fit one CTA's shared memory"};
  int C = s.C;
  if (C <= 0) {
    if (d.cfast) {
      // rows of at least 128 bytes for coalesced strided loads, ~256 threads
      C = s.dbl ? 8 : 16;
      while (C * P < 256 && C < 64) C *= 2;
    } else {
      C = 1;
      while (C * 2 * P <= 256) C *= 2;
    }
  }
  while (C > 1 && (C * P > lb || (size_t)C * col_bytes > smax)) C /= 2;
  if (Q > 0 && C > Q) {
    // do not launch threads for columns that do not exist
    int c2 = 1;
    while (c2 * 2 <= Q) c2 *= 2;
    if (c2 < C) C = c2;
  }
  d.C = C;
  auto tw = twiddle_table(s.dbl, L, 1, 0, L, false);
  p.tables.push_back(tw);
  d.tw = tw->p;
  if (s.epi) {
    auto tw2 = twiddle_table(s.dbl, 2LL * L, 1, 0, L + 1, false);
    p.tables.push_back(tw2);
    d.tw2 = tw2->p;
  }
  const long long nblk = (Q + C - 1) / C;
  if (nblk > 0x7fffffffLL) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "too many columns for one launch"};
  p.grid = dim3((unsigned)nblk);
  p.block = dim3((unsigned)(C * P));
  p.smem = (size_t)C * col_bytes;
  return p;
}

Pass make_slab_pass(int dbl, int L, long long O, int inverse, int v) {
  const SlabKernel* k = find_slab_kernel(dbl, L, v);
  if (!k) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "no fused slab kernel for this length"};
  if (L % k->cs != 0) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab tiling does not divide L"};
  if (O < 1 || O >= (1LL << 31)) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab count out of range"};
  const int esz = dbl ? 16 : 8;
  const std::vector<int> rad(k->radix, k->radix + k->nst);
  Pass p;
  p.slab = true;
  p.is_static = true;
  p.fn = inverse ? k->fn_inv : k->fn;
  int ld = swz_host(L - 1, esz) + 1;
  if ((ld & 1) == 0) ld += 1;
  auto fill = [&](PassDesc& d, long long I) {
    d.L = L;
    d.nst = k->nst;
    int ns = 1;
    for (int i = 0; i < d.nst; ++i) {
      d.radix[i] = rad[i];
      d.ns[i] = ns;
      d.tws[i] = L / (ns * rad[i]);
      ns *= rad[i];
    }
    d.P = k->P;
    d.C = k->cs;
    d.ld = ld;
    d.inverse = inverse;
    d.cfast = I > 1 ? 1 : 0;
    d.Q = (long long)L * O;
    d.I = I;
    d.scale = inverse ? 1.0 / (double)L : 1.0;
    d.in.kind = d.out.kind = IO_CPLX;
    d.in.si = d.out.si = 1;
    d.in.so = d.out.so = I * L;
    d.in.sk = d.out.sk = I;
  };
  fill(p.d, 1);
  fill(p.d2, L);
  // the inverse kernels fold 1/L into the last stage's twiddles
  auto stw = stage_twiddles(dbl, L, rad, inverse ? 1.0 / (double)L : 1.0);
  p.tables.push_back(stw);
  p.d.tw = stw->p;
  auto twl = twiddle_table(dbl, L, 1, 0, L, false);
  p.tables.push_back(twl);
  p.d2.tw2 = twl->p;
  SlabGeom& g = p.sgeom;
  g.nslab = O;
  g.rin = g.rout = L;
  g.zr = O;
  g.tiles = L / k->cs;
  g.xscale = dbl ? 2 : 1;
  g.lb = box_rows(L);
  g.nlb = L / g.lb;
  g.ntw = k->nst > 1 ? L - rad[0] : 0;
  const size_t tile = (size_t)k->cs * L * esz;
  const size_t bstride = (tile + 127) & ~(size_t)127;
  g.bstride = (int)(bstride / esz);
  g.err = device_error_word();
  if (g.nlb > 1 && ((size_t)g.lb * k->cs * esz) % 128 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "TMA box offsets would not be 128-byte aligned"};
  if (((size_t)k->cs * g.xscale * 8) % 16 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "TMA rows would not be 16-byte multiples"};
  // tensor map geometry (encode_map): {L*xscale, L, O}, box {cs*xscale, lb, 1}
  p.geom.C = k->cs;
  p.geom.xscale = g.xscale;
  p.geom.lb = g.lb;
  p.tI = L;
  p.tL = L;
  p.tO = O;
  const size_t tw_bytes = ((size_t)g.ntw * esz + 127) & ~(size_t)127;
  p.smem = kSlabHeader + tw_bytes + (size_t)k->nb * bstride;
  p.block = dim3((unsigned)(k->cs * k->P + 32));  // stage threads + producer warp
  if ((int)p.block.x != k->lb) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab kernel block size mismatch"};
  if (p.smem > max_smem_per_block()) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab tiles do not fit"};
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(slab)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab kernel cannot be resident"};
  const long long jobs = 2LL * g.tiles * O;
  long long nb = (long long)sm_count() * occ;
  if (nb > jobs) nb = jobs;
  p.grid = dim3((unsigned)nb);
  // a CTA holds up to (buffers + claim) jobs: y-jobs trail their slab's
  // x-jobs by more rounds than the jobs in flight span
  g.lag = (int)((nb * (k->nb + kSlabClaim) + 2LL * g.tiles - 1) / (2LL * g.tiles)) + 1;
  p.ctr_bytes = 8 + 4 * (size_t)O;
  return p;
}

// Columns split by rank, y-phase first (kernel MODE 2): the y-phase reads
// the input through a map over its rank blocks of rin columns, the x-phase
// writes pieces of rout elements (both powers of two, multiples of the tile
// width); rin = L / rout = L is the plain side.
static Pass make_slab_cols_pass(int dbl, int L, long long nslab, int inverse, int v, int rin, int rout,
                                long long zr) {
  Pass p = make_slab_pass(dbl, L, nslab, inverse, v);
  SlabGeom& g = p.sgeom;
  const int cs = p.geom.C;
  auto pow2 = [](int x) { return x >= 1 && (x & (x - 1)) == 0; };
  if (!pow2(rin) || !pow2(rout) || rin > L || rout > L || L % rin || L % rout || zr < nslab)
    throw Error{DFFT_ERROR_INVALID_VALUE, "column split: columns per rank must be a power of two dividing L, zr >= slabs"};
  if (rin % cs != 0 || rout % cs != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "column split: columns per rank do not hold whole tiles"};
  const size_t esz = dbl ? 16 : 8;
  if (((size_t)rout * esz) % 16 != 0 || ((size_t)rin * esz) % 16 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "column split: rows of a rank block are not 16-byte multiples"};
  const long long zin = zr * (long long)(L / rin - 1) + nslab;
  const long long zout = zr * (long long)(L / rout - 1) + nslab;
  if (zin >= (1LL << 31) || zout >= (1LL << 31)) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "column split too large"};
  g.rin = rin;
  g.rout = rout;
  g.zr = zr;
  const SlabKernel* k = find_slab_kernel(dbl, L, v);
  p.fn = inverse ? k->fn_inv_cols : k->fn_cols;
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(slab cols)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab column-split kernel cannot be resident"};
  p.cols = true;
  // forward: the intermediate overwrites the (plain) input; inverse: it
  // goes to the (plain) output
  p.cols_mid_in = !inverse;
  p.tI = L;  // tout: the plain intermediate
  p.tL = L;
  p.tO = nslab;
  p.tI2 = rin;  // tin: the input, rin columns per rank block
  p.tL2 = L;
  p.tO2 = zin;
  return p;
}

Pass make_slab_split_pass(int dbl, int L, long long nslab, int inverse, int v, int rin, int rout,
                          long long zr, int split_dim) {
  if (split_dim == 1) return make_slab_cols_pass(dbl, L, nslab, inverse, v, rin, rout, zr);
  Pass p = make_slab_pass(dbl, L, nslab, inverse, v);
  SlabGeom& g = p.sgeom;
  const int cs = p.geom.C;
  auto ok_rows = [&](int R) { return R >= 1 && R <= L && L % R == 0; };
  if (!ok_rows(rin) || !ok_rows(rout) || zr < nslab)
    throw Error{DFFT_ERROR_INVALID_VALUE, "rank split: rows per rank must divide L, zr >= slabs"};
  // a tile's pencils stay contiguous, and no TMA box straddles two ranks'
  // rows (boxes of the largest divisor of rout up to the plain box height)
  if (rin % cs != 0 || rout % cs != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "rank split: rows per rank do not hold whole tiles"};
  while (rout % g.lb != 0) --g.lb;
  g.nlb = L / g.lb;
  p.geom.lb = g.lb;
  const size_t esz = dbl ? 16 : 8;
  if (g.nlb > 1 && ((size_t)g.lb * cs * esz) % 128 != 0)
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "rank split: TMA box offsets would not be 128-byte aligned"};
  const long long zmax = zr * (long long)(L / rout - 1) + nslab;  // slab coordinates the map spans
  const long long zin = zr * (long long)(L / rin - 1) + nslab;
  if (zmax >= (1LL << 31) || zin >= (1LL << 31)) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "rank split too large"};
  g.rin = rin;
  g.rout = rout;
  g.zr = zr;
  const SlabKernel* k = find_slab_kernel(dbl, L, v);
  p.fn = inverse ? k->fn_inv_split : k->fn_split;
  cuda_check(ensure_smem_attr(p.fn, p.smem), "cudaFuncSetAttribute(slab split)");
  int occ = 0;
  cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p.fn, (int)p.block.x, p.smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (occ < 1) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab split kernel cannot be resident"};
  p.tL = rout;
  p.tO = zmax;
  return p;
}

cudaError_t launch_pass(const Pass& p, void* in, void* out, cudaStream_t stream, void* work) {
  if (p.grid.x == 0) return cudaSuccess;
  cudaError_t e = ensure_smem_attr(p.fn, p.smem);
  if (e != cudaSuccess) return e;
  PassDesc d = p.d;
  d.in.p = in;
  d.out.p = out;
  if (p.mixed) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    CUtensorMap tin, tout;
    std::memset(&tin, 0, sizeof(tin));
    std::memset(&tout, 0, sizeof(tout));
    if (p.mstrided) {
      e = encode_map_sw128(&tin, in, p);
      if (e != cudaSuccess) return e;
      e = encode_map_sw128(&tout, out, p);
      if (e != cudaSuccess) return e;
    }
    MixedGeom g = p.mgeom;
    const void* ip = in;
    void* op = out;
    void* args[] = {&ip, &op, &tin, &tout, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.tiled) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    CUtensorMap tin, tout;
    std::memset(&tin, 0, sizeof(tin));
    std::memset(&tout, 0, sizeof(tout));
    if (p.tiled == 2) {
      e = encode_real_map(&tin, in, p, p.tdbl);
      if (e != cudaSuccess) return e;
      e = encode_real_map(&tout, out, p, p.tdbl);
      if (e != cudaSuccess) return e;
    }
    TiledGeom g = p.tgeom;
    g.src = in;
    g.dst = out;
    void* args[] = {&d, &tin, &tout, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.real) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    RealGeom g = p.rgeom;
    void* args[] = {&d, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.async_) {
    // the cp.async kernels move 8-byte (ComplexF32) elements
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 7)
      return cudaErrorMisalignedAddress;
    AsyncGeom g = p.ageom;
    void* args[] = {&d, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.feed) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    CUtensorMap tin, tout;
    std::memset(&tin, 0, sizeof(tin));
    std::memset(&tout, 0, sizeof(tout));
    e = encode_map(&tin, in, p);
    if (e != cudaSuccess) return e;
    e = encode_map(&tout, out, p);
    if (e != cudaSuccess) return e;
    StridedGeom g = p.fgeom;
    void* args[] = {&d, &tin, &tout, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.swap) {
    const void* a = in;
    void* b = out;
    SwapGeom g = p.swg;
    void* args[] = {&a, &b, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, 0, stream);
  }
  if (p.slab) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    if (!work || (reinterpret_cast<uintptr_t>(work) & 7)) return cudaErrorInvalidValue;
    CUtensorMap tin, tout;
    std::memset(&tin, 0, sizeof(tin));
    std::memset(&tout, 0, sizeof(tout));
    void* mid = p.cols && p.cols_mid_in ? in : out;  // what tout covers
    e = encode_map_dims(&tout, mid, p, p.tI, p.tL, p.tO);
    if (e != cudaSuccess) return e;
    if (p.cols) {
      e = encode_map_dims(&tin, in, p, p.tI2, p.tL2, p.tO2);
      if (e != cudaSuccess) return e;
      d.in.p = mid;  // the x-phase reads the intermediate
    } else {
      tin = tout;
    }
    e = cudaMemsetAsync(work, 0, p.ctr_bytes, stream);
    if (e != cudaSuccess) return e;
    PassDesc d2 = p.d2;
    SlabGeom g = p.sgeom;
    g.jobs = static_cast<unsigned long long*>(work);
    g.done = reinterpret_cast<unsigned*>(static_cast<char*>(work) + 8);
    void* args[] = {&d, &d2, &tin, &tout, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  if (p.pipe) {
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15)
      return cudaErrorMisalignedAddress;
    CUtensorMap tin, tout;
    std::memset(&tin, 0, sizeof(tin));
    std::memset(&tout, 0, sizeof(tout));
    if (p.tma) {
      e = encode_map(&tin, in, p);
      if (e != cudaSuccess) return e;
      e = encode_map(&tout, out, p);
      if (e != cudaSuccess) return e;
    }
    TmaGeom g = p.geom;
    void* args[] = {&d, &tin, &tout, &g};
    return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
  }
  void* args[] = {&d};
  return cudaLaunchKernel(p.fn, p.grid, p.block, args, p.smem, stream);
}

}  // namespace dfft

namespace dfft {

// ---------------------------------------------------------------------------
// Four-step decomposition of a complex axis that no single pass handles:
// L = L1 * L2, n = n1 + L1 n2, k = k2 + L2 k1,
//   X[k2 + L2 k1] = sum_n1 W_L1^(n1 k1) [ W_L^(n1 k2) sum_n2 x[n1 + L1 n2] W_L2^(n2 k2) ].
// Pass A: L2-point transforms along the sub-axis of stride I*L1 (columns
// (i, n1, o)), into a scratch in the same layout, times W_L^(n1 k2) on the
// way out; pass B: L1-point transforms along stride I (columns (i, k2, o)),
// written to position k2 + L2 k1 (the output's two-level column split).
// Each factor runs as one pass: a static plan, or the dynamic kernel for
// lengths up to 4096 with prime factors up to 13 that fit one CTA.  Splits
// with two static factors come first, then the most balanced one.
// ---------------------------------------------------------------------------

static int four_step_factor(int dbl, int n) {
  const StaticPlan* sp = find_static(dbl, n);
  if (sp && sp->P <= sp->lb) return VARIANT_DIRECT;
  if (n > 4096) return 0;
  const std::vector<int> rad = dynamic_radices(n);
  if (rad.empty() || (int)rad.size() > kMaxStages) return 0;
  int P = 1;
  for (int R : rad) {
    const int B = 16 / R;
    const int need = (n / R + B - 1) / B;
    if (need > P) P = need;
  }
  return P <= 1024 ? VARIANT_DYNAMIC : 0;
}

static bool four_step_split(int dbl, int L, int* L1, int* L2) {
  int best = 0, best_static = 0;
  for (int d = 2; (long long)d * d <= L; ++d) {
    if (L % d != 0) continue;
    const int va = four_step_factor(dbl, d), vb = four_step_factor(dbl, L / d);
    if (!va || !vb) continue;
    const int st = va == VARIANT_DIRECT && vb == VARIANT_DIRECT;
    if (st >= best_static) {
      best = d;
      best_static = st;
    }
  }
  if (!best) return false;
  *L1 = best;
  *L2 = L / best;
  return true;
}

// The pass pair of a four-step transform of length s.L = L1 * L2 along a
// complex axis with unit inner stride (element (i, n, o) at i + n I + o so).
// Pass A reads s.in (its chirp / mul indexed along the whole axis) and
// writes the scratch (I, L, O) times the twiddle; pass B reads the scratch
// and writes s.out at k2 + L2 k1 (with its chirp and the scale).
static void four_step_pair(const PassSpec& s, int L1, int L2, Pass* pa, Pass* pb) {
  const long long L = (long long)L1 * L2;
  auto tw = twiddle_table(s.dbl, L, 1, 0, (int)L, s.inverse != 0);
  PassSpec a = s;
  a.L = L2;
  a.I = s.I * L1;
  a.O = s.O;
  a.scale = 1.0;
  a.fast_io = false;
  a.epi = false;
  a.C = 0;
  a.variant = four_step_factor(s.dbl, L2);
  a.in.sk = s.I * L1;  // si = 1 and so as for the whole axis
  // sub-axis index j from the column base b = i + j I + o so: (b mod so) / I
  // (so need not be a multiple of I L1: Bluestein's input has L < L1 L2 rows)
  if (a.in.chirp || a.in.mul || a.in.kind == IO_HERM_FULL || a.in.kind == IO_R2R) {
    a.in.t_i = s.I;
    a.in.t_ia = a.in.so;
    a.in.t_m = L1;
  }
  a.out = IoAny{};
  a.out.kind = IO_CPLX_TW;
  a.out.si = 1;
  a.out.so = s.I * L;
  a.out.sk = s.I * L1;
  a.out.w = tw->p;
  a.out.n = (int)L;
  a.out.t_i = s.I;
  a.out.t_ia = s.I * L;
  a.keep.push_back(tw);
  PassSpec b = s;
  b.L = L1;
  b.I = s.I;
  b.O = (long long)L2 * s.O;
  b.fast_io = s.out.kind == IO_CPLX && !s.out.chirp;
  b.epi = false;
  b.C = 0;
  b.variant = four_step_factor(s.dbl, L1);
  b.in = IoAny{};
  b.in.kind = IO_CPLX;
  b.in.si = 1;
  b.in.so = s.I * L1;
  b.in.sk = s.I;
  b.out.sk = s.I * L2;
  b.out.so = s.I;
  b.out.o1 = L2;
  b.out.so2 = s.out.so;
  if (b.out.chirp || b.out.kind == IO_TRUNC || b.out.kind == IO_R2R) {
    b.out.t_i = s.I;
    b.out.t_ia = s.out.so;
    b.out.t_m = L2;
  }
  *pa = make_pass(a);
  *pb = make_pass(b);
}

static bool plain_complex_axis(const PassSpec& s) {
  const long long L = s.L;
  return s.in.kind == IO_CPLX && s.out.kind == IO_CPLX && !s.epi && !s.in.chirp && !s.out.chirp &&
         !s.in.mul && s.in.o1 == 0 && s.out.o1 == 0 && s.in.si == 1 && s.out.si == 1 && s.in.sk == s.I &&
         s.out.sk == s.I && s.in.so == s.I * L && s.out.so == s.I * L;
}

// Sides a four-step pair can split, and the extents of their columns in
// memory: complex, the full-length forms of the real transforms (real in /
// first n/2+1 outputs kept; Hermitian half in / real out) and the r2r
// kinds (n reals each side), with unit inner stride and whole-axis columns.
// A sub-axis column index (n1 < L1 on the input, k2 < L2 on the output)
// must stay inside its column's extent.
static bool four_step_extents(const PassSpec& s, long long* ein, long long* eout) {
  const long long L = s.L;
  auto ext = [&](const IoAny& io, bool out) -> long long {
    switch (io.kind) {
      case IO_CPLX:
      case IO_REAL:
        return L;
      case IO_HERM_FULL:
        return !out && io.n == L ? L / 2 + 1 : -1;
      case IO_TRUNC:
        return out && io.n == L / 2 ? L / 2 + 1 : -1;
      case IO_R2R:
        return io.n;
      default:
        return -1;
    }
  };
  const long long ei = ext(s.in, false), eo = ext(s.out, true);
  if (ei <= 0 || eo <= 0 || s.epi || s.in.chirp || s.out.chirp || s.in.mul || s.in.o1 != 0 || s.out.o1 != 0 ||
      s.in.si != 1 || s.out.si != 1 || s.in.sk != s.I || s.out.sk != s.I || s.in.so != s.I * ei ||
      s.out.so != s.I * eo)
    return false;
  *ein = ei;
  *eout = eo;
  return true;
}

// Axis swap pass (i, a, b, o) -> (i, b, a, o) over an I x A x B x O array.
static Pass make_swap_pass(int dbl, long long I, long long A, long long B, long long O) {
  Pass p;
  p.swap = true;
  p.swg = SwapGeom{I, A, B, O};
  p.d.L = 1;
  p.d.I = I;
  p.d.Q = I * A * B * O;
  p.fn = swap_axes_kernel(dbl, I == 1);
  p.block = dim3(256);
  const long long units = I == 1 ? ((A + 31) / 32) * ((B + 31) / 32) * O : (A * B * O + 7) / 8;
  long long nb = (long long)sm_count() * 8;
  if (nb > units) nb = units;
  p.grid = dim3((unsigned)(nb > 0 ? nb : 1));
  return p;
}

// The fast form of a plain complex four-step axis, three passes through one
// scratch (the strided and contiguous passes keep their pipelined kernels):
//   1. L2-point transforms along n2 (columns (i, n1), stride I L1) with the
//      twiddle W_L^(n1 k2) applied to the transformed tile before its store;
//   2. L1-point transforms along n1 (columns (i) per (k2, o), stride I), in
//      place, leaving (i, k1, k2);
//   3. the swap of the k1 and k2 axes into the output: (i, k2, k1), i.e.
//      index k2 + L2 k1 along the axis.
// Needs the pipelined strided kernel for L2 (else false, nothing added).
// fast_split picks the largest strided factor with such a kernel (so the
// contiguous factor is as short as it can be) whose cofactor is a length
// one pass handles.
static bool fast_split(int dbl, int L, int* Lc, int* Ls) {
  for (int d = dbl ? 512 : 1024; d >= 2; --d) {
    if (L % d != 0) continue;
    const StaticPlan* sp = find_static(dbl, d);
    if (!sp || !sp->pipe_s || sp->P > sp->lb) continue;
    const int c = L / d;
    // (a contiguous factor beyond one static plan runs the one-column
    // dynamic kernel, slower than the two-pass form: 2^24 ComplexF32 1.28
    // against 0.73 ms)
    if (c < 2 || !four_step_factor(dbl, c)) continue;
    *Ls = d;
    *Lc = c;
    return true;
  }
  return false;
}

static bool add_four_step_fast(std::vector<Pass>& out, const PassSpec& s, unsigned flags, int L1, int L2,
                               int src, int dst) {
  const long long L = (long long)L1 * L2;
  PassSpec a;
  a.dbl = s.dbl;
  a.L = L2;
  a.I = s.I * L1;
  a.O = s.O;
  a.inverse = s.inverse;
  a.scale = 1.0;
  a.in = s.in;
  a.in.sk = s.I * L1;  // si = 1 and so = I L as for the whole axis
  a.out = IoAny{};
  a.out.kind = IO_CPLX;
  a.out.si = 1;
  a.out.sk = s.I * L1;
  a.out.so = s.I * L;
  a.fast_io = true;
  a.variant = VARIANT_PIPE;
  Pass pa;
  try {
    pa = make_pass(a);
  } catch (const Error& e) {
    if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE && e.status != DFFT_ERROR_INVALID_VALUE) throw;
    return false;
  }
  if (!pa.tma || !pa.pipe) return false;  // the hook lives in the strided pipelined kernel
  // W_L^m = W_L^(m mod B) * W_L^(B * (m / B)), two small tables
  const int Bt = 1024;
  auto lo = twiddle_table(s.dbl, L, 1, 0, Bt, s.inverse != 0);
  auto hi = twiddle_table(s.dbl, L, Bt, 0, (int)((L + Bt - 1) / Bt), s.inverse != 0);
  pa.tables.push_back(lo);
  pa.tables.push_back(hi);
  pa.geom.tw_lo = lo->p;
  pa.geom.tw_hi = hi->p;
  pa.geom.tw_div = s.I;
  pa.geom.tw_lf = L;
  pa.geom.tw_b = Bt;
  PassSpec b;
  b.dbl = s.dbl;
  b.L = L1;
  b.I = s.I;
  b.O = (long long)L2 * s.O;
  b.inverse = s.inverse;
  b.scale = s.scale;
  b.in.kind = b.out.kind = IO_CPLX;
  b.in.si = b.out.si = 1;
  b.in.sk = b.out.sk = s.I;
  b.in.so = b.out.so = s.I * L1;
  b.fast_io = true;
  Pass pb;
  try {
    pb = plan_pass(b, flags);
  } catch (const Error& e) {
    if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
    return false;
  }
  Pass pc = make_swap_pass(s.dbl, s.I, L1, L2, s.O);
  pa.src = src;
  pa.dst = BUF_CHIRP;
  pb.src = BUF_CHIRP;
  pb.dst = BUF_CHIRP;
  pc.src = BUF_CHIRP;
  pc.dst = dst;
  out.push_back(std::move(pa));
  out.push_back(std::move(pb));
  out.push_back(std::move(pc));
  return true;
}

static size_t add_four_step(std::vector<Pass>& out, const PassSpec& s, int L1, int L2, int src, int dst) {
  Pass pa, pb;
  four_step_pair(s, L1, L2, &pa, &pb);
  pa.src = src;
  pa.dst = BUF_CHIRP;
  pb.src = BUF_CHIRP;
  pb.dst = dst;
  out.push_back(std::move(pa));
  out.push_back(std::move(pb));
  return (size_t)(s.I * s.O) * (size_t)s.L * (s.dbl ? 16 : 8);
}

// One pass, or a four-step pair, for a plain complex axis; no Bluestein.
// Returns the scratch bytes (BUF_CHIRP) the passes need.
static size_t add_direct_passes(std::vector<Pass>& out, const PassSpec& s, unsigned flags, int src, int dst) {
  try {
    Pass p = plan_pass(s, flags);
    p.src = src;
    p.dst = dst;
    out.push_back(std::move(p));
    return 0;
  } catch (const Error& e) {
    if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
  }
  int L1 = 0, L2 = 0;
  if (!plain_complex_axis(s) || !four_step_split(s.dbl, s.L, &L1, &L2))
    throw Error{DFFT_ERROR_UNSUPPORTED_SIZE,
                "length " + std::to_string(s.L) + " has no single-pass or four-step form"};
  return add_four_step(out, s, L1, L2, src, dst);
}

// ---------------------------------------------------------------------------
// Bluestein (chirp-z) for lengths no single pass or four-step pair handles.
//   X_k = w_k sum_n (x_n w_n) b_{k-n},  w_n = exp(s i pi n^2 / L),
//   b_m = conj(w_m), s = -1 (forward) or +1 (inverse);
// the convolution runs as FFT_M, a pointwise multiply by
// Bhat = FFT_M(B) / M (B the wrapped b), and an inverse FFT_M, with M the
// smallest 5-smooth length >= 2L-1.
// ---------------------------------------------------------------------------

static int smooth5_at_least(int n) {
  for (int m = n;; ++m) {
    int r = m;
    for (int p : {2, 3, 5})
      while (r % p == 0) r /= p;
    if (r == 1) return m;
  }
}

static std::shared_ptr<DevTable> upload(int dbl, const std::vector<long double>& re,
                                        const std::vector<long double>& im) {
  const size_t n = re.size(), esz = dbl ? 16 : 8;
  std::vector<unsigned char> host(esz * (n ? n : 1));
  for (size_t k = 0; k < n; ++k) {
    if (dbl) { double v[2] = {(double)re[k], (double)im[k]}; std::memcpy(&host[esz * k], v, esz); }
    else { float v[2] = {(float)re[k], (float)im[k]}; std::memcpy(&host[esz * k], v, esz); }
  }
  auto t = std::make_shared<DevTable>();
  cuda_check(cudaGetDevice(&t->device), "cudaGetDevice");
  t->bytes = host.size();
  cuda_check(cudaMalloc(&t->p, t->bytes), "cudaMalloc(bluestein)");
  cuda_check(cudaMemcpy(t->p, host.data(), t->bytes, cudaMemcpyHostToDevice), "cudaMemcpy(bluestein)");
  return t;
}

struct BluesteinTables {
  int M;
  std::shared_ptr<DevTable> chirp, bhat;
};

static BluesteinTables bluestein_tables(int dbl, int L, int sgn) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int>, std::pair<int, std::pair<std::weak_ptr<DevTable>,
                                                                           std::weak_ptr<DevTable>>>> cache;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  auto key = std::make_tuple(dev, dbl, L, sgn);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(key);
  if (it != cache.end()) {
    auto a = it->second.second.first.lock();
    auto b = it->second.second.second.lock();
    if (a && b) return BluesteinTables{it->second.first, a, b};
  }
  const int M = smooth5_at_least(2 * L - 1);
  const long double pi = acosl(-1.0L);
  // chirp w_n = exp(s i pi n^2 / L), n^2 reduced exactly modulo 2L
  std::vector<long double> wr(L), wi(L);
  for (int n = 0; n < L; ++n) {
    const long long m = ((long long)n * n) % (2LL * L);
    const long double a = pi * (long double)m / (long double)L;
    wr[n] = cosl(a);
    wi[n] = sgn * sinl(a);
  }
  // B (wrapped conj chirp), transformed in double precision on the device
  std::vector<double> B(2 * (size_t)M, 0.0);
  for (int m = 0; m < L; ++m) {
    B[2 * m] = (double)wr[m];
    B[2 * m + 1] = (double)-wi[m];
    if (m > 0) {
      B[2 * (M - m)] = (double)wr[m];
      B[2 * (M - m) + 1] = (double)-wi[m];
    }
  }
  void* dB = nullptr;
  void* dS = nullptr;
  cuda_check(cudaMalloc(&dB, B.size() * sizeof(double)), "cudaMalloc(bluestein B)");
  std::vector<double> F(B.size());
  try {
    cuda_check(cudaMemcpy(dB, B.data(), B.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    PassSpec ps;
    ps.dbl = 1;
    ps.L = M;
    ps.I = 1;
    ps.O = 1;
    ps.in.kind = ps.out.kind = IO_CPLX;
    ps.in.si = ps.out.si = 1;
    ps.in.so = ps.out.so = M;
    ps.in.sk = ps.out.sk = 1;
    ps.fast_io = true;
    std::vector<Pass> fp;
    const size_t sb = add_direct_passes(fp, ps, 0, BUF_IN, BUF_OUT);
    if (sb) cuda_check(cudaMalloc(&dS, sb), "cudaMalloc(bluestein filter scratch)");
    for (const Pass& q : fp) {
      void* bufs[4] = {dB, dB, nullptr, dS};
      cuda_check(launch_pass(q, static_cast<char*>(bufs[q.src]) + q.src_off,
                             static_cast<char*>(bufs[q.dst]) + q.dst_off, 0),
                 "bluestein filter FFT");
    }
    cuda_check(cudaMemcpy(F.data(), dB, F.size() * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
  } catch (...) {
    cudaFree(dB);
    if (dS) cudaFree(dS);
    throw;
  }
  cudaFree(dB);
  if (dS) cudaFree(dS);
  std::vector<long double> br(M), bi(M);
  for (int k = 0; k < M; ++k) {
    br[k] = (long double)F[2 * k] / M;
    bi[k] = (long double)F[2 * k + 1] / M;
  }
  BluesteinTables t{M, upload(dbl, wr, wi), upload(dbl, br, bi)};
  cache[key] = {M, {t.chirp, t.bhat}};
  return t;
}

size_t add_axis_passes(std::vector<Pass>& out, const PassSpec& s, unsigned flags, int src, int dst) {
  try {
    Pass p = plan_pass(s, flags);
    p.src = src;
    p.dst = dst;
    out.push_back(std::move(p));
    return 0;
  } catch (const Error& e) {
    if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
  }
  const int L = s.L;
  {
    long long ein = 0, eout = 0;
    int L1 = 0, L2 = 0;
    if (four_step_extents(s, &ein, &eout) && four_step_split(s.dbl, L, &L1, &L2) && L1 <= ein && L2 <= eout) {
      // plain complex sides: the three-pass form (strided pass on a factor
      // with a pipelined kernel, contiguous pass on its cofactor)
      int Lc = 0, Ls = 0;
      if (plain_complex_axis(s) && fast_split(s.dbl, L, &Lc, &Ls) &&
          add_four_step_fast(out, s, flags, Lc, Ls, src, dst))
        return (size_t)(s.I * s.O) * (size_t)L * (s.dbl ? 16 : 8);
      return add_four_step(out, s, L1, L2, src, dst);
    }
  }
  if (L > (1 << 23)) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "length too large for Bluestein"};
  // the outer direction is in the tables; the inner FFT_M pair is forward
  // then inverse
  BluesteinTables bt = bluestein_tables(s.dbl, L, s.inverse ? +1 : -1);
  const int M = bt.M;
  const size_t csz = s.dbl ? 16 : 8;
  PassSpec a = s;
  a.L = M;
  a.inverse = 0;
  a.scale = 1.0;
  a.fast_io = false;
  a.epi = false;
  a.variant = VARIANT_AUTO;
  a.C = 0;
  a.in.chirp = bt.chirp->p;
  a.in.chirp_n = L;
  a.out = IoAny{};
  a.out.kind = IO_CPLX;
  a.out.si = 1;
  a.out.so = s.I * M;
  a.out.sk = s.I;
  a.keep.push_back(bt.chirp);
  PassSpec b = s;
  b.L = M;
  b.inverse = 1;
  b.fast_io = false;
  b.epi = false;
  b.variant = VARIANT_AUTO;
  b.C = 0;
  b.in = IoAny{};
  b.in.kind = IO_CPLX;
  b.in.si = 1;
  b.in.so = s.I * M;
  b.in.sk = s.I;
  b.in.mul = bt.bhat->p;
  b.out.chirp = bt.chirp->p;
  b.out.chirp_n = L;
  b.keep.push_back(bt.chirp);
  b.keep.push_back(bt.bhat);
  const size_t scratch = (size_t)(s.I * s.O) * (size_t)M * csz;
  Pass pa, pb;
  try {
    pa = make_pass(a);
    pb = make_pass(b);
  } catch (const Error& e) {
    if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
    // FFT_M does not fit one CTA: each FFT_M as a four-step pair, through
    // two scratch halves: x * chirp -> S1 -> S2 (the spectrum),
    // S2 * Bhat -> S1 -> out * chirp.  The last pass's sub-axis index
    // k2 < M2 must stay below L (its column bases lie in the output).
    int M1 = 0, M2 = 0;
    // the sub-axis index of a column must stay inside the column's extent
    // on both sides (n1 < M1 rows of the input, k2 < M2 rows of the output)
    long long ein = 0, eout = 0;
    if (!four_step_extents(s, &ein, &eout) || !four_step_split(s.dbl, M, &M1, &M2) || M2 > eout || M1 > ein)
      throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "length " + std::to_string(L) + " is too long for Bluestein here"};
    Pass p[4];
    four_step_pair(a, M1, M2, &p[0], &p[1]);
    four_step_pair(b, M1, M2, &p[2], &p[3]);
    p[0].src = src;
    p[0].dst = BUF_CHIRP;
    p[1].src = BUF_CHIRP;
    p[1].dst = BUF_CHIRP;
    p[1].dst_off = scratch;
    p[2].src = BUF_CHIRP;
    p[2].src_off = scratch;
    p[2].dst = BUF_CHIRP;
    p[3].src = BUF_CHIRP;
    p[3].dst = dst;
    for (Pass& q : p) out.push_back(std::move(q));
    return 2 * scratch;
  }
  pa.src = src;
  pa.dst = BUF_CHIRP;
  pb.src = BUF_CHIRP;
  pb.dst = dst;
  out.push_back(std::move(pa));
  out.push_back(std::move(pb));
  return scratch;
}

}  // namespace dfft
