// Plans: a transform over a column-major 1-3-D array becomes a list of
// passes (one per transformed axis), executed in the order the reference's
// stage drivers use (src/fft.jl:650-776, src/fftgpu.jl:497-619).
#include <algorithm>
#include <cstring>
#include "dfft.h"
#include "dfft_plan.h"

namespace dfft {

namespace {

bool is_c2c(int t) { return t == DFFT_FFT || t == DFFT_IFFT || t == DFFT_FFT_INPLACE || t == DFFT_IFFT_INPLACE; }
bool is_inverse_c2c(int t) { return t == DFFT_IFFT || t == DFFT_IFFT_INPLACE; }
bool is_rfft(int t) { return t == DFFT_RFFT || t == DFFT_RFFT_INPLACE; }
bool is_irfft(int t) { return t == DFFT_IRFFT || t == DFFT_IRFFT_INPLACE; }

// Column split of axis a of a 3-D shape: I = product of the faster dims,
// O = product of the slower dims.
void split(const int64_t S[3], int a, long long* I, long long* O) {
  long long i = 1, o = 1;
  for (int k = 0; k < a; ++k) i *= S[k];
  for (int k = a + 1; k < 3; ++k) o *= S[k];
  *I = i;
  *O = o;
}

IoAny io(int kind, long long I, long long extent) {
  IoAny x{};
  x.kind = kind;
  x.si = 1;
  x.so = I * extent;
  x.sk = I;
  return x;
}

}  // namespace

Plan* build_plan(int ndim, const int64_t* shape, int precision, int transform, int ndims,
                 const int32_t* dims, const int32_t* r2r_kinds, int64_t irfft_len, int decomp,
                 int method, unsigned flags) {
  if (ndim < 1 || ndim > 3) throw Error{DFFT_ERROR_INVALID_VALUE, "ndim must be 1, 2 or 3"};
  if (!shape) throw Error{DFFT_ERROR_INVALID_VALUE, "shape is NULL"};
  if (precision != DFFT_F32 && precision != DFFT_F64)
    throw Error{DFFT_ERROR_INVALID_VALUE, "precision must be DFFT_F32 or DFFT_F64"};
  if (transform < DFFT_FFT || transform > DFFT_R2R)
    throw Error{DFFT_ERROR_UNKNOWN_TRANSFORM, "Unknown transform type"};
  if (decomp != DFFT_PENCIL && decomp != DFFT_SLAB)
    throw Error{DFFT_ERROR_INVALID_VALUE, "decomp must be DFFT_PENCIL or DFFT_SLAB"};
  if (method != DFFT_PLAIN && method != DFFT_MIXED)
    throw Error{DFFT_ERROR_INVALID_VALUE, "method must be DFFT_PLAIN or DFFT_MIXED"};
  if (ndims < 0 || ndims > ndim || (ndims > 0 && !dims))
    throw Error{DFFT_ERROR_INVALID_VALUE, "dims must list 0..ndim distinct axes"};
  std::vector<int> ax;
  for (int i = 0; i < ndims; ++i) {
    int a = dims[i] - 1;
    if (a < 0 || a >= ndim) throw Error{DFFT_ERROR_INVALID_VALUE, "dims entry out of range"};
    if (std::find(ax.begin(), ax.end(), a) != ax.end())
      throw Error{DFFT_ERROR_INVALID_VALUE, "dims entries must be distinct"};
    ax.push_back(a);
  }
  for (int i = 0; i < ndim; ++i)
    if (shape[i] < 1) throw Error{DFFT_ERROR_INVALID_VALUE, "shape entries must be >= 1"};

  std::unique_ptr<Plan> P(new Plan());
  P->ndim = ndim;
  P->precision = precision;
  P->transform = transform;
  P->decomp = decomp;
  P->method = method;
  P->flags = flags;
  P->dims = ax;
  cuda_check(cudaGetDevice(&P->device), "cudaGetDevice");
  const int dbl = precision == DFFT_F64 ? 1 : 0;
  const size_t rsz = dbl ? 8 : 4, csz = 2 * rsz;
  int64_t S[3] = {1, 1, 1};
  for (int i = 0; i < ndim; ++i) S[i] = shape[i];
  for (int i = 0; i < 3; ++i) { P->in_shape[i] = S[i]; P->out_shape[i] = S[i]; }
  for (int a : ax)
    if (S[a] > 0x7fffffffLL) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "axis too long"};

  // the mixed (tensor-core) form covers complex transforms; its passes run
  // the ComplexF32 axes of length 512, the other axes (and ComplexF64) keep
  // the plain form
  if (method == DFFT_MIXED && !is_c2c(transform))
    throw Error{DFFT_ERROR_INVALID_VALUE, "the mixed form covers complex (FFT / IFFT) transforms"};

  size_t chirp_bytes = 0;
  auto add = [&](const PassSpec& sp, int src, int dst) {
    size_t w = add_axis_passes(P->passes, sp, flags, src, dst);
    if (w > chirp_bytes) chirp_bytes = w;
  };
  // does a single pass handle FFT length L?  (otherwise Bluestein, and the
  // real transforms take their full-length form)
  auto single_ok = [&](int L, long long I, long long O) {
    PassSpec t;
    t.dbl = dbl;
    t.L = L;
    t.I = I;
    t.O = O;
    t.in.kind = t.out.kind = IO_CPLX;
    t.in.si = t.out.si = 1;
    t.in.so = t.out.so = I * L;
    t.in.sk = t.out.sk = I;
    t.variant = VARIANT_AUTO;
    try {
      make_pass(t);
      return true;
    } catch (const Error& e) {
      if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
      return false;
    }
  };

  if (is_c2c(transform)) {
    const bool inv = is_inverse_c2c(transform);
    P->in_elem = P->out_elem = csz;
    std::vector<int> order = ax;
    if (inv) std::reverse(order.begin(), order.end());  // ifft!: dims[3] first
    int src = BUF_IN;
    auto axis_spec = [&](int a) {
      PassSpec s;
      s.dbl = dbl;
      s.L = (int)S[a];
      split(S, a, &s.I, &s.O);
      s.inverse = inv ? 1 : 0;
      s.scale = inv ? 1.0 / (double)S[a] : 1.0;
      s.in = io(IO_CPLX, s.I, S[a]);
      s.out = io(IO_CPLX, s.I, S[a]);
      s.fast_io = true;
      return s;
    };
    for (size_t i = 0; i < order.size(); ++i) {
      const int a = order[i];
      if (method == DFFT_MIXED) {
        PassSpec s = axis_spec(a);
        if (mixed_supported(dbl, s.L, s.I)) {
          Pass m = make_mixed_pass(s.I, s.O, inv ? 1 : 0);
          m.src = src;
          m.dst = BUF_OUT;
          P->passes.push_back(std::move(m));
        } else {
          add(s, src, BUF_OUT);
        }
        src = BUF_OUT;
        continue;
      }
      // dims 1 and 2 adjacent in the stage order of an L x L x O array: one
      // fused 2-D pass per slab (src/fft.jl:735 transforms each slab along
      // dims (1, 2) before the exchange) when it beats the per-axis passes
      if (!(flags & DFFT_FLAG_NO_FUSE) && i + 1 < order.size() && a + order[i + 1] == 1 &&
          S[0] == S[1] && find_slab_kernel(dbl, (int)S[0])) {
        std::vector<Pass> pair;
        size_t w = add_axis_passes(pair, axis_spec(a), flags, src, BUF_OUT);
        w = std::max(w, add_axis_passes(pair, axis_spec(order[i + 1]), flags, BUF_OUT, BUF_OUT));
        const int v = choose_slab(dbl, (int)S[0], S[2], inv ? 1 : 0, pair, flags);
        if (v >= 0) {
          Pass f = make_slab_pass(dbl, (int)S[0], S[2], inv ? 1 : 0, v);
          f.src = src;
          f.dst = BUF_OUT;
          P->work_bytes = std::max(P->work_bytes, f.ctr_bytes);
          P->passes.push_back(std::move(f));
        } else {
          for (Pass& p : pair) P->passes.push_back(std::move(p));
          chirp_bytes = std::max(chirp_bytes, w);
        }
        src = BUF_OUT;
        ++i;
        continue;
      }
      add(axis_spec(a), src, BUF_OUT);
      src = BUF_OUT;
    }
  } else if (is_rfft(transform)) {
    if (ax.empty()) throw Error{DFFT_ERROR_INVALID_VALUE, "rfft needs at least one dim"};
    P->in_elem = rsz;
    P->out_elem = csz;
    const int a0 = ax[0];
    const int64_t n = S[a0];
    int64_t H[3] = {S[0], S[1], S[2]};
    H[a0] = n / 2 + 1;
    for (int i = 0; i < 3; ++i) P->out_shape[i] = H[i];
    PassSpec s;
    s.dbl = dbl;
    split(S, a0, &s.I, &s.O);
    if (n % 2 == 0 && single_ok((int)(n / 2), s.I, s.O)) {
      s.L = (int)(n / 2);
      s.in = io(IO_REAL_PAIR, s.I, n);
      s.out = io(IO_CPLX, s.I, H[a0]);
      s.epi = true;
    } else {
      // odd length (or a half length no single pass handles): the real
      // input as complex, full-length FFT, first n/2+1 outputs kept
      s.L = (int)n;
      s.in = io(IO_REAL, s.I, n);
      s.out = io(IO_TRUNC, s.I, H[a0]);
      s.out.n = (int)(n / 2);
    }
    add(s, BUF_IN, BUF_OUT);
    for (size_t i = 1; i < ax.size(); ++i) {
      const int a = ax[i];
      PassSpec c;
      c.dbl = dbl;
      c.L = (int)H[a];
      split(H, a, &c.I, &c.O);
      c.in = io(IO_CPLX, c.I, H[a]);
      c.out = io(IO_CPLX, c.I, H[a]);
      c.fast_io = true;
      add(c, BUF_OUT, BUF_OUT);
    }
  } else if (is_irfft(transform)) {
    if (ax.empty()) throw Error{DFFT_ERROR_INVALID_VALUE, "irfft needs at least one dim"};
    const int a0 = ax[0];
    const int64_t d = irfft_len;
    if (d < 1 || d / 2 + 1 != S[a0])
      throw Error{DFFT_ERROR_INVALID_VALUE,
                  "irfft: the real length d must satisfy d/2+1 == size(F, dims[1])"};
    P->in_elem = csz;
    P->out_elem = rsz;
    int64_t R[3] = {S[0], S[1], S[2]};
    R[a0] = d;
    for (int i = 0; i < 3; ++i) P->out_shape[i] = R[i];
    const bool destroy = (flags & DFFT_FLAG_DESTROY_INPUT) || transform == DFFT_IRFFT_INPLACE;
    int src = BUF_IN;
    const int work = destroy ? BUF_IN : BUF_WORK;
    // inverse C2C along dims[end..2] (reverse stage order), then C2R on dims[1]
    for (size_t i = ax.size(); i-- > 1;) {
      const int a = ax[i];
      PassSpec c;
      c.dbl = dbl;
      c.L = (int)S[a];
      split(S, a, &c.I, &c.O);
      c.inverse = 1;
      c.scale = 1.0 / (double)S[a];
      c.in = io(IO_CPLX, c.I, S[a]);
      c.out = io(IO_CPLX, c.I, S[a]);
      c.fast_io = true;
      add(c, src, work);
      src = work;
    }
    if (src == BUF_WORK) P->work_bytes = (size_t)(S[0] * S[1] * S[2]) * csz;
    PassSpec s;
    s.dbl = dbl;
    split(S, a0, &s.I, &s.O);
    s.inverse = 1;
    s.scale = 1.0 / (double)d;
    if (d % 2 == 0 && single_ok((int)(d / 2), s.I, s.O)) {
      s.L = (int)(d / 2);
      s.in = io(IO_HERM_PAIR, s.I, S[a0]);
      s.in.n = s.L;
      auto w = twiddle_table(dbl, d, 1, 0, (int)(d / 2) + 1, false);
      s.in.w = w->p;
      s.keep.push_back(w);
      s.out = io(IO_REAL_PAIR, s.I, d);
    } else {
      s.L = (int)d;
      s.in = io(IO_HERM_FULL, s.I, S[a0]);
      s.in.n = (int)d;
      s.out = io(IO_REAL, s.I, d);
    }
    add(s, src, BUF_OUT);
  } else {  // DFFT_R2R
    if (!r2r_kinds && !ax.empty()) throw Error{DFFT_ERROR_INVALID_VALUE, "r2r_kinds is NULL"};
    P->in_elem = P->out_elem = rsz;
    int src = BUF_IN;
    for (size_t i = 0; i < ax.size(); ++i) {
      const int a = ax[i];
      const int kind = r2r_kinds[i];
      const int64_t N = S[a];
      PassSpec s;
      s.dbl = dbl;
      split(S, a, &s.I, &s.O);
      s.in = io(IO_R2R, s.I, N);
      s.out = io(IO_R2R, s.I, N);
      s.in.r2r = s.out.r2r = kind;
      s.in.n = s.out.n = (int)N;
      std::shared_ptr<DevTable> win, wout;
      switch (kind) {
        case DFFT_REDFT10:
        case DFFT_RODFT10:
          s.L = (int)N;
          wout = twiddle_table(dbl, 4 * N, 1, 0, (int)N, false);
          break;
        case DFFT_REDFT01:
        case DFFT_RODFT01:
          s.L = (int)N;
          s.inverse = 1;
          win = twiddle_table(dbl, 4 * N, 1, 0, (int)N, true);
          break;
        case DFFT_REDFT11:
        case DFFT_RODFT11:
          s.L = (int)(2 * N);
          win = twiddle_table(dbl, 4 * N, 1, 0, (int)N, false);
          wout = twiddle_table(dbl, 8 * N, 2, 1, (int)N, false);
          break;
        case DFFT_REDFT00:
          if (N < 2) throw Error{DFFT_ERROR_INVALID_VALUE, "REDFT00 needs n >= 2"};
          s.L = (int)(2 * (N - 1));
          break;
        case DFFT_RODFT00:
          s.L = (int)(2 * (N + 1));
          break;
        case DFFT_DHT:
          s.L = (int)N;
          break;
        default:
          throw Error{DFFT_ERROR_UNKNOWN_TRANSFORM, "Unknown transform type"};
      }
      if (win) { s.in.w = win->p; s.keep.push_back(win); }
      if (wout) { s.out.w = wout->p; s.keep.push_back(wout); }
      add(s, src, BUF_OUT);
      src = BUF_OUT;
    }
  }
  P->chirp_bytes = chirp_bytes;
  if (!(flags & kFlagCallerWorkspace)) {
    if (chirp_bytes) cuda_check(cudaMalloc(&P->chirp, chirp_bytes), "cudaMalloc(bluestein scratch)");
    if (P->work_bytes) cuda_check(cudaMalloc(&P->work, P->work_bytes), "cudaMalloc(workspace)");
  }
  return P.release();
}

Plan* build_slab_split_plan(int precision, int inverse, int64_t L, int64_t nslab, int64_t zr, int nranks,
                            int split_dim, unsigned flags) {
  if (split_dim != 1 && split_dim != 2) throw Error{DFFT_ERROR_INVALID_VALUE, "split_dim must be 1 or 2"};
  if (precision != DFFT_F32 && precision != DFFT_F64)
    throw Error{DFFT_ERROR_INVALID_VALUE, "precision must be DFFT_F32 or DFFT_F64"};
  if (L < 1 || L > 0x7fffffffLL || nslab < 1 || zr < nslab || nranks < 1 || L % nranks != 0)
    throw Error{DFFT_ERROR_INVALID_VALUE, "slab split: need L % nranks == 0, 1 <= nslab <= zr"};
  const int dbl = precision == DFFT_F64 ? 1 : 0;
  const int64_t R = L / nranks;
  std::unique_ptr<Plan> P(new Plan());
  P->ndim = 3;
  P->precision = precision;
  P->transform = inverse ? DFFT_IFFT : DFFT_FFT;
  P->decomp = DFFT_SLAB;
  P->method = DFFT_PLAIN;
  P->flags = flags;
  P->dims = {0, 1};
  cuda_check(cudaGetDevice(&P->device), "cudaGetDevice");
  P->in_elem = P->out_elem = dbl ? 16 : 8;
  const int64_t plain[3] = {L, L, nslab};
  // the span of the rank blocks: rows (split_dim 2) or columns split
  const int64_t split[3] = {split_dim == 2 ? L : R, split_dim == 2 ? R : L, zr * (nranks - 1) + nslab};
  for (int i = 0; i < 3; ++i) {
    P->in_shape[i] = inverse ? split[i] : plain[i];
    P->out_shape[i] = inverse ? plain[i] : split[i];
  }
  const int rin = (int)(inverse ? R : L), rout = (int)(inverse ? L : R);
  bool made = false;
  std::string why = "no fused slab kernel for this length";
  for (int v = 0; const SlabKernel* k = find_slab_kernel(dbl, (int)L, v); ++v) {
    if (!k->dflt) continue;
    try {
      Pass p = make_slab_split_pass(dbl, (int)L, nslab, inverse, v, rin, rout, zr, split_dim);
      p.src = BUF_IN;
      p.dst = BUF_OUT;
      P->work_bytes = p.ctr_bytes;
      P->passes.push_back(std::move(p));
      made = true;
      break;
    } catch (const Error& e) {
      if (e.status != DFFT_ERROR_UNSUPPORTED_SIZE) throw;
      why = e.msg;
    }
  }
  if (!made) throw Error{DFFT_ERROR_UNSUPPORTED_SIZE, "slab split: " + why};
  if (!(flags & kFlagCallerWorkspace))
    cuda_check(cudaMalloc(&P->work, P->work_bytes), "cudaMalloc(workspace)");
  return P.release();
}

Plan::~Plan() {
  if (work || chirp) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    if (work) cudaFree(work);
    if (chirp) cudaFree(chirp);
    if (cur != device && cur >= 0) cudaSetDevice(cur);
  }
}

size_t Plan::in_bytes() const { return (size_t)(in_shape[0] * in_shape[1] * in_shape[2]) * in_elem; }
size_t Plan::out_bytes() const { return (size_t)(out_shape[0] * out_shape[1] * out_shape[2]) * out_elem; }

void execute_plan(const Plan* P, const void* in, void* out, cudaStream_t stream, void* work, void* chirp) {
  if (!in || !out) throw Error{DFFT_ERROR_INVALID_VALUE, "in/out is NULL"};
  if (!work) work = P->work;
  if (!chirp) chirp = P->chirp;
  if ((P->work_bytes && !work) || (P->chirp_bytes && !chirp))
    throw Error{DFFT_ERROR_INVALID_VALUE, "plan has no workspace and none was supplied"};
  int cur = -1;
  cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
  if (cur != P->device) cuda_check(cudaSetDevice(P->device), "cudaSetDevice");
  cudaError_t err = cudaSuccess;
  if (P->passes.empty()) {
    if (in != out) err = cudaMemcpyAsync(out, in, P->in_bytes(), cudaMemcpyDeviceToDevice, stream);
  }
  for (const Pass& p : P->passes) {
    if (err != cudaSuccess) break;
    void* bufs[4] = {const_cast<void*>(in), out, work, chirp};
    err = launch_pass(p, static_cast<char*>(bufs[p.src]) + p.src_off, static_cast<char*>(bufs[p.dst]) + p.dst_off,
                      stream, work);
  }
  if (cur != P->device) cudaSetDevice(cur);
  cuda_check(err, "kernel launch");
}

}  // namespace dfft
