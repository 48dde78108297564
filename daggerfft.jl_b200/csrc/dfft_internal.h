// Host-side declarations shared by the planner, the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <memory>
#include <string>
#include <vector>
#include "async_pass.cuh"
#include "mixed_pass.cuh"

namespace dfft {

// Error reporting: every failing path records a message for dfft_last_error.
void set_error(const std::string& msg);
const char* last_error();

struct Error {
  int status;
  std::string msg;
};

// Throws Error{DFFT_ERROR_CUDA, ...} when e != cudaSuccess.
void cuda_check(cudaError_t e, const char* what);

// A device table owned by the table cache (shared between plans).
struct DevTable {
  void* p = nullptr;
  size_t bytes = 0;
  int device = -1;
  ~DevTable();
};

// Entries exp(-2 pi i (a*k + b) / D) for k = 0..count-1 (exp(+...) if conj),
// evaluated in long double and rounded to the plan precision.
std::shared_ptr<DevTable> twiddle_table(int dbl, long long D, long long a, long long b, int count,
                                        bool conj);

// One kernel launch of a plan.
enum BufId : int { BUF_IN = 0, BUF_OUT = 1, BUF_WORK = 2, BUF_CHIRP = 3 };

// Axis swap of the last four-step pass (transpose_pass.cu): element
// (i, a, b, o) of an I x A x B x O array moves to (i, b, a, o).
struct SwapGeom {
  long long I, A, B, O;
};
const void* swap_axes_kernel(int dbl, bool tiled);

struct Pass {
  PassDesc d{};
  const void* fn = nullptr;
  dim3 grid, block;
  size_t smem = 0;
  int src = BUF_IN, dst = BUF_OUT;
  size_t src_off = 0, dst_off = 0;  // byte offsets into those buffers
  bool is_static = false;
  // persistent pipelined pass (bulk copies); tma: strided, tensor
  // {I*xscale, L, O} of 8-byte elements
  bool pipe = false;
  bool tma = false;
  TmaGeom geom{};
  long long tI = 0, tL = 0, tO = 0;
  // fused 2-D slab pass (dims 1 and 2 of an L x L x O array): d is the
  // x-phase descriptor, d2 the y-phase one; tensor map as for tma with
  // {tI, tL, tO} = {L, L, O} over the output
  bool slab = false;
  bool feed = false;     // axis_pass_strided (tensor maps as for tma)
  StridedGeom fgeom{};
  bool real = false;     // real_pass (R2C / C2R along the contiguous axis)
  RealGeom rgeom{};
  int tiled = 0;         // tiled_pass: 1 contiguous, 2 strided (real tensor maps)
  int tdbl = 0;          // its precision (element type of the tensor maps)
  TiledGeom tgeom{};
  bool async_ = false;   // axis_pass_async (cp.async tiles, strides TMA cannot address)
  AsyncGeom ageom{};
  bool mixed = false;    // mixed_pass (tensor-core radix-32 x 16 stages, L = 512 ComplexF32)
  bool mstrided = false; // its strided variant (128-byte swizzled tensor maps {tI, tL, tO})
  MixedGeom mgeom{};
  size_t ctr_bytes = 0;  // job and per-slab counters (in the plan workspace)
  PassDesc d2{};
  SlabGeom sgeom{};
  // slab pass with the y-phase first and columns split by rank (kernel
  // MODE 2): the y-phase reads `in` through a map {tI2, tL2, tO2} and writes
  // the plain intermediate {L, L, nslab} (in `in` when cols_mid_in, else
  // in `out`), which the x-phase then reads
  bool swap = false;     // swap_axes_* (the last pass of a fast four-step axis)
  SwapGeom swg{};
  bool cols = false;
  bool cols_mid_in = false;
  long long tI2 = 0, tL2 = 0, tO2 = 0;
  std::vector<std::shared_ptr<DevTable>> tables;
};

// A launch shape of the fused slab kernel (slab_pass.cu): tile width x
// threads per pencil.  Variants of one (precision, L) are listed best-first
// for the untuned planner.
struct SlabKernel {
  int dbl, L, P, nst, radix[4];
  int lb;   // threads per CTA
  int cs;   // pencils / columns per tile
  int nb;   // tile buffers
  int dflt; // an untuned plan may pick this variant
  const void* fn;      // forward
  const void* fn_inv;  // inverse
  const void* fn_split;      // forward, rows split by rank
  const void* fn_inv_split;  // inverse, rows split by rank
  const void* fn_cols;       // forward, y-phase first, columns split by rank
  const void* fn_inv_cols;   // inverse, the same
};
// Variant `v` (0-based) for (dbl, L), or null past the last one.
const SlabKernel* find_slab_kernel(int dbl, int L, int v = 0);
// Launch shapes of axis_pass_strided for (dbl, L), same conventions.
const SlabKernel* find_strided_kernel(int dbl, int L, int v = 0);
// Launch shapes of axis_pass_async (async_pass.cu), same conventions.
const SlabKernel* find_async_kernel(int dbl, int L, int v = 0);
// real_pass kernels for half length M (fn: R2C, fn_inv: C2R), or null.
const SlabKernel* find_real_kernel(int dbl, int M);
// A compiled tiled_pass (tiled_pass.cu).
struct TiledKernel {
  int dbl, L, P, nst, radix[4];
  int lb;       // threads per CTA
  int cs;       // pencils / columns per tile
  int strided;  // 0 contiguous axis, 1 strided axis
  int kind;     // FFTW r2r kind (REDFT10 / REDFT01)
  const void* fn;
};
const TiledKernel* find_tiled_kernel(int dbl, int L, int strided, int kind);

// Fused forward or inverse 2-D C2C over dims 1 and 2 of an L x L x O array
// (scales: 1 forward, 1/L per axis inverse) with launch variant v; throws
// Error{DFFT_ERROR_UNSUPPORTED_SIZE} when that variant cannot serve the shape.
Pass make_slab_pass(int dbl, int L, long long O, int inverse, int v = 0);
// The same pass over nslab slabs with rank-split input (rin rows per rank)
// and/or output (rout rows per rank), zr slabs between one rank's blocks
// (SlabGeom); rin = rout = L is make_slab_pass.
// split_dim 2: rows (y) split, x-phase first (MODE 1); split_dim 1: columns
// (x) split, y-phase first (MODE 2; rin / rout count columns, and the
// forward pass overwrites its input with the intermediate).
Pass make_slab_split_pass(int dbl, int L, long long nslab, int inverse, int v, int rin, int rout,
                          long long zr, int split_dim = 2);

// Fused variant to use for dims (1, 2) of an L x L x O array, or -1 for the
// per-axis passes `split` (x then y, already planned): wisdom, then timing
// under DFFT_FLAG_TUNE, else the first default variant that builds (any
// variant under DFFT_FLAG_FUSE).
int choose_slab(int dbl, int L, long long O, int inverse, const std::vector<Pass>& split,
                unsigned flags);

// Mixed (tensor-core) form: does mixed_pass serve this axis (ComplexF32,
// L = 512, rows TMA can address), and the pass for it (one axis of Q = I*O
// pencils; inverse scales by 1/512).
bool mixed_supported(int dbl, int L, long long I);
Pass make_mixed_pass(long long I, long long O, int inverse);

// Device error word of the current device (bounded waits that expire set it).
int* device_error_word();

// VARIANT_FEED: strided C2C pass with a producer warp (axis_pass_strided);
// VARIANT_ASYNC: strided C2C pass copying tiles with cp.async
// (axis_pass_async); PassSpec::C then selects the launch shape (index into
// the kernel's table).
enum Variant : int { VARIANT_AUTO = 0, VARIANT_DIRECT = 1, VARIANT_PIPE = 2, VARIANT_DYNAMIC = 3,
                     VARIANT_FEED = 4, VARIANT_ASYNC = 5 };

// Pass construction.
struct PassSpec {
  int dbl = 0;
  int L = 1;                 // FFT length
  long long I = 1, O = 1;    // column split
  int inverse = 0;
  double scale = 1.0;
  IoAny in{}, out{};         // pointers filled at execute time
  bool epi = false;          // R2C half-length post-pass
  bool fast_io = false;      // plain complex in/out
  int variant = VARIANT_AUTO;
  int C = 0;                 // columns per CTA (0: heuristic)
  std::vector<std::shared_ptr<DevTable>> keep;  // tables the IoAny sides point into
};

// Appends the passes of one axis: a single pass, or the two passes of
// Bluestein's algorithm (via a scratch of Q*M complex elements) when no
// single-pass kernel handles the length.  Returns the scratch bytes needed.
size_t add_axis_passes(std::vector<Pass>& out, const PassSpec& s, unsigned flags, int src, int dst);

// Builds a launchable pass; throws Error on unsupported sizes.
Pass make_pass(const PassSpec& s);

// Planner entry: wisdom lookup, tuning (DFFT_FLAG_TUNE) or heuristics.
Pass plan_pass(const PassSpec& s, unsigned flags);
Pass tune_pass(const PassSpec& s);
int wisdom_export(const char* path);
int wisdom_import(const char* path);
void wisdom_forget();
int wisdom_size();

// Launches one pass on `stream` with the given buffers; `work` holds the
// counters of a fused slab pass (p.ctr_bytes, zeroed here before the launch).
cudaError_t launch_pass(const Pass& p, void* in, void* out, cudaStream_t stream, void* work = nullptr);

// Raise the dynamic shared-memory limit of a kernel on the current device.
cudaError_t ensure_smem_attr(const void* fn, size_t bytes);

const void* dynamic_kernel(int dbl);

}  // namespace dfft
