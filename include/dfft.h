/*
 * dfft.h -- C ABI of libdfft, the B200 (sm_100a) transform hot path of
 * DaggerFFT.jl.
 *
 * Conventions shared by every entry point
 *   - Arrays are column-major (Julia order): dim 1 is contiguous.  Shapes
 *     are given as int64_t[ndim] in that order, ndim in 1..3.
 *   - dims are 1-based axis numbers, as in Julia.
 *   - Complex data is interleaved (re, im): ComplexF32 = 2 x float,
 *     ComplexF64 = 2 x double.
 *   - All device pointers are caller-owned CUDA device memory on the device
 *     that was current when the plan was created.  The library owns plans,
 *     twiddle tables and workspaces; they stay resident until destroyed.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *     Work is enqueued asynchronously; no call synchronises the stream
 *     unless documented.
 *   - Every call returns a dfft_status; 0 is success.  dfft_last_error()
 *     returns a thread-local message describing the last failure.
 *   - Numerical conventions follow AbstractFFTs/FFTW: forward sign -1,
 *     unnormalised; inverse transforms scale by 1/prod(n_i); rfft halves the
 *     FIRST transformed dim to n/2+1; irfft needs the real length d; r2r
 *     kinds are FFTW's and unnormalised.
 *   - Threading: a plan may be used by one stream at a time; distinct plans
 *     may be used concurrently from any thread.
 */
#ifndef DFFT_H
#define DFFT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DFFT_API __attribute__((visibility("default")))
#else
#define DFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef enum {
  DFFT_SUCCESS = 0,
  DFFT_ERROR_INVALID_VALUE = 1,      /* null pointer, bad rank/dims/shape     */
  DFFT_ERROR_UNKNOWN_TRANSFORM = 2,  /* reference: ArgumentError("Unknown transform type") */
  DFFT_ERROR_UNSUPPORTED_SIZE = 3,   /* a length this build cannot transform  */
  DFFT_ERROR_CUDA = 4,               /* a CUDA runtime call failed            */
  DFFT_ERROR_OUT_OF_MEMORY = 5,      /* device allocation failed / over budget */
  DFFT_ERROR_NOT_READY = 6,          /* serving: no completed request yet     */
  DFFT_ERROR_TIMEOUT = 7,            /* a bounded wait gave up                */
  DFFT_ERROR_CANCELLED = 8           /* serving: request cancelled            */
} dfft_status;

/* ---- transform tags (src/fft.jl:17-24) -------------------------------- */
typedef enum {
  DFFT_FFT = 0,          /* FFT    : out-of-place complex forward           */
  DFFT_IFFT = 1,         /* IFFT   : out-of-place complex inverse (1/N)      */
  DFFT_RFFT = 2,         /* RFFT   : real -> half complex                     */
  DFFT_IRFFT = 3,        /* IRFFT  : half complex -> real, needs real length  */
  DFFT_FFT_INPLACE = 4,  /* FFT!                                             */
  DFFT_IFFT_INPLACE = 5, /* IFFT!                                            */
  DFFT_RFFT_INPLACE = 6, /* RFFT!  (separate output buffer, input preserved)  */
  DFFT_IRFFT_INPLACE = 7,/* IRFFT! (input may be overwritten as workspace)    */
  DFFT_R2R = 8           /* R2R((kind,...)) README.md:58-67                   */
} dfft_transform;

/* element precision of the real or complex data */
typedef enum { DFFT_F32 = 0, DFFT_F64 = 1 } dfft_precision;

/* decomposition tags (src/fft.jl:13-15) */
typedef enum { DFFT_PENCIL = 0, DFFT_SLAB = 1 } dfft_decomp;

/* arithmetic form: PLAIN = FP32/FP64 CUDA-core Stockham; MIXED = ComplexF32
 * axes of length 512 as radix-32 x radix-16 complex matrix products on the
 * tensor cores (tcgen05, FP16 hi+lo split operands, FP32 accumulation,
 * per-pencil power-of-two scaling; relative L2 error ~3e-7 per 3-D
 * transform); other axes, ComplexF64 and FFT/IFFT of other lengths run the
 * plain form; real and r2r transforms return DFFT_ERROR_INVALID_VALUE */
typedef enum { DFFT_PLAIN = 0, DFFT_MIXED = 1 } dfft_method;

/* FFTW r2r kinds (fftw_r2r_kind values; src/fft.jl:1-11) */
enum {
  DFFT_R2HC = 0, DFFT_HC2R = 1, DFFT_DHT = 2,
  DFFT_REDFT00 = 3, DFFT_REDFT01 = 4, DFFT_REDFT10 = 5, DFFT_REDFT11 = 6,
  DFFT_RODFT00 = 7, DFFT_RODFT01 = 8, DFFT_RODFT10 = 9, DFFT_RODFT11 = 10
};

/* plan flags */
enum {
  DFFT_FLAG_DESTROY_INPUT = 1u << 0, /* C2R may use its input as workspace   */
  DFFT_FLAG_TUNE = 1u << 1,          /* time launch candidates at creation   */
  DFFT_FLAG_NO_WISDOM = 1u << 2,     /* ignore the tuning cache              */
  DFFT_FLAG_NO_FUSE = 1u << 3,       /* one pass per axis: no fused 2-D slab
                                        pass over dims (1, 2)                */
  DFFT_FLAG_FUSE = 1u << 4           /* use the fused slab pass wherever a
                                        kernel exists (no timing)            */
};

typedef struct dfft_plan_s* dfft_plan;

/*
 * Plan creation.  Replaces the reference's plan layer:
 *   plan_transform / get_or_create_plan   (src/fft.jl:126-166)
 *   gpu_plan_transform / get_or_create_gpu_plan (src/fft.jl: n/a,
 *   src/fftgpu.jl:85-116)
 * shape      : INPUT array shape, column-major, ndim in 1..3.  For IRFFT this
 *              is the half-complex input shape (dims[0] extent d/2+1).
 * ndims,dims : the transformed axes, 1-based, in the order the stages run
 *              (Pencil: one stage per entry; Slab: dims[0],dims[1] form the
 *              2-D slab stage).  Any subset of {1..ndim}.
 * r2r_kinds  : DFFT_R2R only, one FFTW kind per entry of dims.
 * irfft_len  : DFFT_IRFFT(_INPLACE) only: the real length d along dims[0].
 * Unknown `transform` values return DFFT_ERROR_UNKNOWN_TRANSFORM with the
 * message "Unknown transform type" (src/fft.jl:142, src/fftgpu.jl:103).
 */
DFFT_API int dfft_plan_create(dfft_plan* plan, int ndim, const int64_t* shape, int precision,
                     int transform, int ndims, const int32_t* dims, const int32_t* r2r_kinds,
                     int64_t irfft_len, int decomp, int method, unsigned flags);

/*
 * Slab stage of a distributed Slab transform with the exchange's pack and
 * unpack folded into it.  Replaces, for Slab with L % nranks == 0, the
 * separate pack / unpack kernels around the exchange
 * (src/fftgpu.jl:324-415 gpu_flat_redistribute!, :417-480 pack_kernel! /
 * unpack_kernel!) next to the 2-D slab stage (src/fftgpu.jl:534-557 and
 * :596-619).  The plan runs the fused dims-(1, 2) pass over `nslab` L x L
 * slabs, one side in a RANK-SPLIT layout with R = L / nranks:
 *   split_dim = 1 (columns: the reference's Slab layouts, A = Blocks(L, L,
 *     c), B = Blocks(L/P, L, N3)): element (x, y, z) of the local slabs at
 *     (x mod R) + R * (y + L * (z + zr * (x / R))), so rank s = x / R gets
 *     one contiguous (R, L, zr) block -- on arrival exactly its (R, L, N3)
 *     chunk's z-range of the sender.  The y-phase runs first; the FORWARD
 *     overwrites its input with the intermediate (as the reference's
 *     in-place slab stage overwrites A).  R must be a power of two.
 *   split_dim = 2 (rows, B = Blocks(L, L/P, N3)): row y of slab z (L
 *     contiguous elements) at row (y mod R) + R * (z + zr * (y / R)).
 * Forward (inverse = 0): plain L x L x nslab input, split output (block s
 * is what this rank sends to rank s).  Inverse (inverse = 1): split input
 * (the received blocks), plain output.  zr >= nslab is the stride between
 * rank blocks in slabs: running slab groups z0.. of one local array means
 * offsetting the plain side by z0 * L * L and the split side by
 * z0 * R * L elements with the same zr.  Execute with dfft_execute.
 */
DFFT_API int dfft_slab_split_create(dfft_plan* plan, int precision, int inverse, int64_t L, int64_t nslab,
                                    int64_t zr, int nranks, int split_dim, unsigned flags);

/* Output shape (column-major, ndim entries) of a plan. */
DFFT_API int dfft_plan_output_shape(dfft_plan plan, int64_t* shape);

/* Device workspace the plan holds (bytes, twiddles excluded). */
DFFT_API int dfft_plan_workspace_bytes(dfft_plan plan, size_t* bytes);

/* Number of kernel launches one dfft_execute makes. */
DFFT_API int dfft_plan_launches(dfft_plan plan, int* launches);

/* One line per kernel launch of the plan ("<kernel> L=.. I=.. O=.. grid=..
 * block=.. smem=.. radices=AxBx.."), NUL-terminated and truncated to len-1 characters
 * (the analogue of fftw_sprint_plan; for logs and tests). */
DFFT_API int dfft_plan_describe(dfft_plan plan, char* buf, size_t len);

/*
 * Execute: out = T(in).  Replaces apply_fft! / apply_gpu_fft!
 * (`mul!(out, plan, in)`, src/fft.jl:168-174, src/fftgpu.jl:118-124) and
 * the per-stage drivers fft!/ifft!/gpu_fft!/gpu_ifft! on one GPU
 * (src/fft.jl:650-776, src/fftgpu.jl:497-619): every stage and the
 * redistribution between stages run as strided tile passes inside HBM.
 * in == out is allowed for C2C and R2R (in-place).
 */
DFFT_API int dfft_execute(dfft_plan plan, const void* in, void* out, void* stream);

/* Release a plan (gpu_cleanup_workspace!, src/fftgpu.jl:630-634). */
DFFT_API int dfft_plan_destroy(dfft_plan plan);

/*
 * Reads and clears the device error word of the current device.  Kernels
 * whose bounded waits expire (TMA tile pipeline) record a non-zero code there
 * instead of hanging or faulting: 1 = a tile load or a dependency did not
 * complete in time, 2 = a tile buffer was not aligned for the bulk copies
 * (nothing was issued), 3 = a batch work item of a length the persistent
 * kernel does not run (nothing was computed for it).  Synchronises the
 * device.
 */
DFFT_API int dfft_device_error(int* code);

/*
 * Tuning cache ("wisdom"; the reference imports FFTW wisdom at load and
 * exports it after each new plan, src/fft.jl:113-124,162).  Plans created
 * with DFFT_FLAG_TUNE time every launch candidate of each pass and record
 * the fastest; later plans of the same pass shape reuse it.  The file format
 * is text, one pass per line, keyed by the GPU model.
 */
DFFT_API int dfft_wisdom_export(const char* path);
DFFT_API int dfft_wisdom_import(const char* path);
DFFT_API int dfft_wisdom_forget(void);
DFFT_API int dfft_wisdom_size(int* n);

/* ---- batches of uneven transforms -----------------------------------
 *
 * No counterpart in the reference (an addition beyond its API): N independent
 * plans (any shapes/kinds) executed together.  By default the first execute
 * with a set of buffers captures every plan's passes as concurrent branches
 * of a CUDA graph (the branch count keeps the transforms in flight within
 * L2); later executes with the same buffers replay the graph, new buffers
 * update it.  With DFFT_BATCH_PERSISTENT, a batch whose plans are all
 * complex transforms (FFT / IFFT, one precision) of axis lengths the
 * persistent batch kernel runs (16, 24, 32, 40, 48, 60, 64, 72, 80, 96,
 * 100, 120, 128, 144, 160, 192, 256) is instead ONE kernel launch over a
 * work list of every axis pass of every transform (a pass waits, bounded,
 * for its predecessor; bits 8-15 of the flags give the stagger `lag`
 * between a pass and its predecessor in the list, 0 = automatic); other
 * batches keep the graph.  The graph is the faster form on B200 for the
 * shapes measured here; the persistent form is kept for callers that need
 * a single launch.  Plans must outlive the batch and live on the current
 * device.  dfft_batch_launches reports which: 1 for the persistent kernel,
 * else the graph's kernel count.
 */
typedef struct dfft_batch_s* dfft_batch;
enum {
  DFFT_BATCH_GRAPH = 1u << 0,      /* the graph of the plans' own passes (the default) */
  DFFT_BATCH_PERSISTENT = 1u << 1  /* one persistent-kernel launch where eligible */
};
DFFT_API int dfft_batch_create(dfft_batch* batch, int nplans, const dfft_plan* plans);
/* The same with flags (DFFT_BATCH_GRAPH / DFFT_BATCH_PERSISTENT | lag << 8). */
DFFT_API int dfft_batch_create_ex(dfft_batch* batch, int nplans, const dfft_plan* plans, unsigned flags);
DFFT_API int dfft_batch_execute(dfft_batch batch, const void* const* ins, void* const* outs,
                                void* stream);
DFFT_API int dfft_batch_launches(dfft_batch batch, int* launches);
DFFT_API int dfft_batch_destroy(dfft_batch batch);

/* ---- serving: continuous batching of transform requests --------------
 *
 * No counterpart in the reference (an addition beyond its API).  A server owns an
 * HBM arena of `hbm_budget_bytes` (allocated once) and `slots` execution
 * streams.  Requests are admitted in arrival order while a slot is free and
 * their staging memory (host input copied in, host or server-held output)
 * fits the arena; admitted requests run concurrently on their own streams
 * and new ones join as slots and memory free up.  Plans and twiddles stay
 * resident per shape (one plan serves concurrent requests); a request's
 * plan workspace, if any, is taken from the arena with its staging memory.  Every request must be released
 * (dfft_server_release) after it finishes.
 */
enum { DFFT_MEM_DEVICE = 0, DFFT_MEM_HOST = 1, DFFT_MEM_SERVER = 2 };

typedef struct {
  int transform;          /* DFFT_FFT, DFFT_IFFT, DFFT_RFFT, DFFT_IRFFT, DFFT_R2R ... */
  int precision;          /* DFFT_F32 / DFFT_F64 */
  int decomp;             /* DFFT_PENCIL / DFFT_SLAB */
  int ndim;
  int64_t shape[3];       /* input shape, column-major */
  int ndims;
  int32_t dims[3];        /* 1-based */
  int32_t r2r_kinds[3];
  int64_t irfft_len;
  const void* in;
  int in_location;        /* DFFT_MEM_DEVICE or DFFT_MEM_HOST (pinned for overlap) */
  void* out;              /* ignored for DFFT_MEM_SERVER */
  int out_location;       /* DFFT_MEM_DEVICE, DFFT_MEM_HOST or DFFT_MEM_SERVER */
} dfft_request;

typedef struct {
  uint64_t completed, rejected, cancelled, failed, queued;
  double p50_ms, p99_ms, max_ms;   /* submit -> completion latency */
  double bytes_moved;              /* input + output bytes of completed requests */
  double elapsed_s;                /* since creation or the last reset */
  size_t arena_bytes, arena_peak_bytes;
  int peak_running;                /* most requests on the GPU at once */
  int resident_plans;
} dfft_server_stats;

typedef struct dfft_server_s* dfft_server;

DFFT_API int dfft_server_create(dfft_server* server, size_t hbm_budget_bytes, int slots, unsigned flags);
DFFT_API int dfft_server_submit(dfft_server server, const dfft_request* req, uint64_t* id);
/* ids of finished (completed, failed or cancelled) requests, oldest first */
DFFT_API int dfft_server_poll(dfft_server server, uint64_t* ids, int max, int* n);
/* bounded wait for one request; status = its result (DFFT_ERROR_TIMEOUT if not done) */
DFFT_API int dfft_server_wait(dfft_server server, uint64_t id, int timeout_ms, int* status);
/* copy a server-held result out (DFFT_MEM_HOST or DFFT_MEM_DEVICE destination) */
DFFT_API int dfft_server_fetch(dfft_server server, uint64_t id, void* dst, int dst_location, void* stream);
DFFT_API int dfft_server_result_pointer(dfft_server server, uint64_t id, void** ptr);
DFFT_API int dfft_server_release(dfft_server server, uint64_t id);
/* cancel a request that has not been admitted yet */
DFFT_API int dfft_server_cancel(dfft_server server, uint64_t id);
DFFT_API int dfft_server_get_stats(dfft_server server, dfft_server_stats* stats);
DFFT_API int dfft_server_reset_stats(dfft_server server);
DFFT_API int dfft_server_destroy(dfft_server server);

/* ---- redistribution between blockings --------------------------------
 *
 * One sub-block copy: `count` elements per dim from chunk `src` (column-major
 * extents src_dims) starting at src_start (0-based) to chunk `dst` at
 * dst_start.  A flat pack/unpack buffer is a chunk whose extents equal
 * `count` (x fastest, as pack_data!/unpack_data! lay it out,
 * src/fft.jl:180-214).  Replaces the per-pattern launches of
 * local_copy_kernel!, pack_kernel! and unpack_kernel!
 * (src/fftgpu.jl:367-385, 417-495).
 */
typedef struct {
  const void* src;
  void* dst;
  int64_t src_start[3];
  int64_t dst_start[3];
  int64_t src_dims[3];
  int64_t dst_dims[3];
  int64_t count[3];
} dfft_block_copy;

typedef struct dfft_copy_plan_s* dfft_copy_plan;

/* A device-resident list of block copies executed by one launch (the
 * pattern list of create_gpu_workspace, src/fftgpu.jl:126-318). */
DFFT_API int dfft_copy_plan_create(dfft_copy_plan* plan, const dfft_block_copy* blocks, int nblocks,
                                   int elem_bytes);
/* Runs every copy of the plan (the LOCAL_COPIES / PACK_SEND / RECV_UNPACK
 * phases of gpu_flat_redistribute!, src/fftgpu.jl:324-415). */
DFFT_API int dfft_copy_plan_execute(dfft_copy_plan plan, void* stream);
DFFT_API int dfft_copy_plan_bytes(dfft_copy_plan plan, int64_t* bytes);
DFFT_API int dfft_copy_plan_destroy(dfft_copy_plan plan);

/*
 * irfft of a ComplexF32 half-spectrum over all dims (dims = 1..ndim, real
 * length shape[0] along dim 1) that allocates no device memory.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc when they transform (code inside another framework's memory
 * pool, or held to a fixed HBM budget).  The intermediate lives in a static
 * device array of 2^21 ComplexF32 (16 MiB) that every GPU loading the
 * library keeps until exit; larger sizes return DFFT_ERROR_INVALID_VALUE.
 * Calls that overlap on the GPU race on that array.  The first call on a
 * device looks up the array's address, which (CUDA loads modules lazily) is
 * also when the library's device code and the 16 MiB array are loaded on that
 * device: make one small call (ndim = 1 will do) at start-up, before the
 * caller's pool has grown to fill the GPU and before any stream capture.
 * Every length is checked before anything is launched (13-smooth, at most 16
 * radix stages, one CTA per pencil); rejected lengths return
 * DFFT_ERROR_UNSUPPORTED_SIZE and leave the stream untouched.
 * in: (shape[0]/2+1, shape[1], shape[2]) ComplexF32, out: shape Float32,
 * both column-major device memory.
 */
DFFT_API int dfft_irfft_noalloc_f32(const void* in, void* out, int ndim, const int64_t* shape,
                                    void* stream);

/* Thread-local description of the last error. */
DFFT_API const char* dfft_last_error(void);
DFFT_API const char* dfft_status_string(int status);

/* Library version, e.g. "0.1.0". */
DFFT_API const char* dfft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DFFT_H */
