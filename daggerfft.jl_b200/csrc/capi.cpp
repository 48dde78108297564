// extern "C" entry points of libdfft: argument checks, exception -> status.
#include <new>
#include <cstdio>
#include <cstring>
#include <string>
#include "dfft.h"
#include "dfft_plan.h"

using dfft::Error;

namespace {

template <class F> int guarded(F&& f) {
  try {
    f();
    return DFFT_SUCCESS;
  } catch (const Error& e) {
    dfft::set_error(e.msg);
    return e.status;
  } catch (const std::bad_alloc&) {
    dfft::set_error("host allocation failed");
    return DFFT_ERROR_OUT_OF_MEMORY;
  } catch (...) {
    dfft::set_error("unexpected exception");
    return DFFT_ERROR_INVALID_VALUE;
  }
}

dfft::Plan* impl(dfft_plan p) {
  if (!p || !p->impl) throw Error{DFFT_ERROR_INVALID_VALUE, "plan is NULL"};
  return p->impl;
}

}  // namespace

extern "C" {

int dfft_plan_create(dfft_plan* plan, int ndim, const int64_t* shape, int precision, int transform,
                     int ndims, const int32_t* dims, const int32_t* r2r_kinds, int64_t irfft_len,
                     int decomp, int method, unsigned flags) {
  return guarded([&] {
    if (!plan) throw Error{DFFT_ERROR_INVALID_VALUE, "plan is NULL"};
    *plan = nullptr;
    dfft::Plan* p = dfft::build_plan(ndim, shape, precision, transform, ndims, dims, r2r_kinds,
                                     irfft_len, decomp, method, flags);
    *plan = new dfft_plan_s{p};
  });
}

int dfft_slab_split_create(dfft_plan* plan, int precision, int inverse, int64_t L, int64_t nslab, int64_t zr,
                           int nranks, int split_dim, unsigned flags) {
  return guarded([&] {
    if (!plan) throw Error{DFFT_ERROR_INVALID_VALUE, "plan is NULL"};
    *plan = nullptr;
    dfft::Plan* p = dfft::build_slab_split_plan(precision, inverse ? 1 : 0, L, nslab, zr, nranks, split_dim, flags);
    *plan = new dfft_plan_s{p};
  });
}

int dfft_plan_output_shape(dfft_plan plan, int64_t* shape) {
  return guarded([&] {
    dfft::Plan* p = impl(plan);
    if (!shape) throw Error{DFFT_ERROR_INVALID_VALUE, "shape is NULL"};
    for (int i = 0; i < p->ndim; ++i) shape[i] = p->out_shape[i];
  });
}

int dfft_plan_workspace_bytes(dfft_plan plan, size_t* bytes) {
  return guarded([&] {
    dfft::Plan* p = impl(plan);
    if (!bytes) throw Error{DFFT_ERROR_INVALID_VALUE, "bytes is NULL"};
    *bytes = p->work_bytes + p->chirp_bytes;
  });
}

int dfft_plan_launches(dfft_plan plan, int* launches) {
  return guarded([&] {
    dfft::Plan* p = impl(plan);
    if (!launches) throw Error{DFFT_ERROR_INVALID_VALUE, "launches is NULL"};
    *launches = (int)p->passes.size();
  });
}

int dfft_plan_describe(dfft_plan plan, char* buf, size_t len) {
  return guarded([&] {
    dfft::Plan* p = impl(plan);
    if (!buf || len == 0) throw Error{DFFT_ERROR_INVALID_VALUE, "buf is NULL or len is 0"};
    std::string out;
    for (const dfft::Pass& q : p->passes) {
      const char* kind = q.swap ? "axis-swap"
                         : q.mixed ? (q.mstrided ? "mixed-strided" : "mixed-contig")
                         : q.slab ? "slab-xy" : q.feed ? "strided-feed" : q.async_ ? "strided-async"
                         : q.real ? "real-pipe"
                         : q.tiled == 1 ? "tiled-contig" : q.tiled == 2 ? "tiled-strided"
                         : q.pipe ? (q.tma ? "strided-pipe" : "contig-pipe")
                         : q.is_static ? "direct" : "dynamic";
      std::string rad;
      for (int i = 0; i < q.d.nst; ++i) rad += (i ? "x" : "") + std::to_string(q.d.radix[i]);
      if (q.mixed) rad = "32x16(tcgen05 fp16 hi+lo)";
      char line[256];
      // the two passes of a four-step axis: twiddled store, then the split output
      const char* step = q.d.out.kind == dfft::IO_CPLX_TW || q.geom.tw_lo ? " four-step=1"
                         : q.d.out.o1 > 0 || q.swap ? " four-step=2" : "";
      std::snprintf(line, sizeof line, "%s L=%d I=%lld O=%lld grid=%u block=%u smem=%zu radices=%s%s\n", kind,
                    q.d.L, q.d.I, q.d.I > 0 ? q.d.Q / q.d.I : 0LL, q.grid.x, q.block.x, q.smem,
                    rad.empty() ? "-" : rad.c_str(), step);
      out += line;
    }
    const size_t n = out.size() < len - 1 ? out.size() : len - 1;
    std::memcpy(buf, out.data(), n);
    buf[n] = '\0';
  });
}

int dfft_execute(dfft_plan plan, const void* in, void* out, void* stream) {
  return guarded([&] {
    dfft::execute_plan(impl(plan), in, out, reinterpret_cast<cudaStream_t>(stream));
  });
}

int dfft_plan_destroy(dfft_plan plan) {
  return guarded([&] {
    if (!plan) return;
    delete plan->impl;
    delete plan;
  });
}

int dfft_device_error(int* code) {
  return guarded([&] {
    if (!code) throw Error{DFFT_ERROR_INVALID_VALUE, "code is NULL"};
    int* w = dfft::device_error_word();
    int v = 0;
    dfft::cuda_check(cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(error word)");
    dfft::cuda_check(cudaMemset(w, 0, sizeof(int)), "cudaMemset(error word)");
    *code = v;
  });
}

int dfft_wisdom_export(const char* path) {
  if (!path) { dfft::set_error("path is NULL"); return DFFT_ERROR_INVALID_VALUE; }
  int st = dfft::wisdom_export(path);
  if (st) dfft::set_error(std::string("cannot write wisdom file ") + path);
  return st;
}

int dfft_wisdom_import(const char* path) {
  if (!path) { dfft::set_error("path is NULL"); return DFFT_ERROR_INVALID_VALUE; }
  int st = dfft::wisdom_import(path);
  if (st) dfft::set_error(std::string("cannot read wisdom file ") + path);
  return st;
}

int dfft_wisdom_forget(void) {
  dfft::wisdom_forget();
  return DFFT_SUCCESS;
}

int dfft_wisdom_size(int* n) {
  if (!n) { dfft::set_error("n is NULL"); return DFFT_ERROR_INVALID_VALUE; }
  *n = dfft::wisdom_size();
  return DFFT_SUCCESS;
}

const char* dfft_last_error(void) { return dfft::last_error(); }

const char* dfft_status_string(int status) {
  switch (status) {
    case DFFT_SUCCESS: return "success";
    case DFFT_ERROR_INVALID_VALUE: return "invalid value";
    case DFFT_ERROR_UNKNOWN_TRANSFORM: return "Unknown transform type";
    case DFFT_ERROR_UNSUPPORTED_SIZE: return "unsupported size";
    case DFFT_ERROR_CUDA: return "CUDA error";
    case DFFT_ERROR_OUT_OF_MEMORY: return "out of memory";
    case DFFT_ERROR_NOT_READY: return "not ready";
    case DFFT_ERROR_TIMEOUT: return "timeout";
    case DFFT_ERROR_CANCELLED: return "cancelled";
    default: return "unknown status";
  }
}

const char* dfft_version(void) { return "0.1.0"; }

}  // extern "C"
