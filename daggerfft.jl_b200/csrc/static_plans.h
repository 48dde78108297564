// Table of the precompiled static-plan kernels (generated by gen_plans.py).
#pragma once
#include "tma_pass.cuh"

namespace dfft {

struct StaticPlan {
  int L;              // transform length
  int P;              // threads per column
  int nst;            // number of stages
  int radix[8];       // stage radices
  int lb;             // __launch_bounds__ of the kernels (max threads per CTA)
  const void* fast;   // axis_pass_static<T, true, ...>: complex in, complex out
  const void* any;    // axis_pass_static<T, false, ...>: any IoKind, R2C post-pass
  const void* pipe_s; // axis_pass_pipe<T, LB, false, ...>: strided C2C, TMA-pipelined (or null)
  const void* pipe_c; // axis_pass_pipe<T, LB, true, ...>: contiguous C2C, bulk-copy pipelined
  int pipe_lb;        // __launch_bounds__ of the pipelined kernels
  int pipe_cs;        // columns per tile compiled into the strided pipelined kernel
};

struct StaticPlanTable {
  const StaticPlan* plans;
  const int* count;
};

extern const StaticPlanTable kTable_f32[];
extern const StaticPlanTable kTable_f64[];
extern const int kTableParts;

}  // namespace dfft
