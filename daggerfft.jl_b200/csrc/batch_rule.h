// Branch count of a batch graph (no CUDA types: the rule is unit-tested on
// the host).
//
// A batch graph spreads its plans over k concurrent branches.  Enough
// branches fill the GPU with small grids; few enough keep the buffers of the
// transforms in flight resident in L2 between a transform's passes, each of
// which reads what the previous one wrote.  A plan in flight holds its input
// and its output, so the rule divides 0.8 x L2 by the mean per-plan
// (input + output) bytes and clamps the result to 2..max_branches (and to
// the number of plans).
//
// Worked case: 64 uneven ComplexF32 grids (edges 48..192) hold 96.07 M
// elements, 1.50 M per grid: 12.0 MB of input plus 12.0 MB of output, 24.0
// MB per plan.  With B200's L2 of about 126 MB (cudaDevAttrL2CacheSize)
// 0.8 x 126 MB / 24.0 MB = 4.2, so k = 4.  Measured
// on B200 with one graph launch: 1.08 / 0.96 / 0.94 / 0.96 / 1.05 / 1.22 ms
// with 2 / 3 / 4 / 5 / 6 / 8 branches.
#pragma once

namespace dfft {

inline int batch_branch_rule(int nplans, double total_inout_bytes, long long l2_bytes, int max_branches) {
  int k = max_branches;
  if (nplans > 0 && total_inout_bytes > 0 && l2_bytes > 0)
    k = (int)(0.8 * (double)l2_bytes / (total_inout_bytes / nplans));
  if (k < 2) k = 2;
  if (k > max_branches) k = max_branches;
  return k < nplans ? k : nplans;
}

}  // namespace dfft
