// The persistent batch (batch_pass.cu): a work list of every axis pass of
// every transform of a batch, run by one kernel launch.
#pragma once
#include <memory>
#include <vector>
#include "dfft_internal.h"

namespace dfft {

struct Plan;
struct BatchPhase;

struct PersistentBatch {
  int dbl = 0;
  std::vector<BatchPhase> phases;      // host copy (buffers filled at execute)
  std::vector<int> phase_plan;         // transform of each phase
  std::vector<char> phase_first;       // the transform's first pass (reads its input)
  std::vector<std::shared_ptr<DevTable>> tables;
  std::vector<const void*> last_in;
  std::vector<void*> last_out;
  long long total = 0;
  size_t smem = 0, ctr_bytes = 0;
  unsigned grid = 0;
  const void* fn = nullptr;
  void* d_phases = nullptr;
  void* d_ctr = nullptr;
  int* err = nullptr;
  ~PersistentBatch();
};

// The persistent form of a batch, or null when some transform is not a
// complex transform of the kernel's lengths (the batch then replays a graph
// of the plans' own passes).  lag: transforms between a pass and the next
// pass of the same transform in the work list.
std::unique_ptr<PersistentBatch> make_persistent_batch(const std::vector<Plan*>& plans, int lag);

void launch_persistent_batch(PersistentBatch* B, const void* const* ins, void* const* outs, cudaStream_t s);

}  // namespace dfft
