// BATCHED schedule (multi-source BFS over bitmask frontiers). Placeholder
// until the batched kernels land: every entry point reports that the schedule
// is unavailable, so callers fail loudly instead of silently using another path.
#include "batched.h"

namespace bcg {

struct BatchedPlan {};

int batched_create(const bc_bccs *, const BatchedConfig &, const int64_t *, const int32_t *, const int32_t *,
                   const int64_t *, const int32_t *, const int32_t *, const int32_t *, const int32_t *, double *, int *,
                   cudaStream_t, BatchedPlan **, std::string *msg) {
  if (msg) *msg = "the BATCHED schedule is not available in this build";
  return BCGPU_EINVAL;
}
void batched_destroy(BatchedPlan *p) { delete p; }
int64_t batched_device_bytes(const BatchedPlan *) { return 0; }
int batched_width(const BatchedPlan *) { return 0; }
void batched_unit_work(const BatchedPlan *, std::vector<int64_t> &, std::vector<int64_t> &, std::vector<int64_t> &,
                       std::vector<int64_t> &, std::vector<int64_t> &) {}
int batched_run(BatchedPlan *, int64_t, int64_t, cudaStream_t, int *, std::string *msg) {
  if (msg) *msg = "the BATCHED schedule is not available in this build";
  return BCGPU_EINVAL;
}

}  // namespace bcg
