// Host-visible interface of the BATCHED schedule (kernels_batched.cu).
#pragma once
#include <cstdint>
#include <climits>
#include <functional>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "bcgpu.h"

namespace bcg {

struct BatchedConfig {
  int width = 0;            // sources per pass (multiple of 32); 0 = choose
  bool delta_fp32c = true;  // FP32 two-sum compensated dependencies (else FP64)
  int sms = 148;
  int64_t limit_bytes = 0;  // device bytes available to the plan's workspace
  int rescale_exp = 900;    // rescale a level's path counts above 2^rescale_exp
  unsigned long long wait_ns = 60ull * 1000 * 1000 * 1000;  // limit of one device-side wait
  cudaMemPool_t pool = nullptr;  // device memory from this pool, ordered on the plan's stream (null: cudaMalloc)
  const std::vector<char> *bccs_on = nullptr;  // BCCs this plan schedules (null: all)
  const std::vector<int32_t> *ecc0 = nullptr;  // per BCC: eccentricity of local vertex 0 if known (< 0: compute)
  // Passes (global index) whose slot, seed and arming tables are built; the
  // others keep their sizes and offsets but no sources, and must not be run.
  int64_t fill_begin = 0, fill_end = INT64_MAX;
  bool keep_host_tables = false;  // keep host copies of seeds and arming lists (batched_pass_digest)
  // Source order of BCC b (batched_source_order with at least the length the
  // filled passes need), computed by the caller (e.g. alongside its uploads);
  // empty: batched_create computes it.
  std::function<const std::vector<int32_t> &(int32_t b)> order_of;
};

// Sources per pass for a requested width (0: the default).
int batched_width(int requested);
// The source order of BCC b's passes, at least its first `need` entries (a
// prefix of the full order).
void batched_source_order(const bc_bccs *B, int32_t b, int width, int64_t need, std::vector<int32_t> &order);

struct BatchedPlan;

// Builds the passes (host scheduling) and allocates device workspace. The
// device pointers are owned by the caller and must outlive the plan.
int batched_create(const bc_bccs *B, const BatchedConfig &cfg, const int64_t *row, const int32_t *col,
                   const int32_t *reach, const int64_t *vtx_off, const int32_t *chain_start, const int32_t *chain_len,
                   const int32_t *chain_l, const int32_t *chain_r, double *bc, int *err, cudaStream_t stream,
                   BatchedPlan **out, std::string *msg);
void batched_destroy(BatchedPlan *p);
int64_t batched_device_bytes(const BatchedPlan *p);
// Digest of what pass `pass` runs from: its descriptor (less the table
// offsets), its slots, seeds and arming list (tests compare builds with it;
// the plan must have been built with keep_host_tables).
uint64_t batched_pass_digest(const BatchedPlan *p, int64_t pass);
// Bytes batched_create copied host -> device and read back (its row checks' flag);
// bytes batched_failed_batches reads back.
int64_t batched_h2d_bytes(const BatchedPlan *p);
int64_t batched_d2h_bytes(const BatchedPlan *p);
int64_t batched_status_bytes(const BatchedPlan *p);
int batched_width(const BatchedPlan *p);
// Packed ids of the own sources (own BFS + chain slots) of batches [begin, end).
void batched_unit_sources(const BatchedPlan *p, int64_t begin, int64_t end, std::vector<int64_t> &out);
// Prefix sums over passes of sources, TEPS arcs, BFS sources, aux BFS runs
// and vertex visits.
void batched_unit_work(const BatchedPlan *p, std::vector<int64_t> &sources, std::vector<int64_t> &teps,
                       std::vector<int64_t> &bfs, std::vector<int64_t> &aux, std::vector<int64_t> &visits);
// Levels and path counts (level bases applied) of the core vertices for
// every slot of pass `pass`, read from the workspace, which holds the pass
// the plan ran last: d[b * n_core + v], sigma likewise; src[b] = slot b's
// source (local id; a chain source at its own position). For parity tests.
// BCC and slot count of pass `pass`.
int batched_pass_shape(const BatchedPlan *p, int64_t pass, int32_t *bcc, int32_t *nslots);
int batched_pass_rows(const BatchedPlan *p, int64_t pass, const int32_t *chain_start, int32_t n_core,
                      cudaStream_t stream, std::vector<int32_t> &src, std::vector<int32_t> &d, std::vector<double> &sigma,
                      std::string *msg);
int batched_run(BatchedPlan *p, int64_t begin, int64_t end, cudaStream_t stream, int *launches, std::string *msg);
// Batches whose FP32 dependency values left FP32's exponent range (their
// contributions were withheld); synchronises the stream.
int batched_failed_batches(BatchedPlan *p, cudaStream_t stream, int64_t *count);

}  // namespace bcg
