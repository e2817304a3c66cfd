// Shared device-side definitions for libbcgpu kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bcg {

// Device error codes written to a flag the host reads after each run.
enum DevErr : int {
  kDevOk = 0,
  kDevDisconnected = 1,  // a BCC row did not reach every vertex (malformed input)
  kDevWorkspace = 2,     // a BCC larger than the workspace the kernel was given
  kDevTimeout = 3,       // a bounded device-side wait gave up
  kDevBadItem = 4,       // a work item that references data out of range
};

__device__ __forceinline__ void set_err(int *err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// Read-only cached load (the CSR and per-vertex constants never change during a run).
template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// Deterministic warp sum (fixed butterfly order).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace bcg
