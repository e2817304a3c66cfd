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
  kDevOverflow = 5,      // a path count or dependency left FP64's range despite per-level scaling,
                         // or a BC contribution beyond the fixed-point accumulator's range
};

__device__ __forceinline__ void set_err(int *err, int code) {
  if (err) atomicCAS(err, 0, code);
}

// Device wall clock in nanoseconds (%globaltimer).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// The one bounded wait of the library's kernels: spins while *word == seen.
// Returns true once the word changes; false when stop() turns true (another
// CTA flagged an error) or when limit_ns of device time have passed, in which
// case kDevTimeout is recorded in err. No trap, no unbounded loop.
template <class Stop>
__device__ __forceinline__ bool wait_while_equal(const volatile unsigned int *word, unsigned int seen,
                                                 unsigned long long limit_ns, int *err, Stop stop) {
  const unsigned long long t0 = global_ns();
  while (*word == seen) {
    if (stop()) return false;
    if (global_ns() - t0 > limit_ns) {
      set_err(err, kDevTimeout);
      return false;
    }
    __nanosleep(128);
  }
  return true;
}

// wait_while_equal on a word expected to stay 0, with nothing else to stop it
// (bc_wait_probe's kernel).
__device__ __forceinline__ void wait_while_equal_probe(const unsigned int *word, int *err, unsigned long long limit_ns) {
  wait_while_equal(word, 0u, limit_ns, err, [] { return false; });
}

// Default limit of a device-side wait (bc_opts.wait_limit_ms = 0).
constexpr unsigned long long kDefaultWaitNs = 60ull * 1000 * 1000 * 1000;

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
