// Host-visible interface of the small-BCC schedule (kernels_tile.cu): a CTA
// takes a range of sources of one BCC small enough for shared memory, stages
// the BCC's CSR slice there with one bulk copy, and each of its warps runs one
// source at a time (forward BFS + dependency sweep, FP64).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bcg {

// Sources [s0, s1) (local ids) of BCC bcc.
struct TileItem {
  int32_t bcc, s0, s1, pad;
};

constexpr int kTileWarps = 8;  // warps (sources in flight) per CTA

// Byte layout of one BCC's staged slice (all int32, each part starting on a
// 16-byte boundary): local row offsets [n+1], neighbours [arcs], reach [n].
struct TileSlice {
  __host__ __device__ static int64_t pad16(int64_t bytes) { return (bytes + 15) / 16 * 16; }
  __host__ __device__ static int64_t col_at(int64_t n) { return pad16(4 * (n + 1)); }
  __host__ __device__ static int64_t reach_at(int64_t n, int64_t arcs) { return col_at(n) + pad16(4 * arcs); }
  __host__ __device__ static int64_t bytes(int64_t n, int64_t arcs) { return reach_at(n, arcs) + pad16(4 * n); }
};

struct TileArgs {
  const int64_t *vtx_off;        // [n_bcc+1]
  const unsigned char *slices;   // staged slices, 16-byte aligned
  const int64_t *slice_off;      // [n_bcc] byte offset of BCC b's slice (-1: BCC not in this schedule)
  const int32_t *slice_bytes;    // [n_bcc] its size (TileSlice::bytes)
  const TileItem *items;
  int64_t item_begin, item_end;
  unsigned long long *next_item;  // zeroed before each launch
  unsigned long long *acc;        // [n_packed][kAccDigits] fixed-point BC counters (plain.h)
  int32_t *ws_S, *ws_lv;          // per warp slot: visit order, level offsets ([slots][cap])
  double *ws_sq;                  // per warp slot: path counts, then q ([slots][cap])
  int64_t cap;                    // per-slot row capacity (>= largest BCC of the schedule + 2)
  int32_t nmax;                   // largest BCC of the launch (shared-memory rows are sized for it)
  int32_t slice_max;              // largest slice in bytes
  unsigned long long wait_ns;     // limit of the wait for a staged slice
  int *err;
};

// Dynamic shared memory of a launch for BCCs of up to nmax vertices and
// slices of up to slice_max bytes.
size_t tile_smem_bytes(int64_t nmax, int64_t slice_max);
// Largest shared memory a CTA may use (opt-in limit of the device).
size_t tile_smem_limit(int device);
cudaError_t launch_tile(const TileArgs &a, int grid, size_t smem, cudaStream_t stream);
// CTAs of the schedule resident per SM at this shared-memory size.
int tile_ctas_per_sm(size_t smem);

}  // namespace bcg
