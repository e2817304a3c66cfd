// Host-visible interface of the small-BCC schedule (kernels_tile.cu): a CTA
// takes a range of sources of one BCC small enough for shared memory, stages
// the BCC's CSR slice there with one bulk copy, and keeps every per-source
// array in shared memory too. Two classes:
//   kTileWarp  one warp per source (eight sources in flight per CTA), for the
//              smallest BCCs;
//   kTileCta   the whole CTA on one source at a time, for BCCs up to several
//              thousand vertices.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace bcg {

// Sources [s0, s1) (local ids) of BCC bcc.
struct TileItem {
  int32_t bcc, s0, s1, pad;
};

// kTileCta512 / kTileCta1024: the CTA class with 512 / 1024 threads, for the
// BCCs whose shared memory allows only two / one CTA per SM (more lanes on
// each level and more warps per SM than two or one 256-thread CTAs).
// kTileCta1024x2 / kTileCta1024x4: 1024 threads in two groups of 512 / four
// of 256, each group on its own source with its own arrays, every group on
// the one staged slice: two / four sources in flight per SM for BCCs whose
// single-source CTA fits only once or twice per SM.
enum TileClass : int { kTileWarp = 0, kTileCta = 1, kTileCta512 = 2, kTileCta1024 = 3, kTileCta1024x2 = 4,
                       kTileCta1024x4 = 5 };
constexpr int kTileWarps = 8;          // warps per CTA
constexpr int kTileMaxLevels = 1024;   // BFS levels the CTA class records (routing keeps BCCs below)
constexpr int kTileGroupMaxLevels = 256;  // the same for the grouped classes
constexpr int kGroupLongQueue = 256;      // long-row queue of a group in the grouped classes
constexpr int32_t kTileMaxVertices = 65535;  // neighbour ids are 16-bit in the slice

// Byte layout of one BCC's staged slice, each part starting on a 16-byte
// boundary: local row offsets [n+1] -- uint16 when the BCC has fewer than
// 2^16 arcs ("narrow", 2 bytes per vertex less in shared memory), else
// int32 -- then neighbours uint16 [arcs]. A slice's offset in the slice
// buffer is a multiple of 16; bit 0 of the offset recorded for the kernels
// (TileArgs::slice_off) marks a narrow slice.
struct TileSlice {
  __host__ __device__ static int64_t pad16(int64_t bytes) { return (bytes + 15) / 16 * 16; }
  __host__ __device__ static bool narrow(int64_t arcs) { return arcs < 65536; }
  __host__ __device__ static int64_t col_at(int64_t n, bool narrow) { return pad16((narrow ? 2 : 4) * (n + 1)); }
  __host__ __device__ static int64_t bytes(int64_t n, int64_t arcs) {
    return col_at(n, narrow(arcs)) + pad16(2 * arcs);
  }
};

struct TileArgs {
  const int64_t *vtx_off;        // [n_bcc+1]
  const int32_t *reach;          // [n_packed]
  const unsigned char *slices;   // staged slices, 16-byte aligned
  const int64_t *slice_off;      // [n_bcc] byte offset of BCC b's slice, | 1 when narrow (-1: not in this schedule)
  const int32_t *slice_bytes;    // [n_bcc] its size (TileSlice::bytes)
  const TileItem *items;
  int64_t item_begin, item_end;
  unsigned long long *next_item;  // zeroed before each launch
  unsigned long long *acc;        // [n_packed][kAccDigits] fixed-point BC counters (plain.h)
  int32_t *ws_lv;                 // warp class: level offsets per warp slot ([slots][cap])
  int64_t cap;                    // per-slot row capacity (>= largest BCC of the class + 2)
  double *ws_P;                   // CTA class: FP64 partial BC row per source group ([grid * groups][cap_P])
  int64_t cap_P;
  int32_t nmax;                   // largest BCC of the launch (shared-memory rows are sized for it)
  int32_t slice_max;              // largest slice in bytes
  unsigned long long wait_ns;     // limit of the wait for a staged slice
  int *err;
};

// Dynamic shared memory of a launch of class cls for BCCs of up to nmax
// vertices and slices of up to slice_max bytes.
size_t tile_smem_bytes(int cls, int64_t nmax, int64_t slice_max);
// Source groups per CTA of class cls (each with its own FP64 row in ws_P).
int tile_groups(int cls);
// Largest shared memory a CTA may use (opt-in limit of the device).
size_t tile_smem_limit(int device);
// CTAs of class cls resident per SM at this shared-memory size (0: none fits).
int tile_ctas_per_sm(int cls, size_t smem);
cudaError_t launch_tile(int cls, const TileArgs &a, int grid, size_t smem, cudaStream_t stream);

}  // namespace bcg
