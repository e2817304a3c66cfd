// Host-visible interface of the PLAIN schedule kernels (kernels_plain.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bcg {

// One free/endpoint source (BCC-local id) plus chains [c0, c1) of the global
// chain table whose left endpoint it is. A source owning many chains is split
// into several items; only the one with own != 0 accumulates the source's own
// dependencies, the others run its BFS forward only.
struct PlainItem {
  int32_t bcc, src, c0, c1, own;
};

struct PlainArgs {
  const int64_t *row;      // [n_packed+1] global arc offsets
  const int32_t *col;      // local neighbour ids
  const int32_t *reach;    // [n_packed]
  const int64_t *vtx_off;  // [n_bcc+1]
  const int32_t *chain_start, *chain_len, *chain_l, *chain_r;
  const PlainItem *items;
  int64_t item_begin, item_end;
  unsigned long long *next_item;  // zeroed before each launch
  double *bc;                     // [n_packed] accumulator
  int32_t *ws_i;                  // 7 int rows per workspace slot
  double *ws_f;                   // 4 double rows per workspace slot
  int64_t ws_n;                   // row capacity (>= largest BCC + 2)
  int32_t *epochs;                // 2 per slot: level-stamp bases of rows A and B
  int64_t rows_slot;              // workspace slot reserved for launch_rows
  int *err;
};

// block: 256, 512 or 1024 threads (1024 / block CTAs fit an SM).
cudaError_t launch_plain(const PlainArgs &a, int block, int grid, cudaStream_t stream);
// Rows (levels, path counts) of one source of BCC `bcc`; chain >= 0 selects
// the merged rows of chain vertex src on that chain.
cudaError_t launch_rows(const PlainArgs &a, int32_t bcc, int32_t src, int32_t chain, int32_t *d_out, double *s_out,
                        cudaStream_t stream);

}  // namespace bcg
