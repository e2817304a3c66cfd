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

// Deterministic BC accumulation of the per-source schedule. Each (source,
// vertex) contribution c >= 0 is turned into the integer floor(c * 2^kAccFrac)
// and added, split into kAccDigits digits of kAccDigitBits bits, to that
// vertex's kAccDigits 64-bit counters with integer atomics. Integer addition
// is associative, so the counters do not depend on the order in which
// concurrently running CTAs add; launch_fold then turns them into FP64 in a
// fixed order and adds that to the FP64 accumulator. Range of one
// contribution: [2^-kAccFrac, 2^(kAccDigits*kAccDigitBits - kAccFrac));
// larger ones flag kDevOverflow. Each counter takes at most kAccMaxAdds adds
// between two folds (a digit is below 2^kAccDigitBits), so a launch runs at
// most kAccMaxAdds sources.
constexpr int kAccDigits = 4;
constexpr int kAccDigitBits = 40;
constexpr int kAccFrac = 100;
constexpr int64_t kAccMaxAdds = int64_t(1) << (64 - kAccDigitBits);

struct PlainArgs {
  const int64_t *row;      // [n_packed+1] global arc offsets
  const int32_t *col;      // local neighbour ids
  const int32_t *reach;    // [n_packed]
  const int64_t *vtx_off;  // [n_bcc+1]
  const int32_t *chain_start, *chain_len, *chain_l, *chain_r;
  const PlainItem *items;
  int64_t item_begin, item_end;
  unsigned long long *next_item;  // zeroed before each launch
  unsigned long long *acc;        // [n_packed][kAccDigits] fixed-point BC counters
  int32_t *ws_i;                  // kWsIntRows int rows per workspace slot
  double *ws_f;                   // kWsDblRows double rows per workspace slot (16-byte records, 16-byte aligned)
  int64_t ws_n;                   // row capacity (>= largest BCC + 2)
  int32_t *epochs;                // 2 per slot: level-stamp bases of rows A and B
  int64_t rows_slot;              // workspace slot reserved for launch_rows
  int32_t rescale_exp;            // a level whose largest path count passes 2^rescale_exp is rescaled
  int *err;
};

// Workspace per slot: visit orders, level offsets and level exponents of
// rows A and B and the merged row's level exponents (int rows); the records
// (level stamp, path count then q) of rows A, B and merged, 16 bytes per
// vertex each (as double rows: two per record row). The records start zeroed
// (stamp 0: unvisited).
constexpr int kWsIntRows = 7;
constexpr int kWsDblRows = 6;

// block: 64 ... 1024 threads (1024 / block CTAs fit an SM).
cudaError_t launch_plain(const PlainArgs &a, int block, int grid, cudaStream_t stream);
// Adds the fixed-point counters of packed vertices [v0, v1) to bc (FP64) and
// clears them; the value added to each vertex is independent of the order of
// the atomic adds that filled its counters.
cudaError_t launch_fold(unsigned long long *acc, double *bc, int64_t v0, int64_t v1, cudaStream_t stream);
// Rows (levels, path counts) of one source of BCC `bcc`; chain >= 0 selects
// the merged rows of chain vertex src on that chain. Path counts are written
// unscaled (as FP64 values; inf where they exceed FP64's range).
cudaError_t launch_rows(const PlainArgs &a, int32_t bcc, int32_t src, int32_t chain, int32_t *d_out, double *s_out,
                        cudaStream_t stream);

}  // namespace bcg
