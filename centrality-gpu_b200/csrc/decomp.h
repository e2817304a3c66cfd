// Library-internal: the graph and decomposition objects behind bchost.h, and
// the hand-off between the BCC split (host or GPU) and the packing (host).
#pragma once
#include <chrono>
#include <cstdint>
#include <vector>

#include "bchost.h"

struct bc_graph {
  int32_t n = 0;
  std::vector<int64_t> row;
  std::vector<int32_t> col;
};

struct bc_decomp {
  bc_bccs view{};
  bc_decomp_info info{};
  std::vector<int64_t> vtx_off, row, chain_off;
  std::vector<int32_t> col, reach, orig, n_plain, chain_start, chain_len, chain_l, chain_r;
  std::vector<double> art;
};

namespace bcg {

// What the packing needs from the BCC split and the arc-to-member pass.
// BCC b's members are members[mem_off[b], mem_off[b + 1]), its head last; the
// member slot s = mem_off[b] + local id holds that member's arcs inside b as
// local ids, sadj[sdeg[s], sdeg[s + 1]), in the member's arc order. The order
// of the non-head members inside a BCC is free: the packing keys everything
// it writes by vertex id.
struct SplitResult {
  int32_t nbcc = 0, n_art = 0;
  std::vector<int32_t> comp, head, members, sadj;
  std::vector<int64_t> comp_size, below, hang, mem_off, sdeg;
  std::vector<double> art;
};

// Orders and packs every BCC of >= 3 vertices into D (largest first, chains
// found and numbered, adjacency in final local ids, reach per member); t0 is
// the start of the whole decomposition, for bc_decomp_info::host_ms.
int decomp_pack(SplitResult &S, int32_t n, bc_decomp *D, std::chrono::steady_clock::time_point t0);

// Points D's view at its arrays and fills its info (D's vtx_off, row,
// chain_off and chain_len must be final).
void decomp_finish(bc_decomp *D, int32_t n, int32_t n_components, int32_t nbcc, int32_t n_art, int64_t n_cycle_bccs,
                   std::chrono::steady_clock::time_point t0);

// The whole decomposition as data-parallel steps (decomp_steps.cu): on GPU
// `device` (>= 0), or, for a check of the same steps without a GPU, as host
// loops (device < 0). Same result as bc_decompose.
int decomp_gpu(const bc_graph *g, int device, bc_decomp *D, std::chrono::steady_clock::time_point t0, char *err,
               size_t errlen);

}  // namespace bcg
