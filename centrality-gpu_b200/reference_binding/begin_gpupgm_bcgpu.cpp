// begin_gpupgm_bcgpu.cpp — binds the reference's begin_gpu to libbcgpu
#include "ear_graph.h"
#include "bcgpu.h"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

static bc_ctx *ctx() {
  static bc_ctx *c = nullptr;
  if (!c) {
    bc_opts o; bc_default_opts(&o);
    o.mode = BCGPU_MODE_PLAIN;                      // explicit source lists
    if (bc_create(&o, &c)) { fprintf(stderr, "%s\n", bc_last_error(nullptr)); exit(EXIT_FAILURE); }
  }
  return c;
}

void begin_gpu(int *&R, int *&C, int *&F, int n, int m, ear_premble **&, ear_premble **&,
               std::vector<int> &req_nodes, std::vector<int> &artnodes, float *&bc, double &t) {
  if (bc_begin_free(ctx(), R, C, n, m, req_nodes.data(), (int)req_nodes.size(), artnodes.data(), bc, &t))
    { fprintf(stderr, "%s\n", bc_last_error(ctx())); exit(EXIT_FAILURE); }
}

void begin_gpu(int *&R, int *&C, int *&F, int n, int m, ear_premble **&ear_info, std::vector<int> &,
               std::vector<int> &, std::vector<int> &, std::vector<int> &, int, std::vector<int> &artnodes,
               float *&bc, double &t, int *&ear_R, int *&ear_C) {
  // flatten the ears attached to the ear-graph arcs (ear_premble, Codes/ear_graph.h:3-32)
  std::vector<int> act, l, r, cnt, off, nodes, ld, rd;
  for (int v = 0; v < n; ++v)
    for (int j = ear_R[v]; j < ear_R[v + 1]; ++j) {
      ear_premble *e = ear_info[j];
      if (!e || e->lnode != v) continue;
      l.push_back(e->lnode); r.push_back(e->rnode); cnt.push_back(e->cnt); off.push_back((int)nodes.size());
      for (int k = 0; k < e->cnt; ++k) { nodes.push_back(e->nodes[k]); ld.push_back(e->ld[k]); rd.push_back(e->rd[k]); }
      act.push_back(e->lnode); act.push_back(e->rnode);
    }
  std::sort(act.begin(), act.end()); act.erase(std::unique(act.begin(), act.end()), act.end());
  if (bc_begin_active(ctx(), R, C, n, m, act.data(), (int)act.size(), (int)l.size(), l.data(), r.data(),
                      cnt.data(), off.data(), nodes.data(), ld.data(), rd.data(), artnodes.data(), bc, &t))
    { fprintf(stderr, "%s\n", bc_last_error(ctx())); exit(EXIT_FAILURE); }
}
