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
  // Each ear record hangs on the ear-graph arc leaving its left end; parallel
  // ears between one pair of ends share a record, and its ld/rd need not be
  // exact (Codes/readeardata.cpp:50-100,154-182; Codes/bcc_bfs.cpp:100-236).
  // So the chains are rebuilt from the graph: every neighbour of the left end
  // that belongs to the record starts a chain, walked through its degree-2
  // vertices to the right end; positions give the distances.
  std::vector<int> act, l, r, cnt, off, nodes, ld, rd;
  std::vector<char> in_ear((size_t)n, 0);
  for (int v = 0; v < n; ++v)
    for (int j = ear_R[v]; j < ear_R[v + 1]; ++j) {
      ear_premble *e = ear_info[j];
      if (!e || e->lnode != v) continue;
      for (int k = 0; k < e->cnt; ++k) in_ear[e->nodes[k]] = 1;
      for (int a = R[v]; a < R[v + 1]; ++a) {
        int x = C[a], prev = v;
        if (!in_ear[x]) continue;
        const int start = (int)nodes.size();
        while (x != e->rnode && in_ear[x] && R[x + 1] - R[x] == 2) {
          nodes.push_back(x);
          in_ear[x] = 0;
          const int nx = C[R[x]] == prev ? C[R[x] + 1] : C[R[x]];
          prev = x;
          x = nx;
        }
        if (x != e->rnode) { fprintf(stderr, "begin_gpu: an ear that is not a chain of degree-2 vertices\n"); exit(EXIT_FAILURE); }
        const int len = (int)nodes.size() - start;
        l.push_back(v); r.push_back(e->rnode); cnt.push_back(len); off.push_back(start);
        for (int k = 0; k < len; ++k) { ld.push_back(k + 1); rd.push_back(len - k); }
      }
      for (int k = 0; k < e->cnt; ++k)
        if (in_ear[e->nodes[k]]) { fprintf(stderr, "begin_gpu: an ear vertex off every chain\n"); exit(EXIT_FAILURE); }
      act.push_back(e->lnode); act.push_back(e->rnode);
    }
  std::sort(act.begin(), act.end()); act.erase(std::unique(act.begin(), act.end()), act.end());
  if (bc_begin_active(ctx(), R, C, n, m, act.data(), (int)act.size(), (int)l.size(), l.data(), r.data(),
                      cnt.data(), off.data(), nodes.data(), ld.data(), rd.data(), artnodes.data(), bc, &t))
    { fprintf(stderr, "%s\n", bc_last_error(ctx())); exit(EXIT_FAILURE); }
}
