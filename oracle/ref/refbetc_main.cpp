// Test infrastructure only: the reference's own host pipeline driving libbcgpu
// through centrality-gpu_b200/reference_binding/begin_gpupgm_bcgpu.cpp, i.e.
// the reference's `betc` with its GPU files replaced by the binding to
// libbcgpu. Mirrors Codes/main.cpp:26-72 (same run_modified_apsp flags,
// :65) and prints the per-vertex BC that it leaves commented out (:45-49),
// then the "GPU total time" line it prints (:70).
#include "graph.h"
#include "modified_apsp.h"
#include <cstdio>

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: refbetc <edge-list>\n"); return 1; }
  Graph g(argv[1]);
  float *bc = new float[g.n_vertices];
  for (int i = 0; i < g.n_vertices; ++i) bc[i] = 0.f;
  double t = 0;
  int active = 0, free_cnt = 0;
  Modified_APSP m;
  m.run_modified_apsp(g, true, true, false, bc, t, active, free_cnt);
  for (int i = 0; i < g.n_vertices; ++i) printf("%d %f\n", i, (double)bc[i]);
  fprintf(stderr, "GPU total time is %f \n", t);
  delete[] bc;
  return 0;
}
