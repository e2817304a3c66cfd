// Test infrastructure only (oracle): driver for the reference's host pipeline.
// Mirrors run_modified_apsp in the reference's Codes/main.cpp:26-52 (which is
// not linked: it prints nothing per vertex) and prints the articulation cross
// terms that BiCC::reachfunction leaves in bc_result (Codes/modified_apsp.cpp:209),
// the only BC values the reference computes on the host.
#include "graph.h"
#include "modified_apsp.h"
#include <cstdio>
#include <cstdlib>

FILE *dump_fp();  // refdump_stub.cpp: the one stream all records go to

int main(int argc, char **argv) {
  if (argc < 2) { fprintf(stderr, "usage: refdump <edge-list>\n"); return 1; }
  Graph g(argv[1]);
  float *bc = new float[g.n_vertices];
  for (int i = 0; i < g.n_vertices; ++i) bc[i] = 0.f;
  double t = 0; int active = 0, free_cnt = 0;
  Modified_APSP m;
  // Same flags as the reference's main (Codes/main.cpp:65): cpu, gpu, no pendant removal.
  m.run_modified_apsp(g, true, true, false, bc, t, active, free_cnt);
  FILE *fp = dump_fp();
  for (int i = 0; i < g.n_vertices; ++i)
    if (bc[i] != 0.f) fprintf(fp, "ART %d %.1f\n", i, (double)bc[i]);
  fprintf(fp, "COUNTS %d %d\n", active, free_cnt);
  return 0;
}
