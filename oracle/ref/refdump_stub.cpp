// Test infrastructure only (oracle): replaces the reference's two GPU entry
// points with stubs that DUMP what the reference's host pipeline hands to the
// GPU, so the decomposition (BCC split, reach vector, free set, ears) can be
// pinned against this project's oracle and host decomposition.
//
// Replaced interfaces (reference, Codes/ear_graph.h:45-49; bodies in
// Codes/begin_gpupgm.cu:42-71 and :73-89):
//   begin_gpu(R,C,F,n,m, ear_info, self_ear, req_nodes, artnodes, bc, time)   [free sources]
//   begin_gpu(R,C,F,n,m, ear_info, parents, levels, level_order, level_offset,
//             max_earlevel, artnodes, bc, time, ear_R, ear_C)                  [active + chain sources]
//
// The stubs leave bc zeroed, so the reference's bc_result after the run holds
// only the articulation cross terms added by BiCC::reachfunction
// (Codes/modified_apsp.cpp:157-220).
//
// Output (file named by $REFDUMP_OUT), one record per line, ORIGINAL vertex ids:
//   BCC <bcc_index> <n>
//   V <orig> <reach>                 one per BCC vertex (Codes/to_eargraph_construct.cpp:151-160)
//   FREE <orig>...                   free sources (req_nodes, :115-122)
//   EAR <l> <r> <cnt> (<ld> <orig> <rd>)*cnt   ears as attached by read_ear_info (Codes/readeardata.cpp:117-182)
//   LEVELS <level_offset.size()>     number of active batch boundaries (Codes/arrangelevels.cpp:56-146)
#include "ear_graph.h"
#include "bicc.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <map>

FILE *dump_fp() {
  static FILE *fp = nullptr;
  if (!fp) {
    const char *p = getenv("REFDUMP_OUT");
    fp = p ? fopen(p, "w") : stderr;
    if (!fp) { perror("REFDUMP_OUT"); exit(3); }
  }
  return fp;
}

// Which BCC (index into BiCC::bccvertno) the current call belongs to.
static int g_bcc = -1;
static const int *g_last_R = nullptr;
static int g_last_n = -1;
static std::vector<int> g_last_C;

static int orig_of(int local) { return BiCC::bccvertno[g_bcc][local].first; }

static void start_bcc(int n, const int *R, const int *C, int m, const std::vector<int> &reach) {
  // to_eargraph walks BCCs in index order and skips those with <= 2 vertices
  // (Codes/to_eargraph_construct.cpp:54-60).
  do { ++g_bcc; } while (g_bcc < (int)BiCC::bccvertno.size() && (int)BiCC::bccvertno[g_bcc].size() <= 2);
  if (g_bcc >= (int)BiCC::bccvertno.size() || (int)BiCC::bccvertno[g_bcc].size() != n) {
    fprintf(stderr, "refdump: lost track of BCC order (n=%d)\n", n);
    exit(4);
  }
  g_last_R = R; g_last_n = n; g_last_C.assign(C, C + m);
  FILE *fp = dump_fp();
  fprintf(fp, "BCC %d %d\n", g_bcc, n);
  for (int k = 0; k < n; ++k) fprintf(fp, "V %d %d\n", orig_of(k), reach[k]);
}

void begin_gpu(int *&R, int *&C, int *&F, int n, int m, ear_premble **&ear_info, ear_premble **&self_ear,
               std::vector<int> &req_nodes, std::vector<int> &artnodes, float *&bc_gpu, double &g_free_time) {
  (void)F; (void)ear_info; (void)self_ear; (void)g_free_time;
  start_bcc(n, R, C, m, artnodes);  // the free call always comes first for a BCC
  FILE *fp = dump_fp();
  fprintf(fp, "FREE");
  for (int v : req_nodes) fprintf(fp, " %d", orig_of(v));
  fprintf(fp, "\n");
  for (int k = 0; k < n; ++k) bc_gpu[k] = 0.f;
}

void begin_gpu(int *&R, int *&C, int *&F, int n, int m, ear_premble **&ear_info, std::vector<int> &parents,
               std::vector<int> &levels, std::vector<int> &level_order, std::vector<int> &level_offset, int max_earlevel,
               std::vector<int> &artnodes, float *&bc_gpu, double &g_free_time, int *&ear_R, int *&ear_C) {
  (void)F; (void)parents; (void)levels; (void)level_order; (void)max_earlevel; (void)g_free_time;
  bool same = (R == g_last_R && n == g_last_n && (int)g_last_C.size() == m &&
               std::memcmp(g_last_C.data(), C, sizeof(int) * (size_t)m) == 0);
  if (!same) start_bcc(n, R, C, m, artnodes);
  FILE *fp = dump_fp();
  for (int v = 0; v < n; ++v) {
    for (int j = ear_R[v]; j < ear_R[v + 1]; ++j) {
      ear_premble *e = ear_info[j];
      if (!e || e->lnode != v) continue;  // each ear is attached to its (lnode -> rnode) arc
      fprintf(fp, "EAR %d %d %d", orig_of(e->lnode), orig_of(e->rnode), e->cnt);
      for (int c = 0; c < e->cnt; ++c) fprintf(fp, " %d %d %d", e->ld[c], orig_of(e->nodes[c]), e->rd[c]);
      fprintf(fp, "\n");
    }
  }
  fprintf(fp, "LEVELS %zu\n", level_offset.size());
  for (int k = 0; k < n; ++k) bc_gpu[k] = 0.f;
}
