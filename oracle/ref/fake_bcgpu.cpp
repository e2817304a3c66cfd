// Test infrastructure only: a stand-in for the five libbcgpu entry points the
// reference-side binding calls (centrality-gpu_b200/reference_binding/). It
// computes nothing; it records, in ORIGINAL vertex ids, the chains the
// binding hands to bc_begin_active, so a CPU test can compare them with the
// product's own decomposition on the reference's inputs. Records go to the
// file named by $BINDCHECK_OUT:
//   CHAIN <left> <right> (<ld> <vertex> <rd>)*len
#include "bcgpu.h"
#include "bicc.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

FILE *out() {
  static FILE *fp = nullptr;
  if (!fp) {
    const char *p = getenv("BINDCHECK_OUT");
    fp = p ? fopen(p, "w") : stderr;
    if (!fp) { perror("BINDCHECK_OUT"); exit(3); }
  }
  return fp;
}

// The BCC (index into BiCC::bccvertno) of the current call: the reference
// visits BCCs in index order, skipping those of <= 2 vertices
// (Codes/to_eargraph_construct.cpp:54-60); a call with a CSR other than the
// previous call's starts the next one.
int g_bcc = -1;
std::vector<int32_t> g_R, g_C;

void track(const int32_t *R, const int32_t *C, int32_t n, int32_t m) {
  if ((int32_t)g_R.size() == n + 1 && (int32_t)g_C.size() == m && !memcmp(g_R.data(), R, 4 * (n + 1)) &&
      !memcmp(g_C.data(), C, 4 * (size_t)m))
    return;
  do { ++g_bcc; } while (g_bcc < (int)BiCC::bccvertno.size() && (int)BiCC::bccvertno[g_bcc].size() <= 2);
  if (g_bcc >= (int)BiCC::bccvertno.size() || (int)BiCC::bccvertno[g_bcc].size() != n) {
    fprintf(stderr, "fake_bcgpu: lost track of BCC order (n=%d)\n", n);
    exit(4);
  }
  g_R.assign(R, R + n + 1);
  g_C.assign(C, C + m);
}

int orig(int32_t local) { return BiCC::bccvertno[g_bcc][local].first; }
int g_ctx;

}  // namespace

extern "C" void bc_default_opts(bc_opts *o) { memset(o, 0, sizeof *o); }
extern "C" int bc_create(const bc_opts *, bc_ctx **c) {
  *c = reinterpret_cast<bc_ctx *>(&g_ctx);
  return BCGPU_OK;
}
extern "C" const char *bc_last_error(const bc_ctx *) { return "fake_bcgpu"; }

extern "C" int bc_begin_free(bc_ctx *, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *,
                             int32_t, const int32_t *, float *bc, double *) {
  track(R, C, n, m);
  for (int32_t k = 0; k < n; ++k) bc[k] = 0.f;  // overwritten, as the real call does
  return BCGPU_OK;
}

extern "C" int bc_begin_active(bc_ctx *, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *,
                               int32_t, int32_t n_ears, const int32_t *lnode, const int32_t *rnode,
                               const int32_t *cnt, const int32_t *off, const int32_t *nodes, const int32_t *ld,
                               const int32_t *rd, const int32_t *, float *, double *) {
  track(R, C, n, m);
  for (int32_t e = 0; e < n_ears; ++e) {
    fprintf(out(), "CHAIN %d %d", orig(lnode[e]), orig(rnode[e]));
    for (int32_t k = 0; k < cnt[e]; ++k) fprintf(out(), " %d %d %d", ld[off[e] + k], orig(nodes[off[e] + k]), rd[off[e] + k]);
    fprintf(out(), "\n");
  }
  fflush(out());
  return BCGPU_OK;
}
