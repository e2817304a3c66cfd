// Test infrastructure only (linked against the stand-in runtime's library):
// builds a graph's multi-source pass tables in full and restricted to pass
// ranges (BatchedConfig::fill_begin/fill_end, what bc_opts.lazy_tables uses)
// and checks that every filled pass runs from exactly the tables the full
// build gives it, with the same unit accounting for every pass.
// Usage: fill_range_check EDGE_LIST WIDTH [BEGIN END]...  (a negative bound
// counts from the number of passes). Prints one line per range:
// "range B E ok N" (N passes compared) or "range B E mismatch PASS".
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "batched.h"
#include "bchost.h"

static bcg::BatchedPlan *build(const bc_bccs *B, int width, int64_t b, int64_t e) {
  bcg::BatchedConfig cfg;
  cfg.width = width;
  cfg.limit_bytes = (int64_t)1 << 36;
  cfg.fill_begin = b;
  cfg.fill_end = e;
  cfg.keep_host_tables = true;
  bcg::BatchedPlan *p = nullptr;
  std::string msg;
  if (bcg::batched_create(B, cfg, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                          nullptr, nullptr, &p, &msg)) {
    std::printf("build failed: %s\n", msg.c_str());
    std::exit(2);
  }
  return p;
}

int main(int argc, char **argv) {
  if (argc < 3) return 1;
  bc_graph *g = nullptr;
  char err[256];
  if (bc_graph_load(argv[1], &g, err, sizeof err)) { std::printf("load: %s\n", err); return 1; }
  bc_decomp *d = nullptr;
  if (bc_decompose(g, &d)) return 1;
  const bc_bccs *B = bc_decomp_view(d);
  const int width = std::atoi(argv[2]);
  bcg::BatchedPlan *full = build(B, width, 0, INT64_MAX);
  std::vector<int64_t> src, teps, bfs, aux, visits;
  bcg::batched_unit_work(full, src, teps, bfs, aux, visits);
  const int64_t npass = (int64_t)src.size() - 1;
  std::printf("passes %lld\n", (long long)npass);
  for (int a = 3; a + 1 < argc; a += 2) {
    int64_t b = std::atoll(argv[a]), e = std::atoll(argv[a + 1]);
    if (b < 0) b += npass;
    if (e < 0) e += npass;
    bcg::BatchedPlan *part = build(B, width, b, e);
    std::vector<int64_t> s2, t2, b2, a2, v2;
    bcg::batched_unit_work(part, s2, t2, b2, a2, v2);
    long long bad = -1, filled = 0;
    if (s2 != src || t2 != teps) bad = -2;  // the unit accounting never depends on the range
    for (int64_t j = 0; j < npass && bad == -1; ++j) {
      if (j >= b && j < e) {
        const uint64_t dp = bcg::batched_pass_digest(part, j), df = bcg::batched_pass_digest(full, j);
        if (dp == 0 || dp != df) bad = j;  // 0: no host tables to compare
        ++filled;
      }
    }
    if (bad == -1) std::printf("range %lld %lld ok %lld\n", (long long)b, (long long)e, filled);
    else std::printf("range %lld %lld mismatch %lld\n", (long long)b, (long long)e, bad);
    bcg::batched_destroy(part);
  }
  bcg::batched_destroy(full);
  bc_decomp_free(d);
  bc_graph_free(g);
  return 0;
}
