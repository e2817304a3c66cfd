// Test infrastructure only: the libbcgpu entry points the reference-side
// binding calls, computed on the CPU by the oracle's per-BCC Brandes
// (oracle/bc_oracle.c, every listed source by BFS). Linked with the
// reference's host sources and the binding it gives the numbers the
// reference's own betc would print on top of libbcgpu, without a GPU; the
// same binary linked to the real library (refbetc) must print them on a GPU.
// Call semantics are the library's: the free call overwrites bc with its
// contributions, the active call adds those of the active vertices and of
// every chain vertex.
#include "bcgpu.h"

#include <cstring>
#include <vector>

extern "C" {
#include "../bc_oracle.h"
}

namespace {

int g_ctx;

std::vector<double> contributions(const int32_t *R, const int32_t *C, int32_t n, const int32_t *reach,
                                  const std::vector<int32_t> &sources) {
  std::vector<int64_t> R64(R, R + n + 1);
  std::vector<double> out((size_t)n, 0.0);
  orc_bcc_sources(n, R64.data(), C, reach, 0, nullptr, nullptr, nullptr, nullptr, sources.data(),
                  (int64_t)sources.size(), 1, out.data());
  return out;
}

}  // namespace

extern "C" void bc_default_opts(bc_opts *o) { memset(o, 0, sizeof *o); }
extern "C" int bc_create(const bc_opts *, bc_ctx **c) {
  *c = reinterpret_cast<bc_ctx *>(&g_ctx);
  return BCGPU_OK;
}
extern "C" const char *bc_last_error(const bc_ctx *) { return "cpu_bcgpu"; }

extern "C" int bc_begin_free(bc_ctx *, const int32_t *R, const int32_t *C, int32_t n, int32_t, const int32_t *req,
                             int32_t n_req, const int32_t *reach, float *bc, double *) {
  const std::vector<double> out = contributions(R, C, n, reach, std::vector<int32_t>(req, req + n_req));
  for (int32_t k = 0; k < n; ++k) bc[k] = (float)out[k];
  return BCGPU_OK;
}

extern "C" int bc_begin_active(bc_ctx *, const int32_t *R, const int32_t *C, int32_t n, int32_t,
                               const int32_t *active, int32_t n_active, int32_t n_ears, const int32_t *,
                               const int32_t *, const int32_t *cnt, const int32_t *off, const int32_t *nodes,
                               const int32_t *, const int32_t *, const int32_t *reach, float *bc, double *) {
  std::vector<int32_t> src(active, active + n_active);
  for (int32_t e = 0; e < n_ears; ++e) src.insert(src.end(), nodes + off[e], nodes + off[e] + cnt[e]);
  const std::vector<double> out = contributions(R, C, n, reach, src);
  for (int32_t k = 0; k < n; ++k) bc[k] += (float)out[k];
  return BCGPU_OK;
}
