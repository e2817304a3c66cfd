// betc — command-line drop-in for the reference's `./betc input_file`
// (Codes/main.cpp:54-72, Codes/ReadMe:1-13).
//
// Input: the reference's edge list ("n m", then m lines "u v w", 0-based).
// Output: one line "v bc" per vertex (FP64, ordered pairs), the per-vertex
// print the reference has commented out (Codes/main.cpp:45-49), to stdout or
// --out FILE; counts and timings go to stderr ("GPU total time is ...", as
// Codes/main.cpp:70).
#include "bchost.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static void usage() {
  std::fprintf(stderr,
               "usage: betc INPUT_FILE [--out FILE] [--mode plain|batched] [--delta fp64|fp32c]\n"
               "            [--batch WIDTH] [--device ORDINAL] [--quiet] [--save-csr FILE] [--host-decomp]\n"
               "            [--plain-ctas 4|8|16]\n"
               "  INPUT_FILE: the edge list (n m, then u v w per edge) or a CSR written by --save-csr;\n"
               "    the graph is taken as simple and unweighted: repeated edges count once and\n"
               "    self-loops are dropped (the reference keeps repeated edges as parallel arcs,\n"
               "    which multiplies path counts)\n"
               "  --host-decomp: run the BCC/chain decomposition on the host cores instead of the GPU\n"
               "    (same result; the GPU steps are the default, --gpu-decomp names them explicitly)\n"
               "  --plain-ctas: per-source CTAs per SM (more sources in flight on deep BCCs)\n");
}

int main(int argc, char **argv) {
  if (argc < 2) { usage(); return 1; }
  const char *input = nullptr, *out_path = nullptr, *save_path = nullptr;
  bc_opts opts;
  bc_default_opts(&opts);
  bool quiet = false, gpu_decomp = true;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto next = [&]() -> const char * {
      if (i + 1 >= argc) { usage(); std::exit(1); }
      return argv[++i];
    };
    if (a == "--out") out_path = next();
    else if (a == "--mode") {
      std::string m = next();
      if (m == "plain") opts.mode = BCGPU_MODE_PLAIN;
      else if (m == "batched") opts.mode = BCGPU_MODE_BATCHED;
      else { usage(); return 1; }
    } else if (a == "--delta") {
      std::string m = next();
      if (m == "fp64") opts.delta = BCGPU_DELTA_FP64;
      else if (m == "fp32c") opts.delta = BCGPU_DELTA_FP32C;
      else { usage(); return 1; }
    } else if (a == "--batch") opts.batch_width = std::atoi(next());
    else if (a == "--device") opts.device = std::atoi(next());
    else if (a == "--quiet") quiet = true;
    else if (a == "--save-csr") save_path = next();
    else if (a == "--gpu-decomp") gpu_decomp = true;
    else if (a == "--host-decomp") gpu_decomp = false;
    else if (a == "--plain-ctas") opts.plain_ctas_per_sm = std::atoi(next());
    else if (a == "-h" || a == "--help") { usage(); return 0; }
    else if (!input) input = argv[i];
    else { usage(); return 1; }
  }
  if (!input) { usage(); return 1; }

  auto t0 = std::chrono::steady_clock::now();
  char err[512] = {0};
  bc_graph *g = nullptr;
  int rc = bc_graph_load(input, &g, err, sizeof(err));
  if (rc) { std::fprintf(stderr, "betc: %s\n", err); return 2; }
  if (save_path && bc_graph_save(g, save_path, err, sizeof(err))) {
    std::fprintf(stderr, "betc: %s\n", err);
    bc_graph_free(g);
    return 6;
  }
  // the context first: its options are checked (and its GPU chosen) before
  // any decomposition work
  bc_ctx *ctx = nullptr;
  rc = bc_create(&opts, &ctx);
  if (rc) { std::fprintf(stderr, "betc: %s\n", bc_last_error(nullptr)); bc_graph_free(g); return 4; }
  bc_decomp *d = nullptr;
  if (gpu_decomp) {
    // on the --device GPU, else device 0
    rc = bc_decompose_gpu(g, opts.device >= 0 ? opts.device : 0, &d, err, sizeof(err));
    if (rc == BCGPU_ECUDA) { std::fprintf(stderr, "betc: %s\n", err); bc_destroy(ctx); bc_graph_free(g); return 4; }
    if (rc) {
      std::fprintf(stderr, "betc: GPU decomposition failed (code %d): %s\n", rc, err);
      bc_destroy(ctx);
      bc_graph_free(g);
      return 3;
    }
  } else {
    rc = bc_decompose(g, &d);
    if (rc) {
      std::fprintf(stderr, "betc: decomposition failed (code %d)\n", rc);
      bc_destroy(ctx);
      bc_graph_free(g);
      return 3;
    }
  }
  bc_decomp_info info;
  bc_decomp_get_info(d, &info);
  const bc_bccs *view = bc_decomp_view(d);
  std::vector<double> bc((size_t)view->n_orig, 0.0);
  bc_stats st{};
  rc = bc_run_bccs(ctx, view, bc.data(), &st);
  if (rc) {
    std::fprintf(stderr, "betc: %s\n", bc_last_error(ctx));
    bc_destroy(ctx); bc_decomp_free(d); bc_graph_free(g);
    return 5;
  }
  FILE *fp = out_path ? std::fopen(out_path, "w") : stdout;
  if (!fp) { std::fprintf(stderr, "betc: cannot write %s\n", out_path); return 6; }
  std::vector<char> buf(1 << 20);
  std::setvbuf(fp, buf.data(), _IOFBF, buf.size());
  for (int32_t v = 0; v < view->n_orig; ++v) std::fprintf(fp, "%d %.17g\n", v, bc[v]);
  if (out_path) std::fclose(fp);
  else std::fflush(stdout);
  double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (!quiet) {
    std::fprintf(stderr,
                 "bccs %d (packed %d, cycles %lld) articulation %d chains %lld (chain vertices %lld)\n"
                 "sources %lld bfs %lld aux_bfs %lld teps_edges %lld\n"
                 "host decomposition %.3f ms, GPU kernels %.3f ms, GPU call %.3f ms, wall %.3f s\n"
                 "GPU total time is %f \n",
                 info.n_bcc_all, info.n_bcc_packed, (long long)info.n_cycle_bccs, info.n_articulation,
                 (long long)info.n_chains, (long long)info.n_chain_vertices, (long long)st.sources,
                 (long long)st.bfs_sources, (long long)st.aux_bfs, (long long)st.teps_edges, info.host_ms,
                 st.kernel_ms, st.total_ms, wall, st.kernel_ms * 1e-3);
  }
  bc_destroy(ctx);
  bc_decomp_free(d);
  bc_graph_free(g);
  return 0;
}
