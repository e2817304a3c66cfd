// libbcgpu context, plans and the C ABI of include/bcgpu.h.
//
// A plan uploads the packed BCCs once (the reference copies CSR, reach and
// per-source scratch to the device and frees it again inside every begin_gpu
// call, Codes/kernels_free.cu:40-101, Codes/kernels_active.cu:67-211), keeps
// the BC accumulator on the device in FP64 (the reference accumulates FP32,
// Codes/kernels_free.cu:425) and splits the sources into work units that can
// be run in any ranges.
#include "bcgpu.h"
#include "batched.h"
#include "common.cuh"
#include "internal.h"
#include "plain.h"
#include "tile.h"

#include <algorithm>
#include <cmath>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <set>
#include <string>
#include <thread>
#include <vector>

struct bc_plan;

struct bc_ctx {
  bc_opts opts{};
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Stream-ordered pool of the plans' device memory: a destroyed plan's
  // buffers go back to the pool (cudaFreeAsync) and stay reserved for the
  // next plan of this context instead of returning to the device (a plan of
  // RMAT-20 holds ~5 GB; cudaFree of that took ~0.2 s per plan). Released
  // to the device by bc_destroy.
  cudaMemPool_t pool = nullptr;
  std::set<bc_plan *> plans;  // live plans: bc_destroy releases them first
};

struct bc_plan {
  bc_ctx *ctx = nullptr;
  int mode = BCGPU_MODE_PLAIN;
  // host copies needed to read results
  int32_t n_orig = 0;
  int64_t n_packed = 0;
  std::vector<int32_t> orig;
  std::vector<double> art;
  std::vector<int64_t> h_vtx_off, h_chain_off;
  std::vector<int32_t> h_n_plain, h_chain_start, h_chain_len;
  std::vector<bcg::PlainItem> h_items;
  // device graph
  int64_t *row = nullptr, *vtx_off = nullptr;
  int32_t *col = nullptr, *reach = nullptr, *chain_start = nullptr, *chain_len = nullptr, *chain_l = nullptr,
          *chain_r = nullptr;
  double *bc = nullptr;
  int *err = nullptr;
  unsigned long long *counter = nullptr;
  // PLAIN
  unsigned long long *acc = nullptr;  // [n_packed][kAccDigits] fixed-point BC counters (folded into bc per launch)
  bcg::PlainItem *items = nullptr;
  int64_t n_items = 0;
  int32_t *ws_i = nullptr, *epochs = nullptr;
  double *ws_f = nullptr;
  int64_t ws_n = 0;
  int grid = 0, block = 1024;
  // small-BCC schedule (BATCHED plans): units [n_bat + n_items, ...) are its
  // items, those of the warp class first, then those of the CTA class
  bcg::TileItem *titems = nullptr;
  std::vector<bcg::TileItem> h_titems;
  int64_t n_titems = 0;
  unsigned char *slices = nullptr;
  int64_t *slice_off = nullptr;
  int32_t *slice_bytes = nullptr;
  int32_t *tws_lv = nullptr;  // warp class: level offsets per warp slot
  double *tws_P = nullptr;    // CTA class: FP64 partial BC row per CTA
  int64_t tcap_P = 0;
  // one launch per class and shared-memory bucket (the CTA class in buckets
  // by resident CTAs per SM, so that small BCCs are not run at the
  // occupancy of the largest)
  struct TileLaunch {
    int cls = 0;
    int64_t i0 = 0, i1 = 0;  // its items in h_titems
    int32_t nmax = 0, slice_max = 0;
    size_t smem = 0;
    int grid = 0;
  };
  std::vector<TileLaunch> tl;
  int64_t tcap = 0;
  // BATCHED: multi-source passes are units [0, n_bat); the BCCs routed to
  // the per-source schedule follow as PLAIN items
  bcg::BatchedPlan *bp = nullptr;
  int64_t n_bat = 0;
  // per-unit work (prefix sums over units)
  std::vector<int64_t> unit_sources, unit_teps, unit_bfs, unit_aux, unit_visits;
  int64_t device_bytes = 0;
  int64_t h2d_bytes = 0, d2h_bytes = 0;  // copied so far by this plan (batched tables counted in bp)
  std::vector<void *> allocs;
  // graph mode: instantiated graph and kernel-launch count per recorded unit range
  struct Recorded {
    cudaGraphExec_t exec;
    int launches;
  };
  std::map<std::pair<int64_t, int64_t>, Recorded> graphs;
};

#ifdef BCGPU_HOST_TIMERS
namespace bcg {
void host_mark(const char *name) {
  static auto last = std::chrono::steady_clock::now();
  auto now = std::chrono::steady_clock::now();
  fprintf(stderr, "[host] %-28s %9.2f ms\n", name, std::chrono::duration<double, std::milli>(now - last).count());
  last = now;
}
}
#endif
namespace {

thread_local std::string g_create_err;

int fail(bc_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  else g_create_err = msg;
  return code;
}

int cuda_fail(bc_ctx *ctx, cudaError_t e, const char *what) {
  cudaGetLastError();  // clear a sticky launch error of the calling thread
  return fail(ctx, e == cudaErrorMemoryAllocation ? BCGPU_ENOMEM : BCGPU_ECUDA,
              std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CK(ctx, call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// Runs an entry point's body; a host allocation that throws becomes
// BCGPU_ENOMEM, so no C++ exception leaves the C ABI.
template <class F>
int guard(bc_ctx *ctx, F &&body) {
  try {
    return body();
  } catch (const std::bad_alloc &) {
    return fail(ctx, BCGPU_ENOMEM, "host allocation failed");
  }
}

// Device memory from the context's pool, ordered on its stream. When the
// pool cannot grow, its unused reserve is trimmed once and the allocation
// retried (fragments a larger earlier plan left behind).
cudaError_t pool_alloc(bc_ctx *ctx, void **ptr, size_t bytes) {
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, ctx->pool, ctx->stream);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    if (cudaStreamSynchronize(ctx->stream) == cudaSuccess && cudaMemPoolTrimTo(ctx->pool, 0) == cudaSuccess)
      e = cudaMallocFromPoolAsync(ptr, bytes, ctx->pool, ctx->stream);
  }
  return e;
}

// Bytes the context's pool holds in reserve (freed by earlier plans, not
// yet returned to the device): available to a new plan of this context.
int64_t pool_spare(const bc_ctx *ctx) {
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? (int64_t)(reserved - used) : 0;
}

template <typename T>
int dalloc(bc_plan *p, T **ptr, int64_t count) {
  size_t bytes = sizeof(T) * (size_t)std::max<int64_t>(count, 1);
  cudaError_t e = pool_alloc(p->ctx, (void **)ptr, bytes);
  if (e != cudaSuccess) return cuda_fail(p->ctx, e, "cudaMallocFromPoolAsync");
  p->allocs.push_back(*ptr);
  p->device_bytes += (int64_t)bytes;
  return BCGPU_OK;
}

template <typename T>
int upload(bc_plan *p, T **ptr, const T *src, int64_t count) {
  int rc = dalloc(p, ptr, count);
  if (rc) return rc;
  if (count > 0) CK(p->ctx, cudaMemcpyAsync(*ptr, src, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice, p->ctx->stream));
  p->h2d_bytes += (int64_t)sizeof(T) * count;
  return BCGPU_OK;
}

int check_dev_err(bc_plan *p) {
  int h = 0;
  CK(p->ctx, cudaMemcpyAsync(&h, p->err, sizeof(int), cudaMemcpyDeviceToHost, p->ctx->stream));
  CK(p->ctx, cudaStreamSynchronize(p->ctx->stream));
  p->d2h_bytes += (int64_t)sizeof(int);
  if (h != bcg::kDevOk)
    return fail(p->ctx, bcg::dev_err_status(h), bcg::dev_err_text(h));
  if (p->bp) {
    int64_t bad = 0;
    if (bcg::batched_failed_batches(p->bp, p->ctx->stream, &bad) != BCGPU_OK)
      return fail(p->ctx, BCGPU_ECUDA, "reading batch status");
    p->d2h_bytes += bcg::batched_status_bytes(p->bp);
    if (bad)
      return fail(p->ctx, BCGPU_EOVERFLOW,
                  std::to_string(bad) + " batch(es) left FP32's exponent range in the compensated-FP32 mode; "
                  "their contributions were withheld: run with BCGPU_DELTA_FP64");
  }
  return BCGPU_OK;
}

// Structural checks of the packed input (the kernels trust these).
int validate(bc_ctx *ctx, const bc_bccs *B) {
  if (!B || B->n_bcc < 0 || B->n_orig < 0) return fail(ctx, BCGPU_EINVAL, "null or negative bccs");
  if (B->n_bcc > 0 && (!B->vtx_off || !B->row || !B->col || !B->reach || !B->orig || !B->n_plain || !B->chain_off))
    return fail(ctx, BCGPU_EINVAL, "missing bccs array");
  if (B->n_bcc == 0) return BCGPU_OK;
  if (B->vtx_off[0] != 0 || B->vtx_off[B->n_bcc] != B->n_packed || B->row[0] != 0 || B->row[B->n_packed] != B->n_arcs ||
      B->chain_off[0] != 0 || B->chain_off[B->n_bcc] != B->n_chains)
    return fail(ctx, BCGPU_EINVAL, "inconsistent bccs totals");
  // per BCC: the first failing check in the order below (0 = none); the
  // lowest failing BCC is reported, as a sequential scan would
  static const char *const kWhat[] = {"", "BCC size out of range", "n_plain out of range", "chain out of range",
                                      "chains must be sorted by left endpoint",
                                      "chain vertices do not cover the non-plain ids", "orig/reach out of range",
                                      "row offsets decrease", "negative column id", "column id outside its BCC"};
  std::vector<int8_t> bad((size_t)B->n_bcc, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
    if (nb < 3 || nb > INT32_MAX - 4) { bad[b] = 1; continue; }
    if (B->n_plain[b] < 1 || B->n_plain[b] > nb) { bad[b] = 2; continue; }
    int64_t ch = 0;
    for (int64_t c = B->chain_off[b]; c < B->chain_off[b + 1] && !bad[b]; ++c) {
      if (B->chain_start[c] < B->n_plain[b] || B->chain_len[c] < 1 || B->chain_start[c] + B->chain_len[c] > nb ||
          B->chain_l[c] < 0 || B->chain_l[c] >= B->n_plain[b] || B->chain_r[c] < 0 || B->chain_r[c] >= B->n_plain[b])
        bad[b] = 3;
      else if (c > B->chain_off[b] && B->chain_l[c] < B->chain_l[c - 1])
        bad[b] = 4;
      ch += B->chain_len[c];
    }
    if (bad[b]) continue;
    if (ch != nb - B->n_plain[b]) { bad[b] = 5; continue; }
    for (int64_t k = B->vtx_off[b]; k < B->vtx_off[b + 1]; ++k) {
      if (B->orig[k] < 0 || B->orig[k] >= B->n_orig || B->reach[k] < 0) { bad[b] = 6; break; }
      if (B->row[k + 1] < B->row[k]) { bad[b] = 7; break; }
    }
  }
  for (int32_t b = 0; b < B->n_bcc; ++b)
    if (bad[b]) return fail(ctx, BCGPU_EINVAL, kWhat[bad[b]]);
  int neg = 0;
#pragma omp parallel for schedule(static) reduction(| : neg)
  for (int64_t e = 0; e < B->n_arcs; ++e) neg |= B->col[e] < 0;
  if (neg) return fail(ctx, BCGPU_EINVAL, kWhat[8]);
  int out = 0;
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
    const int64_t e0 = B->row[B->vtx_off[b]], e1 = B->row[B->vtx_off[b + 1]];
#pragma omp parallel for schedule(static) reduction(| : out) if (e1 - e0 > (1 << 16))
    for (int64_t e = e0; e < e1; ++e) out |= B->col[e] >= nb;
    if (out) return fail(ctx, BCGPU_EINVAL, kWhat[9]);
  }
  return BCGPU_OK;
}

// Bytes of the fixed-point BC counters of n packed vertices, as dalloc sizes them.
size_t acc_bytes(int64_t n) {
  return sizeof(unsigned long long) * (size_t)std::max<int64_t>(bcg::kAccDigits * n, 1);
}

// Limit of one device-side wait, from bc_opts.wait_limit_ms.
unsigned long long wait_ns(const bc_ctx *ctx) {
  return ctx->opts.wait_limit_ms > 0 ? (unsigned long long)ctx->opts.wait_limit_ms * 1000000ull : bcg::kDefaultWaitNs;
}

// Chain vertices per PLAIN work item: bounds the longest item so the dynamic
// queue stays balanced when a hub owns thousands of chains.
constexpr int64_t kItemChainVertices = 16;

// BATCHED routing: multi-source passes pay off on large, shallow cores; a
// BCC with a core under kBatchedMinCore vertices, or with levels deeper than
// kBatchedMaxLevels (2 x eccentricity of its first vertex + longest chain),
// runs on the per-source schedule, whose rows stay in L2 and whose levels
// need no grid-wide barrier.
constexpr int32_t kBatchedMinCore = 8192;
constexpr int kBatchedMaxLevels = 96;

// Eccentricity of a BCC's local vertex 0 (BFS levels). BCCs of at least
// kParallelBfs vertices expand each level's frontier in parallel: a vertex
// joins the next level once, by compare-and-swap on its level; the levels,
// and so the eccentricity, are those of the sequential BFS.
constexpr int32_t kParallelBfs = 1 << 16;

int bcc_ecc0(const bc_bccs *B, int32_t b, std::vector<int32_t> &dist, std::vector<int32_t> &queue, bool parallel) {
  const int64_t vo = B->vtx_off[b];
  const int32_t nb = (int32_t)(B->vtx_off[b + 1] - vo);
  dist.assign((size_t)nb, -1);
  dist[0] = 0;
  if (parallel) {
    std::vector<int32_t> frontier{0}, next;
    int lev = 0;
    while (true) {
      next.clear();
#pragma omp parallel
      {
        std::vector<int32_t> mine;
#pragma omp for schedule(dynamic, 256) nowait
        for (size_t i = 0; i < frontier.size(); ++i) {
          const int32_t x = frontier[i];
          for (int64_t e = B->row[vo + x]; e < B->row[vo + x + 1]; ++e) {
            const int32_t y = B->col[e];
            if (dist[y] < 0 && __sync_bool_compare_and_swap(&dist[y], -1, lev + 1)) mine.push_back(y);
          }
        }
#pragma omp critical
        next.insert(next.end(), mine.begin(), mine.end());
      }
      if (next.empty()) return lev;
      frontier.swap(next);
      ++lev;
    }
  }
  queue.resize((size_t)nb);
  int head = 0, tail = 0, ecc = 0;
  queue[tail++] = 0;
  while (head < tail) {
    const int32_t x = queue[head++];
    ecc = std::max(ecc, dist[x]);
    for (int64_t e = B->row[vo + x]; e < B->row[vo + x + 1]; ++e) {
      const int32_t y = B->col[e];
      if (dist[y] < 0) { dist[y] = dist[x] + 1; queue[tail++] = y; }
    }
  }
  return ecc;
}

void plain_items(const bc_bccs *B, std::vector<bcg::PlainItem> &items, const std::vector<char> *skip = nullptr) {
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    if (skip && (*skip)[b]) continue;
    int64_t c = B->chain_off[b];
    const int64_t ce = B->chain_off[b + 1];
    for (int32_t s = 0; s < B->n_plain[b]; ++s) {
      int32_t own = 1;
      do {
        const int64_t c0 = c;
        int64_t verts = 0;
        while (c < ce && B->chain_l[c] == s && (verts == 0 || verts + B->chain_len[c] <= kItemChainVertices)) {
          verts += B->chain_len[c];
          ++c;
        }
        items.push_back({b, s, (int32_t)c0, (int32_t)c, own});
        own = 0;
      } while (c < ce && B->chain_l[c] == s);
    }
  }
}

// The fixed-point BC counters (once per plan), cleared.
int alloc_acc(bc_plan *p, int64_t n_packed) {
  if (p->acc) return BCGPU_OK;
  int rc = dalloc(p, &p->acc, bcg::kAccDigits * n_packed);
  if (rc) return rc;
  if (cudaMemsetAsync(p->acc, 0, acc_bytes(n_packed), p->ctx->stream) != cudaSuccess)
    return cuda_fail(p->ctx, cudaGetLastError(), "cudaMemsetAsync");
  return BCGPU_OK;
}

// Sources per small-BCC work item, at most: the CTA runs them (a warp each,
// or one after another) from one staged slice; larger BCCs are split so that
// many CTAs share them, and a class with few sources in all gets smaller
// items, so that it still has several items per resident CTA.
constexpr int32_t kTileItemSources = 128;
constexpr int64_t kTileItemsPerCta = 4;
// BCCs of up to this many vertices take the warp class (a warp per source,
// eight per CTA); larger ones the CTA class (the CTA on one source).
constexpr int64_t kTileWarpMaxVertices = 640;

// Small-BCC class of each BCC (-1: not in the schedule): BCCs off the
// multi-source passes with at most opts.tile_max vertices whose CTA fits the
// device's shared memory and whose path counts cannot overflow FP64 without
// per-level scaling -- a BFS from any vertex has at most 2 ecc(0) + 1 levels
// and a path count on level l is at most maxdeg^l, so
// (2 ecc(0) + 1) log2(maxdeg) <= 1000 keeps every count below 2^1000 (and the
// levels below the CTA class's level table). Within a class, candidates are
// taken smallest first while the launch's shared memory (sized by the class's
// largest BCC and largest slice) still fits.
// The variant whose shared memory bounds a class's (the CTA class's largest
// block has the largest work queue).
int fit_cls(int c) { return c == bcg::kTileWarp ? c : bcg::kTileCta1024; }

void route_tiles(bc_ctx *ctx, const bc_bccs *B, const std::vector<char> &on, std::vector<int8_t> &cls,
                 std::vector<int32_t> &ecc_of) {
  cls.assign((size_t)B->n_bcc, -1);
  ecc_of.assign((size_t)B->n_bcc, -1);
  const size_t lim = bcg::tile_smem_limit(ctx->device);
  if (lim == 0) return;
  const int64_t cap = std::min<int64_t>(ctx->opts.tile_max > 0 ? ctx->opts.tile_max : INT32_MAX, bcg::kTileMaxVertices);
  std::vector<int64_t> bytes((size_t)B->n_bcc, 0);
  std::vector<int8_t> want((size_t)B->n_bcc, -1);
#pragma omp parallel
  {
    std::vector<int32_t> dist, queue;
#pragma omp for schedule(dynamic, 16)
    for (int32_t b = 0; b < B->n_bcc; ++b) {
      if (on[b]) continue;
      const int64_t vo = B->vtx_off[b], nb = B->vtx_off[b + 1] - vo;
      const int64_t arcs = B->row[vo + nb] - B->row[vo];
      bytes[b] = bcg::TileSlice::bytes(nb, arcs);
      if (nb > cap) continue;
      const int c = nb <= kTileWarpMaxVertices ? bcg::kTileWarp : bcg::kTileCta;
      if (bcg::tile_smem_bytes(fit_cls(c), nb, bytes[b]) > lim) continue;
      int64_t maxdeg = 1;
      for (int64_t k = vo; k < vo + nb; ++k) maxdeg = std::max(maxdeg, B->row[k + 1] - B->row[k]);
      const int ecc = bcc_ecc0(B, b, dist, queue, false);
      ecc_of[b] = ecc;
      if ((2.0 * ecc + 1.0) * std::log2((double)std::max<int64_t>(maxdeg, 2)) <= 1000.0) want[b] = (int8_t)c;
    }
  }
  for (int c : {bcg::kTileWarp, bcg::kTileCta}) {
    std::vector<int32_t> cand;
    for (int32_t b = 0; b < B->n_bcc; ++b)
      if (want[b] == c) cand.push_back(b);
    std::stable_sort(cand.begin(), cand.end(), [&](int32_t x, int32_t y) {
      return B->vtx_off[x + 1] - B->vtx_off[x] < B->vtx_off[y + 1] - B->vtx_off[y];
    });
    int64_t nmax = 0, smax = 0;
    for (int32_t b : cand) {
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
      if (bcg::tile_smem_bytes(fit_cls(c), std::max(nmax, nb), std::max(smax, bytes[b])) > lim) break;
      nmax = std::max(nmax, nb);
      smax = std::max(smax, bytes[b]);
      cls[b] = (int8_t)c;
    }
  }
}

// Work items, staged slices and warp workspace of the small-BCC schedule.
// Launches: the warp class, then the CTA class in buckets by sources in
// flight per SM (from each BCC's own shared-memory need): 256-thread CTAs at
// 4 or more / 3 per SM; a 1024-thread CTA of four source groups (when four
// groups' arrays and the slice fit, and the BCC fits that class's level
// table); 512-thread CTAs at 2 per SM; a 1024-thread CTA of two groups; one
// 1024-thread CTA per SM. Each bucket's items are contiguous.
int build_tiles(bc_ctx *ctx, const bc_bccs *B, const std::vector<int8_t> &cls, const std::vector<int32_t> &ecc_of,
                bc_plan *p) {
  int rc = BCGPU_OK;
  std::vector<int64_t> off((size_t)B->n_bcc, -1);
  std::vector<int32_t> size((size_t)B->n_bcc, 0);
  std::vector<int8_t> bucket((size_t)B->n_bcc, -1);
  constexpr int64_t kSmPerSm = 228 * 1024, kReserved = 1024;  // shared memory per SM, per-CTA reserve
  // bucket k -> class: 0 warp, 1 / 2 CTA (4+ / 3 per SM), 3 four groups, 4 CTA-512, 5 two groups, 6 CTA-1024
  constexpr int kBucketCls[7] = {bcg::kTileWarp,    bcg::kTileCta,       bcg::kTileCta,      bcg::kTileCta1024x4,
                                 bcg::kTileCta512, bcg::kTileCta1024x2, bcg::kTileCta1024};
  const int64_t lim = (int64_t)bcg::tile_smem_limit(ctx->device);
  std::vector<int64_t> per((size_t)B->n_bcc, 0);
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    if (cls[b] < 0) continue;
    const int64_t vo = B->vtx_off[b], nb = B->vtx_off[b + 1] - vo;
    size[b] = (int32_t)bcg::TileSlice::bytes(nb, B->row[vo + nb] - B->row[vo]);
    if (cls[b] == bcg::kTileWarp) { bucket[b] = 0; continue; }
    per[b] = kSmPerSm / ((int64_t)bcg::tile_smem_bytes(bcg::kTileCta, nb, size[b]) + kReserved);
    bucket[b] = (int8_t)(per[b] >= 4 ? 1 : per[b] == 3 ? 2 : per[b] == 2 ? 4 : 6);
  }
  // the grouped classes: a BCC moves up when its groups fit and the bucket's
  // launch (sized by its largest BCC and largest slice) still fits, smallest
  // BCCs first
  auto promote = [&](int to, auto &&eligible) {
    std::vector<int32_t> cand;
    for (int32_t b = 0; b < B->n_bcc; ++b) {
      if (cls[b] < 0 || cls[b] == bcg::kTileWarp || !eligible(b)) continue;
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
      if (2 * (int64_t)ecc_of[b] + 3 >= bcg::kTileGroupMaxLevels) continue;  // levels <= 2 ecc + 1
      if ((int64_t)bcg::tile_smem_bytes(kBucketCls[to], nb, size[b]) > lim) continue;
      cand.push_back(b);
    }
    std::stable_sort(cand.begin(), cand.end(), [&](int32_t x, int32_t y) {
      return B->vtx_off[x + 1] - B->vtx_off[x] < B->vtx_off[y + 1] - B->vtx_off[y];
    });
    int64_t nmax = 0, smax = 0;
    for (int32_t b : cand) {
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
      if ((int64_t)bcg::tile_smem_bytes(kBucketCls[to], std::max(nmax, nb), std::max<int64_t>(smax, size[b])) > lim) break;
      nmax = std::max(nmax, nb);
      smax = std::max<int64_t>(smax, size[b]);
      bucket[b] = (int8_t)to;
    }
  };
  promote(3, [&](int32_t b) { return per[b] <= 3; });                    // four sources in flight, not at most three
  promote(5, [&](int32_t b) { return per[b] <= 1 && bucket[b] == 6; });  // two instead of one
  int64_t total = 0, p_rows = 1;
  for (int k = 0; k <= 6; ++k) {
    bc_plan::TileLaunch T;
    T.cls = kBucketCls[k];
    T.i0 = (int64_t)p->h_titems.size();
    int64_t nmax = 0, smax = 0, sources = 0;
    for (int32_t b = 0; b < B->n_bcc; ++b) {
      if (bucket[b] != k) continue;
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
      nmax = std::max(nmax, nb);
      smax = std::max<int64_t>(smax, size[b]);
      sources += nb;
    }
    if (sources == 0) continue;
    T.nmax = (int32_t)nmax;
    T.slice_max = (int32_t)smax;
    T.smem = bcg::tile_smem_bytes(T.cls, nmax, smax);
    const int per_sm = bcg::tile_ctas_per_sm(T.cls, T.smem);
    if (per_sm < 1) return fail(ctx, BCGPU_ECUDA, "small-BCC schedule: no CTA fits an SM");
    T.grid = ctx->sms * per_sm;
    const int groups = bcg::tile_groups(T.cls);
    if (T.cls != bcg::kTileWarp) p_rows = std::max<int64_t>(p_rows, (int64_t)T.grid * groups);
    // a warp-class item feeds 8 warps, a grouped CTA's item its groups
    const int64_t floor_items = T.cls == bcg::kTileWarp ? bcg::kTileWarps : groups;
    const int32_t per_item = (int32_t)std::max<int64_t>(
        floor_items, std::min<int64_t>(kTileItemSources, sources / ((int64_t)T.grid * kTileItemsPerCta)));
    for (int32_t b = 0; b < B->n_bcc; ++b) {
      if (bucket[b] != k) continue;
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b];
      off[b] = total;
      total += size[b];
      for (int32_t s0 = 0; s0 < nb; s0 += per_item)
        p->h_titems.push_back({b, s0, (int32_t)std::min<int64_t>(nb, s0 + per_item), 0});
    }
    T.i1 = (int64_t)p->h_titems.size();
    if (T.cls == bcg::kTileWarp) p->tcap = nmax + 2;
    p->tl.push_back(T);
  }
  // slices: local row offsets (uint16 when narrow, else int32), neighbours
  // (uint16), 16-byte aligned parts; bit 0 of a narrow slice's offset set
  std::vector<unsigned char> blob((size_t)std::max<int64_t>(total, 16), 0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    if (cls[b] < 0) continue;
    const int64_t vo = B->vtx_off[b], nb = B->vtx_off[b + 1] - vo, e0 = B->row[vo];
    const int64_t arcs = B->row[vo + nb] - e0;
    const bool narrow = bcg::TileSlice::narrow(arcs);
    unsigned char *base = blob.data() + off[b];
    uint16_t *C = reinterpret_cast<uint16_t *>(base + bcg::TileSlice::col_at(nb, narrow));
    for (int64_t v = 0; v <= nb; ++v) {
      if (narrow) reinterpret_cast<uint16_t *>(base)[v] = (uint16_t)(B->row[vo + v] - e0);
      else reinterpret_cast<int32_t *>(base)[v] = (int32_t)(B->row[vo + v] - e0);
    }
    for (int64_t e = 0; e < arcs; ++e) C[e] = (uint16_t)B->col[e0 + e];
  }
  std::vector<int64_t> off_flag(off);  // what the kernels read: offset | narrow
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    if (cls[b] < 0) continue;
    const int64_t vo = B->vtx_off[b], nb = B->vtx_off[b + 1] - vo;
    if (bcg::TileSlice::narrow(B->row[vo + nb] - B->row[vo])) off_flag[b] |= 1;
  }
  p->n_titems = (int64_t)p->h_titems.size();
  int warp_grid = 1;
  for (const auto &T : p->tl) {
    if (T.cls == bcg::kTileWarp) warp_grid = T.grid;
    else p->tcap_P = std::max<int64_t>(p->tcap_P, T.nmax);
  }
  const int64_t slots = (int64_t)warp_grid * bcg::kTileWarps;
  p->tcap = std::max<int64_t>(p->tcap, 2);
  if ((rc = upload(p, &p->slices, blob.data(), (int64_t)blob.size())) ||
      (rc = upload(p, &p->slice_off, off_flag.data(), B->n_bcc)) ||
      (rc = upload(p, &p->slice_bytes, size.data(), B->n_bcc)) ||
      (rc = upload(p, &p->titems, p->h_titems.data(), p->n_titems)) || (rc = dalloc(p, &p->tws_lv, slots * p->tcap)) ||
      (rc = dalloc(p, &p->tws_P, p_rows * std::max<int64_t>(p->tcap_P, 1))) ||
      (rc = alloc_acc(p, B->n_packed)))
    return rc;
  for (const auto &it : p->h_titems) {
    const int64_t vo = B->vtx_off[it.bcc], nb = B->vtx_off[it.bcc + 1] - vo;
    const int64_t arcs = B->row[vo + nb] - B->row[vo];
    const int64_t src = it.s1 - it.s0;
    p->unit_sources.push_back(p->unit_sources.back() + src);
    p->unit_teps.push_back(p->unit_teps.back() + src * arcs);
    p->unit_bfs.push_back(p->unit_bfs.back() + src);
    p->unit_aux.push_back(p->unit_aux.back());
    p->unit_visits.push_back(p->unit_visits.back() + src * nb);
  }
  return BCGPU_OK;
}

// Source orders of the BCCs in multi-source passes, computed on one host
// thread (each BCC up to the passes the plan fills, as batched_create would).
// get() waits for the thread; a host allocation that failed there is
// rethrown as std::bad_alloc. The destructor waits too, so no exit path
// leaves the thread running.
struct SourceOrders {
  std::vector<std::vector<int32_t>> by_bcc;
  std::thread th;
  bool failed = false;
  void start(const bc_bccs *B, const std::vector<char> &on, int width, int64_t fill_begin, int64_t fill_end) {
    by_bcc.resize((size_t)B->n_bcc);
    std::vector<std::pair<int32_t, int64_t>> jobs;  // (BCC, entries needed), as batched_build counts passes
    int64_t bat0 = 0;
    for (int32_t b = 0; b < B->n_bcc; ++b) {
      if (!on[b]) continue;
      const int64_t nb = B->vtx_off[b + 1] - B->vtx_off[b], nbat = (nb + width - 1) / width;
      const int64_t jf0 = std::min(nbat, std::max<int64_t>(0, fill_begin - bat0));
      const int64_t jf1 = std::max(jf0, std::min(nbat, fill_end - bat0));
      if (jf1 > 0) jobs.emplace_back(b, std::min<int64_t>(nb, jf1 * width));
      bat0 += nbat;
    }
    th = std::thread([this, B, width, jobs = std::move(jobs)] {
      try {
#ifdef BCGPU_HOST_TIMERS
        auto t0 = std::chrono::steady_clock::now();
#endif
        for (const auto &j : jobs) bcg::batched_source_order(B, j.first, width, j.second, by_bcc[(size_t)j.first]);
#ifdef BCGPU_HOST_TIMERS
        fprintf(stderr, "[host] order thread %.2f ms\n",
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
#endif
      } catch (const std::bad_alloc &) {
        failed = true;
      }
    });
  }
  const std::vector<int32_t> &get(int32_t b) {
    if (th.joinable()) th.join();
    if (failed) throw std::bad_alloc();
    return by_bcc[(size_t)b];
  }
  ~SourceOrders() {
    if (th.joinable()) th.join();
  }
};

// Fills plan p (allocated by create_plan, which releases it on any failure).
// fill_begin/fill_end: the multi-source passes (units) whose tables are built
// (a one-shot call that runs only those); default all.
int build_plan(bc_ctx *ctx, const bc_bccs *B, const std::vector<bcg::PlainItem> *override_items, bc_plan *p,
               int64_t fill_begin = 0, int64_t fill_end = INT64_MAX) {
  int rc = BCGPU_OK;
  auto bail = [](int code) { return code; };
  p->n_orig = B->n_orig;
  p->n_packed = B->n_packed;
  p->orig.assign(B->orig, B->orig + B->n_packed);
  if (B->art) p->art.assign(B->art, B->art + B->n_orig);
  p->h_vtx_off.assign(B->vtx_off, B->vtx_off + B->n_bcc + 1);
  p->h_chain_off.assign(B->chain_off, B->chain_off + B->n_bcc + 1);
  p->h_n_plain.assign(B->n_plain, B->n_plain + B->n_bcc);
  p->h_chain_start.assign(B->chain_start, B->chain_start + B->n_chains);
  p->h_chain_len.assign(B->chain_len, B->chain_len + B->n_chains);
  int64_t nb_max = 0;
  for (int32_t b = 0; b < B->n_bcc; ++b) nb_max = std::max(nb_max, B->vtx_off[b + 1] - B->vtx_off[b]);

  // BATCHED: which BCCs take multi-source passes (the others: per-source items)
  std::vector<char> on;
  std::vector<int32_t> ecc0;  // eccentricity of each BCC's local vertex 0 (the batched plan reuses it)
  int64_t n_on = 0;
  if (p->mode == BCGPU_MODE_BATCHED) {
    on.assign((size_t)B->n_bcc, 1);
    ecc0.assign((size_t)B->n_bcc, -1);
    if (ctx->opts.plain_core >= 0) {
      const int32_t min_core = ctx->opts.plain_core > 0 ? ctx->opts.plain_core : kBatchedMinCore;
      auto route = [&](int32_t b, std::vector<int32_t> &dist, std::vector<int32_t> &queue, bool parallel) {
        if (B->n_plain[b] < min_core) { on[b] = 0; return; }
        int kmax = 0;
        for (int64_t c = B->chain_off[b]; c < B->chain_off[b + 1]; ++c) kmax = std::max(kmax, B->chain_len[c]);
        ecc0[b] = bcc_ecc0(B, b, dist, queue, parallel);
        on[b] = 2 * ecc0[b] + kmax <= kBatchedMaxLevels;
      };
      auto big = [&](int32_t b) { return B->vtx_off[b + 1] - B->vtx_off[b] >= kParallelBfs; };
      {
        std::vector<int32_t> dist, queue;
        for (int32_t b = 0; b < B->n_bcc; ++b)
          if (big(b)) route(b, dist, queue, true);  // one BCC at a time, its levels in parallel
      }
#pragma omp parallel
      {
        std::vector<int32_t> dist, queue;
#pragma omp for schedule(dynamic, 1)
        for (int32_t b = 0; b < B->n_bcc; ++b)
          if (!big(b)) route(b, dist, queue, false);
      }
    }
    for (char x : on) n_on += x;
  }
  HOST_MARK("route");
  // The multi-source passes' source orders (a sequential greedy over each
  // BCC's arcs) are computed on a host thread while the graph is uploaded
  // and the rest of the plan is built; batched_create waits for them.
  SourceOrders orders;
  if (p->mode == BCGPU_MODE_BATCHED && n_on > 0) orders.start(B, on, bcg::batched_width(ctx->opts.batch_width),
                                                              fill_begin, fill_end);
  if ((rc = upload(p, &p->row, B->row, B->n_packed + 1)) || (rc = upload(p, &p->vtx_off, B->vtx_off, B->n_bcc + 1)) ||
      (rc = upload(p, &p->col, B->col, B->n_arcs)) || (rc = upload(p, &p->reach, B->reach, B->n_packed)) ||
      (rc = upload(p, &p->chain_start, B->chain_start, B->n_chains)) ||
      (rc = upload(p, &p->chain_len, B->chain_len, B->n_chains)) ||
      (rc = upload(p, &p->chain_l, B->chain_l, B->n_chains)) || (rc = upload(p, &p->chain_r, B->chain_r, B->n_chains)) ||
      (rc = dalloc(p, &p->bc, B->n_packed)) || (rc = dalloc(p, &p->err, 1)) || (rc = dalloc(p, &p->counter, 1)))
    return bail(rc);
  if (cudaMemsetAsync(p->bc, 0, sizeof(double) * (size_t)std::max<int64_t>(B->n_packed, 1), ctx->stream) != cudaSuccess ||
      cudaMemsetAsync(p->err, 0, sizeof(int), ctx->stream) != cudaSuccess)
    return bail(cuda_fail(ctx, cudaGetLastError(), "cudaMemsetAsync"));
  HOST_MARK("uploads");

  size_t free_b = 0, total_b = 0;
  CK(ctx, cudaMemGetInfo(&free_b, &total_b));
  const double avail_b = (double)free_b + (double)pool_spare(ctx);
  int64_t limit = ctx->opts.workspace_limit > 0 ? ctx->opts.workspace_limit : (int64_t)(0.8 * avail_b);
  // BATCHED: BCCs off the multi-source passes that fit the small-BCC schedule
  std::vector<int8_t> tile;
  std::vector<int32_t> tile_ecc;
  int64_t n_tile = 0;
  if (p->mode == BCGPU_MODE_BATCHED && ctx->opts.tile_max >= 0 && n_on < B->n_bcc) {
    route_tiles(ctx, B, on, tile, tile_ecc);
    for (int8_t x : tile) n_tile += x >= 0;
  }
  HOST_MARK("route_tiles");
  std::vector<bcg::PlainItem> items;
  if (p->mode == BCGPU_MODE_PLAIN) {
    if (override_items) items = *override_items;
    else plain_items(B, items);
  } else if (n_on + n_tile < B->n_bcc) {
    std::vector<char> skip(on);
    for (int32_t b = 0; b < B->n_bcc; ++b) skip[b] |= n_tile ? tile[b] >= 0 : 0;
    plain_items(B, items, &skip);
  }
  if (p->mode == BCGPU_MODE_BATCHED && n_on > 0) {
    bcg::BatchedConfig cfg;
    cfg.width = ctx->opts.batch_width;
    cfg.delta_fp32c = ctx->opts.delta == BCGPU_DELTA_FP32C;
    cfg.sms = ctx->sms;
    cfg.limit_bytes = limit - p->device_bytes;
    cfg.rescale_exp = ctx->opts.rescale_exp;
    cfg.wait_ns = wait_ns(ctx);
    cfg.pool = ctx->pool;
    cfg.order_of = [&orders](int32_t b) -> const std::vector<int32_t> & { return orders.get(b); };
    cfg.bccs_on = &on;
    cfg.ecc0 = &ecc0;
    cfg.fill_begin = fill_begin;
    cfg.fill_end = fill_end;
    std::string msg;
    rc = bcg::batched_create(B, cfg, p->row, p->col, p->reach, p->vtx_off, p->chain_start, p->chain_len, p->chain_l,
                             p->chain_r, p->bc, p->err, ctx->stream, &p->bp, &msg);
    HOST_MARK("batched_create");
    if (rc) return bail(fail(ctx, rc, "batched plan: " + msg));
    p->device_bytes += bcg::batched_device_bytes(p->bp);
    p->d2h_bytes += bcg::batched_d2h_bytes(p->bp);
    bcg::batched_unit_work(p->bp, p->unit_sources, p->unit_teps, p->unit_bfs, p->unit_aux, p->unit_visits);
    p->n_bat = (int64_t)p->unit_sources.size() - 1;
  } else {
    p->unit_sources.assign(1, 0);
    p->unit_teps.assign(1, 0);
    p->unit_bfs.assign(1, 0);
    p->unit_aux.assign(1, 0);
    p->unit_visits.assign(1, 0);
  }
  if (!items.empty() || p->mode == BCGPU_MODE_PLAIN) {
    p->n_items = (int64_t)items.size();
    int64_t nb_plain = 0;
    for (size_t i = 0; i < items.size(); ++i) {
      const auto &it = items[i];
      int64_t src = it.own ? 1 : 0, aux = it.own ? 0 : 1;
      int32_t prev = -1;
      for (int32_t c = it.c0; c < it.c1; ++c) {
        src += B->chain_len[c];
        if (B->chain_r[c] != prev) { ++aux; prev = B->chain_r[c]; }
      }
      const int64_t nb = B->vtx_off[it.bcc + 1] - B->vtx_off[it.bcc];
      nb_plain = std::max(nb_plain, nb);
      const int64_t arcs = B->row[B->vtx_off[it.bcc + 1]] - B->row[B->vtx_off[it.bcc]];
      p->unit_sources.push_back(p->unit_sources.back() + src);
      p->unit_teps.push_back(p->unit_teps.back() + src * arcs);
      p->unit_bfs.push_back(p->unit_bfs.back() + (it.own ? 1 : 0));
      p->unit_aux.push_back(p->unit_aux.back() + aux);
      p->unit_visits.push_back(p->unit_visits.back() + src * nb);
    }
    if ((rc = upload(p, &p->items, items.data(), (int64_t)items.size()))) return bail(rc);
    p->h_items = items;
    p->ws_n = (p->mode == BCGPU_MODE_PLAIN ? nb_max : nb_plain) + 2;
    if ((rc = alloc_acc(p, B->n_packed))) return bail(rc);
    const int64_t per_slot = p->ws_n * (bcg::kWsIntRows * 4 + bcg::kWsDblRows * 8);
    // Four 256-thread CTAs per SM (four sources in flight) when their rows
    // fit the budget, else two of 512, else one of 1024 per SM; with
    // plain_ctas_per_sm 8 or 16, CTAs of 128 or 64 threads are tried first.
    int64_t avail = limit - p->device_bytes - 64 * (int64_t)ctx->sms;
    if (avail < 2 * per_slot) return bail(fail(ctx, BCGPU_ENOMEM, "workspace for the largest BCC exceeds the limit"));
    int grid = 0;
    const int first = ctx->opts.plain_ctas_per_sm > 4 ? 1024 / ctx->opts.plain_ctas_per_sm : 256;
    for (int block : {64, 128, 256, 512, 1024}) {
      if (block < first) continue;
      const int want = ctx->sms * (1024 / block);
      grid = (int)std::min<int64_t>(want, avail / per_slot - 1);
      p->block = block;
      if (grid == want) break;
    }
    p->grid = std::max(1, grid);
    const int64_t slots = p->grid + 1;  // + the row-export slot
    if ((rc = dalloc(p, &p->ws_i, slots * bcg::kWsIntRows * p->ws_n)) ||
        (rc = dalloc(p, &p->ws_f, slots * bcg::kWsDblRows * p->ws_n)) || (rc = dalloc(p, &p->epochs, 2 * slots)))
      return bail(rc);
    if (cudaMemsetAsync(p->ws_f, 0, sizeof(double) * (size_t)(slots * bcg::kWsDblRows * p->ws_n), ctx->stream) !=
        cudaSuccess)  // row records: stamp 0, unvisited
      return bail(cuda_fail(ctx, cudaGetLastError(), "cudaMemsetAsync"));
    std::vector<int32_t> ep((size_t)(2 * slots), 1);
    CK(ctx, cudaMemcpyAsync(p->epochs, ep.data(), sizeof(int32_t) * ep.size(), cudaMemcpyHostToDevice, ctx->stream));
    p->h2d_bytes += (int64_t)(sizeof(int32_t) * ep.size());
  }
  HOST_MARK("plain items+ws");
  if (n_tile && (rc = build_tiles(ctx, B, tile, tile_ecc, p))) return bail(rc);
  CK(ctx, cudaStreamSynchronize(ctx->stream));
  HOST_MARK("tiles+sync");
  return BCGPU_OK;
}

// Validates the input and builds a plan; on any failure -- a status code, or
// a host allocation that throws -- the partial plan and its device buffers are
// released and no C++ exception leaves the library.
int create_plan(bc_ctx *ctx, const bc_bccs *B, const std::vector<bcg::PlainItem> *override_items, bc_plan **out,
                int64_t fill_begin = 0, int64_t fill_end = INT64_MAX) {
  bc_plan *p = nullptr;
  int rc;
  try {
    rc = validate(ctx, B);
    if (rc == BCGPU_OK) {
      const cudaError_t e = cudaSetDevice(ctx->device);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
      p = new bc_plan;
      p->ctx = ctx;
      p->mode = ctx->opts.mode;
      rc = build_plan(ctx, B, override_items, p, fill_begin, fill_end);
      if (rc == BCGPU_OK) ctx->plans.insert(p);
    }
  } catch (const std::bad_alloc &) {
    rc = fail(ctx, BCGPU_ENOMEM, "host allocation failed while building the plan");
  }
  if (rc != BCGPU_OK) {
    if (p) bc_plan_destroy(p);
    return rc;
  }
  *out = p;
  return BCGPU_OK;
}

}  // namespace

namespace bcg {
void ctx_device_stream(const bc_ctx *ctx, int *device, cudaStream_t *stream, cudaEvent_t *ev0, cudaEvent_t *ev1) {
  *device = ctx->device;
  *stream = ctx->stream;
  *ev0 = ctx->ev0;
  *ev1 = ctx->ev1;
}
void ctx_set_error(bc_ctx *ctx, const char *msg) { ctx->err = msg; }
const char *dev_err_text(int code) {
  switch (code) {
    case kDevDisconnected: return "a BCC is not connected (row did not reach every vertex)";
    case kDevWorkspace: return "BCC larger than the kernel workspace";
    case kDevTimeout: return "device-side wait exceeded its iteration limit";
    case kDevBadItem: return "work item references data out of range";
    case kDevOverflow:
      return "a path count or dependency left FP64's range despite per-level power-of-two scaling, or a BC "
             "contribution exceeded the fixed-point accumulator";
    default: return "unknown device error";
  }
}

int dev_err_status(int code) {
  return code == kDevTimeout ? BCGPU_ETIMEOUT : code == kDevOverflow ? BCGPU_EOVERFLOW : BCGPU_EINVAL;
}

}  // namespace bcg

extern "C" void bc_default_opts(bc_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = -1;
  o->mode = BCGPU_MODE_BATCHED;
  o->delta = BCGPU_DELTA_FP32C;
  o->batch_width = 0;
  o->lazy_tables = 1;
}

extern "C" int bc_create(const bc_opts *opts, bc_ctx **out) {
  if (!out) return fail(nullptr, BCGPU_EINVAL, "null out");
  bc_opts o;
  if (opts) o = *opts;
  else bc_default_opts(&o);
  if (o.mode != BCGPU_MODE_PLAIN && o.mode != BCGPU_MODE_BATCHED) return fail(nullptr, BCGPU_EINVAL, "bad mode");
  if (o.delta != BCGPU_DELTA_FP64 && o.delta != BCGPU_DELTA_FP32C) return fail(nullptr, BCGPU_EINVAL, "bad delta");
  if (o.batch_width < 0 || o.batch_width > 1024 || (o.batch_width % 32) != 0)
    return fail(nullptr, BCGPU_EINVAL, "batch_width must be a multiple of 32 in [0, 1024]");
  if (o.plain_ctas_per_sm != 0 && o.plain_ctas_per_sm != 4 && o.plain_ctas_per_sm != 8 && o.plain_ctas_per_sm != 16)
    return fail(nullptr, BCGPU_EINVAL, "plain_ctas_per_sm must be 0, 4, 8 or 16");
  if (o.lazy_tables != 0 && o.lazy_tables != 1) return fail(nullptr, BCGPU_EINVAL, "lazy_tables must be 0 or 1");
  if (o.wait_limit_ms < 0) return fail(nullptr, BCGPU_EINVAL, "wait_limit_ms must be >= 0");
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(nullptr, BCGPU_ECUDA, std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none"));
  int dev = o.device;
  if (dev < 0) {  // highest compute capability, as the reference's choose_device (Codes/begin_gpupgm.cu:8-39)
    int best = -1;
    for (int i = 0; i < count; ++i) {
      cudaDeviceProp pr;
      if (cudaGetDeviceProperties(&pr, i) != cudaSuccess) continue;
      int cc = pr.major * 10 + pr.minor;
      if (cc > best) { best = cc; dev = i; }
    }
  }
  if (dev < 0 || dev >= count) return fail(nullptr, BCGPU_EINVAL, "device ordinal out of range");
  bc_ctx *ctx = new (std::nothrow) bc_ctx;
  if (!ctx) return fail(nullptr, BCGPU_ENOMEM, "host allocation");
  ctx->opts = o;
  ctx->device = dev;
  auto bad = [&](cudaError_t err, const char *what) {
    cuda_fail(nullptr, err, what);
    bc_destroy(ctx);
    return BCGPU_ECUDA;
  };
  if ((e = cudaSetDevice(dev)) != cudaSuccess) return bad(e, "cudaSetDevice");
  cudaDeviceProp pr;
  if ((e = cudaGetDeviceProperties(&pr, dev)) != cudaSuccess) return bad(e, "cudaGetDeviceProperties");
  if (pr.major < 10) {
    g_create_err = std::string("device ") + pr.name + " is not sm_100 (kernels are built for sm_100a only)";
    bc_destroy(ctx);
    return BCGPU_ECUDA;
  }
  ctx->sms = pr.multiProcessorCount;
  if (o.stream) ctx->stream = (cudaStream_t)o.stream;
  else {
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
      return bad(e, "cudaStreamCreate");
    ctx->own_stream = true;
  }
  if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev1)) != cudaSuccess)
    return bad(e, "cudaEventCreate");
  cudaMemPoolProps pp{};
  pp.allocType = cudaMemAllocationTypePinned;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = dev;
  if ((e = cudaMemPoolCreate(&ctx->pool, &pp)) != cudaSuccess) return bad(e, "cudaMemPoolCreate");
  uint64_t keep = ~(uint64_t)0;  // never release reserve at a synchronisation: plans reuse it
  if ((e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
    return bad(e, "cudaMemPoolSetAttribute");
  *out = ctx;
  return BCGPU_OK;
}

extern "C" void bc_destroy(bc_ctx *ctx) {
  if (!ctx) return;
  while (!ctx->plans.empty()) bc_plan_destroy(*ctx->plans.begin());
  cudaSetDevice(ctx->device);
  if (ctx->pool) {
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);  // frees ordered on the stream have completed
    cudaMemPoolDestroy(ctx->pool);
  }
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

extern "C" const char *bc_last_error(const bc_ctx *ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

extern "C" int bc_plan_create(bc_ctx *ctx, const bc_bccs *bccs, bc_plan **out) {
  if (!ctx || !out) return fail(ctx, BCGPU_EINVAL, "null argument");
  return create_plan(ctx, bccs, nullptr, out);
}

extern "C" int bc_autotune_width(bc_ctx *ctx, const bc_bccs *bccs, int32_t passes, int32_t *width, double *gteps_out) {
  if (!ctx || !bccs || !width) return fail(ctx, BCGPU_EINVAL, "null argument");
  if (ctx->opts.mode != BCGPU_MODE_BATCHED) return fail(ctx, BCGPU_EINVAL, "autotuning needs a BATCHED context");
  const int cand[4] = {128, 256, 512, 1024};
  const int32_t saved = ctx->opts.batch_width;
  double best = -1.0;
  *width = 0;
  for (int i = 0; i < 4; ++i) {
    if (gteps_out) gteps_out[i] = 0.0;
    ctx->opts.batch_width = cand[i];
    bc_plan *p = nullptr;
    int rc = create_plan(ctx, bccs, nullptr, &p);
    if (rc == BCGPU_ENOMEM) continue;  // this width does not fit
    if (rc) { ctx->opts.batch_width = saved; return rc; }
    if (p->n_bat == 0) { bc_plan_destroy(p); break; }
    const int64_t k = std::max<int64_t>(1, std::min<int64_t>(std::max(passes, 1), p->n_bat));
    const int64_t b0 = std::max<int64_t>(0, p->n_bat / 2 - k / 2), b1 = std::min(p->n_bat, b0 + k);
    bc_stats st;
    rc = bc_plan_run(p, b0, std::min(b1, b0 + 1), nullptr);  // warm-up
    if (!rc) rc = bc_plan_run(p, b0, b1, &st);
    bc_plan_destroy(p);
    if (rc) { ctx->opts.batch_width = saved; return rc; }
    const double g = st.kernel_ms > 0 ? (double)st.teps_edges / (st.kernel_ms * 1e6) : 0.0;
    if (gteps_out) gteps_out[i] = g;
    if (g > best) { best = g; *width = cand[i]; }
  }
  ctx->opts.batch_width = saved;
  return BCGPU_OK;
}

namespace {

// One thread waits on *flag (which nothing sets) with the library's bounded wait.
__global__ void wait_probe_kernel(const unsigned int *flag, int *err, unsigned long long limit_ns) {
  if (threadIdx.x == 0) bcg::wait_while_equal_probe(flag, err, limit_ns);
}

}  // namespace

extern "C" int bc_wait_probe(bc_ctx *ctx, int32_t limit_ms, double *waited_ms) {
  if (!ctx) return fail(ctx, BCGPU_EINVAL, "null context");
  if (limit_ms <= 0) return fail(ctx, BCGPU_EINVAL, "limit_ms must be > 0");
  CK(ctx, cudaSetDevice(ctx->device));
  unsigned int *buf = nullptr;  // [0]: the flag, [1]: the error word
  CK(ctx, cudaMalloc((void **)&buf, 2 * sizeof(unsigned int)));
  cudaError_t e = cudaMemsetAsync(buf, 0, 2 * sizeof(unsigned int), ctx->stream);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, ctx->stream);
  if (e == cudaSuccess) {
    wait_probe_kernel<<<1, 32, 0, ctx->stream>>>(buf, reinterpret_cast<int *>(buf + 1),
                                                 (unsigned long long)limit_ms * 1000000ull);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, ctx->stream);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, buf + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  cudaFree(buf);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "wait probe");
  if (waited_ms) *waited_ms = ms;
  if (h != bcg::kDevOk) return fail(ctx, bcg::dev_err_status(h), bcg::dev_err_text(h));
  return BCGPU_OK;
}

extern "C" void bc_plan_destroy(bc_plan *p) {
  if (!p) return;
  p->ctx->plans.erase(p);
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  for (auto &g : p->graphs) cudaGraphExecDestroy(g.second.exec);
  if (p->bp) bcg::batched_destroy(p->bp);
  for (void *a : p->allocs) cudaFreeAsync(a, p->ctx->stream);  // back to the context's pool
  delete p;
}

extern "C" int64_t bc_plan_num_units(const bc_plan *p) {
  return p ? (int64_t)p->unit_sources.size() - 1 : 0;
}

extern "C" int bc_plan_unit_work(const bc_plan *p, int64_t begin, int64_t end, int64_t *sources, int64_t *teps,
                                 int64_t *visits) {
  if (!p) return BCGPU_EINVAL;
  const int64_t n = bc_plan_num_units(p);
  if (begin < 0 || end < begin || end > n) return fail(p->ctx, BCGPU_EINVAL, "unit range out of bounds");
  if (sources) *sources = p->unit_sources[end] - p->unit_sources[begin];
  if (teps) *teps = p->unit_teps[end] - p->unit_teps[begin];
  if (visits) *visits = p->unit_visits[end] - p->unit_visits[begin];
  return BCGPU_OK;
}

extern "C" int64_t bc_plan_device_bytes(const bc_plan *p) { return p ? p->device_bytes : 0; }

extern "C" int bc_plan_tile_launches(const bc_plan *p, int32_t *cls, int32_t *grid, int32_t cap) {
  if (!p || cap < 0 || (cap > 0 && (!cls || !grid))) return BCGPU_EINVAL;
  const int32_t n = (int32_t)p->tl.size();
  for (int32_t i = 0; i < std::min(n, cap); ++i) {
    cls[i] = p->tl[(size_t)i].cls;
    grid[i] = p->tl[(size_t)i].grid;
  }
  return n;
}
extern "C" int bc_plan_concurrency(const bc_plan *p) { return !p ? 0 : p->mode == BCGPU_MODE_BATCHED ? 1 : p->grid; }

extern "C" int64_t bc_plan_unit_sources(const bc_plan *p, int64_t begin, int64_t end, int64_t *out, int64_t cap) {
  if (!p) return -BCGPU_EINVAL;
  const int64_t n = bc_plan_num_units(p);
  if (begin < 0 || end < begin || end > n) return -BCGPU_EINVAL;
  std::vector<int64_t> ids;
  try {
    if (p->bp && begin < p->n_bat) bcg::batched_unit_sources(p->bp, begin, std::min(end, p->n_bat), ids);
    for (int64_t i = std::max(begin, p->n_bat) - p->n_bat; i < std::min(end - p->n_bat, p->n_items); ++i) {
      const auto &it = p->h_items[i];  // per-source items
      const int64_t vo = p->h_vtx_off[it.bcc];
      if (it.own) ids.push_back(vo + it.src);
      for (int32_t c = it.c0; c < it.c1; ++c)
        for (int32_t k = 0; k < p->h_chain_len[c]; ++k) ids.push_back(vo + p->h_chain_start[c] + k);
    }
    for (int64_t i = std::max(begin, p->n_bat + p->n_items) - p->n_bat - p->n_items;
         i < end - p->n_bat - p->n_items; ++i) {  // small-BCC items
      const auto &it = p->h_titems[i];
      for (int32_t s = it.s0; s < it.s1; ++s) ids.push_back(p->h_vtx_off[it.bcc] + s);
    }
  } catch (const std::bad_alloc &) {
    return -BCGPU_ENOMEM;
  }
  for (int64_t i = 0; i < (int64_t)ids.size() && i < cap; ++i) out[i] = ids[i];
  return (int64_t)ids.size();
}

extern "C" int bc_plan_reset(bc_plan *p) {
  if (!p) return BCGPU_EINVAL;
  CK(p->ctx, cudaSetDevice(p->ctx->device));
  CK(p->ctx, cudaMemsetAsync(p->bc, 0, sizeof(double) * (size_t)std::max<int64_t>(p->n_packed, 1), p->ctx->stream));
  if (p->acc)  // folded after every launch, so normally zero already; cleared after a failed run
    CK(p->ctx, cudaMemsetAsync(p->acc, 0, acc_bytes(p->n_packed), p->ctx->stream));
  CK(p->ctx, cudaMemsetAsync(p->err, 0, sizeof(int), p->ctx->stream));
  return BCGPU_OK;
}

namespace {

// Arguments of the per-source kernel over this plan's buffers (item range unset).
bcg::PlainArgs plain_args(const bc_plan *p) {
  bcg::PlainArgs a{};
  a.row = p->row; a.col = p->col; a.reach = p->reach; a.vtx_off = p->vtx_off;
  a.chain_start = p->chain_start; a.chain_len = p->chain_len; a.chain_l = p->chain_l; a.chain_r = p->chain_r;
  a.items = p->items; a.next_item = p->counter; a.acc = p->acc;
  a.ws_i = p->ws_i; a.ws_f = p->ws_f; a.ws_n = p->ws_n; a.epochs = p->epochs; a.rows_slot = p->grid;
  a.rescale_exp = p->ctx->opts.rescale_exp > 0 ? p->ctx->opts.rescale_exp : 900;
  a.err = p->err;
  return a;
}

// The device work of units [begin, end) (range already checked), enqueued on
// the context's stream: the multi-source passes, then the per-source items.
int enqueue_units(bc_plan *p, int64_t begin, int64_t end, int *launches) {
  bc_ctx *ctx = p->ctx;
  if (p->bp && begin < p->n_bat) {  // multi-source passes
    std::string msg;
    int rc = bcg::batched_run(p->bp, begin, std::min(end, p->n_bat), ctx->stream, launches, &msg);
    if (rc) return fail(ctx, rc, "batched run: " + msg);
  }
  const int64_t i0 = std::max(begin, p->n_bat) - p->n_bat, i1 = std::min(end - p->n_bat, p->n_items);
  // per-source items, in launches of at most kAccMaxAdds sources (the adds one
  // fixed-point counter takes between folds); each launch is followed by the
  // fold of the counters of the BCCs it touched
  for (int64_t j0 = i0; j0 < i1;) {
    const int64_t *us = p->unit_sources.data() + p->n_bat;
    int64_t j1 = j0 + 1;
    while (j1 < i1 && us[j1 + 1] - us[j0] <= bcg::kAccMaxAdds) ++j1;
    int32_t b0 = INT32_MAX, b1 = -1;
    for (int64_t j = j0; j < j1; ++j) {
      b0 = std::min(b0, p->h_items[j].bcc);
      b1 = std::max(b1, p->h_items[j].bcc);
    }
    CK(ctx, cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), ctx->stream));
    bcg::PlainArgs a = plain_args(p);
    a.item_begin = j0; a.item_end = j1;
    const int grid = (int)std::min<int64_t>(p->grid, j1 - j0);
    CK(ctx, bcg::launch_plain(a, p->block, grid, ctx->stream));
    CK(ctx, bcg::launch_fold(p->acc, p->bc, p->h_vtx_off[b0], p->h_vtx_off[b1 + 1], ctx->stream));
    *launches += 2;
    j0 = j1;
  }
  // small-BCC items: one launch per class (each BCC's sources are far fewer
  // than kAccMaxAdds), then one fold over the BCCs they touched
  const int64_t t0 = std::max(begin, p->n_bat + p->n_items) - p->n_bat - p->n_items;
  const int64_t t1 = end - p->n_bat - p->n_items;
  if (t1 > t0) {
    int32_t b0 = INT32_MAX, b1 = -1;
    for (int64_t j = t0; j < t1; ++j) {
      b0 = std::min(b0, p->h_titems[j].bcc);
      b1 = std::max(b1, p->h_titems[j].bcc);
    }
    for (const bc_plan::TileLaunch &T : p->tl) {
      const int64_t j0 = std::max(t0, T.i0), j1 = std::min(t1, T.i1);
      if (j1 <= j0) continue;
      CK(ctx, cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), ctx->stream));
      bcg::TileArgs a{};
      a.vtx_off = p->vtx_off; a.reach = p->reach; a.slices = p->slices; a.slice_off = p->slice_off;
      a.slice_bytes = p->slice_bytes; a.items = p->titems; a.item_begin = j0; a.item_end = j1;
      a.next_item = p->counter; a.acc = p->acc; a.ws_lv = p->tws_lv; a.cap = p->tcap; a.nmax = T.nmax;
      a.ws_P = p->tws_P; a.cap_P = p->tcap_P;
      a.slice_max = T.slice_max; a.wait_ns = wait_ns(ctx); a.err = p->err;
      CK(ctx, bcg::launch_tile(T.cls, a, (int)std::min<int64_t>(T.grid, j1 - j0), T.smem, ctx->stream));
      ++*launches;
    }
    CK(ctx, bcg::launch_fold(p->acc, p->bc, p->h_vtx_off[b0], p->h_vtx_off[b1 + 1], ctx->stream));
    ++*launches;
  }
  return BCGPU_OK;
}

// Captures enqueue_units of the range into a graph and instantiates it (the
// capture records the work; nothing runs).
int record_units(bc_plan *p, int64_t begin, int64_t end, bc_plan::Recorded *out) {
  bc_ctx *ctx = p->ctx;
  CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int launches = 0;
  const int rc = enqueue_units(p, begin, end, &launches);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc ? rc : cuda_fail(ctx, e, "cudaStreamEndCapture");
  }
  cudaGraphExec_t ex = nullptr;
  const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return cuda_fail(ctx, ei, "cudaGraphInstantiate");
  *out = bc_plan::Recorded{ex, launches};
  return BCGPU_OK;
}

int check_range(bc_plan *p, int64_t begin, int64_t end) {
  const int64_t n = bc_plan_num_units(p);
  if (begin < 0 || end < begin || end > n) return fail(p->ctx, BCGPU_EINVAL, "unit range out of bounds");
  return BCGPU_OK;
}

}  // namespace

extern "C" int bc_plan_record(bc_plan *p, int64_t begin, int64_t end) {
  if (!p) return BCGPU_EINVAL;
  bc_ctx *ctx = p->ctx;
  if (!ctx->opts.graph) return fail(ctx, BCGPU_EINVAL, "bc_plan_record needs a context with bc_opts.graph set");
  int rc = check_range(p, begin, end);
  if (rc) return rc;
  CK(ctx, cudaSetDevice(ctx->device));
  bc_plan::Recorded r{};
  if ((rc = record_units(p, begin, end, &r))) return rc;
  auto it = p->graphs.find({begin, end});
  if (it != p->graphs.end()) {
    CK(ctx, cudaStreamSynchronize(ctx->stream));  // the old graph may still be running
    cudaGraphExecDestroy(it->second.exec);
    it->second = r;
  } else {
    p->graphs.emplace(std::make_pair(begin, end), r);
  }
  return BCGPU_OK;
}

extern "C" int bc_plan_run(bc_plan *p, int64_t begin, int64_t end, bc_stats *stats) {
  if (!p) return BCGPU_EINVAL;
  bc_ctx *ctx = p->ctx;
  int rc = check_range(p, begin, end);
  if (rc) return rc;
  CK(ctx, cudaSetDevice(ctx->device));
  int launches = 0;
  if (ctx->opts.graph) {
    auto it = p->graphs.find({begin, end});
    if (it == p->graphs.end()) {
      if ((rc = bc_plan_record(p, begin, end))) return rc;
      it = p->graphs.find({begin, end});
    }
    if (stats) CK(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    CK(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
    launches = it->second.launches;
  } else {
    if (stats) CK(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
    if ((rc = enqueue_units(p, begin, end, &launches))) return rc;
  }
  if (stats) {
    CK(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
    const int64_t d2h0 = p->d2h_bytes;
    int rc = check_dev_err(p);
    if (rc) return rc;
    float ms = 0.f;
    CK(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    std::memset(stats, 0, sizeof(*stats));
    stats->sources = p->unit_sources[end] - p->unit_sources[begin];
    stats->bfs_sources = p->unit_bfs[end] - p->unit_bfs[begin];
    stats->aux_bfs = p->unit_aux[end] - p->unit_aux[begin];
    stats->teps_edges = p->unit_teps[end] - p->unit_teps[begin];
    stats->kernel_ms = ms;
    stats->total_ms = ms;
    stats->kernel_launches = launches;
    stats->batch_width = p->bp ? bcg::batched_width(p->bp) : 0;
    stats->d2h_bytes = p->d2h_bytes - d2h0;  // the status words read back (the run copies nothing in)
  }
  return BCGPU_OK;
}

extern "C" int bc_plan_read(bc_plan *p, double *bc_out) {
  return guard(p ? p->ctx : nullptr, [&]() -> int {
    if (!p || !bc_out) return BCGPU_EINVAL;
    CK(p->ctx, cudaSetDevice(p->ctx->device));
    int rc = check_dev_err(p);
    if (rc) return rc;
    std::vector<double> packed((size_t)p->n_packed);
    if (p->n_packed)
      CK(p->ctx, cudaMemcpyAsync(packed.data(), p->bc, sizeof(double) * (size_t)p->n_packed, cudaMemcpyDeviceToHost,
                                 p->ctx->stream));
    CK(p->ctx, cudaStreamSynchronize(p->ctx->stream));
    p->d2h_bytes += (int64_t)sizeof(double) * p->n_packed;
    for (int32_t v = 0; v < p->n_orig; ++v) bc_out[v] = p->art.empty() ? 0.0 : p->art[v];
    for (int64_t k = 0; k < p->n_packed; ++k) bc_out[p->orig[k]] += packed[k];  // fixed order: deterministic
    return BCGPU_OK;
  });
}

extern "C" int bc_plan_source_rows(bc_plan *p, int64_t packed, int32_t *d_out, double *sigma_out) {
  if (!p || !d_out || !sigma_out) return BCGPU_EINVAL;
  bc_ctx *ctx = p->ctx;
  if (packed < 0 || packed >= p->n_packed) return fail(ctx, BCGPU_EINVAL, "packed id out of range");
  if (p->mode != BCGPU_MODE_PLAIN) return fail(ctx, BCGPU_EINVAL, "row export needs a PLAIN plan");
  CK(ctx, cudaSetDevice(ctx->device));
  const auto &vo = p->h_vtx_off;
  const int32_t b = (int32_t)(std::upper_bound(vo.begin(), vo.end(), packed) - vo.begin() - 1);
  const int32_t local = (int32_t)(packed - vo[b]);
  const int32_t nb = (int32_t)(vo[b + 1] - vo[b]);
  int32_t chain = -1;
  if (local >= p->h_n_plain[b]) {
    for (int64_t c = p->h_chain_off[b]; c < p->h_chain_off[b + 1]; ++c)
      if (local >= p->h_chain_start[c] && local < p->h_chain_start[c] + p->h_chain_len[c]) chain = (int32_t)c;
    if (chain < 0) return fail(ctx, BCGPU_EINVAL, "chain vertex without a chain");
  }
  int32_t *dd = nullptr;
  double *ds = nullptr;
  CK(ctx, cudaMallocAsync((void **)&dd, sizeof(int32_t) * (size_t)nb, ctx->stream));
  CK(ctx, cudaMallocAsync((void **)&ds, sizeof(double) * (size_t)nb, ctx->stream));
  const bcg::PlainArgs a = plain_args(p);
  cudaError_t e = bcg::launch_rows(a, b, local, chain, dd, ds, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, dd, sizeof(int32_t) * (size_t)nb, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sigma_out, ds, sizeof(double) * (size_t)nb, cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(dd, ctx->stream);
  cudaFreeAsync(ds, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "row export");
  return check_dev_err(p);
}

extern "C" int bc_plan_pass_rows(bc_plan *p, int64_t unit, int32_t *nslots, int32_t *ncore, int32_t *src_out,
                                 int32_t *d_out, double *sigma_out) {
  if (!p || !nslots || !ncore) return BCGPU_EINVAL;
  bc_ctx *ctx = p->ctx;
  int32_t b = 0, ns = 0;
  if (!p->bp || unit < 0 || unit >= p->n_bat || bcg::batched_pass_shape(p->bp, unit, &b, &ns) != BCGPU_OK)
    return fail(ctx, BCGPU_EINVAL, "unit is not a multi-source pass");
  *nslots = ns;
  *ncore = p->h_n_plain[b];
  if (!src_out && !d_out && !sigma_out) return BCGPU_OK;  // sizes only
  if (!src_out || !d_out || !sigma_out) return fail(ctx, BCGPU_EINVAL, "null output");
  int rc = bc_plan_run(p, unit, unit + 1, nullptr);
  if (rc) return rc;
  std::vector<int32_t> src, d;
  std::vector<double> sg;
  std::string msg;
  rc = bcg::batched_pass_rows(p->bp, unit, p->h_chain_start.data(), *ncore, ctx->stream, src, d, sg, &msg);
  if (rc) return fail(ctx, rc, msg.c_str());
  rc = check_dev_err(p);
  if (rc) return rc;
  std::copy(src.begin(), src.end(), src_out);
  std::copy(d.begin(), d.end(), d_out);
  std::copy(sg.begin(), sg.end(), sigma_out);
  return BCGPU_OK;
}

namespace {

int run_units(bc_ctx *ctx, const bc_bccs *bccs, int64_t begin, int64_t end, bool all, bool with_art, double *bc_out,
              bc_stats *stats) {
  if (!ctx || !bccs || !bc_out) return fail(ctx, BCGPU_EINVAL, "null argument");
  CK(ctx, cudaSetDevice(ctx->device));
  cudaEvent_t t0, t1;
  CK(ctx, cudaEventCreate(&t0));
  CK(ctx, cudaEventCreate(&t1));
  CK(ctx, cudaEventRecord(t0, ctx->stream));
  bc_plan *p = nullptr;
  // with lazy_tables, only the passes this call runs get their tables built
  const bool lazy = ctx->opts.lazy_tables && !all;
  HOST_MARK("run_units start");
  int rc = create_plan(ctx, bccs, nullptr, &p, lazy ? begin : 0, lazy ? end : INT64_MAX);
  bc_stats st{};
  if (!rc && all) { begin = 0; end = bc_plan_num_units(p); }
  if (!rc) rc = bc_plan_run(p, begin, end, &st);
  HOST_MARK("run");
  if (!rc) rc = bc_plan_read(p, bc_out);
  HOST_MARK("read");
  if (!rc && !with_art && !p->art.empty())
    for (int32_t v = 0; v < p->n_orig; ++v) bc_out[v] -= p->art[v];
  if (!rc) {
    if (cudaEventRecord(t1, ctx->stream) == cudaSuccess && cudaEventSynchronize(t1) == cudaSuccess) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, t0, t1);
      st.total_ms = ms;
    }
    // everything this call copied: the plan's uploads and every read-back
    st.h2d_bytes = p->h2d_bytes + (p->bp ? bcg::batched_h2d_bytes(p->bp) : 0);
    st.d2h_bytes = p->d2h_bytes;
    if (stats) *stats = st;
  }
  bc_plan_destroy(p);
  HOST_MARK("destroy");
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  return rc;
}

}  // namespace

extern "C" int bc_run_bccs(bc_ctx *ctx, const bc_bccs *bccs, double *bc_out, bc_stats *stats) {
  return guard(ctx, [&]() -> int {
    return run_units(ctx, bccs, 0, 0, true, true, bc_out, stats);
  });
}

extern "C" int bc_run_bccs_units(bc_ctx *ctx, const bc_bccs *bccs, int64_t unit_begin, int64_t unit_end,
                                 int32_t with_art, double *bc_out, bc_stats *stats) {
  return guard(ctx, [&]() -> int {
    return run_units(ctx, bccs, unit_begin, unit_end, false, with_art != 0, bc_out, stats);
  });
}

namespace {

// One-BCC packed input built from a reference-style CSR (int32 offsets).
struct OneBcc {
  std::vector<int64_t> vtx_off, row, chain_off;
  std::vector<int32_t> col, reach, orig, n_plain, chain_start, chain_len, chain_l, chain_r;
  bc_bccs view{};
  void finish(int32_t n) {
    view.n_bcc = 1;
    view.n_orig = n;
    view.n_packed = n;
    view.n_arcs = row[n];
    view.n_chains = (int64_t)chain_start.size();
    view.vtx_off = vtx_off.data(); view.row = row.data(); view.col = col.data(); view.reach = reach.data();
    view.orig = orig.data(); view.n_plain = n_plain.data(); view.chain_off = chain_off.data();
    view.chain_start = chain_start.data(); view.chain_len = chain_len.data(); view.chain_l = chain_l.data();
    view.chain_r = chain_r.data(); view.art = nullptr;
  }
};

int check_csr(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *reach) {
  if (!R || !C || !reach || n < 3 || m < 0) return fail(ctx, BCGPU_EINVAL, "bad CSR arguments (a BCC has >= 3 vertices)");
  if (R[0] != 0 || R[n] != m) return fail(ctx, BCGPU_EINVAL, "R[0] must be 0 and R[n] must equal m (arcs)");
  for (int32_t v = 0; v < n; ++v)
    if (R[v + 1] < R[v]) return fail(ctx, BCGPU_EINVAL, "R decreases");
  for (int32_t e = 0; e < m; ++e)
    if (C[e] < 0 || C[e] >= n) return fail(ctx, BCGPU_EINVAL, "C out of range");
  return BCGPU_OK;
}

int run_one(bc_ctx *ctx, OneBcc &o, const std::vector<bcg::PlainItem> &items, std::vector<double> &packed_bc,
            double *time_s) {
  bc_plan *p = nullptr;
  const int saved = ctx->opts.mode;
  ctx->opts.mode = BCGPU_MODE_PLAIN;  // explicit source lists are run with the per-source schedule
  int rc = create_plan(ctx, &o.view, &items, &p);
  ctx->opts.mode = saved;
  if (rc) return rc;
  bc_stats st{};
  rc = bc_plan_run(p, 0, bc_plan_num_units(p), &st);
  if (!rc) {
    packed_bc.assign((size_t)o.view.n_orig, 0.0);
    rc = bc_plan_read(p, packed_bc.data());  // orig is the identity here
  }
  if (!rc && time_s) *time_s += st.kernel_ms * 1e-3;
  bc_plan_destroy(p);
  return rc;
}

}  // namespace

extern "C" int bc_begin_free(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m,
                             const int32_t *req_nodes, int32_t n_req, const int32_t *reach, float *bc, double *time_s) {
  return guard(ctx, [&]() -> int {
    if (!ctx || !bc || (n_req > 0 && !req_nodes)) return fail(ctx, BCGPU_EINVAL, "null argument");
    int rc = check_csr(ctx, R, C, n, m, reach);
    if (rc) return rc;
    OneBcc o;
    o.vtx_off = {0, n};
    o.row.assign(R, R + n + 1);
    o.col.assign(C, C + m);
    o.reach.assign(reach, reach + n);
    o.orig.resize(n);
    for (int32_t v = 0; v < n; ++v) o.orig[v] = v;
    o.n_plain = {n};
    o.chain_off = {0, 0};
    o.finish(n);
    std::vector<bcg::PlainItem> items;
    for (int32_t i = 0; i < n_req; ++i) {
      if (req_nodes[i] < 0 || req_nodes[i] >= n) return fail(ctx, BCGPU_EINVAL, "req_nodes out of range");
      items.push_back({0, req_nodes[i], 0, 0, 1});
    }
    std::vector<double> out;
    rc = run_one(ctx, o, items, out, time_s);
    if (rc) return rc;
    for (int32_t v = 0; v < n; ++v) bc[v] = (float)out[v];  // overwritten, as the reference's free call
    return BCGPU_OK;
  });
}

extern "C" int bc_begin_active(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m,
                               const int32_t *active, int32_t n_active, int32_t n_ears, const int32_t *lnode,
                               const int32_t *rnode, const int32_t *cnt, const int32_t *off, const int32_t *nodes,
                               const int32_t *ld, const int32_t *rd, const int32_t *reach, float *bc, double *time_s) {
  return guard(ctx, [&]() -> int {
    if (!ctx || !bc || (n_active > 0 && !active) || (n_ears > 0 && (!lnode || !rnode || !cnt || !off || !nodes || !ld || !rd)))
      return fail(ctx, BCGPU_EINVAL, "null argument");
    int rc = check_csr(ctx, R, C, n, m, reach);
    if (rc) return rc;
    // New ids: every vertex not on an ear first (original order), then each ear's
    // vertices from its left end (ld = 1, 2, ...) to its right end.
    std::vector<int32_t> nid((size_t)n, -1), old;
    std::vector<char> on_ear((size_t)n, 0), is_active((size_t)n, 0);
    for (int32_t i = 0; i < n_active; ++i) {
      if (active[i] < 0 || active[i] >= n) return fail(ctx, BCGPU_EINVAL, "active vertex out of range");
      is_active[active[i]] = 1;
    }
    for (int32_t e = 0; e < n_ears; ++e)
      for (int32_t j = 0; j < cnt[e]; ++j) {
        int32_t z = nodes[off[e] + j];
        if (z < 0 || z >= n || on_ear[z]) return fail(ctx, BCGPU_EINVAL, "ear vertex out of range or repeated");
        on_ear[z] = 1;
      }
    for (int32_t v = 0; v < n; ++v)
      if (!on_ear[v]) { nid[v] = (int32_t)old.size(); old.push_back(v); }
    const int32_t nplain = (int32_t)old.size();
    // ears sorted by the new id of their left end (chains are grouped by owner)
    std::vector<int32_t> order((size_t)n_ears);
    for (int32_t e = 0; e < n_ears; ++e) {
      order[e] = e;
      if (lnode[e] < 0 || lnode[e] >= n || rnode[e] < 0 || rnode[e] >= n || on_ear[lnode[e]] || on_ear[rnode[e]] ||
          lnode[e] == rnode[e] || !is_active[lnode[e]] || cnt[e] < 1)
        return fail(ctx, BCGPU_EINVAL, "ear endpoints must be distinct active vertices");
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return std::make_pair(nid[lnode[a]], nid[rnode[a]]) <
                                                        std::make_pair(nid[lnode[b]], nid[rnode[b]]); });
    OneBcc o;
    for (int32_t e : order) {
      std::vector<std::pair<int32_t, int32_t>> byld;
      for (int32_t j = 0; j < cnt[e]; ++j) {
        const int32_t k = off[e] + j;
        if (ld[k] < 1 || ld[k] > cnt[e] || ld[k] + rd[k] != cnt[e] + 1)
          return fail(ctx, BCGPU_EINVAL, "ear distances must be 1..cnt with ld + rd = cnt + 1 (unit weights)");
        byld.push_back({ld[k], nodes[k]});
      }
      std::sort(byld.begin(), byld.end());
      o.chain_start.push_back((int32_t)old.size());
      o.chain_len.push_back(cnt[e]);
      o.chain_l.push_back(nid[lnode[e]]);
      o.chain_r.push_back(nid[rnode[e]]);
      for (auto &pr : byld) { nid[pr.second] = (int32_t)old.size(); old.push_back(pr.second); }
    }
    if ((int32_t)old.size() != n) return fail(ctx, BCGPU_EINVAL, "relabelling failed");
    o.vtx_off = {0, n};
    o.row.assign((size_t)n + 1, 0);
    for (int32_t k = 0; k < n; ++k) o.row[k + 1] = o.row[k] + (R[old[k] + 1] - R[old[k]]);
    o.col.resize((size_t)m);
    o.reach.resize((size_t)n);
    o.orig.resize((size_t)n);
    for (int32_t k = 0; k < n; ++k) {
      int64_t w = o.row[k];
      for (int32_t e = R[old[k]]; e < R[old[k] + 1]; ++e) o.col[w++] = nid[C[e]];
      o.reach[k] = reach[old[k]];
      o.orig[k] = k;  // results are mapped back below
    }
    o.n_plain = {nplain};
    o.chain_off = {0, (int64_t)o.chain_start.size()};
    o.finish(n);
    std::vector<bcg::PlainItem> items;
    size_t c = 0;
    for (int32_t k = 0; k < nplain; ++k) {
      size_t c0 = c;
      while (c < o.chain_l.size() && o.chain_l[c] == k) ++c;
      if (is_active[old[k]] || c > c0) items.push_back({0, k, (int32_t)c0, (int32_t)c, is_active[old[k]] ? 1 : 0});
    }
    std::vector<double> out;
    rc = run_one(ctx, o, items, out, time_s);
    if (rc) return rc;
    for (int32_t k = 0; k < n; ++k) bc[old[k]] += (float)out[k];  // added, as the reference seeds from bc
    return BCGPU_OK;
  });
}
