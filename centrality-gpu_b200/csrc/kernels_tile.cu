// Small-BCC schedule: one CTA per range of sources of one BCC, every array a
// source touches in shared memory.
//
// The reference runs every BCC through the same per-source kernel, one
// source per CTA (Codes/kernels_free.cu:154-473, launch shape
// Codes/begin_gpupgm.cu:52-65), with its rows in global memory, whatever the
// BCC's size; on a batch of thousands of small graphs the CTAs then wait on
// global-memory latency at every arc. Here a BCC that fits shared memory is
// run from shared memory only:
//  * the slice (local row offsets, 16-bit neighbour ids; tile.h TileSlice) is
//    brought in by one cp.async.bulk (a plain bulk copy from this GPU's global
//    memory into this CTA's shared memory, completion on an mbarrier whose wait
//    is bounded) and serves every source of the item;
//  * levels, path counts (then q in place) and the visit order of each source
//    live in shared memory: one set per warp in the warp class (a warp per
//    source, eight in flight), one per source group in the CTA class (the
//    whole CTA on one source, or, for BCCs whose single-source CTA fits only
//    once or twice per SM, two or four groups of a 1024-thread CTA on their
//    own sources from the one slice);
//  * forward: level-synchronous, each frontier vertex pulls sigma from its
//    predecessors and claims its successors in one scan of its row -- a row of
//    up to kLaneDeg arcs by one lane (four arcs' loads in flight), a longer one
//    by a whole warp (lanes over arcs, then a fixed-order warp sum);
//  * backward: successor form, q(w) = (reach(w)+1+delta(w))/sigma(w) and
//    delta(v) = sigma(v) * sum q (Codes/kernels_free.cu:391,409), q
//    overwriting sigma in place;
//  * chain (degree-2) vertices are ordinary vertices and sources here: on a
//    BCC this small their BFS costs about what the endpoint merge of the
//    per-source schedule does;
//  * BC: contributions delta * (reach(s)+1) (Codes/kernels_free.cu:425) go to
//    shared-memory fixed-point counters (warp class: integer atomics, any
//    order) or to an FP64 partial row per source group (CTA class: a group's
//    sources, fixed by the item, run one after another, each vertex written
//    by one thread, so the order is fixed), then once per item into the
//    global fixed-point counters.
// Path counts are FP64 without per-level scaling: the plan routes a BCC here
// only when no path count can pass 2^1000 ((2 ecc + 1) levels of at most
// maxdeg predecessors each); a non-finite value still flags kDevOverflow.
#include "accum.cuh"
#include "common.cuh"
#include "tile.h"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace bcg {

namespace {

constexpr int kThreads = kTileWarps * 32;
constexpr int kLaneDeg = 8;  // rows up to this many arcs: one lane; longer rows: a whole warp
// CTA class: long rows of a level queued for the whole CTA (a row beyond the
// queue's room is scanned at once by the warp that found it).
constexpr int kLongQueue = 1024;

struct Ctl {
  unsigned long long bar;  // mbarrier of the slice copy
  int item, next, bcc, pad;
  int tails[kTileWarps];
};

__host__ __device__ constexpr int64_t align16(int64_t x) { return (x + 15) / 16 * 16; }

// ---- shared-memory layouts (host and device agree through these)
struct WarpLayout {  // ctl | counters [nmax][kAccDigits] | per warp: d [nmax], S [nmax], sq [nmax] | slice
  __host__ __device__ static int64_t cnt() { return align16(sizeof(Ctl)); }
  __host__ __device__ static int64_t per_warp(int64_t nmax) { return align16(8 * nmax) + 2 * align16(4 * nmax); }
  __host__ __device__ static int64_t warps(int64_t nmax) { return cnt() + align16(nmax * kAccDigits * 8); }
  __host__ __device__ static int64_t slice(int64_t nmax) { return warps(nmax) + kTileWarps * per_warp(nmax); }
};
// CTA class: kBlock threads in kBlock / kGroup groups, each group on its own
// sources with its own arrays and barrier, all groups on the one staged slice.
// ctl | per group: sq [nmax] | d int16 [nmax] | S uint16 [nmax] | lv [kLevels]
//     | long-row queue [kQueue] | counters cnt[4], nq[4] | slice
// (one group: levels and queue of the class limits; several: the smaller
// limits of the grouped classes, tile.h).
template <int kBlock, int kGroup>
struct CtaLayout {
  static constexpr int kG = kBlock / kGroup;
  static constexpr int kLevels = kG == 1 ? kTileMaxLevels : kTileGroupMaxLevels;
  static constexpr int kQueue = kG == 1 ? kLongQueue : kGroupLongQueue;
  __host__ __device__ static int64_t d(int64_t nmax) { return align16(8 * nmax); }
  __host__ __device__ static int64_t S(int64_t nmax) { return d(nmax) + align16(2 * nmax); }
  __host__ __device__ static int64_t lv(int64_t nmax) { return S(nmax) + align16(2 * nmax); }
  __host__ __device__ static int64_t q(int64_t nmax) { return lv(nmax) + align16(4 * kLevels); }
  __host__ __device__ static int64_t ctr(int64_t nmax) { return q(nmax) + align16(4 * kQueue); }
  __host__ __device__ static int64_t group_bytes(int64_t nmax) { return ctr(nmax) + align16(8 * sizeof(int)); }
  __host__ __device__ static int64_t group(int g, int64_t nmax) { return align16(sizeof(Ctl)) + g * group_bytes(nmax); }
  __host__ __device__ static int64_t slice(int64_t nmax) { return group(kG, nmax); }
  // the group's barrier: the CTA's own when the group is the CTA, else named barrier g+1
  __device__ __forceinline__ static void sync(int g) {
    if constexpr (kG == 1) {
      __syncthreads();
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(kGroup) : "memory");
    }
  }
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// mbarrier and bulk-copy primitives (PTX ISA: mbarrier, cp.async.bulk).
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Global -> this CTA's shared memory; bytes a multiple of 16, both ends 16-byte aligned.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of dst before the copy's writes
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Waits for phase `parity` of the barrier, at most limit_ns; false on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned long long limit_ns) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// One BCC as the kernels read it: local row offsets (uint16 or int32) and
// neighbours (shared memory), reach (global).
struct View {
  const int32_t *R32;
  const uint16_t *R16;  // set for a narrow slice
  const uint16_t *C;
  const int32_t *rch;
  __device__ __forceinline__ int row(int32_t w) const { return R16 ? (int)R16[w] : R32[w]; }
};

// Pulls the next item for the CTA (thread 0) and stages its BCC's slice if
// the CTA does not hold it already. Returns false when the CTA is done (no
// item left, an error flagged, or the slice did not arrive in time).
__device__ bool next_item(const TileArgs &a, Ctl &ctl, unsigned char *slice, unsigned &phase, TileItem &it,
                          int64_t &vo, int32_t &nb) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    const int64_t k = (int64_t)atomicAdd(a.next_item, 1ull);
    ctl.item = (*(volatile int *)a.err != kDevOk || a.item_begin + k >= a.item_end) ? -1 : (int)k;
    ctl.next = 0;
  }
  __syncthreads();  // also: every thread is done with the previous item's slice and rows
  if (ctl.item < 0) return false;
  it = a.items[a.item_begin + ctl.item];
  vo = a.vtx_off[it.bcc];
  nb = (int32_t)(a.vtx_off[it.bcc + 1] - vo);
  const int64_t soff = a.slice_off[it.bcc] & ~int64_t(15);
  if (nb > a.nmax || a.slice_off[it.bcc] < 0 || it.s0 < 0 || it.s1 > nb) {  // uniform over the CTA
    if (tid == 0) set_err(a.err, kDevBadItem);
    return false;
  }
  if (ctl.bcc != it.bcc) {  // uniform: ctl.bcc was last written before a barrier
    if (tid == 0) {
      const unsigned bytes = (unsigned)a.slice_bytes[it.bcc];
      mbar_expect_tx(&ctl.bar, bytes);
      bulk_copy(slice, a.slices + soff, bytes, &ctl.bar);
    }
    if (!mbar_wait(&ctl.bar, phase, a.wait_ns)) {
      // the copy did not complete in time: record it, wait (again bounded)
      // for the copy in flight to land in this CTA's shared memory, stop
      set_err(a.err, kDevTimeout);
      mbar_wait(&ctl.bar, phase, a.wait_ns);
      return false;
    }
    phase ^= 1u;
  }
  return true;
}

__device__ __forceinline__ View view_of(const TileArgs &a, const unsigned char *slice, int32_t nb, int64_t vo,
                                        int32_t bcc) {
  const bool narrow = (a.slice_off[bcc] & 1) != 0;
  return View{reinterpret_cast<const int32_t *>(slice), narrow ? reinterpret_cast<const uint16_t *>(slice) : nullptr,
              reinterpret_cast<const uint16_t *>(slice + TileSlice::col_at(nb, narrow)), a.reach + vo};
}

// Appends x to the visit order S: one atomic per group of lanes appending at
// once (the lanes that reach this call together), not one per lane.
template <typename ST>
__device__ __forceinline__ void append(ST *S, int *tail, int32_t x) {
  cg::coalesced_group g = cg::coalesced_threads();
  int pos = 0;
  if (g.thread_rank() == 0) pos = atomicAdd(tail, (int)g.size());
  S[g.shfl(pos, 0) + (int)g.thread_rank()] = (ST)x;
}

// Claims unvisited vertex x (level -1) for level lev; true for the one claim
// that wins. Levels are int32 (warp class) or int16 (CTA class).
__device__ __forceinline__ bool claim(int32_t *d, int32_t x, int lev) { return atomicCAS(d + x, -1, lev) == -1; }
__device__ __forceinline__ bool claim(int16_t *d, int32_t x, int lev) {
  return atomicCAS(reinterpret_cast<unsigned short *>(d + x), (unsigned short)0xffffu, (unsigned short)lev) == 0xffffu;
}

// Forward scan of one row by one thread (four arcs' loads in flight, sums in
// arc order): pulls sigma from level dprev, claims unvisited vertices for
// dnext (appended to S at *tail).
template <typename DT, typename ST>
__device__ __forceinline__ double pull_row(const View &g, int e0, int e1, DT *d, const double *sq, ST *S, int *tail,
                                           int dprev, int dnext) {
  double acc = 0.0;
  for (int e = e0; e < e1; e += 4) {
    int32_t x[4], dx[4];
    double sv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = e + j < e1 ? (int32_t)g.C[e + j] : -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) dx[j] = x[j] >= 0 ? (int)d[x[j]] : INT_MAX;
#pragma unroll
    for (int j = 0; j < 4; ++j) sv[j] = dx[j] == dprev ? sq[x[j]] : 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (dx[j] == dprev) acc += sv[j];
      else if (dx[j] == -1 && claim(d, x[j], dnext)) append(S, tail, x[j]);
    }
  }
  return acc;
}

// The same for a long row, by a whole warp (lanes over arcs, fixed-order sum).
template <typename DT, typename ST>
__device__ __forceinline__ double pull_row_warp(const View &g, int e0, int e1, DT *d, const double *sq, ST *S, int *tail,
                                                int dprev, int dnext, int lane) {
  double acc = 0.0;
  for (int e = e0 + lane; e < e1; e += 32) {
    const int32_t x = g.C[e];
    const int dx = d[x];
    if (dx == dprev) acc += sq[x];
    else if (dx == -1 && claim(d, x, dnext)) append(S, tail, x);
  }
  return warp_sum(acc);
}

// Sum of q over the successors (level dsucc) of one row, by one thread.
template <typename DT>
__device__ __forceinline__ double push_row(const View &g, int e0, int e1, const DT *d, const double *sq, int dsucc) {
  double acc = 0.0;
  for (int e = e0; e < e1; e += 4) {
    int32_t x[4];
    bool hit[4];
    double qv[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) x[j] = e + j < e1 ? (int32_t)g.C[e + j] : -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) hit[j] = x[j] >= 0 && (int)d[x[j]] == dsucc;
#pragma unroll
    for (int j = 0; j < 4; ++j) qv[j] = hit[j] ? sq[x[j]] : 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (hit[j]) acc += qv[j];
  }
  return acc;
}

template <typename DT>
__device__ __forceinline__ double push_row_warp(const View &g, int e0, int e1, const DT *d, const double *sq, int dsucc,
                                                int lane) {
  double acc = 0.0;
  for (int e = e0 + lane; e < e1; e += 32) {
    const int32_t x = g.C[e];
    if ((int)d[x] == dsucc) acc += sq[x];
  }
  return warp_sum(acc);
}

// delta and q of w from the successors' sum; returns delta (q overwrites sigma).
__device__ __forceinline__ double finish(const View &g, int32_t w, double sum, double *sq, int *err) {
  const double sw = sq[w];
  const double delta = sw * sum;
  const double qw = ((double)__ldg(g.rch + w) + 1.0 + delta) / sw;
  if (exp_bits(qw) == 0x7ff || exp_bits(delta) == 0x7ff || exp_bits(sw) == 0) set_err(err, kDevOverflow);
  sq[w] = qw;
  return delta;
}

// ======================================================= warp per source ===

// BFS of one warp from s (rows in this warp's shared memory, level offsets lv
// in global memory). Returns the number of levels.
__device__ int warp_bfs(const View &g, int32_t nb, int32_t s, int32_t *d, double *sq, int32_t *S, int32_t *lv,
                        int *tail, int lane) {
  for (int v = lane; v < nb; v += 32) d[v] = -1;
  __syncwarp();
  if (lane == 0) {
    d[s] = 0;
    S[0] = s;
    sq[s] = 1.0;
    lv[0] = 0;
    lv[1] = 1;
    *tail = 1;
  }
  __syncwarp();
  int lev = 0, f0 = 0, f1 = 1;
  while (true) {
    const int dprev = lev == 0 ? INT_MIN : lev - 1, dnext = lev + 1;
    for (int c0 = f0; c0 < f1; c0 += 32) {
      const int i = c0 + lane;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < f1) {
        w = S[i];
        e0 = g.row(w);
        e1 = g.row(w + 1);
      }
      const bool big = e1 - e0 > kLaneDeg;
      if (w >= 0 && !big) {
        const double acc = pull_row(g, e0, e1, d, sq, S, tail, dprev, dnext);
        if (lev > 0) sq[w] = acc;
      }
      uint32_t bigs = __ballot_sync(0xffffffffu, w >= 0 && big);
      while (bigs) {
        const int j = __ffs(bigs) - 1;
        bigs &= bigs - 1;
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        const int a0 = __shfl_sync(0xffffffffu, e0, j), a1 = __shfl_sync(0xffffffffu, e1, j);
        const double acc = pull_row_warp(g, a0, a1, d, sq, S, tail, dprev, dnext, lane);
        if (lane == 0 && lev > 0) sq[wj] = acc;
      }
    }
    __syncwarp();
    const int t = *(volatile int *)tail;
    if (t == f1) break;
    if (lane == 0) lv[lev + 2] = t;
    f0 = f1;
    f1 = t;
    ++lev;
    __syncwarp();
  }
  return lev + 1;
}

__device__ void warp_sweep(const View &g, int nlev, const int32_t *d, double *sq, const int32_t *S, const int32_t *lv,
                           double wsrc, unsigned long long *cnt, int lane, int *err) {
  for (int lev = nlev - 1; lev >= 1; --lev) {
    const int dsucc = lev + 1, a0 = lv[lev], a1 = lv[lev + 1];
    for (int c0 = a0; c0 < a1; c0 += 32) {
      const int i = c0 + lane;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < a1) {
        w = S[i];
        e0 = g.row(w);
        e1 = g.row(w + 1);
      }
      const bool big = e1 - e0 > kLaneDeg;
      double sum = 0.0;
      if (w >= 0 && !big) sum = push_row(g, e0, e1, d, sq, dsucc);
      uint32_t bigs = __ballot_sync(0xffffffffu, w >= 0 && big);
      while (bigs) {
        const int j = __ffs(bigs) - 1;
        bigs &= bigs - 1;
        const int b0 = __shfl_sync(0xffffffffu, e0, j), b1 = __shfl_sync(0xffffffffu, e1, j);
        const double part = push_row_warp(g, b0, b1, d, sq, dsucc, lane);
        if (lane == j) sum = part;
      }
      if (w >= 0) {
        const double delta = finish(g, w, sum, sq, err);  // this level's q: read by the level above only
        if (delta != 0.0) acc_add(cnt + (int64_t)kAccDigits * w, delta * wsrc, err);
      }
    }
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kThreads, 1) tile_warp_kernel(TileArgs a) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  Ctl &ctl = *reinterpret_cast<Ctl *>(s_raw);
  unsigned long long *cnt = reinterpret_cast<unsigned long long *>(s_raw + WarpLayout::cnt());
  unsigned char *slice = s_raw + WarpLayout::slice(a.nmax);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned char *mine = s_raw + WarpLayout::warps(a.nmax) + (int64_t)warp * WarpLayout::per_warp(a.nmax);
  double *sq = reinterpret_cast<double *>(mine);
  int32_t *d = reinterpret_cast<int32_t *>(mine + align16(8 * (int64_t)a.nmax));
  int32_t *S = d + align16(4 * (int64_t)a.nmax) / 4;
  int32_t *lv = a.ws_lv + ((int64_t)blockIdx.x * kTileWarps + warp) * a.cap;
  if (tid == 0) {
    mbar_init(&ctl.bar, 1);
    ctl.bcc = -1;
  }
  __syncthreads();
  unsigned phase = 0;
  TileItem it;
  int64_t vo;
  int32_t nb;
  while (next_item(a, ctl, slice, phase, it, vo, nb)) {
    for (int64_t k = tid; k < (int64_t)kAccDigits * nb; k += kThreads) cnt[k] = 0ull;
    __syncthreads();
    if (tid == 0) ctl.bcc = it.bcc;  // read again only after the next barrier
    const View g = view_of(a, slice, nb, vo, it.bcc);
    while (true) {  // the warps take the item's sources one at a time
      int k = 0;
      if (lane == 0) k = atomicAdd(&ctl.next, 1);
      k = __shfl_sync(0xffffffffu, k, 0);
      const int32_t s = it.s0 + k;
      if (s >= it.s1) break;
      const int nlev = warp_bfs(g, nb, s, d, sq, S, lv, &ctl.tails[warp], lane);
      warp_sweep(g, nlev, d, sq, S, lv, (double)__ldg(g.rch + s) + 1.0, cnt, lane, a.err);
    }
    __syncthreads();
    unsigned long long *acc = a.acc + (int64_t)kAccDigits * vo;  // integer adds: any order
    for (int64_t k = tid; k < (int64_t)kAccDigits * nb; k += kThreads) {
      const unsigned long long c = cnt[k];
      if (c) atomicAdd(acc + k, c);
    }
  }
}

// ======================================================== CTA per source ===

// BFS of one group (the whole CTA, or a fixed share of its threads) from s,
// two group barriers per level: the frontier's rows of up to kLaneDeg arcs
// are scanned by one thread each (chunks of a level are independent: they
// read the previous level only) while longer rows are queued; after a
// barrier the group's warps share the queued rows; a second barrier ends the
// level. Queue and tail counters of level l are cnt[l % 3] and nq[l % 3];
// those of level l+1 are cleared at the start of level l, two barriers after
// their last reader.
template <int kBlock, int kGroup>
__device__ int cta_bfs(const View &g, int32_t nb, int32_t s, int16_t *d, double *sq, uint16_t *S, int32_t *lv,
                       int32_t *q, int *cnt, int *nq, int *err, int grp, int tid) {
  using L = CtaLayout<kBlock, kGroup>;
  constexpr int kWarps = kGroup / 32;
  const int lane = tid & 31, warp = tid >> 5;
  for (int v = tid; v < nb; v += kGroup) d[v] = -1;
  if (tid == 0) {
    cnt[0] = 0;
    cnt[1] = 0;
    nq[0] = 0;
    nq[1] = 0;
  }
  L::sync(grp);
  if (tid == 0) {
    d[s] = 0;
    S[0] = (uint16_t)s;
    sq[s] = 1.0;
    lv[0] = 0;
    lv[1] = 1;
  }
  L::sync(grp);
  int lev = 0, f0 = 0, f1 = 1;
  while (true) {
    const int dprev = lev == 0 ? INT_MIN : lev - 1, dnext = lev + 1;
    int *tail = cnt + lev % 3, *nql = nq + lev % 3;
    if (tid == 0) {
      cnt[(lev + 1) % 3] = 0;
      nq[(lev + 1) % 3] = 0;
    }
    for (int c0 = f0; c0 < f1; c0 += kGroup) {  // uniform over the group
      const int i = c0 + tid;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < f1) {
        w = S[i];
        e0 = g.row(w);
        e1 = g.row(w + 1);
      }
      const bool big = e1 - e0 > kLaneDeg;
      if (w >= 0 && !big) {
        const double acc = pull_row(g, e0, e1, d, sq, S + f1, tail, dprev, dnext);
        if (lev > 0) sq[w] = acc;
      }
      bool mine = false;  // a long row the queue had no room for
      if (w >= 0 && big) {
        const int pos = atomicAdd(nql, 1);
        if (pos < L::kQueue) q[pos] = w;
        else mine = true;
      }
      uint32_t over = __ballot_sync(0xffffffffu, mine);
      while (over) {
        const int j = __ffs(over) - 1;
        over &= over - 1;
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        const double acc = pull_row_warp(g, g.row(wj), g.row(wj + 1), d, sq, S + f1, tail, dprev, dnext, lane);
        if (lane == 0 && lev > 0) sq[wj] = acc;
      }
    }
    L::sync(grp);
    const int nlong = min(*(volatile int *)nql, L::kQueue);
    for (int k = warp; k < nlong; k += kWarps) {
      const int32_t w = q[k];
      const double acc = pull_row_warp(g, g.row(w), g.row(w + 1), d, sq, S + f1, tail, dprev, dnext, lane);
      if (lane == 0 && lev > 0) sq[w] = acc;
    }
    L::sync(grp);
    const int t = f1 + *(volatile int *)tail;
    if (t == f1) break;
    if (lev + 2 >= L::kLevels) {  // uniform; routing keeps BCCs below this depth
      if (tid == 0) set_err(err, kDevWorkspace);
      return -1;
    }
    if (tid == 0) lv[lev + 2] = t;
    f0 = f1;
    f1 = t;
    ++lev;
  }
  return lev + 1;
}

// Dependency sweep of one group, two group barriers per level as in cta_bfs;
// contributions go to the group's FP64 row P, each vertex written by one
// thread.
template <int kBlock, int kGroup>
__device__ void cta_sweep(const View &g, int nlev, const int16_t *d, double *sq, const uint16_t *S, const int32_t *lv,
                          int32_t *q, int *nq, double wsrc, double *P, int *err, int grp, int tid) {
  using L = CtaLayout<kBlock, kGroup>;
  constexpr int kWarps = kGroup / 32;
  const int lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    nq[0] = 0;
    nq[1] = 0;
  }
  L::sync(grp);
  for (int lev = nlev - 1, k3 = 0; lev >= 1; --lev, k3 = (k3 + 1) % 3) {
    const int dsucc = lev + 1, a0 = lv[lev], a1 = lv[lev + 1];
    int *nql = nq + k3;
    if (tid == 0) nq[(k3 + 1) % 3] = 0;
    for (int c0 = a0; c0 < a1; c0 += kGroup) {  // uniform over the group
      const int i = c0 + tid;
      int32_t w = -1, e0 = 0, e1 = 0;
      if (i < a1) {
        w = S[i];
        e0 = g.row(w);
        e1 = g.row(w + 1);
      }
      const bool big = e1 - e0 > kLaneDeg;
      if (w >= 0 && !big) P[w] += finish(g, w, push_row(g, e0, e1, d, sq, dsucc), sq, err) * wsrc;
      bool mine = false;
      if (w >= 0 && big) {
        const int pos = atomicAdd(nql, 1);
        if (pos < L::kQueue) q[pos] = w;
        else mine = true;
      }
      uint32_t over = __ballot_sync(0xffffffffu, mine);
      while (over) {
        const int j = __ffs(over) - 1;
        over &= over - 1;
        const int32_t wj = __shfl_sync(0xffffffffu, w, j);
        const double sum = push_row_warp(g, g.row(wj), g.row(wj + 1), d, sq, dsucc, lane);
        if (lane == 0) P[wj] += finish(g, wj, sum, sq, err) * wsrc;
      }
    }
    L::sync(grp);
    const int nlong = min(*(volatile int *)nql, L::kQueue);
    for (int k = warp; k < nlong; k += kWarps) {
      const int32_t w = q[k];
      const double sum = push_row_warp(g, g.row(w), g.row(w + 1), d, sq, dsucc, lane);
      if (lane == 0) P[w] += finish(g, w, sum, sq, err) * wsrc;
    }
    L::sync(grp);
  }
}

// 1024 / kBlock CTAs per SM at most (the shared-memory buckets), so 64
// registers per thread whatever the block size. Group grp of the CTA takes
// the item's sources s0 + grp, s0 + grp + G, ... one after another (a fixed
// assignment: its FP64 row P is summed in a fixed order), then flushes P into
// the integer counters (any order).
template <int kBlock, int kGroup>
__global__ void __launch_bounds__(kBlock, 1024 / kBlock) tile_cta_kernel(TileArgs a) {
  using L = CtaLayout<kBlock, kGroup>;
  extern __shared__ __align__(16) unsigned char s_raw[];
  const int64_t nmax = a.nmax;
  Ctl &ctl = *reinterpret_cast<Ctl *>(s_raw);
  const int grp = threadIdx.x / kGroup, gtid = threadIdx.x % kGroup;
  unsigned char *mine = s_raw + L::group(grp, nmax);
  double *P = a.ws_P + ((int64_t)blockIdx.x * L::kG + grp) * a.cap_P;  // the group's FP64 row (global, L2-resident)
  double *sq = reinterpret_cast<double *>(mine);
  int16_t *d = reinterpret_cast<int16_t *>(mine + L::d(nmax));
  uint16_t *S = reinterpret_cast<uint16_t *>(mine + L::S(nmax));
  int32_t *lv = reinterpret_cast<int32_t *>(mine + L::lv(nmax));
  int32_t *q = reinterpret_cast<int32_t *>(mine + L::q(nmax));
  int *cnt = reinterpret_cast<int *>(mine + L::ctr(nmax)), *nq = cnt + 4;
  unsigned char *slice = s_raw + L::slice(nmax);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&ctl.bar, 1);
    ctl.bcc = -1;
  }
  __syncthreads();
  unsigned phase = 0;
  TileItem it;
  int64_t vo;
  int32_t nb;
  while (next_item(a, ctl, slice, phase, it, vo, nb)) {
    for (int v = gtid; v < nb; v += kGroup) P[v] = 0.0;
    __syncthreads();
    if (tid == 0) ctl.bcc = it.bcc;  // read again only after the next barrier
    const View g = view_of(a, slice, nb, vo, it.bcc);
    for (int32_t s = it.s0 + grp; s < it.s1; s += L::kG) {  // the group's sources in order: P's sums are fixed
      const int nlev = cta_bfs<kBlock, kGroup>(g, nb, s, d, sq, S, lv, q, cnt, nq, a.err, grp, gtid);
      if (nlev < 0) break;
      cta_sweep<kBlock, kGroup>(g, nlev, d, sq, S, lv, q, nq, (double)__ldg(g.rch + s) + 1.0, P, a.err, grp, gtid);
    }
    __syncthreads();
    unsigned long long *acc = a.acc + (int64_t)kAccDigits * vo;
    for (int v = gtid; v < nb; v += kGroup)
      if (P[v] != 0.0) acc_add(acc + (int64_t)kAccDigits * v, P[v], a.err);
  }
}

}  // namespace

int block_of(int cls) { return cls >= kTileCta1024 ? 1024 : cls == kTileCta512 ? 512 : kThreads; }

size_t tile_smem_bytes(int cls, int64_t nmax, int64_t slice_max) {
  const int64_t head = cls == kTileWarp       ? WarpLayout::slice(nmax)
                       : cls == kTileCta      ? CtaLayout<256, 256>::slice(nmax)
                       : cls == kTileCta512   ? CtaLayout<512, 512>::slice(nmax)
                       : cls == kTileCta1024  ? CtaLayout<1024, 1024>::slice(nmax)
                       : cls == kTileCta1024x2 ? CtaLayout<1024, 512>::slice(nmax)
                                              : CtaLayout<1024, 256>::slice(nmax);
  return (size_t)(head + align16(slice_max));
}

int tile_groups(int cls) { return cls == kTileCta1024x2 ? 2 : cls == kTileCta1024x4 ? 4 : 1; }

size_t tile_smem_limit(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return 0;
  return (size_t)v;
}

namespace {
const void *tile_fn(int cls) {
  return cls == kTileWarp       ? reinterpret_cast<const void *>(tile_warp_kernel)
         : cls == kTileCta      ? reinterpret_cast<const void *>(tile_cta_kernel<256, 256>)
         : cls == kTileCta512   ? reinterpret_cast<const void *>(tile_cta_kernel<512, 512>)
         : cls == kTileCta1024  ? reinterpret_cast<const void *>(tile_cta_kernel<1024, 1024>)
         : cls == kTileCta1024x2 ? reinterpret_cast<const void *>(tile_cta_kernel<1024, 512>)
                                : reinterpret_cast<const void *>(tile_cta_kernel<1024, 256>);
}
}  // namespace

int tile_ctas_per_sm(int cls, size_t smem) {
  int n = 0;
  if (cudaFuncSetAttribute(tile_fn(cls), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tile_fn(cls), block_of(cls), smem) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_tile(int cls, const TileArgs &a, int grid, size_t smem, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(tile_fn(cls), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  switch (cls) {
    case kTileWarp: tile_warp_kernel<<<grid, kThreads, smem, stream>>>(a); break;
    case kTileCta: tile_cta_kernel<256, 256><<<grid, 256, smem, stream>>>(a); break;
    case kTileCta512: tile_cta_kernel<512, 512><<<grid, 512, smem, stream>>>(a); break;
    case kTileCta1024: tile_cta_kernel<1024, 1024><<<grid, 1024, smem, stream>>>(a); break;
    case kTileCta1024x2: tile_cta_kernel<1024, 512><<<grid, 1024, smem, stream>>>(a); break;
    case kTileCta1024x4: tile_cta_kernel<1024, 256><<<grid, 1024, smem, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace bcg
