// BATCHED schedule: many sources per pass as a bitmask multi-source BFS.
//
// One pass ("batch") covers up to B = 32*W sources ("slots") of one BCC:
//   own BFS slots   free vertices / chain endpoints whose dependencies count,
//   aux BFS slots   chain endpoints BFS'd only so their chains can merge,
//   chain slots     degree-2 chain vertices: rows merged from the two endpoint
//                   columns, d = min(dL+ld, dR+rd) (reference
//                   Codes/postprocesses.cu:329-351, chain walk :205-274).
// State is vertex-major, slot-minor ([v][B]) so a warp reads the 32 slots of
// a word as one coalesced row segment, and every neighbour's row serves all
// slots at once:
//   d[v][b]     level (int32)            sigma[v][b] path count (FP64, scaled)
//   q[v][b]     (reach(v)+1+delta)/sigma (FP64, or FP32 in the compensated mode)
//   lm[t][v][w] bitmask of the slots that reach v at level t: the frontier of
//               the forward phase and the successor test of the backward phase
// Forward: level-synchronous pull. For every vertex still unseen by some BFS
// slot, the warp scans its neighbours once per 32-slot word, ORs their level-t
// masks and sums the path counts of the slots that hit (the reference's
// per-source atomicCAS/atomicAdd BFS, Codes/kernels_free.cu:286-362).
// Backward: successor form (Codes/kernels_free.cu:377-421) with the level
// masks as successor test: delta(v) = sigma(v) * sum over successors of q.
// Path counts carry a per-(slot, level) power-of-two base X so deep graphs do
// not overflow FP64: a level is rescaled when its largest count passes
// 2^rescale_exp (900 by default).
// BC: per (vertex, word) FP64 partials summed over levels in fixed order, then
// over words in fixed order -> deterministic (the reference uses FP32
// atomics, Codes/kernels_free.cu:423-426).
// The whole GPU works on one batch at a time: a cooperative persistent kernel
// with a grid barrier whose waits are bounded (error flag, no hang).
#include "batched.h"
#include "common.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

namespace bcg {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerCta = kThreads / 32;
constexpr int kHeavyDeg = 256;     // vertices above this degree are scanned in chunks by whole CTAs
constexpr int kChunkArcs = 2048;   // arcs per heavy chunk
constexpr long long kSpinLimit = 1ll << 28;  // ~1 min of polling before giving up

enum SlotKind : int32_t { kOwn = 0, kAux = 1, kChain = 2, kUnused = 3 };

struct Slot {
  int32_t kind, src;        // src: BFS source (local id) or the chain vertex itself
  int32_t sl, sr, ld, rd;   // chain slots: endpoint slots and distances
  int32_t cstart, clen, cpos;
  int32_t pad;
};

struct Batch {
  int32_t bcc, nslots, words, max_off;  // max_off: largest chain distance ld/rd in the batch
  int64_t slot_off;   // into the slot table
  int64_t mask_off;   // 3 mask rows (bfs, own, chain), each padded to whole 4-word groups
};

// Control block in global memory (one per plan).
struct Ctrl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int more;          // forward: some slot found a new vertex this level
  int rescale;       // forward: some slot needs a rescale at this level
  int tmax;          // deepest level of the batch (all slots)
  int tbfs;          // deepest BFS level
  int range_err;     // FP32 q left FP32's exponent range in this batch
  int pad;
};

struct Args {
  const int64_t *row;
  const int32_t *col;
  const int32_t *reach;
  const int64_t *vtx_off;
  const int64_t *heavy_off;  // per BCC range in heavy[] (heavy vertices: degree > kHeavyDeg)
  const int32_t *heavy;      // local ids
  const int64_t *hchunk_off; // per BCC range in the chunk table
  const int32_t *hchunk_v;   // chunk -> heavy index (within its BCC's heavy list)
  const int64_t *hchunk_e0;  // chunk arc range [e0, e1) (global arc offsets)
  const int64_t *hchunk_e1;
  const int32_t *hfirst;     // heavy index -> first chunk (BCC-relative), hfirst[h+1] ends it
  double *hacc;              // [chunks][W][32] partial sums
  uint32_t *hmask;           // [chunks][W] partial masks
  const Batch *batches;
  const Slot *slots;
  const uint32_t *masks;
  int64_t b0, b1;
  // workspace
  int32_t *d;
  double *sig;
  void *q;
  uint32_t *lm;     // [tcap+2][n][W]
  uint32_t *seen;   // [n][W]
  int32_t *lmin, *lmax;
  int32_t *gdone;   // [n] groups of the vertex already seen by all their BFS slots
  int *wq;          // [2*(tcap+3)] work counters of the forward (t) and backward (tcap+3+lev) phases
  double *bcpart;   // [n][W]
  int32_t *X;       // [B][tcap+2]
  int32_t *rexp;    // [B] per-level max exponent (rescale)
  int64_t n_cap;    // rows allocated (>= largest BCC)
  int32_t W;        // words per row (row stride)
  int32_t tcap;     // levels allocated
  int32_t rescale_exp;  // rescale a level's path counts above 2^rescale_exp
  double *bc;
  Ctrl *ctrl;
  int *err;
  int *redo;        // per batch: 1 = FP32 range exceeded, contributions not added
};

__device__ __forceinline__ bool failed(const Args &a) { return *(volatile int *)a.err != kDevOk; }

// The same answer for every thread of the CTA (thread 0 decides).
__device__ __forceinline__ bool cta_failed(const Args &a) {
  __shared__ int s_fail;
  __syncthreads();
  if (threadIdx.x == 0) s_fail = failed(a) ? 1 : 0;
  __syncthreads();
  return s_fail != 0;
}

// Grid-wide barrier for a cooperative launch. Waits are bounded: after
// kSpinLimit polls the CTA records kDevTimeout and continues; once any error
// is flagged every barrier returns at once so the kernel drains quickly.
__device__ void grid_sync(const Args &a) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *gen = &a.ctrl->bar_gen;
    const unsigned int g = *gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(&a.ctrl->bar_count, 1u);
    if (arrived == gridDim.x - 1) {
      a.ctrl->bar_count = 0;
      __threadfence();
      atomicAdd(&a.ctrl->bar_gen, 1u);
    } else {
      long long it = 0;
      while (*gen == g) {
        if (failed(a)) break;
        if (++it > kSpinLimit) { set_err(a.err, kDevTimeout); break; }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Phase timers for profiling builds only (-DBCGPU_PHASE_TIMERS): CTA 0's
// thread 0 accumulates %globaltimer deltas between grid barriers.
#ifdef BCGPU_PHASE_TIMERS
__device__ unsigned long long g_phase_ns[32];
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
#define PHASE_INIT() unsigned long long ph_t = (blockIdx.x == 0 && threadIdx.x == 0) ? gtimer() : 0ull
#define PHASE_MARK(id)                                             \
  do {                                                             \
    if (blockIdx.x == 0 && threadIdx.x == 0) {                     \
      const unsigned long long ph_n = gtimer();                    \
      g_phase_ns[id] += ph_n - ph_t;                               \
      ph_t = ph_n;                                                 \
    }                                                              \
  } while (0)
#define PHASE_COUNT(id) do { if (blockIdx.x == 0 && threadIdx.x == 0) g_phase_ns[id] += 1; } while (0)
#else
#define PHASE_INIT() do {} while (0)
#define PHASE_MARK(id) do {} while (0)
#define PHASE_COUNT(id) do {} while (0)
#endif

__device__ __forceinline__ int64_t gwarp() { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t nwarps() { return ((int64_t)gridDim.x * blockDim.x) >> 5; }


// ---- compensated FP32 accumulation (Neumaier's two-sum variant)
struct Comp32 {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float x) {
    const float t = s + x;
    c += fabsf(s) >= fabsf(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

// ============================================================== forward ====
// A task is one vertex's whole row: lane j loads neighbour j's mask words for
// up to kHalf words at once (aligned 16-byte loads, all in flight), the
// (word, neighbour) pairs that hit are listed in shared memory, and the
// neighbours' path-count rows are gathered eight at a time (lane = slot,
// coalesced) into per-(word, slot) accumulators in shared memory. Adds to an
// accumulator follow neighbour order, so sums are deterministic.

constexpr int kHalf = 8;  // words per pass over a vertex row

struct WarpScratch {
  uint32_t f[32][kHalf + 1];  // neighbour masks of the current 32-arc chunk (padded against bank conflicts)
  uint16_t pairs[32 * kHalf]; // (word << 5 | neighbour lane) of the hits
  double acc[kHalf][32];      // per (word, slot) sums (FP64, or two FP32 halves in the compensated mode)
};

__device__ __forceinline__ uint4 and4(uint4 a, uint4 b) { return make_uint4(a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w); }
__device__ __forceinline__ uint4 ld4(const uint32_t *p) { return __ldcg(reinterpret_cast<const uint4 *>(p)); }

// Loads the kHalf-word mask row at p (first nw words, nw a multiple of 4).
__device__ __forceinline__ void load_row(const uint32_t *p, int nw, uint32_t (&m)[kHalf]) {
#pragma unroll
  for (int g = 0; g < kHalf / 4; ++g) {
    const uint4 x = 4 * g < nw ? ld4(p + 4 * g) : make_uint4(0, 0, 0, 0);
    m[4 * g] = x.x; m[4 * g + 1] = x.y; m[4 * g + 2] = x.z; m[4 * g + 3] = x.w;
  }
}

template <typename T>
__device__ __forceinline__ T warp_or(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One pull / successor pass over arcs [e0, e1) for words [w0, w0+nw):
//   filt[k]  the slots of word w0+k that are looked for (uniform)
//   masks    level masks of the neighbours (level t for the forward, t+1 for the backward)
//   vals     per-slot values gathered on a hit (sigma, or q)
// Accumulates into S.acc (ACC::add) and ORs the hits into any[k] (per lane).
template <typename T, bool kComp>
__device__ __forceinline__ void row_pass(const Args &a, WarpScratch &S, const uint32_t *masks, const T *vals,
                                         int64_t e0, int64_t e1, int w0, int nw, const uint32_t (&filt)[kHalf],
                                         uint32_t (&any)[kHalf], int lane) {
  const int W = a.W;
  for (int64_t base = e0; base < e1; base += 32) {
    const int64_t e = base + lane;
    const bool valid = e < e1;
    const int32_t u = valid ? ldg(a.col + e) : 0;
    uint32_t f[kHalf];
    load_row(masks + (int64_t)u * W + w0, valid ? nw : 0, f);
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < kHalf; ++k) {
      f[k] &= filt[k];
      S.f[lane][k] = f[k];
      any[k] |= f[k];
      cnt += f[k] != 0u;
    }
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int pos = incl - cnt;
#pragma unroll
    for (int k = 0; k < kHalf; ++k)
      if (f[k]) S.pairs[pos++] = (uint16_t)((k << 5) | lane);
    __syncwarp();
    for (int i = 0; i < total; i += 8) {
      T x[8];
      int kk[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        x[r] = (T)0;
        kk[r] = -1;
        if (i + r < total) {  // uniform
          const int p = S.pairs[i + r];
          const int k = p >> 5, j = p & 31;
          const uint32_t fj = S.f[j][k];
          const int32_t uj = __shfl_sync(0xffffffffu, u, j);
          if ((fj >> lane) & 1u) x[r] = __ldcg(vals + ((int64_t)uj * W + w0 + k) * 32 + lane);
          kk[r] = ((fj >> lane) & 1u) ? k : -1;
        }
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        if (kk[r] < 0) continue;
        if (kComp) {
          float2 *c = reinterpret_cast<float2 *>(&S.acc[kk[r]][lane]);
          Comp32 cc;
          cc.s = c->x;
          cc.c = c->y;
          cc.add((float)x[r]);
          *c = make_float2(cc.s, cc.c);
        } else {
          S.acc[kk[r]][lane] += (double)x[r];
        }
      }
    }
    __syncwarp();
  }
}

__device__ __forceinline__ double acc_value(const WarpScratch &S, int k, int lane, bool comp) {
  if (!comp) return S.acc[k][lane];
  const float2 c = *reinterpret_cast<const float2 *>(&S.acc[k][lane]);
  return (double)c.x + (double)c.y;
}

// Stores the result of one (vertex, word) of the forward step.
__device__ __forceinline__ void finish_pull(const Args &a, int32_t v, int w, int t, uint32_t newm, uint32_t own,
                                            int lane, double acc) {
  if (!newm) return;
  const int64_t idx = ((int64_t)v * a.W + w) * 32 + lane;
  if ((newm >> lane) & 1u) {
    a.d[idx] = t + 1;
    a.sig[idx] = acc;
    if (acc > ldexp(1.0, a.rescale_exp)) {
      atomicMax(a.rexp + w * 32 + lane, ilogb(acc));
      a.ctrl->rescale = 1;
    }
  }
  if (lane == 0) {
    a.lm[((int64_t)(t + 1) * a.n_cap + v) * a.W + w] = newm;
    a.seen[(int64_t)v * a.W + w] |= newm;
    a.ctrl->more = 1;
    if (newm & own) {
      atomicMin(a.lmin + v, t + 1);
      atomicMax(a.lmax + v, t + 1);
    }
  }
}

// ============================================================== backward ===

// delta, q and the BC partial of one (vertex, word) at level lev.
template <typename QT>
__device__ __forceinline__ void finish_dep(const Args &a, const Slot *slots, const int32_t *rch, int32_t v, int w,
                                           int lev, uint32_t act, int lane, double sum) {
  constexpr bool kF32 = sizeof(QT) == 4;
  if (!act) return;
  const int W = a.W;
  double contrib = 0.0;
  if ((act >> lane) & 1u) {
    const int b = w * 32 + lane;
    const int64_t idx = ((int64_t)v * W + w) * 32 + lane;
    const double sv = a.sig[idx];
    const int xd = a.X[(int64_t)b * (a.tcap + 2) + lev] - a.X[(int64_t)b * (a.tcap + 2) + lev + 1];
    const double delta = ldexp(sv * sum, xd);
    const double qv = ((double)rch[v] + 1.0 + delta) / sv;
    if (kF32) {
      const double aq = fabs(qv);
      if (!(aq >= (double)FLT_MIN * 0x1p24 && aq <= (double)FLT_MAX * 0x1p-24)) atomicExch(&a.ctrl->range_err, 1);
    }
    reinterpret_cast<QT *>(a.q)[idx] = (QT)qv;
    contrib = delta * ((double)rch[slots[b].src] + 1.0);
  }
  contrib = warp_sum(contrib);  // fixed-order reduction of this word's slots
  if (lane == 0) a.bcpart[(int64_t)v * W + w] += contrib;
}

// Next block of 32 vertices for this warp from the phase's work counter.
__device__ __forceinline__ int64_t next_block(int *counter, int lane) {
  int b = 0;
  if (lane == 0) b = atomicAdd(counter, 1);
  return __shfl_sync(0xffffffffu, b, 0);
}

}  // namespace

// --------------------------------------------------------------- kernel ----

template <typename QT>
__global__ void __launch_bounds__(kThreads, 4) batched_kernel(Args a) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  WarpScratch *scratch = reinterpret_cast<WarpScratch *>(s_raw);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WarpScratch &S = scratch[wib];
  const int W = a.W;
  constexpr bool kComp = sizeof(QT) == 4;
  PHASE_INIT();

  for (int64_t bi = a.b0; bi < a.b1; ++bi) {
    if (cta_failed(a)) return;
    const Batch bt = a.batches[bi];
    const Slot *slots = a.slots + bt.slot_off;
    const uint32_t *bfs_mask = a.masks + bt.mask_off;
    const int words = bt.words;
    const int groups = (words + 3) / 4;
    const int wpad = groups * 4;                 // masks are padded to whole groups
    const uint32_t *own_mask = bfs_mask + wpad;
    const uint32_t *chain_mask = own_mask + wpad;
    const int64_t vo = a.vtx_off[bt.bcc];
    const int32_t n = (int32_t)(a.vtx_off[bt.bcc + 1] - vo);
    const int64_t *R = a.row + vo;
    const int32_t *rch = a.reach + vo;
    const int32_t *hv = a.heavy + a.heavy_off[bt.bcc];
    const int32_t nheavy = (int32_t)(a.heavy_off[bt.bcc + 1] - a.heavy_off[bt.bcc]);
    const int64_t hc0 = a.hchunk_off[bt.bcc];
    const int64_t nchunks = a.hchunk_off[bt.bcc + 1] - hc0;
    const int32_t *hcv = a.hchunk_v + hc0;
    const int64_t *hce0 = a.hchunk_e0 + hc0, *hce1 = a.hchunk_e1 + hc0;
    const int32_t *hfst = a.hfirst + a.heavy_off[bt.bcc] + bt.bcc;  // nheavy+1 entries per BCC
    const int64_t gthreads = (int64_t)gridDim.x * blockDim.x;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nblk = ((int64_t)n + 31) / 32;  // vertex blocks of 32 (lane l takes vertex blk + l*nblk)
    const int halves = (wpad + kHalf - 1) / kHalf;

    // ---- init: seen = non-BFS slots, spans, partials, level-0/1 masks, X, rexp, work counters
    for (int64_t i = gtid; i < (int64_t)n * W; i += gthreads) {
      const int w = (int)(i % W);
      a.seen[i] = w < wpad ? ~bfs_mask[w] : 0xffffffffu;
      a.bcpart[i] = 0.0;
      a.lm[i] = 0;                         // level 0
      a.lm[(int64_t)a.n_cap * W + i] = 0;  // level 1
      if (w == 0) { a.lmin[i / W] = INT_MAX; a.lmax[i / W] = -1; a.gdone[i / W] = 0; }
    }
    for (int64_t i = gtid; i < (int64_t)W * 32; i += gthreads) {
      a.rexp[i] = INT_MIN;
      a.X[i * (a.tcap + 2)] = 0;
    }
    for (int64_t i = gtid; i < 2 * ((int64_t)a.tcap + 3); i += gthreads) a.wq[i] = 0;
    if (gtid == 0) {
      a.ctrl->more = 0;
      a.ctrl->rescale = 0;
      a.ctrl->tmax = 0;
      a.ctrl->range_err = 0;
    }
    grid_sync(a);
    for (int64_t b = gtid; b < bt.nslots; b += gthreads) {  // sources at level 0
      const Slot s = slots[b];
      if (s.kind != kOwn && s.kind != kAux) continue;
      const int64_t idx = ((int64_t)s.src * W + (b >> 5)) * 32 + (b & 31);
      a.d[idx] = 0;
      a.sig[idx] = 1.0;
      atomicOr(a.lm + (int64_t)s.src * W + (b >> 5), 1u << (b & 31));
      atomicOr(a.seen + (int64_t)s.src * W + (b >> 5), 1u << (b & 31));
      if (s.kind == kOwn) { atomicMin(a.lmin + s.src, 0); atomicMax(a.lmax + s.src, 0); }
    }
    grid_sync(a);
    PHASE_MARK(0);

    // ---- forward: levels t -> t+1
    int t = 0;
    while (true) {
      if (t + 1 > a.tcap) { set_err(a.err, kDevWorkspace); break; }
      const uint32_t *lmt = a.lm + (int64_t)t * a.n_cap * W;
      // heavy vertices: chunks of their arcs, one CTA per (chunk, half); partials
      // are combined across the CTA's warps, then across chunks after the barrier
      for (int64_t task = blockIdx.x; task < nchunks * halves; task += gridDim.x) {
        const int64_t c = task / halves;
        const int w0 = (int)(task % halves) * kHalf;
        const int nw = min(kHalf, wpad - w0);
        const int32_t v = hv[hcv[c]];
        uint32_t unseen[kHalf], any[kHalf];
        load_row(a.seen + (int64_t)v * W + w0, nw, unseen);
        uint32_t u_any = 0;
#pragma unroll
        for (int k = 0; k < kHalf; ++k) { unseen[k] = k < nw ? ~unseen[k] : 0u; any[k] = 0; u_any |= unseen[k]; }
#pragma unroll
        for (int k = 0; k < kHalf; ++k) S.acc[k][lane] = 0.0;
        if (u_any) {  // uniform over the CTA
          const int64_t e0 = hce0[c], e1 = hce1[c];
          const int64_t per = (e1 - e0 + kWarpsPerCta - 1) / kWarpsPerCta;
          const int64_t s0 = e0 + wib * per, s1 = min(e1, s0 + per);
          if (s0 < s1) row_pass<double, false>(a, S, lmt, a.sig, s0, s1, w0, nw, unseen, any, lane);
        }
#pragma unroll
        for (int k = 0; k < kHalf; ++k) {
          any[k] = warp_or(any[k]);
          if (lane == 0) S.f[0][k] = any[k];  // this warp's hit masks, for the combine
        }
        __syncthreads();
        for (int k = wib; k < nw; k += kWarpsPerCta) {  // fixed warp order
          double tot = 0.0;
          uint32_t mm = 0;
          for (int x = 0; x < kWarpsPerCta; ++x) { tot += scratch[x].acc[k][lane]; mm |= scratch[x].f[0][k]; }
          a.hacc[((hc0 + c) * W + w0 + k) * 32 + lane] = tot;
          if (lane == 0) a.hmask[(hc0 + c) * W + w0 + k] = mm;
        }
        __syncthreads();
      }
      // light vertices: dynamic blocks of 32, lane-parallel activity check
      for (int64_t vb = next_block(a.wq + t, lane); vb < nblk; vb = next_block(a.wq + t, lane)) {
        const int64_t vl = vb + (int64_t)lane * nblk;
        int64_t e0l = 0, e1l = 0;
        bool on = false;
        if (vl < n) {
          e0l = R[vl];
          e1l = R[vl + 1];
          on = e1l - e0l <= kHeavyDeg && __ldcg(a.gdone + vl) < groups;
        }
        uint32_t todo = __ballot_sync(0xffffffffu, on);
        while (todo) {
          const int j = __ffs(todo) - 1;
          todo &= todo - 1;
          const int32_t v = (int32_t)(vb + (int64_t)j * nblk);
          const int64_t e0 = __shfl_sync(0xffffffffu, e0l, j), e1 = __shfl_sync(0xffffffffu, e1l, j);
          for (int w0 = 0; w0 < wpad; w0 += kHalf) {
            const int nw = min(kHalf, wpad - w0);
            uint32_t seen[kHalf], unseen[kHalf], any[kHalf];
            load_row(a.seen + (int64_t)v * W + w0, nw, seen);
            uint32_t u_any = 0;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) { unseen[k] = k < nw ? ~seen[k] : 0u; any[k] = 0; u_any |= unseen[k]; }
            if (!u_any) continue;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) S.acc[k][lane] = 0.0;
            row_pass<double, false>(a, S, lmt, a.sig, e0, e1, w0, nw, unseen, any, lane);
#pragma unroll
            for (int k = 0; k < kHalf; ++k) {
              if (k >= nw) continue;
              const uint32_t m = warp_or(any[k]);
              finish_pull(a, v, w0 + k, t, m, own_mask[w0 + k], lane, S.acc[k][lane]);
              any[k] = m;
            }
#pragma unroll
            for (int g = 0; g < kHalf / 4; ++g) {  // groups now seen by all their BFS slots
              if (4 * g >= nw || lane != 0) continue;
              bool was = true, now = true;
#pragma unroll
              for (int k = 4 * g; k < 4 * g + 4; ++k) {
                was = was && unseen[k] == 0u;
                now = now && (unseen[k] & ~any[k]) == 0u;
              }
              if (now && !was) atomicAdd(a.gdone + v, 1);
            }
          }
        }
      }
      grid_sync(a);
      PHASE_MARK(1);
      PHASE_COUNT(16);
      if (nheavy) {
        for (int64_t task = gwarp(); task < (int64_t)nheavy * wpad; task += nwarps()) {
          const int32_t h = (int32_t)(task / wpad);
          const int w = (int)(task % wpad);
          const int32_t v = hv[h];
          if (!~__ldcg(a.seen + (int64_t)v * W + w)) continue;
          double acc = 0.0;
          uint32_t m = 0;
          for (int32_t c = hfst[h]; c < hfst[h + 1]; ++c) {
            acc += __ldcg(a.hacc + ((hc0 + c) * W + w) * 32 + lane);
            m |= __ldcg(a.hmask + (hc0 + c) * W + w);
          }
          finish_pull(a, v, w, t, m, own_mask[w], lane, acc);
        }
        grid_sync(a);
        PHASE_MARK(2);
      }
      const int more = *(volatile int *)&a.ctrl->more;
      const int resc = *(volatile int *)&a.ctrl->rescale;
      // base exponent of level t+1; rescale it when some slot's counts passed 2^rescale_exp
      for (int64_t b = gtid; b < (int64_t)W * 32; b += gthreads) {
        const int re = __ldcg(a.rexp + b);
        a.X[b * (a.tcap + 2) + t + 1] = a.X[b * (a.tcap + 2) + t] + (re > a.rescale_exp ? re : 0);
      }
      if (resc) {
        for (int64_t task = gwarp(); task < (int64_t)n * words; task += nwarps()) {
          const int32_t v = (int32_t)(task / words);
          const int w = (int)(task % words);
          const uint32_t m = __ldcg(a.lm + ((int64_t)(t + 1) * a.n_cap + v) * W + w);
          const int re = __ldcg(a.rexp + w * 32 + lane);
          if (((m >> lane) & 1u) && re > a.rescale_exp) {
            const int64_t idx = ((int64_t)v * W + w) * 32 + lane;
            a.sig[idx] = ldexp(a.sig[idx], -re);
          }
        }
      }
      grid_sync(a);  // everyone has read more/rescale/rexp
      if (resc)
        for (int64_t b = gtid; b < (int64_t)W * 32; b += gthreads) a.rexp[b] = INT_MIN;
      if (gtid == 0) {
        a.ctrl->more = 0;
        a.ctrl->rescale = 0;
      }
      if (!more || cta_failed(a)) break;
      ++t;
      for (int64_t i = gtid; i < (int64_t)n * W; i += gthreads) a.lm[(int64_t)(t + 1) * a.n_cap * W + i] = 0;
      grid_sync(a);
      PHASE_MARK(3);
    }
    PHASE_MARK(3);
    if (cta_failed(a)) return;
    const int tbfs = t;  // deepest level with BFS vertices

    // ---- chain slots: clear the levels above the BFS depth they may use,
    // per-level base exponents, then the merge
    const int top = min(a.tcap + 1, tbfs + bt.max_off + 1);
    for (int lv = tbfs + 2; lv <= top; ++lv)
      for (int64_t i = gtid; i < (int64_t)n * W; i += gthreads) a.lm[(int64_t)lv * a.n_cap * W + i] = 0;
    for (int64_t i = gtid; i < (int64_t)bt.nslots * (a.tcap + 1); i += gthreads) {
      const int b = (int)(i / (a.tcap + 1));
      const int lv = (int)(i % (a.tcap + 1));
      const Slot s = slots[b];
      if (s.kind != kChain) continue;
      int x = INT_MIN;
      if (lv - s.ld >= 0 && lv - s.ld <= tbfs) x = max(x, a.X[(int64_t)s.sl * (a.tcap + 2) + lv - s.ld]);
      if (lv - s.rd >= 0 && lv - s.rd <= tbfs) x = max(x, a.X[(int64_t)s.sr * (a.tcap + 2) + lv - s.rd]);
      a.X[(int64_t)b * (a.tcap + 2) + lv] = x == INT_MIN ? 0 : x;
    }
    grid_sync(a);
    int tmax_local = tbfs;
    for (int64_t task = gwarp(); task < (int64_t)n * words; task += nwarps()) {
      const int32_t v = (int32_t)(task / words);
      const int w = (int)(task % words);
      // every BFS slot must have reached every vertex of the BCC
      if (lane == 0 && ~__ldcg(a.seen + (int64_t)v * W + w) != 0u) set_err(a.err, kDevDisconnected);
      const uint32_t cm = chain_mask[w];
      if (!cm) continue;
      const int b = w * 32 + lane;
      int lvl = -1;
      if ((cm >> lane) & 1u) {
        const Slot s = slots[b];
        const int64_t il = ((int64_t)v * W + (s.sl >> 5)) * 32 + (s.sl & 31);
        const int64_t ir = ((int64_t)v * W + (s.sr >> 5)) * 32 + (s.sr & 31);
        int dl = a.d[il], dr = a.d[ir];
        if (dl < 0 || dl > tbfs || dr < 0 || dr > tbfs) {  // unreached (flagged above): keep indices in range
          set_err(a.err, kDevDisconnected);
          dl = dr = 0;
        }
        const int x1 = dl + s.ld, x2 = dr + s.rd;
        lvl = min(x1, x2);
        if (lvl > a.tcap) {  // cannot happen within the eccentricity bound; keep indices in range
          set_err(a.err, kDevWorkspace);
          lvl = a.tcap;
        }
        const int xz = a.X[(int64_t)b * (a.tcap + 2) + lvl];
        double sg = 0.0;
        if (x1 <= x2) sg += ldexp(a.sig[il], a.X[(int64_t)s.sl * (a.tcap + 2) + dl] - xz);
        if (x2 <= x1) sg += ldexp(a.sig[ir], a.X[(int64_t)s.sr * (a.tcap + 2) + dr] - xz);
        const int64_t iz = ((int64_t)v * W + w) * 32 + lane;
        a.d[iz] = lvl;
        a.sig[iz] = sg;
        tmax_local = max(tmax_local, lvl);
      }
      // set level bits: one writer per (vertex, word) in this phase
      uint32_t todo = __ballot_sync(0xffffffffu, lvl >= 0);
      while (todo) {
        const int leader = __ffs(todo) - 1;
        const int L = __shfl_sync(0xffffffffu, lvl, leader);
        const uint32_t grp = __ballot_sync(0xffffffffu, lvl == L);
        if (lane == leader) {
          a.lm[((int64_t)L * a.n_cap + v) * W + w] |= grp;
          atomicMin(a.lmin + v, L);
          atomicMax(a.lmax + v, L);
        }
        todo &= ~grp;
      }
    }
    tmax_local = warp_max(tmax_local);
    if (lane == 0) atomicMax(&a.ctrl->tmax, tmax_local);
    grid_sync(a);
    // same-chain vertices: the direct distance along the chain wins or ties
    for (int64_t b = gtid; b < bt.nslots; b += gthreads) {
      const Slot s = slots[b];
      if (s.kind != kChain) continue;
      for (int j = 0; j < s.clen; ++j) {
        const int32_t k = s.cstart + j;
        const int dist = j > s.cpos ? j - s.cpos : s.cpos - j;
        const int64_t iz = ((int64_t)k * W + (b >> 5)) * 32 + (b & 31);
        const int cur = a.d[iz];
        const double one = ldexp(1.0, -a.X[b * (a.tcap + 2) + dist]);
        if (cur > dist) {
          atomicAnd(a.lm + ((int64_t)cur * a.n_cap + k) * W + (b >> 5), ~(1u << (b & 31)));
          atomicOr(a.lm + ((int64_t)dist * a.n_cap + k) * W + (b >> 5), 1u << (b & 31));
          atomicMin(a.lmin + k, dist);
          a.d[iz] = dist;
          a.sig[iz] = one;
        } else if (cur == dist) {
          a.sig[iz] += one;
        }
      }
    }
    grid_sync(a);
    const int tmax = *(volatile int *)&a.ctrl->tmax;
    if (tmax + 1 > a.tcap) set_err(a.err, kDevWorkspace);
    if (cta_failed(a)) return;
    PHASE_MARK(4);

    // ---- backward: t = tmax .. 1
    for (int lev = tmax; lev >= 1; --lev) {
      const uint32_t *lm_here = a.lm + (int64_t)lev * a.n_cap * W;
      const uint32_t *lm_next = a.lm + (int64_t)(lev + 1) * a.n_cap * W;
      const QT *q = reinterpret_cast<const QT *>(a.q);
      // heavy vertices: chunked successor sums, combined below
      for (int64_t task = blockIdx.x; task < nchunks * halves; task += gridDim.x) {
        const int64_t c = task / halves;
        const int w0 = (int)(task % halves) * kHalf;
        const int nw = min(kHalf, wpad - w0);
        const int32_t v = hv[hcv[c]];
        uint32_t act[kHalf], any[kHalf];
        load_row(lm_here + (int64_t)v * W + w0, nw, act);
        const bool in_span = lev >= __ldcg(a.lmin + v) && lev <= __ldcg(a.lmax + v);
        uint32_t a_any = 0;
#pragma unroll
        for (int k = 0; k < kHalf; ++k) {
          act[k] = (in_span && k < nw) ? act[k] & own_mask[w0 + k] : 0u;
          any[k] = 0;
          a_any |= act[k];
        }
#pragma unroll
        for (int k = 0; k < kHalf; ++k) S.acc[k][lane] = 0.0;
        if (a_any) {  // uniform over the CTA
          const int64_t e0 = hce0[c], e1 = hce1[c];
          const int64_t per = (e1 - e0 + kWarpsPerCta - 1) / kWarpsPerCta;
          const int64_t s0 = e0 + wib * per, s1 = min(e1, s0 + per);
          if (s0 < s1) row_pass<QT, kComp>(a, S, lm_next, q, s0, s1, w0, nw, act, any, lane);
        }
        __syncthreads();
        for (int k = wib; k < nw; k += kWarpsPerCta) {  // fixed warp order
          double tot = 0.0;
          for (int x = 0; x < kWarpsPerCta; ++x) tot += acc_value(scratch[x], k, lane, kComp);
          a.hacc[((hc0 + c) * W + w0 + k) * 32 + lane] = tot;
        }
        __syncthreads();
      }
      const int wqi = a.tcap + 3 + lev;
      for (int64_t vb = next_block(a.wq + wqi, lane); vb < nblk; vb = next_block(a.wq + wqi, lane)) {
        const int64_t vl = vb + (int64_t)lane * nblk;
        int64_t e0l = 0, e1l = 0;
        bool on = false;
        if (vl < n && lev >= __ldcg(a.lmin + vl) && lev <= __ldcg(a.lmax + vl)) {
          e0l = R[vl];
          e1l = R[vl + 1];
          on = e1l - e0l <= kHeavyDeg;
        }
        uint32_t todo = __ballot_sync(0xffffffffu, on);
        while (todo) {
          const int j = __ffs(todo) - 1;
          todo &= todo - 1;
          const int32_t v = (int32_t)(vb + (int64_t)j * nblk);
          const int64_t e0 = __shfl_sync(0xffffffffu, e0l, j), e1 = __shfl_sync(0xffffffffu, e1l, j);
          for (int w0 = 0; w0 < wpad; w0 += kHalf) {
            const int nw = min(kHalf, wpad - w0);
            uint32_t act[kHalf], any[kHalf];
            load_row(lm_here + (int64_t)v * W + w0, nw, act);
            uint32_t a_any = 0;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) {
              act[k] = k < nw ? act[k] & own_mask[w0 + k] : 0u;
              any[k] = 0;
              a_any |= act[k];
            }
            if (!a_any) continue;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) S.acc[k][lane] = 0.0;
            row_pass<QT, kComp>(a, S, lm_next, q, e0, e1, w0, nw, act, any, lane);
#pragma unroll
            for (int k = 0; k < kHalf; ++k)
              if (k < nw) finish_dep<QT>(a, slots, rch, v, w0 + k, lev, act[k], lane, acc_value(S, k, lane, kComp));
          }
        }
      }
      if (nheavy) {
        grid_sync(a);
        PHASE_MARK(5);
        for (int64_t task = gwarp(); task < (int64_t)nheavy * wpad; task += nwarps()) {
          const int32_t h = (int32_t)(task / wpad);
          const int w = (int)(task % wpad);
          const int32_t v = hv[h];
          if (lev < __ldcg(a.lmin + v) || lev > __ldcg(a.lmax + v)) continue;
          const uint32_t act = __ldcg(lm_here + (int64_t)v * W + w) & own_mask[w];
          if (!act) continue;
          double sum = 0.0;
          for (int32_t c = hfst[h]; c < hfst[h + 1]; ++c) sum += __ldcg(a.hacc + ((hc0 + c) * W + w) * 32 + lane);
          finish_dep<QT>(a, slots, rch, v, w, lev, act, lane, sum);
        }
      }
      grid_sync(a);
      PHASE_MARK(6);
      PHASE_COUNT(17);
    }
    // ---- fold the batch into BC (fixed word order), unless FP32 range failed
    const int bad = *(volatile int *)&a.ctrl->range_err;
    if (bad) {
      if (gtid == 0) a.redo[bi] = 1;
    } else {
      for (int64_t v = gtid; v < n; v += gthreads) {
        double s = 0.0;
        for (int w = 0; w < words; ++w) s += a.bcpart[v * W + w];
        a.bc[vo + v] += s;
      }
    }
    grid_sync(a);
    PHASE_MARK(7);
  }
}

// ================================================================= host ====

struct BatchedPlan {
  int width = 0;       // B
  int W = 0;           // words
  int tcap = 0;
  int64_t n_cap = 0;
  bool f32 = true;
  int grid = 0;
  size_t smem = 0;
  int64_t bytes = 0;
  std::vector<void *> allocs;
  Args args{};
  std::vector<int64_t> u_src, u_teps, u_bfs, u_aux, u_visits;
  std::vector<Batch> h_batches;
  std::vector<Slot> h_slots;
  std::vector<int64_t> h_vtx_off;
  int64_t n_batches = 0;
};

namespace {

// Eccentricity bound of a BCC (BFS from local vertex 0): every level of every
// source is < 2 * ecc + 1.
int bcc_ecc(const int64_t *row, const int32_t *col, int64_t vo, int32_t nb, std::vector<int32_t> &dist,
            std::vector<int32_t> &queue) {
  dist.assign((size_t)nb, -1);
  queue.resize((size_t)nb);
  int head = 0, tail = 0;
  queue[tail++] = 0;
  dist[0] = 0;
  int ecc = 0;
  while (head < tail) {
    const int32_t x = queue[head++];
    ecc = std::max(ecc, dist[x]);
    for (int64_t e = row[vo + x]; e < row[vo + x + 1]; ++e) {
      const int32_t y = col[e];
      if (dist[y] < 0) { dist[y] = dist[x] + 1; queue[tail++] = y; }
    }
  }
  return ecc;
}

}  // namespace

int batched_create(const bc_bccs *B, const BatchedConfig &cfg, const int64_t *row, const int32_t *col,
                   const int32_t *reach, const int64_t *vtx_off, const int32_t *chain_start, const int32_t *chain_len,
                   const int32_t *chain_l, const int32_t *chain_r, double *bc, int *err, cudaStream_t stream,
                   BatchedPlan **out, std::string *msg) {
  (void)chain_start; (void)chain_len; (void)chain_l; (void)chain_r;
  auto *P = new BatchedPlan;
  auto bail = [&](int code, const std::string &m) {
    if (msg) *msg = m;
    batched_destroy(P);
    return code;
  };
  P->f32 = cfg.delta_fp32c;
  int width = cfg.width > 0 ? cfg.width : 512;
  width = std::max(32, std::min(1024, (width + 31) / 32 * 32));
  P->width = width;
  P->W = (width / 32 + 3) / 4 * 4;  // row stride: whole 4-word groups (16-byte mask loads)
  const int W = P->W;

  // ---- host scheduling: batches of slots per BCC
  std::vector<Slot> slots;
  std::vector<uint32_t> masks;
  std::vector<int64_t> heavy_off{0}, hchunk_off{0}, hchunk_e0, hchunk_e1;
  std::vector<int32_t> heavy, hchunk_v, hfirst;
  std::vector<int32_t> dist, queue;
  int64_t nmax = 0;
  int tcap = 2;
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    const int64_t vo = B->vtx_off[b];
    const int32_t nb = (int32_t)(B->vtx_off[b + 1] - vo);
    const int32_t npl = B->n_plain[b];
    nmax = std::max<int64_t>(nmax, nb);
    const int64_t arcs = B->row[vo + nb] - B->row[vo];
    int32_t hidx = 0;
    for (int32_t k = 0; k < nb; ++k) {
      const int64_t e0 = B->row[vo + k], e1 = B->row[vo + k + 1];
      if (e1 - e0 <= kHeavyDeg) continue;
      heavy.push_back(k);
      hfirst.push_back((int32_t)((int64_t)hchunk_v.size() - hchunk_off.back()));
      for (int64_t e = e0; e < e1; e += kChunkArcs) {
        hchunk_v.push_back(hidx);
        hchunk_e0.push_back(e);
        hchunk_e1.push_back(std::min<int64_t>(e1, e + kChunkArcs));
      }
      ++hidx;
    }
    hfirst.push_back((int32_t)((int64_t)hchunk_v.size() - hchunk_off.back()));
    heavy_off.push_back((int64_t)heavy.size());
    hchunk_off.push_back((int64_t)hchunk_v.size());
    int maxchain = 0;
    for (int64_t c = B->chain_off[b]; c < B->chain_off[b + 1]; ++c) maxchain = std::max(maxchain, B->chain_len[c]);
    tcap = std::max(tcap, 2 * bcc_ecc(B->row, B->col, vo, nb, dist, queue) + maxchain + 3);

    // greedy packing: each plain source with the chains it owns
    std::vector<Slot> cur;
    std::vector<int32_t> slot_of((size_t)nb, -1);
    const bool merge = cfg.chain_merge;
    const int32_t nsrc_bfs = merge ? npl : nb;  // vertices that become BFS slots
    std::vector<int32_t> touched;
    int64_t c = B->chain_off[b];
    const int64_t ce = B->chain_off[b + 1];
    int64_t src_cnt = 0, bfs_cnt = 0, aux_cnt = 0;
    auto flush = [&]() {
      if (cur.empty()) return;
      Batch bt{};
      bt.bcc = b;
      bt.nslots = (int32_t)cur.size();
      bt.max_off = 0;
      for (const Slot &z : cur)
        if (z.kind == kChain) bt.max_off = std::max(bt.max_off, std::max(z.ld, z.rd));
      bt.words = (bt.nslots + 31) / 32;
      bt.slot_off = (int64_t)slots.size();
      bt.mask_off = (int64_t)masks.size();
      const int wpad = (bt.words + 3) / 4 * 4;  // masks padded to whole groups, 16-byte aligned
      std::vector<uint32_t> mb((size_t)wpad, 0), mo((size_t)wpad, 0), mc((size_t)wpad, 0);
      for (int32_t i = 0; i < bt.nslots; ++i) {
        const uint32_t bit = 1u << (i & 31);
        if (cur[i].kind == kOwn || cur[i].kind == kAux) mb[i >> 5] |= bit;
        if (cur[i].kind == kOwn || cur[i].kind == kChain) mo[i >> 5] |= bit;
        if (cur[i].kind == kChain) mc[i >> 5] |= bit;
      }
      masks.insert(masks.end(), mb.begin(), mb.end());
      masks.insert(masks.end(), mo.begin(), mo.end());
      masks.insert(masks.end(), mc.begin(), mc.end());
      slots.insert(slots.end(), cur.begin(), cur.end());
      P->h_batches.push_back(bt);
      const int64_t prev = P->u_src.empty() ? 0 : P->u_src.back();
      (void)prev;
      P->u_src.push_back(src_cnt);
      P->u_teps.push_back(src_cnt * arcs);
      P->u_bfs.push_back(bfs_cnt);
      P->u_aux.push_back(aux_cnt);
      P->u_visits.push_back(src_cnt * nb);
      for (int32_t x : touched) slot_of[x] = -1;
      touched.clear();
      cur.clear();
      src_cnt = bfs_cnt = aux_cnt = 0;
    };
    auto bfs_slot = [&](int32_t x, int32_t kind) -> int32_t {
      if (slot_of[x] >= 0) {
        if (kind == kOwn && cur[slot_of[x]].kind == kAux) {
          cur[slot_of[x]].kind = kOwn;
          ++src_cnt; ++bfs_cnt; --aux_cnt;
        }
        return slot_of[x];
      }
      Slot s{};
      s.kind = kind;
      s.src = x;
      slot_of[x] = (int32_t)cur.size();
      touched.push_back(x);
      cur.push_back(s);
      if (kind == kOwn) { ++src_cnt; ++bfs_cnt; }
      else ++aux_cnt;
      return slot_of[x];
    };
    // Source order: bounded BFS balls of nearby plain vertices, so a pass's
    // sources see every vertex within a narrow band of levels (few active
    // levels per vertex, dense 32-slot hits) and the right endpoints of the
    // chains they own are mostly own slots of the same pass.
    // Each chain is owned (scheduled with) its lower-degree endpoint: a pass
    // then holds many small owners whose chains lead to the same few hubs,
    // which appear once each as helper BFS slots.
    auto degb = [&](int32_t x) { return B->row[vo + x + 1] - B->row[vo + x]; };
    std::vector<int64_t> own_off((size_t)npl + 1, 0);
    std::vector<int64_t> owned((size_t)(ce - B->chain_off[b]));
    auto owner = [&](int64_t cc) {
      const int32_t l = B->chain_l[cc], r = B->chain_r[cc];
      return degb(l) <= degb(r) ? l : r;
    };
    for (int64_t cc = B->chain_off[b]; cc < ce; ++cc) own_off[owner(cc) + 1]++;
    for (int32_t x = 0; x < npl; ++x) own_off[x + 1] += own_off[x];
    {
      std::vector<int64_t> fill(own_off.begin(), own_off.end() - 1);
      for (int64_t cc = B->chain_off[b]; cc < ce; ++cc) owned[fill[owner(cc)]++] = cc;
    }
    auto slots_of = [&](int32_t s) {
      int64_t k = 1;
      if (merge && s < npl)
        for (int64_t i = own_off[s]; i < own_off[s + 1]; ++i) k += B->chain_len[owned[i]];
      return k;
    };
    std::vector<int32_t> order;
    order.reserve((size_t)nsrc_bfs);
    {
      std::vector<char> done((size_t)nsrc_bfs, 0);
      std::vector<int32_t> stamp((size_t)nb, -1), q;
      int32_t ball = 0;
      const int64_t arc_budget = 16 * (int64_t)width;  // bounds the host work per ball
      // A ball grows only through vertices it can still take (and, in the
      // merge form, through chain vertices): each source's arcs are scanned
      // once, so late balls cost no rescans of finished regions.
      for (int32_t seed = 0; seed < nsrc_bfs; ++seed) {
        if (done[seed]) continue;
        q.clear();
        q.push_back(seed);
        stamp[seed] = ball;
        int64_t got = 0, scanned = 0;
        for (size_t h = 0; h < q.size() && got < width; ++h) {
          const int32_t x = q[h];
          if (x < nsrc_bfs) {
            done[x] = 1;
            order.push_back(x);
            got += slots_of(x);
          }
          if (scanned >= arc_budget) continue;  // keep draining the queue, stop growing it
          const int64_t e0 = B->row[vo + x], e1 = std::min(B->row[vo + x + 1], e0 + arc_budget - scanned);
          scanned += e1 - e0;
          for (int64_t e = e0; e < e1; ++e) {
            const int32_t y = B->col[e];
            if (stamp[y] != ball && (y >= nsrc_bfs || !done[y])) { stamp[y] = ball; q.push_back(y); }
          }
        }
        ++ball;
      }
    }
    for (int32_t s : order) {
      if ((int)cur.size() + 1 > width) flush();
      bfs_slot(s, kOwn);
      if (!merge) continue;
      for (int64_t oi = own_off[s]; oi < own_off[s + 1]; ++oi) {
        c = owned[oi];
        const int32_t len = B->chain_len[c];
        const int32_t other = B->chain_l[c] == s ? B->chain_r[c] : B->chain_l[c];
        const int need = len + (slot_of[other] >= 0 ? 0 : 1);
        if ((int)cur.size() + need > width) {
          flush();
          bfs_slot(s, kAux);  // the owner returns as a forward-only slot
        }
        if ((int)cur.size() + len + (slot_of[other] >= 0 ? 0 : 1) > width) {
          if (msg) *msg = "chain longer than the batch width";
          delete P;
          return BCGPU_EINVAL;
        }
        bfs_slot(other, kAux);
        const int32_t sl = slot_of[B->chain_l[c]], sr = slot_of[B->chain_r[c]];
        for (int32_t pos = 0; pos < len; ++pos) {
          Slot z{};
          z.kind = kChain;
          z.src = B->chain_start[c] + pos;
          z.sl = sl; z.sr = sr;
          z.ld = pos + 1; z.rd = len - pos;
          z.cstart = B->chain_start[c]; z.clen = len; z.cpos = pos;
          cur.push_back(z);
          ++src_cnt;
        }
      }
    }
    flush();
  }
  P->tcap = tcap;
  P->n_cap = std::max<int64_t>(nmax, 1);
  P->n_batches = (int64_t)P->h_batches.size();
  // prefix sums over batches
  auto prefix = [](std::vector<int64_t> &v) {
    std::vector<int64_t> p(v.size() + 1, 0);
    for (size_t i = 0; i < v.size(); ++i) p[i + 1] = p[i] + v[i];
    v.swap(p);
  };
  prefix(P->u_src); prefix(P->u_teps); prefix(P->u_bfs); prefix(P->u_aux); prefix(P->u_visits);

  // ---- device workspace
  const int64_t n = P->n_cap;
  const int64_t qb = P->f32 ? 4 : 8;
  const int64_t need = n * W * 32 * (4 + 8 + qb) + (int64_t)(tcap + 2) * n * W * 4 + n * W * (4 + 8) + n * 12 +
                       (int64_t)W * 32 * (tcap + 2) * 4;
  if (need > cfg.limit_bytes)
    return bail(BCGPU_ENOMEM, "batched workspace " + std::to_string(need >> 20) + " MiB exceeds the limit " +
                                  std::to_string(cfg.limit_bytes >> 20) + " MiB (lower the batch width)");
  auto alloc = [&](void **p, int64_t bytes) -> bool {
    if (cudaMalloc(p, (size_t)std::max<int64_t>(bytes, 16)) != cudaSuccess) return false;
    P->allocs.push_back(*p);
    P->bytes += bytes;
    return true;
  };
  Args &a = P->args;
  void *p = nullptr;
  bool ok = true;
  ok &= alloc(&p, n * W * 32 * 4); a.d = (int32_t *)p;
  ok &= ok && alloc(&p, n * W * 32 * 8); a.sig = (double *)p;
  ok &= ok && alloc(&p, n * W * 32 * qb); a.q = p;
  ok &= ok && alloc(&p, (int64_t)(tcap + 2) * n * W * 4); a.lm = (uint32_t *)p;
  ok &= ok && alloc(&p, n * W * 4); a.seen = (uint32_t *)p;
  ok &= ok && alloc(&p, n * 4); a.lmin = (int32_t *)p;
  ok &= ok && alloc(&p, n * 4); a.lmax = (int32_t *)p;
  ok &= ok && alloc(&p, n * 4); a.gdone = (int32_t *)p;
  ok &= ok && alloc(&p, 2 * ((int64_t)tcap + 3) * 4); a.wq = (int *)p;
  ok &= ok && alloc(&p, n * W * 8); a.bcpart = (double *)p;
  ok &= ok && alloc(&p, (int64_t)W * 32 * (tcap + 2) * 4); a.X = (int32_t *)p;
  ok &= ok && alloc(&p, (int64_t)W * 32 * 4); a.rexp = (int32_t *)p;
  ok &= ok && alloc(&p, sizeof(Ctrl)); a.ctrl = (Ctrl *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<int64_t>(P->n_batches, 1) * 4); a.redo = (int *)p;
  ok &= ok && alloc(&p, (int64_t)heavy_off.size() * 8); a.heavy_off = (int64_t *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<size_t>(heavy.size(), 1) * 4); a.heavy = (int32_t *)p;
  const int64_t nch = (int64_t)hchunk_v.size();
  ok &= ok && alloc(&p, (int64_t)hchunk_off.size() * 8); a.hchunk_off = (int64_t *)p;
  ok &= ok && alloc(&p, std::max<int64_t>(nch, 1) * 4); a.hchunk_v = (int32_t *)p;
  ok &= ok && alloc(&p, std::max<int64_t>(nch, 1) * 8); a.hchunk_e0 = (int64_t *)p;
  ok &= ok && alloc(&p, std::max<int64_t>(nch, 1) * 8); a.hchunk_e1 = (int64_t *)p;
  ok &= ok && alloc(&p, (int64_t)hfirst.size() * 4); a.hfirst = (int32_t *)p;
  ok &= ok && alloc(&p, std::max<int64_t>(nch, 1) * W * 32 * 8); a.hacc = (double *)p;
  ok &= ok && alloc(&p, std::max<int64_t>(nch, 1) * W * 4); a.hmask = (uint32_t *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<size_t>(P->h_batches.size(), 1) * sizeof(Batch)); a.batches = (Batch *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<size_t>(slots.size(), 1) * sizeof(Slot)); a.slots = (Slot *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<size_t>(masks.size(), 1) * 4); a.masks = (uint32_t *)p;
  if (!ok) return bail(BCGPU_ENOMEM, "cudaMalloc of the batched workspace failed");
  cudaError_t e = cudaSuccess;
  e = cudaMemsetAsync(a.ctrl, 0, sizeof(Ctrl), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.redo, 0, (size_t)std::max<int64_t>(P->n_batches, 1) * 4, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)a.heavy_off, heavy_off.data(), heavy_off.size() * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !heavy.empty()) e = cudaMemcpyAsync((void *)a.heavy, heavy.data(), heavy.size() * 4, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)a.hchunk_off, hchunk_off.data(), hchunk_off.size() * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && nch) e = cudaMemcpyAsync((void *)a.hchunk_v, hchunk_v.data(), nch * 4, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && nch) e = cudaMemcpyAsync((void *)a.hchunk_e0, hchunk_e0.data(), nch * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && nch) e = cudaMemcpyAsync((void *)a.hchunk_e1, hchunk_e1.data(), nch * 8, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)a.hfirst, hfirst.data(), hfirst.size() * 4, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !P->h_batches.empty())
    e = cudaMemcpyAsync((void *)a.batches, P->h_batches.data(), P->h_batches.size() * sizeof(Batch), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !slots.empty())
    e = cudaMemcpyAsync((void *)a.slots, slots.data(), slots.size() * sizeof(Slot), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess && !masks.empty())
    e = cudaMemcpyAsync((void *)a.masks, masks.data(), masks.size() * 4, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // the host vectors go out of scope
  P->h_slots = slots;
  P->h_vtx_off.assign(B->vtx_off, B->vtx_off + B->n_bcc + 1);
  if (e != cudaSuccess) return bail(BCGPU_ECUDA, std::string("batched upload: ") + cudaGetErrorString(e));
  a.row = row; a.col = col; a.reach = reach; a.vtx_off = vtx_off;
  a.n_cap = P->n_cap; a.W = W; a.tcap = tcap; a.bc = bc; a.err = err;
  a.rescale_exp = cfg.rescale_exp > 0 ? cfg.rescale_exp : 900;

  // cooperative grid: every CTA resident
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (!coop) return bail(BCGPU_ECUDA, "device lacks cooperative launch");
  const size_t smem = sizeof(WarpScratch) * kWarpsPerCta;
  if (cudaFuncSetAttribute(batched_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(batched_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return bail(BCGPU_ECUDA, "cannot reserve shared memory for the batched kernel");
  if (P->f32) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_kernel<float>, kThreads, smem);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_kernel<double>, kThreads, smem);
  P->smem = smem;
  if (per_sm < 1) return bail(BCGPU_ECUDA, "batched kernel does not fit an SM");
  P->grid = sms * per_sm;
  *out = P;
  return BCGPU_OK;
}

void batched_destroy(BatchedPlan *p) {
  if (!p) return;
  for (void *a : p->allocs) cudaFree(a);
  delete p;
}

int64_t batched_device_bytes(const BatchedPlan *p) { return p ? p->bytes : 0; }
int batched_width(const BatchedPlan *p) { return p ? p->width : 0; }

void batched_unit_sources(const BatchedPlan *p, int64_t begin, int64_t end, std::vector<int64_t> &out) {
  for (int64_t bi = begin; bi < end; ++bi) {
    const Batch &bt = p->h_batches[bi];
    const int64_t vo = p->h_vtx_off[bt.bcc];
    for (int32_t i = 0; i < bt.nslots; ++i) {
      const Slot &s = p->h_slots[bt.slot_off + i];
      if (s.kind == kOwn || s.kind == kChain) out.push_back(vo + s.src);
    }
  }
}

void batched_unit_work(const BatchedPlan *p, std::vector<int64_t> &sources, std::vector<int64_t> &teps,
                       std::vector<int64_t> &bfs, std::vector<int64_t> &aux, std::vector<int64_t> &visits) {
  sources = p->u_src; teps = p->u_teps; bfs = p->u_bfs; aux = p->u_aux; visits = p->u_visits;
}

#ifdef BCGPU_PHASE_TIMERS
}  // namespace bcg
extern "C" int bc_debug_phase_times(unsigned long long *out, int reset) {
  if (cudaMemcpyFromSymbol(out, bcg::g_phase_ns, sizeof(unsigned long long) * 32) != cudaSuccess) return 2;
  if (reset) {
    unsigned long long z[32] = {0};
    cudaMemcpyToSymbol(bcg::g_phase_ns, z, sizeof(z));
  }
  return 0;
}
namespace bcg {
#endif

int batched_failed_batches(BatchedPlan *p, cudaStream_t stream, int64_t *count) {
  std::vector<int> h((size_t)std::max<int64_t>(p->n_batches, 1), 0);
  cudaError_t e = cudaMemcpyAsync(h.data(), p->args.redo, h.size() * sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return BCGPU_ECUDA;
  int64_t c = 0;
  for (int x : h) c += x != 0;
  *count = c;
  return BCGPU_OK;
}

int batched_run(BatchedPlan *p, int64_t begin, int64_t end, cudaStream_t stream, int *launches, std::string *msg) {
  if (end <= begin) return BCGPU_OK;
  Args a = p->args;
  a.b0 = begin;
  a.b1 = end;
  void *params[] = {&a};
  cudaError_t e = cudaMemsetAsync(&p->args.ctrl->bar_count, 0, 2 * sizeof(unsigned int), stream);
  if (e == cudaSuccess) {
    if (p->f32) e = cudaLaunchCooperativeKernel((void *)batched_kernel<float>, p->grid, kThreads, params, p->smem, stream);
    else e = cudaLaunchCooperativeKernel((void *)batched_kernel<double>, p->grid, kThreads, params, p->smem, stream);
  }
  if (e != cudaSuccess) {
    if (msg) *msg = std::string("cooperative launch: ") + cudaGetErrorString(e);
    return BCGPU_ECUDA;
  }
  if (launches) *launches += 1;
  return BCGPU_OK;
}

}  // namespace bcg
