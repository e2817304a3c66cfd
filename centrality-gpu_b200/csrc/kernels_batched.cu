// BATCHED schedule: many sources per pass as a bitmask multi-source BFS over
// each BCC with its degree-2 chains contracted.
//
// Contracted graph. Within a BCC the core vertices (local ids < n_plain) keep
// their arcs to each other ("unit arcs"); a chain c of k degree-2 vertices
// between the core endpoints L and R becomes one arc L-R of length k+1 in
// both endpoint rows ("chain arcs", listed after the unit arcs of a row).
// Chain vertices never enter the level-synchronous phases: their levels, path
// counts and dependencies follow in closed form from the two endpoint columns
// (the reference's ear postprocessing, Codes/postprocesses.cu:205-351, done
// here for every source of the pass at once).
//
// Slots. One pass ("batch") covers up to B = 32*W sources of one BCC:
//   core source     level 0 at the vertex;
//   chain source    the vertex at position p (0-based from L) of a chain of
//                   k vertices: seeded at L on level p+1 and at R on level
//                   k-p, one path each (its two directions along the chain).
// State of the core vertices, vertex-major and slot-minor ([v][B]) so a warp
// reads the 32 slots of a word as one coalesced row segment:
//   d[v][b]     level (int32)            sigma[v][b] path count (FP64, scaled)
//   q[v][b]     (reach(v)+1+delta)/sigma (FP64, or FP32 in the compensated mode)
//   lm[t][v][w] bitmask of the slots that reach v at level t: the frontier of
//               the forward phase and the successor test of the backward phase
// Forward: level-synchronous pull. A core vertex still unseen by some slot
// scans its row once per 32-slot word: a unit arc to u hits the slots in
// lm[t][u], a chain arc of length k+1 hits those in lm[t-k][u]; the hits'
// path counts are summed (the reference's per-source atomicCAS/atomicAdd BFS,
// Codes/kernels_free.cu:286-362).
// Backward: successor form (Codes/kernels_free.cu:377-421), delta(v) =
// sigma(v) * sum of q over successors, where a chain arc of length k+1 is a
// successor arc when the chain carries the far end's shortest paths (the far
// end sits on level lev+k+1), plus what v receives from the chain vertices
// themselves: a closed form in prefix sums of reach+1 along the chain and the
// two ends' path counts, evaluated for every (vertex, slot) in one parallel
// phase between the forward and the backward sweeps.
// Chain vertices: one warp per (chain, 32-slot word) evaluates every chain
// vertex's dependency for the 32 slots from the endpoint columns.
// Path counts carry a per-(slot, level) power-of-two base X so deep graphs do
// not overflow FP64: a level is rescaled when its largest count passes
// 2^rescale_exp (900 by default).
// BC: per (vertex, word) FP64 partials, summed over words in fixed order ->
// deterministic (the reference uses FP32 atomics, Codes/kernels_free.cu:423-426).
// The whole GPU works on one batch at a time: a cooperative persistent kernel
// with a grid barrier whose waits are bounded (error flag, no hang).
#include "accum.cuh"
#include "batched.h"
#include "common.cuh"
#include "internal.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <type_traits>
#include <utility>
#include <vector>

namespace bcg {

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerCta = kThreads / 32;
// Core rows longer than kHeavyDeg arcs are scanned in chunks by whole CTAs
// (RMAT-20 at 512 sources per pass: 143.7 / 153.7 / 160.4 / 160.4 / 162.3 /
// 156.1 GTEPS for 128 / 256 / 512 / 1024 / 2048 / 4096) ...
#ifndef BCGPU_BATCHED_HEAVY_DEG
#define BCGPU_BATCHED_HEAVY_DEG 1024
#endif
constexpr int kHeavyDeg = BCGPU_BATCHED_HEAVY_DEG;
constexpr int kHeavyDegSmall = 32; // ... or than this, on cores small enough that one row is a level's critical path
constexpr int kSmallCore = 16384;  // cores below this many vertices use kHeavyDegSmall
#ifndef BCGPU_BATCHED_CHUNK
#define BCGPU_BATCHED_CHUNK 2048
#endif
constexpr int kChunkArcs = BCGPU_BATCHED_CHUNK;  // arcs per heavy chunk
constexpr int kHalf = 4;           // words per pass over a vertex row
// Resident CTAs per SM the kernel is compiled for (registers per thread =
// 65536 / (kThreads * kMinCtas)) and hit values gathered at once per lane in
// a row pass; profiling builds may override both. Six CTAs (40 registers,
// some spilled to local memory) with the one-arc hit walk measured fastest
// on RMAT-20 at 512 sources per pass: 135 / 139 / 147 / 124 GTEPS for 4 / 5 /
// 6 / 8 CTAs per SM.
#ifndef BCGPU_BATCHED_MIN_CTAS
#define BCGPU_BATCHED_MIN_CTAS 6
#endif
#ifndef BCGPU_BATCHED_GATHER
#define BCGPU_BATCHED_GATHER 4
#endif
// Hit walk of a row pass: n >= 1 = an arc is walked once for all kHalf
// words of the task (one shuffle of its neighbour), n arcs' values loaded at
// once (n * kHalf loads in flight); 0 = word by word, BCGPU_BATCHED_GATHER
// hits at a time. The same terms are added in the same order either way.
#ifndef BCGPU_BATCHED_WALK
#define BCGPU_BATCHED_WALK 1
#endif
constexpr int kMinCtas = BCGPU_BATCHED_MIN_CTAS;
// Light-row tasks per warp and level at least (smaller vertex blocks when
// the core is small), so the slowest tasks at a level's end are short: on
// RMAT-20 (512 sources per pass) 8 / 16 / 32 gave 147.2 / 150.4 / 151.8 GTEPS.
#ifndef BCGPU_BATCHED_TASKS
#define BCGPU_BATCHED_TASKS 32
#endif
constexpr int kTasksPerWarp = BCGPU_BATCHED_TASKS;
constexpr int kGatherHits = BCGPU_BATCHED_GATHER;

// One source of a pass. chain < 0: the core vertex src (level 0). Otherwise
// src is the chain vertex at position pos of chain `chain` (global index).
struct Slot {
  int32_t src, chain, pos, pad;
};

// Where a chain source enters the core: slot reaches core vertex v on `level`
// with one path along its chain.
struct Seed {
  int32_t v, level, slot, pad;
};

struct Batch {
  int32_t bcc, nslots, words, nseeds;
  int32_t max_seed;  // deepest seed level (0: none)
  int32_t kmax;      // longest chain of the BCC: the longest arc is kmax+1
  int32_t heavy_deg; // rows longer than this are chunked over whole CTAs
  int32_t narm;      // entries of the pass's arming list
  int64_t slot_off, seed_off;
  int64_t arm_off;   // arming list: (vertex, level) of the core sources and seeded vertices
};

// Control block in global memory (one per plan).
struct Ctrl {
  unsigned int bar_count;
  unsigned int bar_gen;
  int more[2];    // forward, by level parity: some slot found a new vertex on the level
  int rescale[2]; // forward, by level parity: some slot needs a rescale on the level
  int range_err;  // FP32 q left FP32's exponent range in this batch
  int pad;
  unsigned long long found;  // forward: (core vertex, slot) pairs reached so far
};

struct Args {
  // contracted rows of the core vertices; BCC b's rows start at hvo[b]
  const int64_t *hvo;
  const int64_t *hrow;    // [n_core_rows + n_bcc] global arc offsets
  const int64_t *hsplit;  // first chain arc of each row
  const int32_t *hcol;    // neighbour (local core id)
  const int32_t *hk;      // chain arcs: vertices on the chain (the arc is one longer)
  const int32_t *hcid;    // chain arcs: chain index * 2 + (the row's vertex is the chain's right end)
  const int32_t *reach;
  const int64_t *vtx_off;
  const int32_t *n_plain;
  // chains (global index)
  const int64_t *chain_off;
  const int32_t *chain_start, *chain_len, *chain_l, *chain_r;
  const int64_t *cpre_off;  // chain -> its k+1 prefix sums of reach+1 (from the left end) in cpre; -1: all reach 0
  const double *cpre;
  // heavy rows (contracted degree > kHeavyDeg), chunked
  const int64_t *heavy_off;  // per BCC range in heavy[]
  const int32_t *heavy;      // local ids
  const int64_t *hchunk_off; // per BCC range in the chunk table
  const int32_t *hchunk_v;   // chunk -> heavy index (within its BCC's heavy list)
  const int64_t *hchunk_e0;  // chunk arc range [e0, e1) (global arc offsets)
  const int64_t *hchunk_e1;
  const int32_t *hfirst;     // heavy index -> first chunk (BCC-relative), hfirst[h+1] ends it
  double *hacc;              // [chunks][W][32] partial successor / path-count sums
  uint32_t *hmask;           // [chunks][W] partial masks
  const Batch *batches;
  const Slot *slots;
  const Seed *seeds;
  const int2 *arms;
  int64_t b0, b1;
  // workspace (core rows)
  int32_t *d;
  double *sig;
  void *q;
  uint32_t *lm;     // [tcap+2][n_cap][W]
  uint32_t *seen;   // [n_cap][W]
  int32_t *lmin, *lmax;
  int32_t *gdone;   // [n_cap] groups of 4 words already seen by all their slots (a lower bound)
  int32_t *armed;   // [n_cap] first level on which some slot can reach the vertex (a neighbour was reached)
  int *wq;          // [4*(tcap+3)+2] work counters: light rows forward (t), backward (tcap+3+lev); heavy chunks (2*(tcap+3)+t, 3*(tcap+3)+lev); chain in-flow (4*(tcap+3)); chain vertices (4*(tcap+3)+1)
  double *bcpart;   // [n_cap][W] BC partials of the core vertices
  double *cdep;     // [n_cap][W][32] dependency a core vertex receives from its chains' vertices
  double *wsrc;     // [B] reach(source)+1 of each slot of the pass
  int32_t *X;       // [B][tcap+2]
  int32_t *rexp;    // [B] per-level max exponent (rescale)
  int64_t n_cap;    // core rows allocated (>= largest core)
  int32_t W;        // words per row (row stride)
  int32_t tcap;     // levels allocated
  int32_t rescale_exp;
  unsigned long long wait_ns;  // limit of one grid-barrier wait
  int32_t pad;
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
// a.wait_ns of device time the CTA records kDevTimeout and continues; once
// any error is flagged every barrier returns at once so the kernel drains
// quickly.
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
      wait_while_equal(gen, g, a.wait_ns, a.err, [&] { return failed(a); });
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

// ============================================================ chain math ===
// A stretch of a chain between two ends A and B holding m chain vertices,
// seen from A: its vertex i (0 <= i < m) lies i+1 arcs from A and m-i from B.
// pre(x) is the sum of reach+1 over its first x vertices counted from A.
// Prefix sum x of a chain: P[x], or x itself on a chain whose vertices have
// nothing hanging off them (P null: no table, no load).
__device__ __forceinline__ double chain_pre(const double *P, int x) { return P ? __ldg(P + x) : (double)x; }

struct Stretch {
  const double *P;  // the chain's prefix sums from its left end (k+1 entries), or null (all reach 0)
  int lo, hi;       // chain positions [lo, hi) of the stretch
  bool rev;         // A is the right-hand end (position hi)
  __device__ __forceinline__ int m() const { return hi - lo; }
  __device__ __forceinline__ double pre(int x) const {
    return rev ? chain_pre(P, hi) - chain_pre(P, hi - x) : chain_pre(P, lo + x) - chain_pre(P, lo);
  }
  __device__ __forceinline__ double wt(int i) const { return pre(i + 1) - pre(i); }
  __device__ __forceinline__ Stretch flip() const { return Stretch{P, lo, hi, !rev}; }
};

// An end of a stretch for one slot, as loaded: its level d, path count
// sigma = s * 2^x and q = qs * 2^-x (qs only read when the stretch carries
// the end's shortest paths). The slot's own source is {0, 0, 1, 0}.
struct End {
  int d, x;
  double s, qs;
};
__device__ __forceinline__ End source_end() { return End{0, 0, 1.0, 0.0}; }

// Dependency of stretch vertex i on the slot's source when i takes its
// shortest paths from A (2i < D): the chain vertices beyond i on the A-fed
// side each add reach+1; the last A-fed vertex either ties (shares its paths
// with B: adds its reach+1 times sigma_A / (sigma_A + sigma_B)) or, when it is
// the vertex next to B and B's shortest paths run through the stretch, passes
// on sigma_A * q(B) (kTail). i = -1 gives what A itself receives.
template <bool kTail>
__device__ __forceinline__ double fed_dep(const Stretch &s, int i, const End &A, const End &B, int D) {
  const int m = s.m();
  const int P = min(m - 1, D / 2);  // last vertex fed from A
  if ((D & 1) == 0 && D / 2 <= m - 1) return s.pre(P) - s.pre(i + 1) + s.wt(P) / (1.0 + scale2(B.s / A.s, B.x - A.x));
  double v = s.pre(P + 1) - s.pre(i + 1);
  if (kTail && P == m - 1 && B.d == A.d + m + 1) v += scale2(A.s * B.qs, A.x - B.x);
  return v;
}

// Dependency of stretch vertex i (0 <= i < m) on the slot's source (out of
// line: only the rare slots whose source sits on the chain take this path).
__device__ __noinline__ double stretch_dep(const Stretch &s, int i, const End &A, const End &B) {
  const int m = s.m();
  const int D = B.d + m - A.d - 1;  // vertex i is fed from A iff 2i <= D, from B iff 2i >= D
  if (2 * i < D) return fed_dep<true>(s, i, A, B, D);
  if (2 * i > D) return fed_dep<true>(s.flip(), m - 1 - i, B, A, A.d + m - B.d - 1);
  return 0.0;  // fed from both ends: no successor on the chain
}

// What end A receives from the stretch's vertices (its neighbour on the
// stretch is its successor iff that neighbour is fed from A: D >= 0), less
// the term through B (sigma_A * q(B) when B's paths run through the
// stretch), which the backward sweep adds as a successor arc.
__device__ __forceinline__ double end_dep(const Stretch &s, const End &A, const End &B) {
  const int D = B.d + s.m() - A.d - 1;
  if (s.m() == 0 || D < 0) return 0.0;
  return fed_dep<false>(s, -1, A, B, D);
}

// ============================================================== forward ====
// A task is one vertex row for kHalf 32-slot words: lane j loads arc j's
// neighbour and its mask words (one aligned 16-byte load), then, word by
// word, the arcs that hit (a ballot) are walked in arc order and their value
// rows gathered four at a time (lane = slot, coalesced) into per-(word,
// slot) accumulators held in registers. Adds follow arc order, so sums are
// deterministic.

// Per-(word, slot) accumulator of a row pass: FP64, or compensated FP32.
template <bool kComp>
struct Acc {
  double s = 0.0;
  __device__ __forceinline__ void add(double x) { s += x; }
  __device__ __forceinline__ double value() const { return s; }
};
template <>
struct Acc<true> {
  Comp32 c;
  __device__ __forceinline__ void add(double x) { c.add((float)x); }
  __device__ __forceinline__ double value() const { return c.value(); }
};

// Per-warp shared memory: partial sums and hit masks of the heavy-row chunks,
// combined across the CTA's warps in fixed order.
struct WarpScratch {
  double acc[kHalf][32];
  uint32_t any[kHalf];
};

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
//   masks    level masks: of level t (unit arcs, kLev == 0), or the
//            level-0 base of lm for chain arcs, whose arc e reads level
//            t - hk[e] (kLev == 1, forward: sigma rebased from that level's
//            X to level t's) or level t + hk[e] (kLev == 2, backward: q
//            rebased to level t's X; levels above tend are empty)
//   vals     per-slot values gathered on a hit (sigma, or q)
// Adds into acc[k] and ORs the hits into any[k] (per lane).
template <typename T, bool kComp, int kLev>
__device__ __forceinline__ void row_pass(const Args &a, const uint32_t *masks, const T *vals, int64_t e0, int64_t e1,
                                         int w0, int nw, const uint32_t (&filt)[kHalf], uint32_t (&any)[kHalf],
                                         Acc<kComp> (&acc)[kHalf], int lane, int t, int tend = 0) {
  const int W = a.W;
  for (int64_t base = e0; base < e1; base += 32) {
    const int64_t e = base + lane;
    bool valid = e < e1;
    const int32_t u = valid ? ldg(a.hcol + e) : 0;
    int lvl = t;
    if (kLev == 1) {
      lvl = valid ? t - ldg(a.hk + e) : -1;
      valid = valid && lvl >= 0;
    } else if (kLev == 2) {
      lvl = valid ? t + ldg(a.hk + e) : INT_MAX;
      valid = valid && lvl <= tend;
    }
    uint32_t f[kHalf];
    const uint32_t *mrow = kLev ? masks + ((int64_t)(valid ? lvl : 0) * a.n_cap + u) * W + w0 : masks + (int64_t)u * W + w0;
    load_row(mrow, valid ? nw : 0, f);
#pragma unroll
    for (int k = 0; k < kHalf; ++k) {
      f[k] &= filt[k];
      any[k] |= f[k];
    }
#if BCGPU_BATCHED_WALK
    uint32_t fo = 0;
#pragma unroll
    for (int k = 0; k < kHalf; ++k) fo |= f[k];
    uint32_t hits = __ballot_sync(0xffffffffu, fo != 0u);
    // level exponent bases of the task's slots: word k's at xb0 + k * xs
    const int64_t xs = (int64_t)32 * (a.tcap + 2);
    const int32_t *xb0 = kLev ? a.X + (int64_t)(w0 * 32 + lane) * (a.tcap + 2) : nullptr;
    int xt[kHalf];
#pragma unroll
    for (int k = 0; k < kHalf; ++k) xt[k] = (kLev && hits) ? __ldcg(xb0 + k * xs + t) : 0;
    const T *vrow = vals + (int64_t)w0 * 32 + lane;
    constexpr int kArcs = BCGPU_BATCHED_WALK;  // hit arcs whose values are loaded at once
    while (hits) {  // uniform: arcs with a hit in some word, in arc order
      T x[kArcs][kHalf];
#pragma unroll
      for (int r = 0; r < kArcs; ++r) {
#pragma unroll
        for (int k = 0; k < kHalf; ++k) x[r][k] = (T)0;
        if (!hits) continue;  // uniform
        const int j = __ffs(hits) - 1;
        hits &= hits - 1;
        const int32_t uj = __shfl_sync(0xffffffffu, u, j);
        const int lj = kLev ? __shfl_sync(0xffffffffu, lvl, j) : 0;
        const T *vu = vrow + (int64_t)uj * W * 32;
#pragma unroll
        for (int k = 0; k < kHalf; ++k) {
          const uint32_t fj = __shfl_sync(0xffffffffu, f[k], j);
          if ((fj >> lane) & 1u) {
            x[r][k] = __ldcg(vu + k * 32);
            if (kLev) {
              const int xl = __ldcg(xb0 + k * xs + lj);
              x[r][k] = (T)scale2((double)x[r][k], kLev == 1 ? xl - xt[k] : xt[k] - xl);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < kArcs; ++r)
#pragma unroll
        for (int k = 0; k < kHalf; ++k) acc[k].add((double)x[r][k]);
    }
#else
#pragma unroll
    for (int k = 0; k < kHalf; ++k) {
      uint32_t hits = __ballot_sync(0xffffffffu, f[k] != 0u);
      const T *vk = vals + (int64_t)(w0 + k) * 32 + lane;
      const int32_t *xb = kLev ? a.X + (int64_t)((w0 + k) * 32 + lane) * (a.tcap + 2) : nullptr;
      const int xt = kLev ? __ldcg(xb + t) : 0;
      while (hits) {  // uniform
        T x[kGatherHits];
#pragma unroll
        for (int r = 0; r < kGatherHits; ++r) {
          x[r] = (T)0;
          if (hits) {  // uniform
            const int j = __ffs(hits) - 1;
            hits &= hits - 1;
            const uint32_t fj = __shfl_sync(0xffffffffu, f[k], j);
            const int32_t uj = __shfl_sync(0xffffffffu, u, j);
            const int lj = kLev ? __shfl_sync(0xffffffffu, lvl, j) : 0;
            if ((fj >> lane) & 1u) {
              x[r] = __ldcg(vk + (int64_t)uj * W * 32);
              if (kLev) x[r] = (T)scale2((double)x[r], kLev == 1 ? __ldcg(xb + lj) - xt : xt - __ldcg(xb + lj));
            }
          }
        }
#pragma unroll
        for (int r = 0; r < kGatherHits; ++r) acc[k].add((double)x[r]);
      }
    }
#endif
  }
}

// Stores the result of one (vertex, word) of the forward step; returns the
// number of slots that reached the vertex, plus 256 when this is the first
// time any slot reached it (uniform over the warp).
__device__ __forceinline__ int finish_pull(const Args &a, int32_t v, int w, int t, uint32_t newm, int lane,
                                           double acc) {
  if (!newm) return 0;
  int first = 0;
  const int64_t idx = ((int64_t)v * a.W + w) * 32 + lane;
  if ((newm >> lane) & 1u) {
    a.d[idx] = t + 1;
    a.sig[idx] = acc;
    if (exp_bits(acc) - 1023 >= a.rescale_exp && acc > pow2(a.rescale_exp)) {  // acc > 2^rescale_exp, acc normal
      atomicMax(a.rexp + w * 32 + lane, exp_bits(acc) - 1023);
      a.ctrl->rescale[t & 1] = 1;
    }
  }
  if (lane == 0) {
    a.lm[((int64_t)(t + 1) * a.n_cap + v) * a.W + w] = newm;
    a.seen[(int64_t)v * a.W + w] |= newm;
    a.ctrl->more[t & 1] = 1;
    first = atomicMin(a.lmin + v, t + 1) == INT_MAX;
    atomicMax(a.lmax + v, t + 1);
  }
  return __popc(newm) + (__shfl_sync(0xffffffffu, first, 0) << 8);
}

// Arms the neighbours of a vertex first reached on level lvl: a neighbour
// across an arc of length k+1 can be reached from it on level lvl+k+1.
__device__ __forceinline__ void arm_arcs(const Args &a, int64_t e0, int64_t e1, int lvl, int64_t tid, int64_t nthr) {
  for (int64_t e = e0 + tid; e < e1; e += nthr) atomicMin(a.armed + ldg(a.hcol + e), lvl + 1 + ldg(a.hk + e));
}

// ============================================================== backward ===

// What core vertex v receives from the vertices of its chains, for the 32
// slots of word w (the part that needs only forward results): cdep[v][w][.].
// Chain-arc data are loaded lane-parallel, 32 arcs at a time; then, four arcs
// at a time, the far ends' levels and path counts in one batch of loads (a
// tie needs the path counts on about half the slots, so a warp nearly always
// needs them: loading them with the levels takes one memory round trip per
// group instead of one more per tying arc), then their level exponents.
constexpr int kArcGroup = 4;
__device__ __forceinline__ int level_index(const Args &a, int d) { return min(max(d, 0), a.tcap + 1); }
__device__ __forceinline__ void chain_in(const Args &a, const Slot *slots, int nslots, int32_t v, int w, int64_t c0,
                                         int64_t c1, int lane) {
  const int W = a.W;
  const int b = w * 32 + lane;
  const bool live = b < nslots;
  const int64_t iv = ((int64_t)v * W + w) * 32 + lane;
  const int32_t *xb = a.X + (int64_t)b * (a.tcap + 2);
  End A{0, 0, 1.0, 0.0};
  Slot sl{0, -1, 0, 0};
  if (live) {
    A.d = __ldcg(a.d + iv);
    A.s = __ldcg(a.sig + iv);
    sl = slots[b];
    A.x = __ldcg(xb + level_index(a, A.d));
  }
  double sum = 0.0;
  for (int64_t base = c0; base < c1; base += 32) {
    const int64_t e = base + lane;
    int32_t u = 0, cid = 0, k = 0;
    int64_t poff = 0;
    if (e < c1) {
      u = ldg(a.hcol + e);
      cid = ldg(a.hcid + e);
      k = ldg(a.hk + e);
      poff = ldg(a.cpre_off + (cid >> 1));
    }
    const int cnt = (int)min((int64_t)32, c1 - base);
    for (int j0 = 0; j0 < cnt; j0 += kArcGroup) {
      int32_t uj[kArcGroup], cj[kArcGroup], kj[kArcGroup], dB[kArcGroup], xB[kArcGroup];
      int64_t pj[kArcGroup];
      double sB[kArcGroup];
#pragma unroll
      for (int r = 0; r < kArcGroup; ++r) {  // the far ends' levels and path counts, all in flight
        const int j = (j0 + r) & 31;
        uj[r] = __shfl_sync(0xffffffffu, u, j);
        cj[r] = __shfl_sync(0xffffffffu, cid, j);
        kj[r] = __shfl_sync(0xffffffffu, k, j);
        pj[r] = __shfl_sync(0xffffffffu, poff, j);
        const int64_t ib = ((int64_t)uj[r] * W + w) * 32 + lane;
        const bool ld = live && j0 + r < cnt;
        dB[r] = ld ? __ldcg(a.d + ib) : 0;
        sB[r] = ld ? __ldcg(a.sig + ib) : 1.0;
      }
#pragma unroll
      for (int r = 0; r < kArcGroup; ++r) xB[r] = (live && j0 + r < cnt) ? __ldcg(xb + level_index(a, dB[r])) : 0;
#pragma unroll
      for (int r = 0; r < kArcGroup; ++r) {
        if (!live || j0 + r >= cnt) continue;
        const bool same = sl.chain == (cj[r] >> 1);  // the source sits on this chain
        if (pj[r] < 0 && !same) {
          // nothing hangs off the chain: prefix sums are positions; the
          // vertices up to P = D/2 are fed from A, the one at D/2 ties when D is even
          const int D = dB[r] + kj[r] - A.d - 1;
          if (D < 0) continue;
          const int P = D >> 1;
          if ((D & 1) == 0 && P <= kj[r] - 1)
            sum += (double)P + 1.0 / (1.0 + scale2(sB[r] / A.s, xB[r] - A.x));
          else
            sum += (double)(min(kj[r] - 1, P) + 1);
          continue;
        }
        const bool right = cj[r] & 1;
        const double *Pj = pj[r] < 0 ? nullptr : a.cpre + pj[r];
        Stretch st{Pj, 0, kj[r], right};
        End B{dB[r], xB[r], sB[r], 0.0};
        if (same) {  // the stretch ends at the source
          B = source_end();
          st = right ? Stretch{Pj, sl.pos + 1, kj[r], true} : Stretch{Pj, 0, sl.pos, false};
        }
        sum += end_dep(st, A, B);
      }
    }
  }
  a.cdep[iv] = sum;
}

// delta, q and the BC partial of one (vertex, word) at level lev.
template <typename QT>
__device__ __forceinline__ void finish_dep(const Args &a, const Slot *slots, const int32_t *rch, int32_t v, int w,
                                           int lev, uint32_t act, int lane, double sum, bool chains) {
  constexpr bool kF32 = sizeof(QT) == 4;
  if (!act) return;
  const int W = a.W;
  double contrib = 0.0;
  if ((act >> lane) & 1u) {
    const int b = w * 32 + lane;
    const int64_t idx = ((int64_t)v * W + w) * 32 + lane;
    const double sv = a.sig[idx];
    const int xd = a.X[(int64_t)b * (a.tcap + 2) + lev] - a.X[(int64_t)b * (a.tcap + 2) + lev + 1];
    const double delta = scale2(sv * sum, xd) + (chains ? __ldcg(a.cdep + idx) : 0.0);
    const double qv = ((double)rch[v] + 1.0 + delta) / sv;
    if (kF32) {
      const double aq = fabs(qv);
      if (!(aq >= (double)FLT_MIN * 0x1p24 && aq <= (double)FLT_MAX * 0x1p-24)) atomicExch(&a.ctrl->range_err, 1);
    }
    reinterpret_cast<QT *>(a.q)[idx] = (QT)qv;
    contrib = delta * a.wsrc[b];
  }
  contrib = warp_sum(contrib);  // fixed-order reduction of this word's slots
  if (lane == 0) a.bcpart[(int64_t)v * W + w] += contrib;
}

// Vertex blocks of a phase: each warp's first block is its own index, later
// ones come from the phase's work counter (no atomics at all when the level
// has no more blocks than the grid has warps).
__device__ __forceinline__ int64_t next_block(int *counter, int lane) {
  int b = 0;
  if (lane == 0) b = atomicAdd(counter, 1);
  return nwarps() + __shfl_sync(0xffffffffu, b, 0);
}

// Vertex of lane l in light-row block vb (bs vertices per block, nblk
// blocks): strided over the core (BCGPU_BATCHED_CONTIG 0: every block mixes
// early, high-degree vertices of the BFS order with late ones) or
// consecutive (1: neighbouring rows share cached mask rows, and with blocks
// handed out in order a level ends on the cheap late vertices; 177.3
// against 172.0 GTEPS on RMAT-20).
#ifndef BCGPU_BATCHED_CONTIG
#define BCGPU_BATCHED_CONTIG 1
#endif
__device__ __forceinline__ int64_t block_vertex(int64_t vb, int l, int bs, int64_t nblk) {
#if BCGPU_BATCHED_CONTIG
  (void)nblk;
  return vb * bs + l;
#else
  (void)bs;
  return vb + (int64_t)l * nblk;
#endif
}

// Heavy-row chunk tasks of a phase: each CTA's first task is its own index;
// later ones in a fixed stride (BCGPU_BATCHED_HEAVY_DYN 0) or from the
// phase's work counter (1: a CTA that drew short chunks takes more; 153.0
// against 151.3-151.4 GTEPS on RMAT-20 at 512 sources per pass).
#ifndef BCGPU_BATCHED_HEAVY_DYN
#define BCGPU_BATCHED_HEAVY_DYN 1
#endif
// Chain in-flow tasks (core vertex, word): a fixed warp stride (0) or a
// work counter (1), as the light rows (168.7 against 161.9 GTEPS on
// RMAT-20: a hub's words carry thousands of chain arcs each). Chain-vertex
// tasks (one chain, every word) likewise (BCGPU_BATCHED_CHAINV_DYN: 167.9-
// 168.0 against 165.5).
#ifndef BCGPU_BATCHED_CHAININ_DYN
#define BCGPU_BATCHED_CHAININ_DYN 1
#endif
#ifndef BCGPU_BATCHED_CHAINV_DYN
#define BCGPU_BATCHED_CHAINV_DYN 1
#endif
__device__ __forceinline__ int64_t next_chunk_task(int64_t task, int *counter) {
#if BCGPU_BATCHED_HEAVY_DYN
  __shared__ int s_next;
  __syncthreads();  // every thread has read the previous s_next
  if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
  __syncthreads();
  return (int64_t)gridDim.x + s_next;
#else
  (void)counter;
  return task + gridDim.x;
#endif
}

}  // namespace

// --------------------------------------------------------------- kernel ----

template <typename QT>
__global__ void __launch_bounds__(kThreads, kMinCtas) batched_kernel(Args a) {
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
    const Seed *seeds = a.seeds + bt.seed_off;
    const int words = bt.words;
    const int groups = (words + 3) / 4;
    const int wpad = groups * 4;  // rows are processed in whole 4-word groups
    const int64_t vo = a.vtx_off[bt.bcc];
    const int32_t n = a.n_plain[bt.bcc];  // core vertices
    const int64_t *HR = a.hrow + a.hvo[bt.bcc];
    const int64_t *HS = a.hsplit + a.hvo[bt.bcc];
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
    // Warp tasks of the light rows: (vertex block, kHalf-word quarter of the
    // row), so a row's quarters run on different warps. Blocks hold bs <= 32
    // vertices (lane l < bs takes vertex blk + l*nblk): whole 32-vertex blocks
    // on large cores, smaller ones on small cores so that every warp of the
    // grid gets work on a level.
    const int halves = wpad / kHalf;
    const int64_t bs_want = ((int64_t)n * halves + nwarps() * kTasksPerWarp - 1) / (nwarps() * kTasksPerWarp);
    const int bs = bs_want >= 32 ? 32 : bs_want < 1 ? 1 : (int)bs_want;
    const int64_t nblk = ((int64_t)n + bs - 1) / bs;
    const int64_t ntask = nblk * halves;

    // ---- init: seen = slots beyond the batch, partials, level-0/1 masks, X, rexp, work counters
    for (int64_t i = gtid; i < (int64_t)n * W; i += gthreads) {
      const int w = (int)(i % W);
      const int live = min(32, max(0, bt.nslots - 32 * w));
      a.seen[i] = live == 32 ? 0u : ~((1u << live) - 1u);
      a.bcpart[i] = 0.0;
      a.lm[i] = 0;                         // level 0
      a.lm[(int64_t)a.n_cap * W + i] = 0;  // level 1
      if (w == 0) { a.lmin[i / W] = INT_MAX; a.lmax[i / W] = -1; a.gdone[i / W] = 0; a.armed[i / W] = INT_MAX; }
    }
    for (int64_t i = gtid; i < (int64_t)W * 32; i += gthreads) {
      a.rexp[i] = INT_MIN;
      a.X[i * (a.tcap + 2)] = 0;
      a.wsrc[i] = i < bt.nslots ? (double)rch[slots[i].src] + 1.0 : 0.0;
    }
    for (int64_t i = gtid; i < 4 * ((int64_t)a.tcap + 3) + 2; i += gthreads) a.wq[i] = 0;
    if (gtid == 0) {
      a.ctrl->more[0] = a.ctrl->more[1] = 0;
      a.ctrl->rescale[0] = a.ctrl->rescale[1] = 0;
      a.ctrl->range_err = 0;
      a.ctrl->found = 0;
    }
    grid_sync(a);
    for (int64_t b = gtid; b < bt.nslots; b += gthreads) {  // core sources at level 0
      const Slot s = slots[b];
      if (s.chain >= 0) continue;
      const int64_t idx = ((int64_t)s.src * W + (b >> 5)) * 32 + (b & 31);
      a.d[idx] = 0;
      a.sig[idx] = 1.0;
      atomicOr(a.lm + (int64_t)s.src * W + (b >> 5), 1u << (b & 31));
      atomicOr(a.seen + (int64_t)s.src * W + (b >> 5), 1u << (b & 31));
      atomicMin(a.lmin + s.src, 0);
      atomicMax(a.lmax + s.src, 0);
      atomicAdd(&a.ctrl->found, 1ull);
    }
    for (int64_t i = gwarp(); i < bt.narm; i += nwarps()) {  // neighbours of sources and seeded vertices
      const int2 m = a.arms[bt.arm_off + i];
      arm_arcs(a, HR[m.x], HR[m.x + 1], m.y, lane, 32);
    }
    grid_sync(a);
    PHASE_MARK(0);

    // ---- forward: levels t -> t+1
    int t = 0, tlast = 0;
    const unsigned long long all_found = (unsigned long long)n * (unsigned long long)bt.nslots;
    while (true) {
      unsigned long long nf = 0;  // pairs this warp found on this level
      if (t + 1 > a.tcap) { set_err(a.err, kDevWorkspace); break; }
      const uint32_t *lmt = a.lm + (int64_t)t * a.n_cap * W;
      // the next level's flags and masks start clear (nothing reads them on this level)
      if (gtid == 0) {
        a.ctrl->more[(t + 1) & 1] = 0;
        a.ctrl->rescale[(t + 1) & 1] = 0;
      }
      for (int64_t i = gtid; i < (int64_t)n * W; i += gthreads) a.lm[(int64_t)(t + 2) * a.n_cap * W + i] = 0;
      // heavy rows: chunks of their arcs, one CTA per (chunk, half); partials
      // are combined across the CTA's warps, then across chunks after the barrier
      for (int64_t task = blockIdx.x; task < nchunks * halves;
           task = next_chunk_task(task, a.wq + 2 * (a.tcap + 3) + t)) {
        const int64_t c = task / halves;
        const int w0 = (int)(task % halves) * kHalf;
        const int nw = min(kHalf, wpad - w0);
        const int32_t v = hv[hcv[c]];
        uint32_t unseen[kHalf], any[kHalf];
        load_row(a.seen + (int64_t)v * W + w0, nw, unseen);
        uint32_t u_any = 0;
#pragma unroll
        for (int k = 0; k < kHalf; ++k) { unseen[k] = k < nw ? ~unseen[k] : 0u; any[k] = 0; u_any |= unseen[k]; }
        Acc<false> acc[kHalf];
        if (u_any && __ldcg(a.armed + v) <= t + 1) {  // uniform over the CTA
          const int64_t e0 = hce0[c], e1 = hce1[c], sp = HS[v];
          const int64_t per = (e1 - e0 + kWarpsPerCta - 1) / kWarpsPerCta;
          const int64_t s0 = e0 + wib * per, s1 = min(e1, s0 + per);
          if (s0 < min(s1, sp)) row_pass<double, false, 0>(a, lmt, a.sig, s0, min(s1, sp), w0, nw, unseen, any, acc, lane, t);
          if (max(s0, sp) < s1) row_pass<double, false, 1>(a, a.lm, a.sig, max(s0, sp), s1, w0, nw, unseen, any, acc, lane, t);
        }
#pragma unroll
        for (int k = 0; k < kHalf; ++k) {
          any[k] = warp_or(any[k]);
          S.acc[k][lane] = acc[k].value();
          if (lane == 0) S.any[k] = any[k];  // this warp's hit masks, for the combine
        }
        __syncthreads();
        for (int k = wib; k < nw; k += kWarpsPerCta) {  // fixed warp order
          double tot = 0.0;
          uint32_t mm = 0;
          for (int x = 0; x < kWarpsPerCta; ++x) { tot += scratch[x].acc[k][lane]; mm |= scratch[x].any[k]; }
          a.hacc[((hc0 + c) * W + w0 + k) * 32 + lane] = tot;
          if (lane == 0) a.hmask[(hc0 + c) * W + w0 + k] = mm;
        }
        __syncthreads();
      }
      // light rows: (vertex block, quarter) tasks, lane-parallel activity check
      for (int64_t tk = gwarp(); tk < ntask; tk = next_block(a.wq + t, lane)) {
        const int64_t vb = tk / halves;
        const int w0 = (int)(tk % halves) * kHalf;
        const int nw = kHalf;
        const int64_t vl = block_vertex(vb, lane, bs, nblk);
        int64_t e0l = 0, e1l = 0, spl = 0;
        bool on = false;
        if (lane < bs && vl < n) {
          e0l = HR[vl];
          e1l = HR[vl + 1];
          spl = HS[vl];
          on = e1l - e0l <= bt.heavy_deg && __ldcg(a.gdone + vl) < groups && __ldcg(a.armed + vl) <= t + 1;
        }
        uint32_t todo = __ballot_sync(0xffffffffu, on);
        while (todo) {
          const int j = __ffs(todo) - 1;
          todo &= todo - 1;
          const int32_t v = (int32_t)block_vertex(vb, j, bs, nblk);
          const int64_t e0 = __shfl_sync(0xffffffffu, e0l, j), e1 = __shfl_sync(0xffffffffu, e1l, j);
          const int64_t sp = __shfl_sync(0xffffffffu, spl, j);
          {
            uint32_t seen[kHalf], unseen[kHalf], any[kHalf];
            load_row(a.seen + (int64_t)v * W + w0, nw, seen);
            uint32_t u_any = 0;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) { unseen[k] = k < nw ? ~seen[k] : 0u; any[k] = 0; u_any |= unseen[k]; }
            if (!u_any) continue;
            Acc<false> acc[kHalf];
            if (e0 < sp) row_pass<double, false, 0>(a, lmt, a.sig, e0, sp, w0, nw, unseen, any, acc, lane, t);
            if (sp < e1) row_pass<double, false, 1>(a, a.lm, a.sig, sp, e1, w0, nw, unseen, any, acc, lane, t);
            int first = 0;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) {
              if (k >= nw) continue;
              const uint32_t m = warp_or(any[k]);
              const int r = finish_pull(a, v, w0 + k, t, m, lane, acc[k].value());
              nf += r & 255;
              first |= r >> 8;
              any[k] = m;
            }
            if (first) arm_arcs(a, e0, e1, t + 1, lane, 32);
#pragma unroll
            for (int g = 0; g < kHalf / 4; ++g) {  // groups now seen by all their slots
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
      if (lane == 0 && nf) atomicAdd(&a.ctrl->found, nf);
      nf = 0;
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
          nf += finish_pull(a, v, w, t, m, lane, acc) & 255;  // heavy rows arm in the next phase
        }
        if (lane == 0 && nf) atomicAdd(&a.ctrl->found, nf);
        grid_sync(a);
        PHASE_MARK(2);
      }
      if (bt.nseeds) {  // chain sources entering the core at level t+1 (one path each)
        for (int64_t i = gtid; i < bt.nseeds; i += gthreads) {
          const Seed s = seeds[i];
          if (s.level != t + 1) continue;
          const int b = s.slot, w = b >> 5;
          const uint32_t bit = 1u << (b & 31);
          const int64_t idx = ((int64_t)s.v * W + w) * 32 + (b & 31);
          const double one = scale2(1.0, -a.X[(int64_t)b * (a.tcap + 2) + t]);
          const uint32_t old = atomicOr(a.seen + (int64_t)s.v * W + w, bit);
          if (!(old & bit)) {
            a.d[idx] = t + 1;
            a.sig[idx] = one;
            atomicOr(a.lm + ((int64_t)(t + 1) * a.n_cap + s.v) * W + w, bit);
            atomicMin(a.lmin + s.v, t + 1);
            atomicMax(a.lmax + s.v, t + 1);
            a.ctrl->more[t & 1] = 1;
            atomicAdd(&a.ctrl->found, 1ull);
          } else if (a.d[idx] == t + 1) {
            a.sig[idx] += one;  // reached on this level from the core as well
          }
        }
        grid_sync(a);
      }
      const int more = *(volatile int *)&a.ctrl->more[t & 1];
      const int resc = *(volatile int *)&a.ctrl->rescale[t & 1];
      const unsigned long long found = *(volatile unsigned long long *)&a.ctrl->found;
      // heavy rows first reached on level t+1 arm their neighbours, one CTA per chunk
      for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x)
        if (__ldcg(a.lmin + hv[hcv[c]]) == t + 1) arm_arcs(a, hce0[c], hce1[c], t + 1, threadIdx.x, blockDim.x);
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
            a.sig[idx] = scale2(a.sig[idx], -re);
          }
        }
      }
      grid_sync(a);  // level t+1's base and counts are final; everyone has read the flags
      if (resc) {
        for (int64_t b = gtid; b < (int64_t)W * 32; b += gthreads) a.rexp[b] = INT_MIN;
        grid_sync(a);
      }
      if (more) tlast = t + 1;
      if (cta_failed(a)) break;
      // done when every slot has reached every core vertex (later seeds then
      // reach seen vertices only); else level t+2 needs a non-empty level
      // within the longest arc, or a seed
      if (found >= all_found) break;
      if (t + 1 - tlast > bt.kmax && t + 2 > bt.max_seed) break;
      ++t;
      PHASE_MARK(3);
    }
    PHASE_MARK(3);
    if (cta_failed(a)) return;
    // every slot must have reached every core vertex of the BCC
    for (int64_t i = gtid; i < (int64_t)n * words; i += gthreads) {
      const int32_t v = (int32_t)(i / words);
      const int w = (int)(i % words);
      if (~__ldcg(a.seen + (int64_t)v * W + w) != 0u) set_err(a.err, kDevDisconnected);
    }
    // what the core vertices receive from their chains' vertices
    if (bt.kmax) {
#if BCGPU_BATCHED_CHAININ_DYN
      for (int64_t task = gwarp(); task < (int64_t)n * words; task = next_block(a.wq + 4 * (a.tcap + 3), lane)) {
#else
      for (int64_t task = gwarp(); task < (int64_t)n * words; task += nwarps()) {
#endif
        const int32_t v = (int32_t)(task / words);
        const int w = (int)(task % words);
        const int64_t c0 = HS[v], c1 = HR[v + 1];
        if (c0 < c1) chain_in(a, slots, bt.nslots, v, w, c0, c1, lane);
      }
      grid_sync(a);
    }
    PHASE_MARK(4);

    // ---- backward: lev = tlast .. 1 (level tlast+1 is empty and not cleared:
    // the deepest level has no unit-arc successors)
    for (int lev = tlast; lev >= 1; --lev) {
      const uint32_t *lm_here = a.lm + (int64_t)lev * a.n_cap * W;
      const uint32_t *lm_next = a.lm + (int64_t)(lev + 1) * a.n_cap * W;
      const QT *q = reinterpret_cast<const QT *>(a.q);
      // heavy rows: chunked successor sums, combined below
      for (int64_t task = blockIdx.x; task < nchunks * halves;
           task = next_chunk_task(task, a.wq + 3 * (a.tcap + 3) + lev)) {
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
          act[k] = (in_span && k < nw) ? act[k] : 0u;
          any[k] = 0;
          a_any |= act[k];
        }
        Acc<kComp> acc[kHalf];
        if (a_any) {  // uniform over the CTA
          const int64_t e0 = hce0[c], e1 = hce1[c], sp = HS[v];
          const int64_t per = (e1 - e0 + kWarpsPerCta - 1) / kWarpsPerCta;
          const int64_t s0 = e0 + wib * per, s1 = min(e1, s0 + per);
          if (lev < tlast && s0 < min(s1, sp))
            row_pass<QT, kComp, 0>(a, lm_next, q, s0, min(s1, sp), w0, nw, act, any, acc, lane, lev + 1);
          if (max(s0, sp) < s1) row_pass<QT, kComp, 2>(a, a.lm, q, max(s0, sp), s1, w0, nw, act, any, acc, lane, lev + 1, tlast);
        }
#pragma unroll
        for (int k = 0; k < kHalf; ++k) S.acc[k][lane] = acc[k].value();
        __syncthreads();
        for (int k = wib; k < nw; k += kWarpsPerCta) {  // fixed warp order
          double tot = 0.0;
          for (int x = 0; x < kWarpsPerCta; ++x) tot += scratch[x].acc[k][lane];
          a.hacc[((hc0 + c) * W + w0 + k) * 32 + lane] = tot;
        }
        __syncthreads();
      }
      const int wqi = a.tcap + 3 + lev;
      for (int64_t tk = gwarp(); tk < ntask; tk = next_block(a.wq + wqi, lane)) {
        const int64_t vb = tk / halves;
        const int w0 = (int)(tk % halves) * kHalf;
        const int nw = kHalf;
        const int64_t vl = block_vertex(vb, lane, bs, nblk);
        int64_t e0l = 0, e1l = 0, spl = 0;
        bool on = false;
        if (lane < bs && vl < n && lev >= __ldcg(a.lmin + vl) && lev <= __ldcg(a.lmax + vl)) {
          e0l = HR[vl];
          e1l = HR[vl + 1];
          spl = HS[vl];
          on = e1l - e0l <= bt.heavy_deg;
        }
        uint32_t todo = __ballot_sync(0xffffffffu, on);
        while (todo) {
          const int j = __ffs(todo) - 1;
          todo &= todo - 1;
          const int32_t v = (int32_t)block_vertex(vb, j, bs, nblk);
          const int64_t e0 = __shfl_sync(0xffffffffu, e0l, j), e1 = __shfl_sync(0xffffffffu, e1l, j);
          const int64_t sp = __shfl_sync(0xffffffffu, spl, j);
          {
            uint32_t act[kHalf], any[kHalf];
            load_row(lm_here + (int64_t)v * W + w0, nw, act);
            uint32_t a_any = 0;
#pragma unroll
            for (int k = 0; k < kHalf; ++k) {
              act[k] = k < nw ? act[k] : 0u;
              any[k] = 0;
              a_any |= act[k];
            }
            if (!a_any) continue;
            Acc<kComp> acc[kHalf];
            if (lev < tlast && e0 < sp) row_pass<QT, kComp, 0>(a, lm_next, q, e0, sp, w0, nw, act, any, acc, lane, lev + 1);
            if (sp < e1) row_pass<QT, kComp, 2>(a, a.lm, q, sp, e1, w0, nw, act, any, acc, lane, lev + 1, tlast);
#pragma unroll
            for (int k = 0; k < kHalf; ++k)
              if (k < nw) finish_dep<QT>(a, slots, rch, v, w0 + k, lev, act[k], lane, acc[k].value(), sp < e1);
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
          const uint32_t act = __ldcg(lm_here + (int64_t)v * W + w);
          if (!act) continue;
          double sum = 0.0;
          for (int32_t c = hfst[h]; c < hfst[h + 1]; ++c) sum += __ldcg(a.hacc + ((hc0 + c) * W + w) * 32 + lane);
          finish_dep<QT>(a, slots, rch, v, w, lev, act, lane, sum, HS[v] < HR[v + 1]);
        }
      }
      grid_sync(a);
      PHASE_MARK(6);
      PHASE_COUNT(17);
    }

    // ---- chain vertices: one warp per chain, every word; each lane sums its
    // slots' contributions over the words (registers for chains of up to
    // kRegVerts vertices), then one warp reduction per chain vertex goes
    // straight into BC (one writer per vertex: fixed order)
    {
      constexpr int kRegVerts = 8;
      const int bad = *(volatile int *)&a.ctrl->range_err;
      const int64_t ch0 = a.chain_off[bt.bcc];
      const int64_t nch = a.chain_off[bt.bcc + 1] - ch0;
#if BCGPU_BATCHED_CHAINV_DYN
      for (int64_t task = gwarp(); task < nch; task = next_block(a.wq + 4 * (a.tcap + 3) + 1, lane)) {
#else
      for (int64_t task = gwarp(); task < nch; task += nwarps()) {
#endif
        const int64_t c = ch0 + task;
        const int32_t L = a.chain_l[c], R = a.chain_r[c], cs = a.chain_start[c], k = a.chain_len[c];
        const int64_t poff = a.cpre_off[c];
        const double *P = poff < 0 ? nullptr : a.cpre + poff;
        double part[kRegVerts];
#pragma unroll
        for (int j = 0; j < kRegVerts; ++j) part[j] = 0.0;
        for (int w = 0; w < words; ++w) {
          const int b = w * 32 + lane;
          const bool live = b < bt.nslots;
          const int64_t iL = ((int64_t)L * W + w) * 32 + lane, iR = ((int64_t)R * W + w) * 32 + lane;
          End eL{0, 0, 1.0, 0.0}, eR{0, 0, 1.0, 0.0};
          int on = -1;
          if (live) {  // the ends' levels, then only the path counts / q the closed forms use
            eL.d = __ldcg(a.d + iL);
            eR.d = __ldcg(a.d + iR);
            const Slot sl = slots[b];
            on = sl.chain == c ? sl.pos : -1;
            // stretches: [L, R] or, with the source on the chain, [L, source] and [source, R]
            const int mL = on < 0 ? k : on, dBL = on < 0 ? eR.d : 0;           // seen from L
            const int mR = on < 0 ? k : k - 1 - on, dBR = on < 0 ? eL.d : 0;  // seen from R
            const int DL = dBL + mL - eL.d - 1, DR = dBR + mR - eR.d - 1;
            const bool tieL = mL > 0 && DL >= 0 && (DL & 1) == 0 && DL / 2 <= mL - 1;
            const bool tieR = mR > 0 && DR >= 0 && (DR & 1) == 0 && DR / 2 <= mR - 1;
            // B's paths through the stretch: R fed via the chain from L, or L from R
            const bool viaL = on < 0 && eR.d == eL.d + k + 1, viaR = on < 0 && eL.d == eR.d + k + 1;
            const bool srcL = on >= 0 && eL.d == on + 1, srcR = on >= 0 && eR.d == k - on;  // fed from the source
            const int32_t *xb = a.X + (int64_t)b * (a.tcap + 2);
            const QT *qq = reinterpret_cast<const QT *>(a.q);
            const bool sig = tieL || tieR || viaL || viaR;
            if (sig) {
              eL.s = __ldcg(a.sig + iL);
              eL.x = __ldcg(xb + level_index(a, eL.d));
              eR.s = __ldcg(a.sig + iR);
              eR.x = __ldcg(xb + level_index(a, eR.d));
            }
            if (viaR || srcL) {
              eL.qs = (double)__ldcg(qq + iL);
              if (!sig) eL.x = __ldcg(xb + level_index(a, eL.d));
            }
            if (viaL || srcR) {
              eR.qs = (double)__ldcg(qq + iR);
              if (!sig) eR.x = __ldcg(xb + level_index(a, eR.d));
            }
          }
          const double wsrc = live ? a.wsrc[b] : 0.0;
          // Source off the chain (the common case), in prefix sums from L:
          // vertex j is fed from L iff 2j <= D; a tie vertex t = D/2 shares
          // its reach+1 between the sides in proportion to sigma_L, sigma_R;
          // else the L-fed vertices end at pl, and the far end's q enters
          // when the chain carries its shortest paths.
          int tv = -1, pl = -1;
          double fL = 0.0, fR = 0.0;  // L-side and R-side constants
          if (live && on < 0) {
            const int D = eR.d + k - eL.d - 1;
            if (D >= 0 && (D & 1) == 0 && D / 2 <= k - 1) {
              tv = D / 2;
              const double p0 = chain_pre(P, tv), p1 = chain_pre(P, tv + 1), wt = p1 - p0;
              fL = p0 + wt / (1.0 + scale2(eR.s / eL.s, eR.x - eL.x));
              fR = -p1 + wt / (1.0 + scale2(eL.s / eR.s, eL.x - eR.x));
            } else {
              pl = D >= 0 ? min(k - 1, D / 2) : -1;
              const double p1 = chain_pre(P, pl + 1);
              fL = p1 + (eR.d == eL.d + k + 1 ? scale2(eL.s * eR.qs, eL.x - eR.x) : 0.0);
              fR = -p1 + (eL.d == eR.d + k + 1 ? scale2(eR.s * eL.qs, eR.x - eL.x) : 0.0);
            }
          }
          auto dep_of = [&](int j) -> double {
            if (!live) return 0.0;
            if (on < 0) {
              if (j == tv) return 0.0;
              const bool from_l = tv >= 0 ? j < tv : j <= pl;
              return (from_l ? fL - chain_pre(P, j + 1) : chain_pre(P, j) + fR) * wsrc;
            }
            if (j < on) return stretch_dep(Stretch{P, 0, on, false}, j, eL, source_end()) * wsrc;
            if (j > on) return stretch_dep(Stretch{P, on + 1, k, false}, j - on - 1, source_end(), eR) * wsrc;
            return 0.0;
          };
          if (k <= kRegVerts) {
#pragma unroll
            for (int j = 0; j < kRegVerts; ++j)
              if (j < k) part[j] += dep_of(j);
          } else {
            for (int j = 0; j < k; ++j) {
              const double tot = warp_sum(dep_of(j));
              if (lane == 0 && !bad) a.bc[vo + cs + j] += tot;
            }
          }
        }
        if (k <= kRegVerts) {
#pragma unroll
          for (int j = 0; j < kRegVerts; ++j) {
            if (j >= k) continue;
            const double tot = warp_sum(part[j]);
            if (lane == 0 && !bad) a.bc[vo + cs + j] += tot;
          }
        }
      }
    }
    grid_sync(a);
    PHASE_MARK(8);

    // ---- fold the batch into BC (fixed word order), unless FP32 range failed
    const int bad = *(volatile int *)&a.ctrl->range_err;
    if (bad) {
      if (gtid == 0) a.redo[bi] = 1;
    } else {
      for (int64_t v = gtid; v < n; v += gthreads) {  // core vertices (chain vertices were added above)
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

// An allocator whose value-initialising construct leaves trivially
// constructible elements uninitialised: table vectors that are resized and
// then fully overwritten by parallel loops skip a sequential zero fill (and
// their pages are first touched by the parallel writers).
template <class T>
struct NoInit : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInit<U>;
  };
  NoInit() = default;
  template <class U>
  NoInit(const NoInit<U> &) {}
  template <class U>
  void construct(U *p) noexcept {
    ::new ((void *)p) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new ((void *)p) U(std::forward<A>(a)...);
  }
};
template <class T>
using HostBuf = std::vector<T, NoInit<T>>;

struct BatchedPlan {
  int width = 0;       // B
  int W = 0;           // words
  int tcap = 0;
  int64_t n_cap = 0;
  bool f32 = true;
  int grid = 0;
  size_t smem = 0;
  int64_t bytes = 0;
  int64_t h2d = 0;  // bytes uploaded by batched_create
  int64_t d2h = 0;  // bytes batched_create read back (the row checks' flag)
  cudaMemPool_t pool = nullptr;  // allocs come from this pool on `stream` (null: cudaMalloc)
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  Args args{};
  std::vector<int64_t> u_src, u_teps, u_bfs, u_aux, u_visits;
  std::vector<Batch> h_batches;
  HostBuf<Slot> h_slots;
  HostBuf<Seed> h_seeds;
  std::vector<int2> h_arms;
  std::vector<int64_t> h_vtx_off;
  int64_t n_batches = 0;
};

namespace {

// Eccentricity of local vertex 0 in the BCC: every level of every source is
// at most 2 * ecc.
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

int batched_width(int requested) {
  const int width = requested > 0 ? requested : 512;
  return std::max(32, std::min(1024, (width + 31) / 32 * 32));
}

// Source order of BCC b: bounded BFS balls of nearby vertices (chain vertices
// included), so a pass's sources see every vertex within a narrow band of
// levels: few active levels per vertex, dense 32-slot hits. A ball grows only
// through vertices not yet taken, so each vertex's arcs are scanned once and
// late balls cost no rescans of finished regions. The greedy stops at the
// first ball boundary at or after `need` vertices: the order of a larger
// `need` extends it (a lazy plan that fills only some passes needs a prefix).
void batched_source_order(const bc_bccs *B, int32_t b, int width, int64_t need, std::vector<int32_t> &order) {
  const int64_t vo = B->vtx_off[b];
  const int32_t nb = (int32_t)(B->vtx_off[b + 1] - vo);
  order.clear();
  need = std::min<int64_t>(need, nb);
  if (need <= 0) return;
  order.reserve((size_t)need + (size_t)width);
  // taken: one bit per vertex (small enough to stay in the host's caches).
  // A ball's queue may list a vertex more than once (every taken vertex
  // queues its untaken neighbours); it is taken at its first listing and
  // skipped at the later ones, so the order is that of a queue holding each
  // vertex once. A vertex queued by an earlier ball but not taken may join
  // a later one.
  std::vector<uint64_t> taken(((size_t)nb + 63) / 64, 0);
  auto is_taken = [&](int32_t y) { return (taken[(size_t)y >> 6] >> (y & 63)) & 1u; };
  std::vector<int32_t> q;
  const int64_t arc_budget = 16 * (int64_t)width;  // bounds the host work per ball
  for (int32_t seed = 0; seed < nb && (int64_t)order.size() < need; ++seed) {
    if (is_taken(seed)) continue;
    q.clear();
    q.push_back(seed);
    int64_t got = 0, scanned = 0;
    for (size_t h = 0; h < q.size() && got < width; ++h) {
      // software pipeline over the queue: row offsets 16 entries ahead, the
      // row's arcs 8 ahead (rows are short: ~9 arcs on RMAT)
      if (h + 16 < q.size()) __builtin_prefetch(&B->row[vo + q[h + 16]]);
      if (h + 8 < q.size()) __builtin_prefetch(&B->col[B->row[vo + q[h + 8]]]);
      const int32_t x = q[h];
      if (is_taken(x)) continue;
      taken[(size_t)x >> 6] |= 1ull << (x & 63);
      order.push_back(x);
      ++got;
      if (scanned >= arc_budget) continue;  // keep draining the queue, stop growing it
      const int64_t e0 = B->row[vo + x], e1 = std::min(B->row[vo + x + 1], e0 + arc_budget - scanned);
      scanned += e1 - e0;
      for (int64_t e = e0; e < e1; ++e) {
        const int32_t y = B->col[e];
        if (!is_taken(y)) q.push_back(y);
      }
    }
  }
}

namespace {

// The contracted rows of the core vertices of the BCCs in multi-source
// passes, built on the device from the packed CSR already there (the host
// computes only the row offsets hrow and, per packed chain vertex, its chain
// and position): one thread per row writes the row's unit arcs, then its chain
// arcs, each in the order of the vertex's CSR row -- so the rows are those a
// sequential fill gives. Entries of rbcc < 0 are a BCC's end offsets. A
// non-core neighbour outside every chain sets bit 1 of *bad, a core vertex
// next to the inside of a chain bit 2.
__global__ void contract_rows_kernel(const int64_t *row, const int32_t *col, const int64_t *vtx_off,
                                     const int32_t *n_plain, const int32_t *rbcc, const int64_t *hvo,
                                     const int64_t *hrow, int64_t nrows, const int32_t *gcof, const int32_t *gcpos,
                                     const int32_t *chain_len, const int32_t *chain_l, const int32_t *chain_r,
                                     int64_t *hsplit, int32_t *hcol, int32_t *hk, int32_t *hcid, int *bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = rbcc[i];
    if (b < 0) {
      hsplit[i] = hrow[i];
      continue;
    }
    const int64_t vo = vtx_off[b];
    const int32_t npl = n_plain[b], x = (int32_t)(i - hvo[b]);
    const int64_t e0 = row[vo + x], e1 = row[vo + x + 1];
    int64_t o = hrow[i];
    for (int64_t e = e0; e < e1; ++e) {
      const int32_t y = col[e];
      if (y < npl) {
        hcol[o] = y;
        hk[o] = 0;
        hcid[o] = -1;
        ++o;
      }
    }
    hsplit[i] = o;
    for (int64_t e = e0; e < e1; ++e) {
      const int32_t y = col[e];
      if (y < npl) continue;
      const int32_t c = gcof[vo + y];
      if (c < 0) {
        atomicOr(bad, 1);
        continue;
      }
      const int32_t k = chain_len[c], pos = gcpos[vo + y];
      int right;
      if (x == chain_l[c] && pos == 0) right = 0;
      else if (x == chain_r[c] && pos == k - 1) right = 1;
      else {
        atomicOr(bad, 2);
        continue;
      }
      hcol[o] = right ? chain_l[c] : chain_r[c];
      hk[o] = k;
      hcid[o] = c * 2 + right;
      ++o;
    }
  }
}

// Fills P (allocated by batched_create, which releases it on any failure).
int batched_build(const bc_bccs *B, const BatchedConfig &cfg, const int64_t *row, const int32_t *col,
                  const int32_t *reach, const int64_t *vtx_off, const int32_t *chain_start, const int32_t *chain_len,
                  const int32_t *chain_l, const int32_t *chain_r, double *bc, int *err, cudaStream_t stream,
                  BatchedPlan *P, std::string *msg) {
  auto bail = [&](int code, const std::string &m) {
    if (msg) *msg = m;
    return code;
  };
  P->f32 = cfg.delta_fp32c;
  const int width = batched_width(cfg.width);
  P->width = width;
  P->W = (width / 32 + 3) / 4 * 4;  // row stride: whole 4-word groups (16-byte mask loads)
  const int W = P->W;

  // ---- contracted rows, chain prefix sums, heavy chunks, passes
  std::vector<int64_t> hvo, hrow, cpre_off;
  std::vector<int32_t> rbcc;          // per hrow entry: its BCC, -1 for a BCC's end offset
  HostBuf<int32_t> gcof, gcpos;       // per packed vertex of a BCC in passes: chain (global, -1: core), position
  int64_t narcs = 0;                  // contracted arcs so far
  std::vector<double> cpre;
  HostBuf<Slot> slots;  // every entry written by the pass fill
  HostBuf<Seed> seeds;
  std::vector<int2> arms;
  std::vector<int64_t> heavy_off{0}, hchunk_off{0}, hchunk_e0, hchunk_e1;
  std::vector<int32_t> heavy, hchunk_v, hfirst;
  std::vector<int32_t> dist, queue;
  std::vector<int32_t> cof, cpos;  // chain vertex -> chain (global), position
  int64_t ncap = 1;
  int tcap = 2;
  cpre_off.resize((size_t)B->n_chains);
  gcof.resize((size_t)std::max<int64_t>(B->n_packed, 1));
  gcpos.resize(gcof.size());
  for (int32_t b = 0; b < B->n_bcc; ++b) {
    const int64_t vo = B->vtx_off[b];
    const int32_t nb = (int32_t)(B->vtx_off[b + 1] - vo);
    const int32_t npl = B->n_plain[b];
    const int64_t ce0 = B->chain_off[b], ce1 = B->chain_off[b + 1];
    if (cfg.bccs_on && !(*cfg.bccs_on)[b]) {  // scheduled elsewhere: empty per-BCC table entries
      hvo.push_back((int64_t)hrow.size());
      hfirst.push_back((int32_t)((int64_t)hchunk_v.size() - hchunk_off.back()));
      heavy_off.push_back((int64_t)heavy.size());
      hchunk_off.push_back((int64_t)hchunk_v.size());
      continue;
    }
    ncap = std::max<int64_t>(ncap, npl);
    const int64_t arcs = B->row[vo + nb] - B->row[vo];
    // chain membership, and the shape the closed forms rely on: each chain
    // vertex has exactly its two chain neighbours, the ends are distinct core
    // vertices. Checked in parallel; the error reported is the one a pass in
    // chain order meets first (per chain: equal ends, then a vertex an
    // earlier chain holds, then the neighbours).
    const int64_t nchb = ce1 - ce0;
    std::vector<int32_t> first((size_t)nb, INT32_MAX);  // smallest chain (BCC-relative) holding each vertex
    std::vector<int32_t> csize((size_t)nchb + 1, 0);     // prefix-sum entries of each chain (0: nothing hangs off it)
    std::vector<uint8_t> cerr((size_t)nchb, 0);          // 1 equal ends, 3 bad neighbours (2 = overlap, below)
    int kmax = 0;
#pragma omp parallel for schedule(static) reduction(max : kmax)
    for (int64_t i = 0; i < nchb; ++i) {
      const int64_t c = ce0 + i;
      const int32_t st = B->chain_start[c], k = B->chain_len[c], L = B->chain_l[c], R = B->chain_r[c];
      kmax = std::max(kmax, k);
      if (L == R) { cerr[(size_t)i] = 1; continue; }
      bool flat = true;
      for (int32_t j = 0; j < k; ++j) {
        int32_t *f = &first[(size_t)(st + j)];
        int32_t cur = __atomic_load_n(f, __ATOMIC_RELAXED);
        while ((int32_t)i < cur && !__atomic_compare_exchange_n(f, &cur, (int32_t)i, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
        }
        const int32_t x = st + j, prev = j == 0 ? L : x - 1, next = j == k - 1 ? R : x + 1;
        const int64_t e0 = B->row[vo + x], e1 = B->row[vo + x + 1];
        if (e1 - e0 != 2 || !((B->col[e0] == prev && B->col[e0 + 1] == next) || (B->col[e0] == next && B->col[e0 + 1] == prev)))
          cerr[(size_t)i] = 3;
        flat = flat && B->reach[vo + x] == 0;
      }
      csize[(size_t)i + 1] = flat ? 0 : k + 1;
    }
    int64_t bad_chain = nchb;  // the first chain with an error
#pragma omp parallel for schedule(static) reduction(min : bad_chain)
    for (int64_t i = 0; i < nchb; ++i) {
      if (cerr[(size_t)i] != 1) {
        const int32_t st = B->chain_start[ce0 + i], k = B->chain_len[ce0 + i];
        for (int32_t j = 0; j < k; ++j)
          if (first[(size_t)(st + j)] < (int32_t)i) cerr[(size_t)i] = 2;  // an earlier chain holds the vertex
      }
      if (cerr[(size_t)i]) bad_chain = std::min(bad_chain, i);
    }
    if (bad_chain < nchb) {
      const int e = cerr[(size_t)bad_chain];
      return bail(BCGPU_EINVAL, e == 1 ? "a chain whose two ends are the same vertex"
                                 : e == 2 ? "chains overlap"
                                          : "a chain vertex whose neighbours are not its chain neighbours");
    }
    for (int64_t i = 0; i < nchb; ++i) csize[(size_t)i + 1] += csize[(size_t)i];
    const int64_t cpre0 = (int64_t)cpre.size();
    cpre.resize((size_t)(cpre0 + csize[(size_t)nchb]));
    cof.assign((size_t)nb, -1);
    cpos.assign((size_t)nb, -1);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nchb; ++i) {
      const int64_t c = ce0 + i;
      const int32_t st = B->chain_start[c], k = B->chain_len[c];
      for (int32_t j = 0; j < k; ++j) {
        cof[(size_t)(st + j)] = (int32_t)c;
        cpos[(size_t)(st + j)] = j;
      }
      const bool flat = csize[(size_t)i + 1] == csize[(size_t)i];
      cpre_off[c] = flat ? -1 : cpre0 + csize[(size_t)i];
      if (!flat) {
        double *P = cpre.data() + cpre0 + csize[(size_t)i], acc = 0.0;
        P[0] = 0.0;
        for (int32_t j = 0; j < k; ++j) {
          acc += (double)B->reach[vo + st + j] + 1.0;
          P[j + 1] = acc;
        }
      }
    }
    HOST_MARK("b: chains");
    // contracted rows: unit arcs first, then chain arcs
    hvo.push_back((int64_t)hrow.size());
    const int heavy_deg = npl < kSmallCore ? kHeavyDegSmall : kHeavyDeg;
    // Every arc of a core vertex becomes one contracted arc (a unit arc, or
    // the chain arc of the chain vertex it leads to), so the contracted rows
    // have the original degrees: offsets first, then the rows in parallel.
    std::copy(cof.begin(), cof.end(), gcof.begin() + vo);  // the device fill reads them per packed vertex
    std::copy(cpos.begin(), cpos.end(), gcpos.begin() + vo);
    const size_t rb = hrow.size();
    hrow.resize(rb + (size_t)npl + 1);
    hrow[rb] = narcs;
    for (int32_t x = 0; x < npl; ++x) hrow[rb + x + 1] = hrow[rb + x] + (B->row[vo + x + 1] - B->row[vo + x]);
    narcs = hrow[rb + npl];
    rbcc.resize(rb + (size_t)npl, b);
    hrow.pop_back();  // the BCC's end offset is pushed below, after its heavy rows
    int32_t hidx = 0;
    for (int32_t x = 0; x < npl; ++x) {
      const int64_t r0 = hrow[rb + x], r1 = x + 1 < npl ? hrow[rb + x + 1] : narcs;
      if (r1 - r0 <= heavy_deg) continue;
      heavy.push_back(x);
      hfirst.push_back((int32_t)((int64_t)hchunk_v.size() - hchunk_off.back()));
      for (int64_t e = r0; e < r1; e += kChunkArcs) {
        hchunk_v.push_back(hidx);
        hchunk_e0.push_back(e);
        hchunk_e1.push_back(std::min<int64_t>(r1, e + kChunkArcs));
      }
      ++hidx;
    }
    hrow.push_back(narcs);
    rbcc.push_back(-1);
    hfirst.push_back((int32_t)((int64_t)hchunk_v.size() - hchunk_off.back()));
    heavy_off.push_back((int64_t)heavy.size());
    hchunk_off.push_back((int64_t)hchunk_v.size());
    const int32_t ecc = cfg.ecc0 && (*cfg.ecc0)[b] >= 0 ? (*cfg.ecc0)[b] : bcc_ecc(B->row, B->col, vo, nb, dist, queue);
    tcap = std::max(tcap, 2 * ecc + kmax + 3);

    const int64_t bat0g = (int64_t)P->h_batches.size(), nbat = ((int64_t)nb + width - 1) / width;
    const int64_t jf0 = std::min(nbat, std::max<int64_t>(0, cfg.fill_begin - bat0g));
    const int64_t jf1 = std::max(jf0, std::min(nbat, cfg.fill_end - bat0g));
    const size_t need = (size_t)std::min<int64_t>(nb, jf1 * (int64_t)width);
    std::vector<int32_t> own_order;
    const std::vector<int32_t> *order_p = cfg.order_of ? &cfg.order_of(b) : nullptr;
    if (!order_p) {
      batched_source_order(B, b, width, (int64_t)need, own_order);
      order_p = &own_order;
    }
    const std::vector<int32_t> &order = *order_p;
    if (order.size() < need) return bail(BCGPU_EINVAL, "source order shorter than the passes need");
    HOST_MARK("b: order");
    // Passes of `width` consecutive sources of the order. Slots and seeds are
    // sized up front (a chain source has two seeds), then every pass fills
    // its own ranges in parallel; the arming lists (variable length after
    // deduplication) are built per pass and concatenated in pass order.
    const size_t bat0 = P->h_batches.size(), slot0 = slots.size(), seed0 = seeds.size();
    std::vector<int64_t> seed_at((size_t)nbat + 1, 0);
#pragma omp parallel for schedule(static)
    for (int64_t j = jf0; j < jf1; ++j) {
      const size_t i0 = (size_t)j * width, i1 = std::min(order.size(), i0 + (size_t)width);
      int64_t cnt = 0;
      for (size_t i = i0; i < i1; ++i) cnt += order[i] >= npl ? 2 : 0;
      seed_at[j + 1] = cnt;
    }
    for (int64_t j = 0; j < nbat; ++j) seed_at[j + 1] += seed_at[j];
    P->h_batches.resize(bat0 + (size_t)nbat);
    slots.resize(slot0 + (size_t)nb);
    seeds.resize(seed0 + (size_t)seed_at[nbat]);
    std::vector<std::vector<int2>> arm_of((size_t)nbat);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < nbat; ++j) {
      const size_t i0 = (size_t)j * width, i1 = std::min((size_t)nb, i0 + (size_t)width);
      const bool fill = j >= jf0 && j < jf1;
      Batch bt{};
      bt.bcc = b;
      bt.nslots = (int32_t)(i1 - i0);
      bt.words = (bt.nslots + 31) / 32;
      bt.kmax = kmax;
      bt.heavy_deg = heavy_deg;
      bt.slot_off = (int64_t)(slot0 + i0);
      bt.seed_off = (int64_t)seed0 + seed_at[j];
      int64_t sd = bt.seed_off;
      std::vector<int2> &arm = arm_of[j];
      if (fill) arm.reserve((size_t)bt.nslots * 2);
      for (size_t i = i0; fill && i < i1; ++i) {
        const int32_t s = order[i];
        const int32_t slot = (int32_t)(i - i0);
        if (s < npl) {
          slots[slot0 + i] = Slot{s, -1, 0, 0};
          arm.push_back(make_int2(s, 0));
          continue;
        }
        const int64_t c = cof[s];
        const int32_t p = cpos[s], k = B->chain_len[c];
        slots[slot0 + i] = Slot{s, (int32_t)c, p, 0};
        seeds[sd++] = Seed{B->chain_l[c], p + 1, slot, 0};
        seeds[sd++] = Seed{B->chain_r[c], k - p, slot, 0};
        bt.max_seed = std::max(bt.max_seed, std::max(p + 1, k - p));
      }
      bt.nseeds = (int32_t)(sd - bt.seed_off);
      // arming list: each core source (level 0) and seeded vertex (its lowest seed level), once
      for (int64_t i = bt.seed_off; i < sd; ++i) arm.push_back(make_int2(seeds[i].v, seeds[i].level));
      std::sort(arm.begin(), arm.end(), [](const int2 &x, const int2 &y) { return x.x != y.x ? x.x < y.x : x.y < y.y; });
      size_t u = 0;
      for (size_t i = 0; i < arm.size(); ++i)
        if (i == 0 || arm[i].x != arm[i - 1].x) arm[u++] = arm[i];
      arm.resize(u);
      bt.narm = (int32_t)u;
      P->h_batches[bat0 + j] = bt;
    }
    for (int64_t j = 0; j < nbat; ++j) {
      Batch &bt = P->h_batches[bat0 + j];
      bt.arm_off = (int64_t)arms.size();
      arms.insert(arms.end(), arm_of[j].begin(), arm_of[j].end());
      std::vector<int2>().swap(arm_of[j]);
      P->u_src.push_back(bt.nslots);
      P->u_teps.push_back((int64_t)bt.nslots * arcs);
      P->u_bfs.push_back(bt.nslots);
      P->u_aux.push_back(0);
      P->u_visits.push_back((int64_t)bt.nslots * nb);
    }
  }
  HOST_MARK("b: passes");
  P->tcap = tcap;
  P->n_cap = ncap;
  P->n_batches = (int64_t)P->h_batches.size();
  auto prefix = [](std::vector<int64_t> &v) {
    std::vector<int64_t> p(v.size() + 1, 0);
    for (size_t i = 0; i < v.size(); ++i) p[i + 1] = p[i] + v[i];
    v.swap(p);
  };
  prefix(P->u_src); prefix(P->u_teps); prefix(P->u_bfs); prefix(P->u_aux); prefix(P->u_visits);

  // ---- device workspace
  const int64_t n = P->n_cap;
  const int64_t qb = P->f32 ? 4 : 8;
  const int64_t nch = (int64_t)hchunk_v.size();
  const int64_t need = n * W * 32 * (4 + 8 + 8 + qb) + (int64_t)(tcap + 2) * n * W * 4 + n * W * 4 + n * 12 +
                       n * W * 8 + (int64_t)W * 32 * (tcap + 2) * 4 + nch * W * 32 * 8;
  if (need > cfg.limit_bytes)
    return bail(BCGPU_ENOMEM, "batched workspace " + std::to_string(need >> 20) + " MiB exceeds the limit " +
                                  std::to_string(cfg.limit_bytes >> 20) + " MiB (lower the batch width)");
  P->pool = cfg.pool;
  P->stream = stream;
  auto alloc = [&](void **p, int64_t bytes) -> bool {
    const size_t sz = (size_t)std::max<int64_t>(bytes, 16);
    cudaError_t e = P->pool ? cudaMallocFromPoolAsync(p, sz, P->pool, stream) : cudaMalloc(p, sz);
    if (e == cudaErrorMemoryAllocation && P->pool) {  // trim the pool's unused reserve once and retry
      cudaGetLastError();
      if (cudaStreamSynchronize(stream) == cudaSuccess && cudaMemPoolTrimTo(P->pool, 0) == cudaSuccess)
        e = cudaMallocFromPoolAsync(p, sz, P->pool, stream);
    }
    if (e != cudaSuccess) return false;
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
  ok &= ok && alloc(&p, n * 4); a.armed = (int32_t *)p;
  ok &= ok && alloc(&p, (4 * ((int64_t)tcap + 3) + 2) * 4); a.wq = (int *)p;
  ok &= ok && alloc(&p, n * W * 8); a.bcpart = (double *)p;
  ok &= ok && alloc(&p, n * W * 32 * 8); a.cdep = (double *)p;
  ok &= ok && alloc(&p, (int64_t)W * 32 * 8); a.wsrc = (double *)p;
  ok &= ok && alloc(&p, (int64_t)W * 32 * (tcap + 2) * 4); a.X = (int32_t *)p;
  ok &= ok && alloc(&p, (int64_t)W * 32 * 4); a.rexp = (int32_t *)p;
  ok &= ok && alloc(&p, sizeof(Ctrl)); a.ctrl = (Ctrl *)p;
  ok &= ok && alloc(&p, (int64_t)std::max<int64_t>(P->n_batches, 1) * 4); a.redo = (int *)p;
  HOST_MARK("b: ws alloc");
  // tables
  auto upload = [&](const void **dst, const void *src, int64_t bytes) -> bool {
    if (!alloc(&p, bytes)) return false;
    *dst = p;
    if (bytes == 0) return true;
    if (cudaMemcpyAsync(p, src, (size_t)bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess) return false;
    P->h2d += bytes;
    return true;
  };
  ok = ok && upload((const void **)&a.hvo, hvo.data(), (int64_t)hvo.size() * 8);
  ok = ok && upload((const void **)&a.hrow, hrow.data(), (int64_t)hrow.size() * 8);
  ok = ok && upload((const void **)&a.n_plain, B->n_plain, (int64_t)B->n_bcc * 4);
  // the contracted rows themselves: filled on the device from the packed CSR
  const int32_t *d_rbcc = nullptr, *d_gcof = nullptr, *d_gcpos = nullptr;
  int *d_bad = nullptr;
  ok = ok && upload((const void **)&d_rbcc, rbcc.data(), (int64_t)rbcc.size() * 4);
  ok = ok && upload((const void **)&d_gcof, gcof.data(), (int64_t)gcof.size() * 4);
  ok = ok && upload((const void **)&d_gcpos, gcpos.data(), (int64_t)gcpos.size() * 4);
  ok = ok && alloc(&p, (int64_t)hrow.size() * 8); a.hsplit = (const int64_t *)p;
  ok = ok && alloc(&p, narcs * 4); a.hcol = (const int32_t *)p;
  ok = ok && alloc(&p, narcs * 4); a.hk = (const int32_t *)p;
  ok = ok && alloc(&p, narcs * 4); a.hcid = (const int32_t *)p;
  ok = ok && alloc(&p, 4); d_bad = (int *)p;
  if (ok && !hrow.empty()) {
    ok = cudaMemsetAsync(d_bad, 0, sizeof(int), stream) == cudaSuccess;
    const int64_t nr = (int64_t)hrow.size();
    const int blocks = (int)std::min<int64_t>((nr + 255) / 256, 148 * 16);
    if (ok) {
      contract_rows_kernel<<<blocks, 256, 0, stream>>>(row, col, vtx_off, a.n_plain, d_rbcc, a.hvo, a.hrow, nr, d_gcof,
                                                       d_gcpos, chain_len, chain_l, chain_r, (int64_t *)a.hsplit,
                                                       (int32_t *)a.hcol, (int32_t *)a.hk, (int32_t *)a.hcid, d_bad);
      ok = cudaGetLastError() == cudaSuccess;
    }
  }
  ok = ok && upload((const void **)&a.chain_off, B->chain_off, (int64_t)(B->n_bcc + 1) * 8);
  ok = ok && upload((const void **)&a.cpre_off, cpre_off.data(), (int64_t)cpre_off.size() * 8);
  ok = ok && upload((const void **)&a.cpre, cpre.data(), (int64_t)cpre.size() * 8);
  ok = ok && upload((const void **)&a.heavy_off, heavy_off.data(), (int64_t)heavy_off.size() * 8);
  ok = ok && upload((const void **)&a.heavy, heavy.data(), (int64_t)heavy.size() * 4);
  ok = ok && upload((const void **)&a.hchunk_off, hchunk_off.data(), (int64_t)hchunk_off.size() * 8);
  ok = ok && upload((const void **)&a.hchunk_v, hchunk_v.data(), nch * 4);
  ok = ok && upload((const void **)&a.hchunk_e0, hchunk_e0.data(), nch * 8);
  ok = ok && upload((const void **)&a.hchunk_e1, hchunk_e1.data(), nch * 8);
  ok = ok && upload((const void **)&a.hfirst, hfirst.data(), (int64_t)hfirst.size() * 4);
  ok = ok && upload((const void **)&a.batches, P->h_batches.data(), (int64_t)P->h_batches.size() * (int64_t)sizeof(Batch));
  {  // slots: only those of the filled passes are copied (the rest are never read)
    int64_t s0 = (int64_t)slots.size(), s1 = 0;
    for (int64_t j = std::max<int64_t>(0, cfg.fill_begin); j < std::min(P->n_batches, cfg.fill_end); ++j) {
      s0 = std::min(s0, P->h_batches[(size_t)j].slot_off);
      s1 = std::max(s1, P->h_batches[(size_t)j].slot_off + P->h_batches[(size_t)j].nslots);
    }
    ok = ok && alloc(&p, (int64_t)slots.size() * (int64_t)sizeof(Slot));
    a.slots = (const Slot *)p;
    if (ok && s1 > s0) {
      const size_t bytes = (size_t)(s1 - s0) * sizeof(Slot);
      ok = cudaMemcpyAsync((Slot *)p + s0, slots.data() + s0, bytes, cudaMemcpyHostToDevice, stream) == cudaSuccess;
      P->h2d += (int64_t)bytes;
    }
  }
  ok = ok && upload((const void **)&a.seeds, seeds.data(), (int64_t)seeds.size() * (int64_t)sizeof(Seed));
  ok = ok && upload((const void **)&a.arms, arms.data(), (int64_t)arms.size() * (int64_t)sizeof(int2));
  ok = ok && alloc(&p, std::max<int64_t>(nch, 1) * W * 32 * 8); a.hacc = (double *)p;
  ok = ok && alloc(&p, std::max<int64_t>(nch, 1) * W * 4); a.hmask = (uint32_t *)p;
  if (!ok) return bail(BCGPU_ENOMEM, "cudaMalloc or upload of the batched workspace failed");
  cudaError_t e = cudaMemsetAsync(a.ctrl, 0, sizeof(Ctrl), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.redo, 0, (size_t)std::max<int64_t>(P->n_batches, 1) * 4, stream);
  int h_bad = 0;
  if (e == cudaSuccess && !hrow.empty()) {
    e = cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, stream);
    P->d2h += (int64_t)sizeof(int);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // the host vectors go out of scope
  HOST_MARK("b: uploads+sync");
  P->h_slots = std::move(slots);
  if (cfg.keep_host_tables) {
    P->h_seeds = std::move(seeds);
    P->h_arms = std::move(arms);
  }
  P->h_vtx_off.assign(B->vtx_off, B->vtx_off + B->n_bcc + 1);
  if (e != cudaSuccess) return bail(BCGPU_ECUDA, std::string("batched upload: ") + cudaGetErrorString(e));
  if (h_bad & 1) return bail(BCGPU_EINVAL, "a non-core vertex outside every chain");
  if (h_bad & 2) return bail(BCGPU_EINVAL, "a core vertex adjacent to the inside of a chain");
  a.reach = reach; a.vtx_off = vtx_off;
  a.chain_start = chain_start; a.chain_len = chain_len; a.chain_l = chain_l; a.chain_r = chain_r;
  a.n_cap = P->n_cap; a.W = W; a.tcap = tcap; a.bc = bc; a.err = err;
  a.rescale_exp = cfg.rescale_exp > 0 ? cfg.rescale_exp : 900;
  a.wait_ns = cfg.wait_ns;

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
  return BCGPU_OK;
}

}  // namespace

int batched_create(const bc_bccs *B, const BatchedConfig &cfg, const int64_t *row, const int32_t *col,
                   const int32_t *reach, const int64_t *vtx_off, const int32_t *chain_start, const int32_t *chain_len,
                   const int32_t *chain_l, const int32_t *chain_r, double *bc, int *err, cudaStream_t stream,
                   BatchedPlan **out, std::string *msg) {
  BatchedPlan *P = nullptr;
  int rc;
  try {  // a host allocation that throws releases the partial plan like any other failure
    P = new BatchedPlan;
    rc = batched_build(B, cfg, row, col, reach, vtx_off, chain_start, chain_len, chain_l, chain_r, bc, err, stream, P,
                       msg);
  } catch (const std::bad_alloc &) {
    if (msg) *msg = "host allocation failed while building the passes";
    rc = BCGPU_ENOMEM;
  }
  if (rc != BCGPU_OK) {
    batched_destroy(P);
    return rc;
  }
  *out = P;
  return BCGPU_OK;
}

void batched_destroy(BatchedPlan *p) {
  if (!p) return;
  for (void *a : p->allocs) {
    if (p->pool) cudaFreeAsync(a, p->stream);
    else cudaFree(a);
  }
  delete p;
}

int64_t batched_device_bytes(const BatchedPlan *p) { return p ? p->bytes : 0; }

uint64_t batched_pass_digest(const BatchedPlan *p, int64_t pass) {
  if (!p || pass < 0 || pass >= (int64_t)p->h_batches.size()) return 0;
  const Batch &b = p->h_batches[(size_t)pass];
  if ((int64_t)p->h_seeds.size() < b.seed_off + b.nseeds || (int64_t)p->h_arms.size() < b.arm_off + b.narm) return 0;
  uint64_t h = 1469598103934665603ull;  // FNV-1a
  auto mix = [&h](const void *q, size_t n) {
    const unsigned char *c = (const unsigned char *)q;
    for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
  };
  const int32_t head[8] = {b.bcc, b.nslots, b.words, b.nseeds, b.max_seed, b.kmax, b.heavy_deg, b.narm};
  mix(head, sizeof head);
  mix(p->h_slots.data() + b.slot_off, sizeof(Slot) * (size_t)b.nslots);
  mix(p->h_seeds.data() + b.seed_off, sizeof(Seed) * (size_t)b.nseeds);
  mix(p->h_arms.data() + b.arm_off, sizeof(int2) * (size_t)b.narm);
  return h;
}
int64_t batched_h2d_bytes(const BatchedPlan *p) { return p ? p->h2d : 0; }
int64_t batched_d2h_bytes(const BatchedPlan *p) { return p ? p->d2h : 0; }
int64_t batched_status_bytes(const BatchedPlan *p) {
  return p ? (int64_t)sizeof(int) * std::max<int64_t>(p->n_batches, 1) : 0;
}
int batched_width(const BatchedPlan *p) { return p ? p->width : 0; }

void batched_unit_sources(const BatchedPlan *p, int64_t begin, int64_t end, std::vector<int64_t> &out) {
  for (int64_t bi = begin; bi < end; ++bi) {
    const Batch &bt = p->h_batches[bi];
    const int64_t vo = p->h_vtx_off[bt.bcc];
    for (int32_t i = 0; i < bt.nslots; ++i) out.push_back(vo + p->h_slots[bt.slot_off + i].src);
  }
}

int batched_pass_shape(const BatchedPlan *p, int64_t pass, int32_t *bcc, int32_t *nslots) {
  if (!p || pass < 0 || pass >= p->n_batches) return BCGPU_EINVAL;
  *bcc = p->h_batches[pass].bcc;
  *nslots = p->h_batches[pass].nslots;
  return BCGPU_OK;
}

int batched_pass_rows(const BatchedPlan *p, int64_t pass, const int32_t *chain_start, int32_t n_core,
                      cudaStream_t stream, std::vector<int32_t> &src, std::vector<int32_t> &d, std::vector<double> &sigma,
                      std::string *msg) {
  if (pass < 0 || pass >= p->n_batches) {
    *msg = "not a multi-source pass";
    return BCGPU_EINVAL;
  }
  const Batch &bt = p->h_batches[pass];
  const int B = bt.nslots, WB = p->W * 32, L = p->tcap + 2;
  std::vector<int32_t> hd((size_t)n_core * WB), hx((size_t)WB * L);
  std::vector<double> hs((size_t)n_core * WB);
  cudaError_t e = cudaMemcpyAsync(hd.data(), p->args.d, hd.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hs.data(), p->args.sig, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hx.data(), p->args.X, hx.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    *msg = std::string("pass row read-back: ") + cudaGetErrorString(e);
    return BCGPU_ECUDA;
  }
  src.resize((size_t)B);
  d.resize((size_t)B * n_core);
  sigma.resize((size_t)B * n_core);
  for (int b = 0; b < B; ++b) {
    const Slot &sl = p->h_slots[bt.slot_off + b];
    src[b] = sl.chain < 0 ? sl.src : chain_start[sl.chain] + sl.pos;
    for (int32_t v = 0; v < n_core; ++v) {
      const size_t i = (size_t)v * WB + b;
      const int lv = hd[i];
      d[(size_t)b * n_core + v] = lv;
      // stored count s at level lv stands for s * 2^X(slot, lv)
      sigma[(size_t)b * n_core + v] = std::ldexp(hs[i], hx[(size_t)b * L + std::min(std::max(lv, 0), L - 1)]);
    }
  }
  return BCGPU_OK;
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
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (e == cudaSuccess) e = cudaStreamIsCapturing(stream, &cap);
  const void *fn = p->f32 ? (const void *)batched_kernel<float> : (const void *)batched_kernel<double>;
  if (e == cudaSuccess && cap == cudaStreamCaptureStatusActive) {
    // recorded into a CUDA graph: a kernel node carrying the cooperative attribute
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(p->grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = p->smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelExC(&cfg, fn, params);
  } else if (e == cudaSuccess) {
    e = cudaLaunchCooperativeKernel(fn, p->grid, kThreads, params, p->smem, stream);
  }
  if (e != cudaSuccess) {
    if (msg) *msg = std::string("cooperative launch: ") + cudaGetErrorString(e);
    return BCGPU_ECUDA;
  }
  if (launches) *launches += 1;
  return BCGPU_OK;
}

}  // namespace bcg
