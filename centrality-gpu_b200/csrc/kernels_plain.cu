// PLAIN schedule: one source per CTA at a time, FP64 path counts (with
// per-level power-of-two scaling) and dependencies; BC accumulated in
// fixed-point integer counters, so the result does not depend on the order
// in which CTAs finish their sources.
//
// Follows the reference's per-source Brandes (bc_kgpu_free / bc_kgpu_active,
// Codes/kernels_free.cu:154-473, Codes/kernels_active.cu:263-602) and its
// chain postprocessing (Codes/postprocesses.cu:205-470), re-designed:
//  * no O(n) row reset per source: levels are stamped with a per-row epoch
//    (level + base; anything below base is unvisited), the reference clears
//    d/sigma/delta for every source (Codes/kernels_free.cu:205-218);
//  * each vertex's adjacency is read once in the forward phase: when a
//    frontier vertex is expanded it pulls sigma from its predecessors (all one
//    level up, already final) and discovers its successors in the same scan,
//    so sigma needs no atomics and its sum order is fixed;
//  * neighbour scans are switched by degree: a thread per vertex up to 8 arcs,
//    a warp up to 2048, the whole CTA above (the reference gives each frontier
//    vertex one thread, Codes/kernels_free.cu:316-335);
//  * the dependency sweep stores q(w) = (reach(w)+1+delta(w)) / sigma(w) so a
//    predecessor reads one value per successor: delta(v) = sigma(v) * sum q(w)
//    (same quantity as Codes/kernels_free.cu:391,409);
//  * path counts are stored per level relative to a power of two 2^X(level):
//    a level whose largest count passes 2^rescale_exp is divided by a power
//    of two (exact), so deep, high-diameter BCCs do not overflow FP64 (the
//    reference keeps sigma in uint64 / int32, Codes/kernels_free.cu:161,
//    Codes/kernels_active.cu:274, and overflows silently); the backward
//    sweep rescales by 2^(X(l) - X(l+1)) between levels. Counts or
//    dependencies that still leave FP64's range flag kDevOverflow;
//  * BC: the reference adds FP32 dependencies with atomicAdd
//    (Codes/kernels_free.cu:423-426), whose result depends on the order of
//    the adds; here each contribution goes into fixed-point integer counters
//    (see PlainArgs::acc) that launch_fold turns into FP64;
//  * a chain vertex's rows are the merge of its endpoints' rows
//    (Codes/postprocesses.cu:329-351) and its dependency sweep walks the
//    endpoints' level buckets directly instead of radix-sorting n distance
//    keys per source (Codes/postprocesses.cu:143-155).
// A work item is one free/endpoint source plus (a bounded share of) the
// chains whose left endpoint it is, so the left endpoint's BFS serves all of
// them and only the right endpoint's BFS is repeated (forward only) per
// distinct right endpoint.
#include "accum.cuh"
#include "common.cuh"
#include "plain.h"

#include <algorithm>
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace bcg {

namespace {

constexpr int kSmallDeg = 8;
constexpr int kWarpDeg = 2048;

template <int kBlock>
struct Shared {
  static constexpr int kWarps = kBlock / 32;
  int tail;          // next free slot of the visit order S
  int nwq, ncq;      // warp-tier / CTA-tier queue lengths
  int flag;
  int imax;
  int item;
  int base_a, base_b;  // epochs of rows A and B
  int emax[2];         // largest biased FP64 exponent of the path counts of a level (by level parity)
  double red[kWarps];
  int wq[kBlock];
  int cq[kBlock];
};

// A vertex's entry in a BFS row: its level stamp and its path count -- q
// once the dependency sweep has passed the vertex (q(w) replaces sigma(w) in
// place: nothing reads sigma(w) after w's own sweep step) -- so that one
// 16-byte load gives a neighbour's level and value (one sector instead of one
// in each of two rows).
struct __align__(16) Rec {
  int32_t d;
  int32_t pad;
  double v;
};
__device__ __forceinline__ Rec ld_rec(const Rec *p) {
  const int4 x = __ldcg(reinterpret_cast<const int4 *>(p));
  return Rec{x.x, 0, __hiloint2double(x.w, x.z)};
}

// Per-CTA workspace (capacity ws_n each), addressed from two base pointers so
// that the row pointers are recomputed where used instead of being held in
// registers. Records: A (own BFS), B (right endpoint BFS), M (merged chain
// rows). Int rows: visit orders and level offsets of A and B, and the
// power-of-two exponent X of each level of A, B and M (path count = stored
// value * 2^X).
struct Rows {
  int32_t *wi;
  Rec *wr;
  int64_t n;
  __device__ __forceinline__ int32_t *SA() const { return wi; }
  __device__ __forceinline__ int32_t *lvA() const { return wi + n; }
  __device__ __forceinline__ int32_t *SB() const { return wi + 2 * n; }
  __device__ __forceinline__ int32_t *lvB() const { return wi + 3 * n; }
  __device__ __forceinline__ int32_t *lxA() const { return wi + 4 * n; }
  __device__ __forceinline__ int32_t *lxB() const { return wi + 5 * n; }
  __device__ __forceinline__ int32_t *lxM() const { return wi + 6 * n; }
  __device__ __forceinline__ Rec *A() const { return wr; }
  __device__ __forceinline__ Rec *B() const { return wr + n; }
  __device__ __forceinline__ Rec *M() const { return wr + 2 * n; }
};

__device__ __forceinline__ Rows rows_of(const PlainArgs &a, int64_t slot) {
  return Rows{a.ws_i + slot * kWsIntRows * a.ws_n,
              reinterpret_cast<Rec *>(a.ws_f + slot * kWsDblRows * a.ws_n), a.ws_n};
}

// Appends x to S (warp-aggregated atomic on the shared tail).
template <class SH>
__device__ __forceinline__ void append(SH &sh, int32_t *S, int32_t x) {
  cg::coalesced_group g = cg::coalesced_threads();
  int pos = 0;
  if (g.thread_rank() == 0) pos = atomicAdd(&sh.tail, (int)g.size());
  pos = g.shfl(pos, 0) + (int)g.thread_rank();
  S[pos] = x;
}

// Forward step for one arc (w -> x) at level lev: accumulate sigma from a
// predecessor, or claim an unvisited vertex for level lev+1.
template <class SH>
__device__ __forceinline__ void fwd_arc(SH &sh, Rec *r, int32_t *S, int32_t x, int dprev, int dnext, int base,
                                        double &acc) {
  const Rec rx = ld_rec(r + x);
  if (rx.d == dprev) {
    acc += rx.v;
  } else if (rx.d < base) {
    int old = atomicMax(&r[x].d, dnext);
    if (old < base) append(sh, S, x);
  }
}

// Forward scan of a low-degree vertex by one thread, kGather arcs at a time:
// the neighbour ids, then their records (level and path count in one load)
// are each issued as independent loads (one memory round trip per group
// instead of one per arc). Sums and claims follow arc order, so sigma is the
// same value the arc-by-arc form computes.
constexpr int kGather = 4;

template <class SH>
__device__ __forceinline__ double fwd_small(SH &sh, const int32_t *Ce, int deg, Rec *r, int32_t *S, int dprev,
                                            int dnext, int base) {
  double acc = 0.0;
  for (int g = 0; g < deg; g += kGather) {
    int32_t x[kGather];
    Rec rx[kGather];
#pragma unroll
    for (int j = 0; j < kGather; ++j) x[j] = g + j < deg ? ldg(Ce + g + j) : -1;
#pragma unroll
    for (int j = 0; j < kGather; ++j) rx[j] = x[j] >= 0 ? ld_rec(r + x[j]) : Rec{INT_MAX, 0, 0.0};  // INT_MAX: skipped
#pragma unroll
    for (int j = 0; j < kGather; ++j) {
      if (rx[j].d == dprev) {
        acc += rx[j].v;
      } else if (rx[j].d < base) {
        const int old = atomicMax(&r[x[j]].d, dnext);
        if (old < base) append(sh, S, x[j]);
      }
    }
  }
  return acc;
}

template <int kBlock>
__device__ __forceinline__ double block_sum(Shared<kBlock> &sh, double v) {
  constexpr int kWarps = kBlock / 32;
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh.red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kWarps; ++i) t += sh.red[i];  // fixed order
    sh.red[0] = t;
  }
  __syncthreads();
  t = sh.red[0];
  __syncthreads();
  return t;
}

// CTA-wide BFS from s over one BCC: fills the records r (level stamps from
// epoch base, scaled path counts), the level order S, level offsets
// lv[0..nlev] and the level exponents lx[0..nlev) (path count of a vertex on
// level l = sigma * 2^lx[l]). Returns nlev (number of levels).
template <int kBlock>
__device__ int cta_bfs(Shared<kBlock> &sh, const int64_t *R, const int32_t *C, int32_t s, Rec *r, int32_t *S,
                       int32_t *lv, int32_t *lx, int base, int rescale_exp, int *err) {
  constexpr int kWarps = kBlock / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    r[s].d = base;
    S[0] = s;
    lv[0] = 0;
    lv[1] = 1;
    sh.tail = 1;
    sh.emax[0] = 0;
    sh.emax[1] = 0;
  }
  __syncthreads();
  int lev = 0, xprev = 0;
  while (true) {
    const int f0 = lv[lev], f1 = lv[lev + 1];
    // the source has no predecessors; stale stamps are < base so they never match base+lev-1
    const int dprev = lev == 0 ? INT_MIN : base + lev - 1, dnext = base + lev + 1;
    int emax = 0;  // largest exponent field among the path counts this thread writes on this level
    for (int c0 = f0; c0 < f1; c0 += kBlock) {
      if (tid == 0) { sh.nwq = 0; sh.ncq = 0; }
      __syncthreads();
      const int i = c0 + tid;
      if (i < f1) {
        const int32_t w = S[i];
        const int64_t e0 = R[w], e1 = R[w + 1];
        const int64_t deg = e1 - e0;
        if (deg <= kSmallDeg) {
          const double acc = fwd_small(sh, C + e0, (int)deg, r, S, dprev, dnext, base);
          const double v = lev == 0 ? 1.0 : acc;
          r[w].v = v;
          emax = max(emax, exp_bits(v));
        } else if (deg <= kWarpDeg) {
          sh.wq[atomicAdd(&sh.nwq, 1)] = w;
        } else {
          sh.cq[atomicAdd(&sh.ncq, 1)] = w;
        }
      }
      __syncthreads();
      for (int k = warp; k < sh.nwq; k += kWarps) {
        const int32_t w = sh.wq[k];
        const int64_t e0 = R[w], e1 = R[w + 1];
        double acc = 0.0;
        for (int64_t e = e0 + lane; e < e1; e += 32) fwd_arc(sh, r, S, ldg(C + e), dprev, dnext, base, acc);
        acc = warp_sum(acc);
        if (lane == 0) {
          const double v = lev == 0 ? 1.0 : acc;
          r[w].v = v;
          emax = max(emax, exp_bits(v));
        }
      }
      const int ncq = sh.ncq;
      for (int k = 0; k < ncq; ++k) {
        const int32_t w = sh.cq[k];
        const int64_t e0 = R[w], e1 = R[w + 1];
        double acc = 0.0;
        for (int64_t e = e0 + tid; e < e1; e += kBlock) fwd_arc(sh, r, S, ldg(C + e), dprev, dnext, base, acc);
        acc = block_sum(sh, acc);
        if (tid == 0) {
          const double v = lev == 0 ? 1.0 : acc;
          r[w].v = v;
          emax = max(emax, exp_bits(v));
        }
      }
      emax = __reduce_max_sync(0xffffffffu, emax);
      if (lane == 0) atomicMax(&sh.emax[lev & 1], emax);
      __syncthreads();
    }
    // the level's path counts are final: rescale them if the largest passed 2^rescale_exp
    const int ebig = sh.emax[lev & 1];
    int x = xprev;
    if (ebig == 0x7ff) {
      set_err(err, kDevOverflow);
    } else if (rescale_exp > 0 && ebig - 1023 > rescale_exp) {
      const int k = ebig - 1023;  // brings the largest count to [1, 2)
      x += k;
      bool lost = false;
      for (int i = f0 + tid; i < f1; i += kBlock) {
        const int32_t w = S[i];
        const double v = scale2(r[w].v, -k);
        lost |= exp_bits(v) == 0;  // a count of this level fell out of the normal range
        r[w].v = v;
      }
      if (lost) set_err(err, kDevOverflow);
    }
    if (tid == 0) {
      lx[lev] = x;
      sh.emax[(lev + 1) & 1] = 0;
    }
    xprev = x;
    const int tail = sh.tail;
    if (tail == f1) break;
    if (tid == 0) lv[lev + 2] = tail;
    ++lev;
    __syncthreads();
  }
  __syncthreads();  // rescaled counts and lx visible to the caller's next phase
  return lev + 1;
}

// Dependency of w at level lev of a row (d stamped as base + level):
// delta(w) = sigma(w) * sum over successors x of q(x); then q(w) and BC.
// (one thread; ids, then the successors' records gathered kGather at a time,
// summed in arc order as in fwd_small)
__device__ __forceinline__ double bwd_arcs_thread(const int64_t *R, const int32_t *C, const Rec *r, int32_t w,
                                                  int dsucc) {
  double acc = 0.0;
  const int64_t e0 = R[w];
  const int deg = (int)(R[w + 1] - e0);
  for (int g = 0; g < deg; g += kGather) {
    int32_t x[kGather];
    Rec rx[kGather];
#pragma unroll
    for (int j = 0; j < kGather; ++j) x[j] = g + j < deg ? ldg(C + e0 + g + j) : -1;
#pragma unroll
    for (int j = 0; j < kGather; ++j) rx[j] = x[j] >= 0 ? ld_rec(r + x[j]) : Rec{INT_MIN, 0, 0.0};
#pragma unroll
    for (int j = 0; j < kGather; ++j)
      if (rx[j].d == dsucc) acc += rx[j].v;
  }
  return acc;
}

// Successor sums arrive in the scale of the next level: 2^sdiff =
// 2^(X(level) - X(level+1)) brings them to this level's, so that
// delta = sig * sum is the unscaled dependency and q = (reach+1+delta)/sig is
// in this level's scale (stored over sigma).
__device__ __forceinline__ void finish_vertex(int32_t w, double acc, int sdiff, const int32_t *rch, Rec *r,
                                              unsigned long long *accb, double wsrc, int *err) {
  const double sw = r[w].v;
  const double delta = sw * scale2(acc, sdiff);
  const double qw = ((double)rch[w] + 1.0 + delta) / sw;
  r[w].v = qw;
  if (exp_bits(qw) == 0x7ff || exp_bits(delta) == 0x7ff) set_err(err, kDevOverflow);
  if (delta != 0.0) acc_add(accb + (int64_t)kAccDigits * w, delta * wsrc, err);
}

// Vertex list of one backward level: up to three index ranges with filters.
struct LevelList {
  const int32_t *S0; int a0, b0;  // primary list
  const int32_t *S1; int a1, b1;  // secondary list (merged rows: right endpoint's bucket)
  int ck0, ck1;                   // chain vertices at direct distance (merged rows; -1 = none)
};

// mode 0: BFS row, every listed vertex is at this level.
// mode 1: merged row: keep w iff dM(w) == lev, with duplicates removed
//         (tie vertices listed in both buckets are taken from the primary one).
struct MergeFilter {
  const Rec *A; int baseA; int ld;
  const Rec *B; int baseB; int rd;
};

__device__ __forceinline__ bool keep_vertex(int mode, int list, int32_t w, int lev, const Rec *rM,
                                            const MergeFilter &mf) {
  if (mode == 0) return true;
  if (rM[w].d != lev) return false;
  if (list == 0) return true;
  const bool inA = (mf.A[w].d - mf.baseA) + mf.ld == lev;
  if (list == 1) return !inA;
  const bool inB = (mf.B[w].d - mf.baseB) + mf.rd == lev;
  return !inA && !inB;
}

template <int kBlock>
__device__ void cta_bwd_level(Shared<kBlock> &sh, const int64_t *R, const int32_t *C, Rec *r, const int32_t *rch,
                              unsigned long long *accb, double wsrc, int dsucc, int lev, int sdiff, int mode,
                              const LevelList &L, const MergeFilter &mf, int *err) {
  constexpr int kWarps = kBlock / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int list = 0; list < 3; ++list) {
    const int32_t *S = list == 0 ? L.S0 : list == 1 ? L.S1 : nullptr;
    int a = list == 0 ? L.a0 : list == 1 ? L.a1 : 0;
    int b = list == 0 ? L.b0 : list == 1 ? L.b1 : (L.ck0 >= 0) + (L.ck1 >= 0);
    if (b <= a) continue;
    for (int c0 = a; c0 < b; c0 += kBlock) {
      if (tid == 0) { sh.nwq = 0; sh.ncq = 0; }
      __syncthreads();
      const int i = c0 + tid;
      if (i < b) {
        int32_t w = list < 2 ? S[i] : (i == 0 && L.ck0 >= 0 ? L.ck0 : L.ck1);
        if (keep_vertex(mode, list, w, lev, r, mf)) {
          const int64_t deg = R[w + 1] - R[w];
          if (deg <= kSmallDeg) {
            finish_vertex(w, bwd_arcs_thread(R, C, r, w, dsucc), sdiff, rch, r, accb, wsrc, err);
          } else if (deg <= kWarpDeg) {
            sh.wq[atomicAdd(&sh.nwq, 1)] = w;
          } else {
            sh.cq[atomicAdd(&sh.ncq, 1)] = w;
          }
        }
      }
      __syncthreads();
      for (int k = warp; k < sh.nwq; k += kWarps) {
        const int32_t w = sh.wq[k];
        double acc = 0.0;
        for (int64_t e = R[w] + lane; e < R[w + 1]; e += 32) {
          const Rec rx = ld_rec(r + ldg(C + e));
          if (rx.d == dsucc) acc += rx.v;
        }
        acc = warp_sum(acc);
        if (lane == 0) finish_vertex(w, acc, sdiff, rch, r, accb, wsrc, err);
      }
      const int ncq = sh.ncq;
      for (int k = 0; k < ncq; ++k) {
        const int32_t w = sh.cq[k];
        double acc = 0.0;
        for (int64_t e = R[w] + tid; e < R[w + 1]; e += kBlock) {
          const Rec rx = ld_rec(r + ldg(C + e));
          if (rx.d == dsucc) acc += rx.v;
        }
        acc = block_sum(sh, acc);
        if (tid == 0) finish_vertex(w, acc, sdiff, rch, r, accb, wsrc, err);
      }
      __syncthreads();
    }
  }
}

// Keeps epochs below 2^30: wraps the whole row (every BCC this CTA may see)
// back to all-unvisited when the next BFS could overflow.
__device__ void ensure_epoch(Rec *r, int64_t cap, int &base, int span) {
  if (base + span + 2 < (1 << 30)) return;
  for (int64_t k = threadIdx.x; k < cap; k += blockDim.x) r[k].d = 0;
  __syncthreads();
  base = 1;
}

// Level exponents of a merged row: level l of the merged row holds vertices
// from level l-ld of row A and level l-rd of row B; its exponent is the larger
// of theirs (0 when neither exists: chain vertices only).
struct MergedExp {
  const int32_t *lxA, *lxB;
  int nlevA, nlevB, ld, rd;
  __device__ __forceinline__ int operator()(int l) const {
    int x = 0;
    const int a = l - ld, b = l - rd;
    if (a >= 0 && a < nlevA) x = max(x, lxA[a]);
    if (b >= 0 && b < nlevB) x = max(x, lxB[b]);
    return x;
  }
};

// Rows of chain vertex (start+pos) from the endpoint rows A (left) and B
// (right): d = min(dA+ld, dB+rd), sigma from the strictly shorter side or the
// sum on ties (Codes/postprocesses.cu:334-350), each brought to the merged
// level's exponent; then the chain's own vertices are fixed along the chain
// (Codes/postprocesses.cu:205-274). Returns max level.
template <int kBlock>
__device__ int merge_rows(Shared<kBlock> &sh, const Rows &r, int baseA, int baseB, int32_t nb, int32_t start, int32_t len,
                          int32_t pos, const MergedExp &xm, int *err) {
  const int ld = pos + 1, rd = len - pos;
  int mx = 0;
  bool bad = false;
  for (int k = threadIdx.x; k < nb; k += kBlock) {
    const Rec ra = ld_rec(r.A() + k), rb = ld_rec(r.B() + k);
    const int la = ra.d - baseA, lb = rb.d - baseB;
    if ((la < 0) | (lb < 0) | (la >= xm.nlevA) | (lb >= xm.nlevB)) {
      bad = true;
      continue;
    }
    const int a = la + ld, b = lb + rd;
    int dm;
    double sm;
    if (a < b) { dm = a; sm = scale2(ra.v, xm.lxA[la] - xm(a)); }
    else if (a > b) { dm = b; sm = scale2(rb.v, xm.lxB[lb] - xm(b)); }
    else {
      dm = b;
      const int x = xm(b);
      sm = scale2(ra.v, xm.lxA[la] - x) + scale2(rb.v, xm.lxB[lb] - x);
    }
    r.M()[k].d = dm;
    r.M()[k].v = sm;
    mx = max(mx, dm);
  }
  if (bad) set_err(err, kDevDisconnected);
  mx = warp_max(mx);
  if (threadIdx.x == 0) sh.imax = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) atomicMax(&sh.imax, mx);
  __syncthreads();
  const int maxlev = sh.imax;
  if (threadIdx.x == 0) {
    for (int j = 0; j < len; ++j) {
      const int k = start + j;
      const int dist = j > pos ? j - pos : pos - j;
      const double one = scale2(1.0, -xm(dist));  // one path, in the merged level's scale
      Rec &m = r.M()[k];
      if (m.d > dist) { m.d = dist; m.v = one; }
      else if (m.d == dist) m.v += one;
    }
  }
  for (int l = threadIdx.x; l <= maxlev; l += kBlock) r.lxM()[l] = xm(l);
  __syncthreads();
  return maxlev;
}

template <int kBlock>
__device__ void process_item(Shared<kBlock> &sh, const PlainArgs &a, const Rows &r, const PlainItem &it) {
  const int32_t b = it.bcc;
  const int64_t vo = a.vtx_off[b];
  const int32_t nb = (int32_t)(a.vtx_off[b + 1] - vo);
  if ((int64_t)nb + 2 > a.ws_n) { set_err(a.err, kDevWorkspace); return; }
  const int64_t *R = a.row + vo;
  const int32_t *rch = a.reach + vo;
  unsigned long long *accb = a.acc + (int64_t)kAccDigits * vo;
  const MergeFilter none{nullptr, 0, 0, nullptr, 0, 0};

  // own source: BFS into row A (its dependency sweep comes after the chains:
  // their merged rows read row A's path counts, which the sweep replaces by q)
  int baseA = sh.base_a;
  ensure_epoch(r.A(), a.ws_n, baseA, nb);
  const int nlevA = cta_bfs(sh, R, a.col, it.src, r.A(), r.SA(), r.lvA(), r.lxA(), baseA, a.rescale_exp, a.err);

  int baseB = sh.base_b, nlevB = 0, prevR = -1;
  for (int32_t c = it.c0; c < it.c1; ++c) {
    const int32_t start = a.chain_start[c], len = a.chain_len[c], cr = a.chain_r[c];
    if (a.chain_l[c] != it.src || start < 0 || start + len > nb) { set_err(a.err, kDevBadItem); break; }
    if (cr != prevR) {
      if (prevR >= 0) baseB += nlevB + 1;
      ensure_epoch(r.B(), a.ws_n, baseB, nb);
      nlevB = cta_bfs(sh, R, a.col, cr, r.B(), r.SB(), r.lvB(), r.lxB(), baseB, a.rescale_exp, a.err);
      prevR = cr;
    }
    for (int32_t pos = 0; pos < len; ++pos) {
      const int32_t z = start + pos;
      const int ld = pos + 1, rd = len - pos;
      const MergedExp xm{r.lxA(), r.lxB(), nlevA, nlevB, ld, rd};
      const int maxlev = merge_rows(sh, r, baseA, baseB, nb, start, len, pos, xm, a.err);
      const double wz = (double)rch[z] + 1.0;
      const MergeFilter mf{r.A(), baseA, ld, r.B(), baseB, rd};
      for (int lev = maxlev; lev >= 1; --lev) {
        LevelList L{r.SA(), 0, 0, r.SB(), 0, 0, -1, -1};
        const int la = lev - ld, lb = lev - rd;
        if (la >= 0 && la < nlevA) { L.a0 = r.lvA()[la]; L.b0 = r.lvA()[la + 1]; }
        if (lb >= 0 && lb < nlevB) { L.a1 = r.lvB()[lb]; L.b1 = r.lvB()[lb + 1]; }
        if (pos - lev >= 0) L.ck0 = start + pos - lev;
        if (pos + lev < len) L.ck1 = start + pos + lev;
        const int sdiff = lev < maxlev ? r.lxM()[lev] - r.lxM()[lev + 1] : 0;
        cta_bwd_level(sh, R, a.col, r.M(), rch, accb, wz, lev + 1, lev, sdiff, 1, L, mf, a.err);
      }
    }
  }
  if (prevR >= 0) baseB += nlevB + 1;

  const double wsrc = (double)rch[it.src] + 1.0;
  for (int lev = it.own ? nlevA - 1 : 0; lev >= 1; --lev) {
    LevelList L{r.SA(), r.lvA()[lev], r.lvA()[lev + 1], nullptr, 0, 0, -1, -1};
    const int sdiff = lev + 1 < nlevA ? r.lxA()[lev] - r.lxA()[lev + 1] : 0;  // the deepest level has no successors
    cta_bwd_level(sh, R, a.col, r.A(), rch, accb, wsrc, baseA + lev + 1, lev, sdiff, 0, L, none, a.err);
  }
  if (threadIdx.x == 0) {
    sh.base_a = baseA + nlevA + 1;
    sh.base_b = baseB;
  }
  __syncthreads();
}

template <int kBlock>
__global__ void __launch_bounds__(kBlock, 1024 / kBlock) plain_kernel(PlainArgs a) {
  __shared__ Shared<kBlock> sh;
  const Rows r = rows_of(a, blockIdx.x);
  if (threadIdx.x == 0) {
    sh.base_a = a.epochs[2 * blockIdx.x];
    sh.base_b = a.epochs[2 * blockIdx.x + 1];
  }
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) {
      // stop early (uniformly for the CTA) once any CTA has flagged an error
      const int64_t k = (int64_t)atomicAdd(a.next_item, 1ull);
      sh.item = (*(volatile int *)a.err != kDevOk || a.item_begin + k >= a.item_end) ? -1 : (int)k;
    }
    __syncthreads();
    if (sh.item < 0) break;
    const PlainItem it = a.items[a.item_begin + sh.item];
    process_item(sh, a, r, it);
  }
  if (threadIdx.x == 0) {
    a.epochs[2 * blockIdx.x] = sh.base_a;
    a.epochs[2 * blockIdx.x + 1] = sh.base_b;
  }
}

// Rows of one source for the parity tests (one CTA).
template <int kBlock>
__global__ void __launch_bounds__(kBlock, 1) rows_kernel(PlainArgs a, int32_t bcc, int32_t src, int32_t chain,
                                                         int32_t *d_out, double *s_out) {
  __shared__ Shared<kBlock> sh;
  const Rows r = rows_of(a, a.rows_slot);  // a slot no plain_kernel CTA uses
  const int64_t vo = a.vtx_off[bcc];
  const int32_t nb = (int32_t)(a.vtx_off[bcc + 1] - vo);
  if ((int64_t)nb + 2 > a.ws_n) { set_err(a.err, kDevWorkspace); return; }
  const int64_t *R = a.row + vo;
  for (int k = threadIdx.x; k < nb; k += kBlock) { r.A()[k].d = 0; r.B()[k].d = 0; }
  __syncthreads();
  if (chain < 0) {
    cta_bfs(sh, R, a.col, src, r.A(), r.SA(), r.lvA(), r.lxA(), 1, a.rescale_exp, a.err);
    for (int k = threadIdx.x; k < nb; k += kBlock) {
      const int l = r.A()[k].d - 1;
      d_out[k] = l;
      s_out[k] = l >= 0 ? scale2(r.A()[k].v, r.lxA()[l]) : 0.0;
    }
  } else {
    const int32_t start = a.chain_start[chain], len = a.chain_len[chain], pos = src - start;
    const int nlevA = cta_bfs(sh, R, a.col, a.chain_l[chain], r.A(), r.SA(), r.lvA(), r.lxA(), 1, a.rescale_exp, a.err);
    const int nlevB = cta_bfs(sh, R, a.col, a.chain_r[chain], r.B(), r.SB(), r.lvB(), r.lxB(), 1, a.rescale_exp, a.err);
    const MergedExp xm{r.lxA(), r.lxB(), nlevA, nlevB, pos + 1, len - pos};
    merge_rows(sh, r, 1, 1, nb, start, len, pos, xm, a.err);
    for (int k = threadIdx.x; k < nb; k += kBlock) {
      const Rec m = r.M()[k];
      d_out[k] = m.d;
      s_out[k] = scale2(m.v, xm(m.d));
    }
  }
}

// Counters -> FP64, one vertex per thread: carries propagated exactly (each
// counter is below 2^64 - 2^(64-kAccDigitBits), so counter + carry fits), then
// the digits summed from the most significant down; the order of the FP64
// operations is fixed, so equal counters give equal values.
__global__ void __launch_bounds__(256) fold_kernel(unsigned long long *acc, double *bc, int64_t v0, int64_t v1) {
  static_assert(kAccDigits == 4, "fold_kernel reads four counters per vertex");
  constexpr unsigned long long kMask = (1ull << kAccDigitBits) - 1;
  for (int64_t v = v0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < v1; v += (int64_t)gridDim.x * blockDim.x) {
    ulonglong2 *p = reinterpret_cast<ulonglong2 *>(acc + kAccDigits * v);
    const ulonglong2 lo = p[0], hi = p[1];
    if ((lo.x | lo.y | hi.x | hi.y) == 0) continue;
    const unsigned long long c[4] = {lo.x, lo.y, hi.x, hi.y};
    unsigned long long dg[5], carry = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const unsigned long long t = c[i] + carry;
      dg[i] = t & kMask;
      carry = t >> kAccDigitBits;
    }
    dg[4] = carry;
    double r = 0.0;
#pragma unroll
    for (int i = 4; i >= 0; --i) r += (double)dg[i] * pow2(i * kAccDigitBits - kAccFrac);
    bc[v] += r;
    p[0] = make_ulonglong2(0, 0);
    p[1] = make_ulonglong2(0, 0);
  }
}

}  // namespace

cudaError_t launch_fold(unsigned long long *acc, double *bc, int64_t v0, int64_t v1, cudaStream_t stream) {
  if (v1 <= v0) return cudaSuccess;
  const int64_t blocks = std::min<int64_t>((v1 - v0 + 255) / 256, 148 * 8);
  fold_kernel<<<(int)blocks, 256, 0, stream>>>(acc, bc, v0, v1);
  return cudaGetLastError();
}

cudaError_t launch_plain(const PlainArgs &a, int block, int grid, cudaStream_t stream) {
  switch (block) {
    case 64: plain_kernel<64><<<grid, 64, 0, stream>>>(a); break;
    case 128: plain_kernel<128><<<grid, 128, 0, stream>>>(a); break;
    case 256: plain_kernel<256><<<grid, 256, 0, stream>>>(a); break;
    case 512: plain_kernel<512><<<grid, 512, 0, stream>>>(a); break;
    case 1024: plain_kernel<1024><<<grid, 1024, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_rows(const PlainArgs &a, int32_t bcc, int32_t src, int32_t chain, int32_t *d_out, double *s_out,
                        cudaStream_t stream) {
  rows_kernel<1024><<<1, 1024, 0, stream>>>(a, bcc, src, chain, d_out, s_out);
  return cudaGetLastError();
}

}  // namespace bcg
