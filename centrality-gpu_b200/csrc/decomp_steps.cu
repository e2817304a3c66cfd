// The decomposition as data-parallel steps, for the GPU (bc_decompose_gpu):
// the BCC split (Tarjan and Vishkin's method over a BFS forest, the same
// mathematics as the host split in host_decomp.cpp), the arc-to-member pass
// and the packing (exact-order BFS of every BCC at once, chains, packed CSR),
// written as one functor per step over vertices, frontier positions, member
// slots or BCCs. A backend runs the steps: DevBackend as a grid-stride kernel
// per step on one GPU, HostBackend as OpenMP loops over the very same
// functors -- a check of the GPU steps on a machine without one. Prefix sums
// run on the device in DevBackend (three scan kernels) and as a host loop in
// HostBackend; the stable regrouping of the BFS order by BCC and the sort of
// packed rows longer than 4096 arcs run on the host (DevBackend sorts rows of
// 33 to 4096 arcs on the GPU, HostBackend leaves every row beyond 32 arcs to
// that host sort). Steps over whole rows run per arc where the arcs are
// independent, else with a warp per long row.
//
// Steps (vertex ids int32, counts int64):
//   components   union-find over the edges, roots the smallest vertices
//                (link the larger root under the smaller with compare-and-swap);
//   forest       BFS from all roots at once, one launch per level: a vertex's
//                parent is whichever frontier vertex claims it first;
//   sweeps       per level, deepest first: subtree sizes; top down: preorder
//                intervals (a child takes the next range of its parent's);
//                then low/high over subtrees and non-tree neighbours;
//   tree edges   union-find over the tree edges (named by their child vertex)
//                joining an unrelated non-tree edge's two tree edges, and a
//                child's with its parent's when the child's subtree escapes
//                the parent's -- the sets are the BCCs, named by their
//                smallest member, numbered in that order;
//   heads        head(b) = parent of b's topmost tree edges, below(b) = the
//                vertices under them, hang(x) = sum of below over the BCCs x
//                heads; articulation terms S^2 - sum of squared parts;
//   members      per-BCC member lists (head last) and, per member slot, the
//                member's arcs inside the BCC as local ids in arc order;
//   packing      as host_decomp.cpp's decomp_pack writes it: BCCs of >= 3
//                vertices largest first, each in BFS order from its max-degree
//                vertex (plain vertices first, then chains numbered from the
//                end met first), adjacency in the new local ids.
// The split and reach follow Codes/bicc.cpp:81-161 and
// Codes/modified_apsp.cpp:77-220 in what they compute (not how).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "decomp.h"
#include "internal.h"

namespace bcg {
namespace decomp_steps {

// ---- atomics and loads that compile for both sides (relaxed on the host:
// each step ends at a barrier -- a kernel boundary or the end of an OpenMP loop)
__host__ __device__ inline int32_t ld32(const int32_t *p) {
#ifdef __CUDA_ARCH__
  return __ldcg(p);
#else
  return __atomic_load_n(p, __ATOMIC_RELAXED);
#endif
}
__host__ __device__ inline void st32(int32_t *p, int32_t v) {
#ifdef __CUDA_ARCH__
  *(volatile int32_t *)p = v;
#else
  __atomic_store_n(p, v, __ATOMIC_RELAXED);
#endif
}
// Compare-and-swap; returns the value found.
__host__ __device__ inline int32_t cas32(int32_t *p, int32_t expect, int32_t v) {
#ifdef __CUDA_ARCH__
  return atomicCAS((int *)p, expect, v);
#else
  __atomic_compare_exchange_n(p, &expect, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
  return expect;
#endif
}
__host__ __device__ inline int64_t add64(int64_t *p, int64_t v) {
#ifdef __CUDA_ARCH__
  return (int64_t)atomicAdd((unsigned long long *)p, (unsigned long long)v);
#else
  return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
#endif
}
__host__ __device__ inline void add32(int32_t *p, int32_t v) {
#ifdef __CUDA_ARCH__
  atomicAdd((int *)p, v);
#else
  __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
#endif
}
__host__ __device__ inline void min32(int32_t *p, int32_t v) {
#ifdef __CUDA_ARCH__
  atomicMin((int *)p, v);
#else
  int32_t c = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v < c && !__atomic_compare_exchange_n(p, &c, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
#endif
}
__host__ __device__ inline void max32(int32_t *p, int32_t v) {
#ifdef __CUDA_ARCH__
  atomicMax((int *)p, v);
#else
  int32_t c = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v > c && !__atomic_compare_exchange_n(p, &c, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
#endif
}

// Union-find whose set roots are the sets' smallest members: p[x] <= x at
// all times, so finds (path halving) and links need only compare-and-swap
// and every loop ends.
__host__ __device__ inline int32_t uf_find(int32_t *p, int32_t x) {
  for (;;) {
    const int32_t y = ld32(&p[x]);
    if (y == x) return x;
    const int32_t z = ld32(&p[y]);
    if (z != y) cas32(&p[x], y, z);
    x = z;
  }
}
__host__ __device__ inline void uf_union(int32_t *p, int32_t a, int32_t b) {
  for (;;) {
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a == b) return;
    if (a > b) {
      const int32_t t = a;
      a = b;
      b = t;
    }
    if (cas32(&p[b], b, a) == b) return;
  }
}

// ---- warp helpers of the warp-per-row forms of the steps (device only)
__device__ __forceinline__ unsigned lanes_below() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ int64_t warp_sum64(int64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Inclusive prefix sum over the warp's lanes.
__device__ __forceinline__ int64_t warp_incl64(int64_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}
// Ascending bitonic sort of one value per lane across the warp.
__device__ __forceinline__ int32_t warp_sort32(int32_t v, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int32_t o = __shfl_xor_sync(0xffffffffu, v, j);
      v = (((lane & j) == 0) == ((lane & k) == 0)) ? min(v, o) : max(v, o);
    }
  return v;
}

// ---- the steps; operator()(i) handles item i. Steps over a vertex's whole
// row come in two forms: per arc (operator()(e) over every arc, its vertex
// from src[e]) where the row's arcs are independent, else per item with a
// warp form (len(i), warp(i, lane)) that the GPU runs for rows longer than
// kLightArcs, keeping the row's arc order wherever the output depends on it.
// Packed rows of at most kSmallRow arcs are sorted as they are written
// (ColFill); longer ones by the backend (sort_rows) and the host.
constexpr int32_t kSmallRow = 32;

struct ArcSrc {  // src[e] = the vertex whose row holds arc e
  const int64_t *R;
  int32_t *src;
  __host__ __device__ void operator()(int64_t i) const {
    for (int64_t e = R[i]; e < R[i + 1]; ++e) src[e] = (int32_t)i;
  }
  __device__ int64_t len(int64_t i) const { return R[i + 1] - R[i]; }
  __device__ void warp(int64_t i, int lane) const {
    for (int64_t e = R[i] + lane; e < R[i + 1]; e += 32) src[e] = (int32_t)i;
  }
};
struct Iota {
  int32_t *p;
  __host__ __device__ void operator()(int64_t i) const { p[i] = (int32_t)i; }
};
struct Fill32 {
  int32_t *p;
  int32_t v;
  __host__ __device__ void operator()(int64_t i) const { p[i] = v; }
};
struct Fill64 {
  int64_t *p;
  int64_t v;
  __host__ __device__ void operator()(int64_t i) const { p[i] = v; }
};
struct Copy64 {
  int64_t *dst;
  const int64_t *src;
  __host__ __device__ void operator()(int64_t i) const { dst[i] = src[i]; }
};
struct Hook {  // components: one union per edge, from its larger end (per arc)
  const int32_t *C, *src;
  int32_t *uf;
  __host__ __device__ void operator()(int64_t e) const {
    const int32_t x = src[e], y = C[e];
    if (y < x) uf_union(uf, x, y);
  }
};
struct Compress {
  int32_t *uf;
  __host__ __device__ void operator()(int64_t i) const { st32(&uf[i], uf_find(uf, (int32_t)i)); }
};
struct RootFlag {  // 1 for a component's smallest vertex
  const int32_t *uf;
  int64_t *flag;
  __host__ __device__ void operator()(int64_t i) const { flag[i] = uf[i] == (int32_t)i; }
};
struct RootScatter {  // rank = exclusive prefix of RootFlag
  const int32_t *uf;
  const int64_t *rank;
  int32_t *roots, *comp, *order, *par;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t r = uf[i];
    comp[i] = (int32_t)rank[r];
    if (r == (int32_t)i) {
      roots[rank[i]] = (int32_t)i;
      order[rank[i]] = (int32_t)i;
      par[i] = -1;
    }
  }
};
struct BfsLevel {  // frontier position i: claim undiscovered neighbours
  const int64_t *R;
  const int32_t *C;
  int32_t *order, *par;
  int64_t *tail;
  int64_t f0;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = order[f0 + i];
    for (int64_t e = R[x]; e < R[x + 1]; ++e) {
      const int32_t y = C[e];
      if (ld32(&par[y]) == -2 && cas32(&par[y], -2, x) == -2) order[add64(tail, 1)] = y;
    }
  }
  __device__ int64_t len(int64_t i) const {
    const int32_t x = order[f0 + i];
    return R[x + 1] - R[x];
  }
  __device__ void warp(int64_t i, int lane) const {  // claims appended with one atomic per 32 arcs
    const int32_t x = order[f0 + i];
    const int64_t e1 = R[x + 1];
    for (int64_t b = R[x]; b < e1; b += 32) {
      const int64_t e = b + lane;
      int32_t y = 0;
      bool got = false;
      if (e < e1) {
        y = C[e];
        got = ld32(&par[y]) == -2 && cas32(&par[y], -2, x) == -2;
      }
      const unsigned m = __ballot_sync(0xffffffffu, got);
      if (!m) continue;
      const int lead = __ffs(m) - 1;
      int64_t at = 0;
      if (lane == lead) at = add64(tail, __popc(m));
      at = __shfl_sync(0xffffffffu, at, lead);
      if (got) order[at + __popc(m & lanes_below())] = y;
    }
  }
};
struct NdUp {  // level items: add the subtree size to the parent's
  const int32_t *order, *par;
  int64_t *nd;
  int64_t off;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = order[off + i];
    add64(&nd[par[x]], nd[x]);
  }
};
struct RootSizes {
  const int32_t *roots;
  const int64_t *nd;
  int64_t *size;
  __host__ __device__ void operator()(int64_t i) const { size[i] = nd[roots[i]]; }
};
struct RootPre {  // start = exclusive prefix of the component sizes
  const int32_t *roots;
  const int64_t *start;
  int32_t *pre;
  int64_t *cur;
  __host__ __device__ void operator()(int64_t i) const {
    pre[roots[i]] = (int32_t)start[i];
    cur[roots[i]] = start[i] + 1;
  }
};
struct PreDown {  // level items: take the next range of the parent's interval
  const int32_t *order, *par;
  const int64_t *nd;
  int32_t *pre;
  int64_t *cur;
  int64_t off;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = order[off + i];
    const int64_t q = add64(&cur[par[x]], nd[x]);
    pre[x] = (int32_t)q;
    cur[x] = q + 1;
  }
};
struct LoHiInit {  // pre range over x ...
  const int32_t *pre;
  int32_t *lo, *hi;
  __host__ __device__ void operator()(int64_t x) const { lo[x] = hi[x] = pre[x]; }
};
struct LoHiArc {  // ... and its neighbours other than its parent (per arc)
  const int32_t *C, *src, *par, *pre;
  int32_t *lo, *hi;
  __host__ __device__ void operator()(int64_t e) const {
    const int32_t x = src[e], y = C[e];
    if (y == par[x]) return;
    const int32_t q = pre[y];
    if (q < ld32(&lo[x])) min32(&lo[x], q);
    if (q > ld32(&hi[x])) max32(&hi[x], q);
  }
};
struct LoHiUp {
  const int32_t *order, *par;
  int32_t *lo, *hi;
  int64_t off;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = order[off + i];
    min32(&lo[par[x]], lo[x]);
    max32(&hi[par[x]], hi[x]);
  }
};
// Tree edges named by their child vertex: a child's with its parent's when
// the child's subtree escapes the parent's (per vertex) ...
struct TreeEdgeUnion {
  const int32_t *par, *pre, *lo, *hi;
  const int64_t *nd;
  int32_t *uf;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t w = (int32_t)i, v = par[w];
    if (v >= 0 && par[v] >= 0 && (lo[w] < pre[v] || (int64_t)hi[w] >= (int64_t)pre[v] + nd[v])) uf_union(uf, v, w);
  }
};
// ... and the two tree edges of an unrelated non-tree edge (per arc, from
// its larger end)
struct TreeArcUnion {
  const int32_t *C, *src, *par, *pre;
  const int64_t *nd;
  int32_t *uf;
  __host__ __device__ void operator()(int64_t e) const {
    const int32_t w = src[e], y = C[e];
    if (y <= w || y == par[w] || w == par[y]) return;
    const int32_t a = pre[w] < pre[y] ? w : y, b = a == w ? y : w;
    if ((int64_t)pre[b] >= (int64_t)pre[a] + nd[a]) uf_union(uf, w, y);
  }
};
struct NameFlag {  // 1 for a BCC's name: a tree edge that is its set's root
  const int32_t *par, *uf;
  int64_t *flag;
  __host__ __device__ void operator()(int64_t i) const { flag[i] = par[i] >= 0 && uf[i] == (int32_t)i; }
};
struct BccOf {  // id = exclusive prefix of NameFlag
  const int32_t *par, *uf;
  const int64_t *id;
  int32_t *tbcc;
  __host__ __device__ void operator()(int64_t i) const { tbcc[i] = par[i] >= 0 ? (int32_t)id[uf[i]] : -1; }
};
struct HeadBelow {
  const int32_t *par, *tbcc;
  const int64_t *nd;
  int32_t *head;
  int64_t *below;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t p = par[i], b = tbcc[i];
    if (p >= 0 && tbcc[p] != b) {  // a topmost tree edge of b (a root's tbcc is -1)
      st32(&head[b], p);
      add64(&below[b], nd[i]);
    }
  }
};
struct Hang {
  const int32_t *head;
  const int64_t *below;
  int64_t *hang, *sq;
  __host__ __device__ void operator()(int64_t b) const {
    add64(&hang[head[b]], below[b]);
    add64(&sq[head[b]], below[b] * below[b]);
  }
};
struct Art {
  const int32_t *comp;
  const int64_t *comp_size, *hang, *sq;
  double *art;
  int32_t *n_art;
  __host__ __device__ void operator()(int64_t x) const {
    const int64_t S = comp_size[comp[x]] - 1, up = S - hang[x];
    const int64_t a = S * S - sq[x] - up * up;
    art[x] = (double)a;
    if (a > 0) add32(n_art, 1);
  }
};
struct LocalId {  // a free position in the BCC's member list
  const int32_t *tbcc;
  int64_t *cnt;
  int32_t *locid;
  __host__ __device__ void operator()(int64_t i) const {
    if (tbcc[i] >= 0) locid[i] = (int32_t)add64(&cnt[tbcc[i]], 1);
  }
};
struct PlusOne {  // the head's place
  int64_t *cnt;
  __host__ __device__ void operator()(int64_t b) const { cnt[b] += 1; }
};
struct Members {
  const int32_t *tbcc, *locid;
  const int64_t *mem_off;
  int32_t *members;
  __host__ __device__ void operator()(int64_t i) const {
    if (tbcc[i] >= 0) members[mem_off[tbcc[i]] + locid[i]] = (int32_t)i;
  }
};
struct HeadLast {
  const int32_t *head;
  const int64_t *mem_off;
  int32_t *members;
  __host__ __device__ void operator()(int64_t b) const { members[mem_off[b + 1] - 1] = head[b]; }
};
// Arcs of x by BCC: the BCC of the tree edge into the endpoint with the larger
// pre. x's slot in BCC b receives x's arcs only, so one item (x) fills all its
// slots without atomics, in arc order.
struct SlotArcs {
  const int64_t *R;
  const int32_t *C, *src, *tbcc, *pre, *head, *locid;
  const int64_t *mem_off;
  int64_t *cnt;           // count pass (per arc): arcs per slot
  int64_t *cursor;        // fill pass (per vertex): next free position per slot
  int32_t *sadj;
  __host__ __device__ int32_t local_of(int32_t x, int32_t b) const {
    return x == head[b] ? (int32_t)(mem_off[b + 1] - mem_off[b] - 1) : locid[x];
  }
  __host__ __device__ int32_t bcc_of(int32_t x, int32_t y) const { return tbcc[pre[x] > pre[y] ? x : y]; }
  __host__ __device__ void operator()(int64_t i) const {
    if (!cursor) {  // count: i is an arc
      const int32_t x = src[i], b = bcc_of(x, C[i]);
      add64(&cnt[mem_off[b] + local_of(x, b)], 1);
      return;
    }
    const int32_t x = (int32_t)i;
    for (int64_t e = R[x]; e < R[x + 1]; ++e) {
      const int32_t y = C[e];
      const int32_t b = bcc_of(x, y);
      const int64_t s = mem_off[b] + local_of(x, b);
      sadj[cursor[s]++] = local_of(y, b);
    }
  }
  __device__ int64_t len(int64_t i) const { return R[i + 1] - R[i]; }
  // fill pass, 32 arcs at a time: the lanes of one slot write in arc order
  // from the slot's cursor, which the slot's lowest lane then advances
  __device__ void warp(int64_t i, int lane) const {
    const int32_t x = (int32_t)i;
    const int64_t e1 = R[x + 1];
    for (int64_t base = R[x]; base < e1; base += 32) {
      const int64_t e = base + lane;
      const bool on = e < e1;
      const unsigned act = __ballot_sync(0xffffffffu, on);
      if (on) {
        const int32_t y = C[e], b = bcc_of(x, y);
        const int64_t s = mem_off[b] + local_of(x, b);
        const unsigned peers = __match_any_sync(act, s);
        const int lead = __ffs(peers) - 1;
        int64_t at = lane == lead ? cursor[s] : 0;
        at = __shfl_sync(peers, at, lead);
        sadj[at + __popc(peers & lanes_below())] = local_of(y, b);
        if (lane == lead) cursor[s] = at + __popc(peers);
      }
      __syncwarp();
    }
  }
};

template <class F>
__global__ void each_kernel(int64_t n, F f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) f(i);
}

// Items with a row each, 32 per warp at a time: a lane runs its item's row
// alone when it has at most kLightArcs arcs; longer rows then run one at a
// time on the whole warp (f.warp), so a hub's row is spread over 32 lanes
// instead of holding one thread while the rest of the grid idles.
constexpr int64_t kLightArcs = 16;
template <class F>
__global__ void rows_kernel(int64_t n, F f) {
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = w * 32; base < n; base += nw * 32) {
    const int64_t i = base + lane;
    const bool heavy = i < n && f.len(i) > kLightArcs;
    if (i < n && !heavy) f(i);
    uint32_t todo = __ballot_sync(0xffffffffu, heavy);
    while (todo) {
      const int j = __ffs(todo) - 1;
      todo &= todo - 1;
      f.warp(base + j, lane);
    }
  }
}

// Exclusive prefix sum on the device, in place, in three kernels: each tile
// of kScanTile elements (kScanItems consecutive ones per thread) is summed;
// one CTA scans the tile sums (and writes the total after them); each tile
// then writes its elements' prefix sums from its tile's offset.
constexpr int kScanBlock = 512, kScanItems = 8, kScanTile = kScanBlock * kScanItems;

// Exclusive scan of v over the CTA (kScanBlock threads); *total gets the sum.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t *warp_sums, int64_t *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < kScanBlock / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < kScanBlock / 32) warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const int64_t before = (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
  *total = warp_sums[kScanBlock / 32 - 1];
  __syncthreads();  // warp_sums is reused by the caller's next scan
  return before;
}

__global__ void __launch_bounds__(kScanBlock) scan_tile_sums(const int64_t *a, int64_t n, int64_t *sums) {
  __shared__ int64_t ws[kScanBlock / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t t = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) t += base + j < n ? a[base + j] : 0;
  int64_t total;
  block_exclusive_scan(t, ws, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) scan_sums_kernel(int64_t *sums, int64_t m) {
  __shared__ int64_t ws[kScanBlock / 32];
  int64_t carry = 0;
  for (int64_t c0 = 0; c0 < m; c0 += kScanBlock) {
    const int64_t i = c0 + threadIdx.x;
    const int64_t v = i < m ? sums[i] : 0;
    int64_t total;
    const int64_t before = block_exclusive_scan(v, ws, &total);
    if (i < m) sums[i] = carry + before;
    carry += total;
  }
  if (threadIdx.x == 0) sums[m] = carry;
}

__global__ void __launch_bounds__(kScanBlock) scan_apply(int64_t *a, int64_t n, const int64_t *sums) {
  __shared__ int64_t ws[kScanBlock / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems], t = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = base + j < n ? a[base + j] : 0;
    t += v[j];
  }
  int64_t total;
  int64_t run = sums[blockIdx.x] + block_exclusive_scan(t, ws, &total);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) a[base + j] = run;
    run += v[j];
  }
}

// Exclusive prefix sum of a[0, n) in place; returns the total.
int64_t scan_host(int64_t *a, int64_t n) {
  int64_t s = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t v = a[i];
    a[i] = s;
    s += v;
  }
  return s;
}

struct StepError {
  int code;
  std::string what;
};

// Host loops over the functors.
struct HostBackend {
  std::vector<void *> owned;
  ~HostBackend() {
    for (void *p : owned) std::free(p);
  }
  template <class T>
  T *alloc(size_t n) {
    void *p = std::malloc(std::max<size_t>(n, 1) * sizeof(T));
    if (!p) throw StepError{BCGPU_ENOMEM, "host allocation failed"};
    owned.push_back(p);
    return (T *)p;
  }
  template <class F>
  void each(int64_t n, const F &f) {
    if (n < kSerialItems) {  // a deep BFS's thin levels: no thread team per level
      for (int64_t i = 0; i < n; ++i) f(i);
      return;
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) f(i);
  }
  static constexpr int64_t kSerialItems = 2048;
  template <class F>
  void rows(int64_t n, const F &f) { each(n, f); }
  // Sorts packed rows on the backend; returns the longest row length it
  // covers (here none beyond the rows ColFill sorts itself).
  int64_t sort_rows(const int64_t *, int32_t *, int64_t) { return kSmallRow; }
  template <class T>
  void upload(T *dst, const T *src, size_t n) { std::memcpy(dst, src, n * sizeof(T)); }
  template <class T>
  void download(T *dst, const T *src, size_t n) { std::memcpy(dst, src, n * sizeof(T)); }
  int64_t scan(int64_t *a, int64_t n) { return scan_host(a, n); }
};

// One GPU: a grid-stride kernel per step on the backend's stream.
struct DevBackend {
  int device = 0, grid_cap = 1024;
  cudaStream_t stream = nullptr;
  std::vector<void *> owned;
  int64_t *scan_sums = nullptr;  // tile sums of scan(), grown on demand
  size_t scan_cap = 0;
  void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
      throw StepError{e == cudaErrorMemoryAllocation ? BCGPU_ENOMEM : BCGPU_ECUDA,
                      std::string(what) + ": " + cudaGetErrorString(e)};
  }
  explicit DevBackend(int dev) : device(dev) {
    check(cudaSetDevice(dev), "cudaSetDevice");
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    grid_cap = std::max(1, sms) * 8;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
  }
  ~DevBackend() {
    if (stream) cudaStreamSynchronize(stream);
    for (void *p : owned) cudaFree(p);
    if (scan_sums) cudaFree(scan_sums);
    for (int i = 0; i < 2; ++i) {
      if (stage[i]) cudaFreeHost(stage[i]);
      if (staged[i]) cudaEventDestroy(staged[i]);
    }
    if (stream) cudaStreamDestroy(stream);
  }
  template <class T>
  T *alloc(size_t n) {
    void *p = nullptr;
    check(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
    return (T *)p;
  }
  template <class F>
  void each(int64_t n, const F &f) {
    if (n <= 0) return;
    constexpr int kBlock = 256;
    const int64_t blocks = std::min<int64_t>((n + kBlock - 1) / kBlock, grid_cap);
    each_kernel<<<(unsigned)blocks, kBlock, 0, stream>>>(n, f);
    check(cudaGetLastError(), "step launch");
  }
  template <class F>
  void rows(int64_t n, const F &f) {
    if (n <= 0) return;
    constexpr int kBlock = 256;
    const int64_t blocks = std::min<int64_t>((n + kBlock - 1) / kBlock, grid_cap);
    rows_kernel<<<(unsigned)blocks, kBlock, 0, stream>>>(n, f);
    check(cudaGetLastError(), "step launch");
  }
  int64_t sort_rows(const int64_t *row, int32_t *col, int64_t npk);  // below the steps
  template <class T>
  void upload(T *dst, const T *src, size_t n) {
    if (n) check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
    check(cudaStreamSynchronize(stream), "upload");
  }
  template <class T>
  void download(T *dst, const T *src, size_t n) {
    const size_t bytes = n * sizeof(T);
    if (bytes >= kStageMin && stage_ok()) {
      download_staged(reinterpret_cast<unsigned char *>(dst), reinterpret_cast<const unsigned char *>(src), bytes);
      return;
    }
    if (n) check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream), "download");
    check(cudaStreamSynchronize(stream), "step");
  }
  // Large results come back through two pinned buffers: the copy of chunk
  // k+1 runs while chunk k is spread into the (pageable) destination by the
  // host threads.
  static constexpr size_t kStageMin = size_t(8) << 20, kStageChunk = size_t(16) << 20;
  unsigned char *stage[2] = {nullptr, nullptr};
  cudaEvent_t staged[2] = {nullptr, nullptr};
  bool stage_tried = false;
  bool stage_ok() {
    if (!stage_tried) {
      stage_tried = true;
      for (int i = 0; i < 2; ++i)
        if (cudaMallocHost(reinterpret_cast<void **>(&stage[i]), kStageChunk) != cudaSuccess ||
            cudaEventCreateWithFlags(&staged[i], cudaEventDisableTiming) != cudaSuccess) {
          cudaGetLastError();
          return false;
        }
    }
    return stage[1] && staged[1];
  }
  void download_staged(unsigned char *dst, const unsigned char *src, size_t bytes) {
    const size_t chunks = (bytes + kStageChunk - 1) / kStageChunk;
    auto issue = [&](size_t c) {
      const size_t off = c * kStageChunk, len = std::min(kStageChunk, bytes - off);
      check(cudaMemcpyAsync(stage[c & 1], src + off, len, cudaMemcpyDeviceToHost, stream), "download");
      check(cudaEventRecord(staged[c & 1], stream), "download");
    };
    issue(0);
    for (size_t c = 0; c < chunks; ++c) {
      if (c + 1 < chunks) issue(c + 1);  // the other buffer: its previous chunk was spread last iteration
      check(cudaEventSynchronize(staged[c & 1]), "download");
      const size_t off = c * kStageChunk, len = std::min(kStageChunk, bytes - off);
      const unsigned char *from = stage[c & 1];
      constexpr size_t kPiece = size_t(1) << 20;
#pragma omp parallel for schedule(static)
      for (int64_t q = 0; q < (int64_t)((len + kPiece - 1) / kPiece); ++q) {
        const size_t a = (size_t)q * kPiece;
        std::memcpy(dst + off + a, from + a, std::min(kPiece, len - a));
      }
    }
  }
  // Exclusive prefix sum of a[0, n) in place on the device; returns the total.
  int64_t scan(int64_t *a, int64_t n) {
    if (n <= 0) return 0;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if ((int64_t)scan_cap < tiles + 1) {
      if (scan_sums) cudaFree(scan_sums);
      scan_sums = nullptr;
      check(cudaMalloc(&scan_sums, sizeof(int64_t) * (size_t)(tiles + 1)), "cudaMalloc");
      scan_cap = (size_t)(tiles + 1);
    }
    scan_tile_sums<<<(unsigned)tiles, kScanBlock, 0, stream>>>(a, n, scan_sums);
    scan_sums_kernel<<<1, kScanBlock, 0, stream>>>(scan_sums, tiles);
    scan_apply<<<(unsigned)tiles, kScanBlock, 0, stream>>>(a, n, scan_sums);
    check(cudaGetLastError(), "scan launch");
    int64_t total = 0;
    download(&total, scan_sums + tiles, 1);
    return total;
  }
};

// Profiling builds (-DBCGPU_HOST_TIMERS): the wall time of each step group,
// the device's queue drained first.
template <class BE>
void step_mark(BE &be, const char *name) {
#ifdef BCGPU_HOST_TIMERS
  if constexpr (std::is_same<BE, DevBackend>::value) cudaStreamSynchronize(be.stream);
  HOST_MARK(name);
#else
  (void)be;
  (void)name;
#endif
}

// The split's results, resident where the backend runs (owned by it).
struct DevSplit {
  int32_t n = 0;
  int64_t arcs = 0, nroots = 0, nbcc = 0, n_slots = 0;
  int32_t *comp, *head, *members, *sadj, *n_art;
  int64_t *csize, *below, *hang, *mem_off, *sdeg;
  double *art;
};

template <class BE>
DevSplit run_split(BE &be, const bc_graph *g) {
  step_mark(be, "d: start");
  const int32_t n = g->n;
  const int64_t arcs = g->row.empty() ? 0 : g->row[n];
  int64_t *R = be.template alloc<int64_t>((size_t)n + 1);
  int32_t *C = be.template alloc<int32_t>((size_t)arcs);
  be.upload(R, g->row.data(), (size_t)n + 1);
  be.upload(C, g->col.data(), (size_t)arcs);
  int32_t *uf = be.template alloc<int32_t>(n), *comp = be.template alloc<int32_t>(n);
  int32_t *par = be.template alloc<int32_t>(n), *order = be.template alloc<int32_t>(n);
  int32_t *roots = be.template alloc<int32_t>(n), *pre = be.template alloc<int32_t>(n);
  int32_t *lo = be.template alloc<int32_t>(n), *hi = be.template alloc<int32_t>(n);
  int32_t *tbcc = be.template alloc<int32_t>(n), *locid = be.template alloc<int32_t>(n);
  int64_t *flag = be.template alloc<int64_t>(n), *nd = be.template alloc<int64_t>(n);
  int64_t *cur = be.template alloc<int64_t>(n), *hang = be.template alloc<int64_t>(n);
  int64_t *sq = be.template alloc<int64_t>(n), *tail = be.template alloc<int64_t>(1);
  int32_t *n_art = be.template alloc<int32_t>(1);
  double *art = be.template alloc<double>(n);
  int32_t *src = be.template alloc<int32_t>((size_t)arcs);
  be.rows(n, ArcSrc{R, src});

  step_mark(be, "d: upload+alloc");
  // components
  be.each(n, Iota{uf});
  be.each(arcs, Hook{C, src, uf});
  be.each(n, Compress{uf});
  be.each(n, RootFlag{uf, flag});
  const int64_t nroots = be.scan(flag, n);
  be.each(n, Fill32{par, -2});
  be.each(n, RootScatter{uf, flag, roots, comp, order, par});

  step_mark(be, "d: components");
  // BFS forest, one launch per level; tail (the end of the listed vertices)
  // carries over from level to level, so each level costs one read-back
  std::vector<int64_t> lvl{0, nroots};
  be.upload(tail, &nroots, 1);
  for (int64_t f0 = 0, f1 = nroots; f1 > f0;) {
    be.rows(f1 - f0, BfsLevel{R, C, order, par, tail, f0});
    int64_t f2 = 0;
    be.download(&f2, tail, 1);
    if (f2 < f1 || f2 > n) throw StepError{BCGPU_EINVAL, "BFS forest: inconsistent frontier"};
    f0 = f1;
    f1 = f2;
    lvl.push_back(f1);
  }
  lvl.pop_back();
  if (lvl.back() != n) throw StepError{BCGPU_EINVAL, "BFS forest does not cover the graph"};
  const int64_t nlev = (int64_t)lvl.size() - 1;

  step_mark(be, "d: forest bfs");
  // subtree sizes, preorder, low/high
  be.each(n, Fill64{nd, 1});
  for (int64_t L = nlev - 1; L >= 1; --L) be.each(lvl[L + 1] - lvl[L], NdUp{order, par, nd, lvl[L]});
  int64_t *csize = be.template alloc<int64_t>((size_t)nroots), *cstart = be.template alloc<int64_t>((size_t)nroots);
  be.each(nroots, RootSizes{roots, nd, csize});
  be.each(nroots, Copy64{cstart, csize});
  be.scan(cstart, nroots);
  be.each(nroots, RootPre{roots, cstart, pre, cur});
  for (int64_t L = 1; L < nlev; ++L) be.each(lvl[L + 1] - lvl[L], PreDown{order, par, nd, pre, cur, lvl[L]});
  be.each(n, LoHiInit{pre, lo, hi});
  be.each(arcs, LoHiArc{C, src, par, pre, lo, hi});
  for (int64_t L = nlev - 1; L >= 1; --L) be.each(lvl[L + 1] - lvl[L], LoHiUp{order, par, lo, hi, lvl[L]});

  step_mark(be, "d: sweeps");
  // BCCs: union-find over tree edges
  be.each(n, Iota{uf});
  be.each(n, TreeEdgeUnion{par, pre, lo, hi, nd, uf});
  be.each(arcs, TreeArcUnion{C, src, par, pre, nd, uf});
  be.each(n, Compress{uf});
  be.each(n, NameFlag{par, uf, flag});
  const int64_t nbcc = be.scan(flag, n);
  be.each(n, BccOf{par, uf, flag, tbcc});

  step_mark(be, "d: bcc union");
  // heads, reach terms, articulation terms
  int32_t *head = be.template alloc<int32_t>((size_t)nbcc);
  int64_t *below = be.template alloc<int64_t>((size_t)nbcc), *mem_off = be.template alloc<int64_t>((size_t)nbcc + 1);
  be.each(nbcc, Fill64{below, 0});
  be.each(n, Fill64{hang, 0});
  be.each(n, Fill64{sq, 0});
  be.each(n, HeadBelow{par, tbcc, nd, head, below});
  be.each(nbcc, Hang{head, below, hang, sq});
  const int32_t zero = 0;
  be.upload(n_art, &zero, 1);
  be.each(n, Art{comp, csize, hang, sq, art, n_art});

  step_mark(be, "d: heads");
  // members (head last) and their arcs per BCC
  be.each(nbcc + 1, Fill64{mem_off, 0});
  be.each(n, LocalId{tbcc, mem_off, locid});
  be.each(nbcc, PlusOne{mem_off});
  const int64_t n_slots = be.scan(mem_off, nbcc + 1);
  int32_t *members = be.template alloc<int32_t>((size_t)n_slots);
  be.each(n, Members{tbcc, locid, mem_off, members});
  be.each(nbcc, HeadLast{head, mem_off, members});
  int64_t *sdeg = be.template alloc<int64_t>((size_t)n_slots + 1), *cursor = be.template alloc<int64_t>((size_t)n_slots);
  be.each(n_slots + 1, Fill64{sdeg, 0});
  be.each(arcs, SlotArcs{R, C, src, tbcc, pre, head, locid, mem_off, sdeg, nullptr, nullptr});
  const int64_t slot_arcs = be.scan(sdeg, n_slots + 1);
  if (slot_arcs != arcs) throw StepError{BCGPU_EINVAL, "member slots do not hold every arc once"};
  int32_t *sadj = be.template alloc<int32_t>((size_t)arcs);
  be.each(n_slots, Copy64{cursor, sdeg});
  be.rows(n, SlotArcs{R, C, src, tbcc, pre, head, locid, mem_off, nullptr, cursor, sadj});

  DevSplit d;
  d.n = n;
  d.arcs = arcs;
  d.nroots = nroots;
  d.nbcc = nbcc;
  d.n_slots = n_slots;
  d.comp = comp;
  d.head = head;
  d.members = members;
  d.sadj = sadj;
  d.n_art = n_art;
  d.csize = csize;
  d.below = below;
  d.hang = hang;
  d.mem_off = mem_off;
  d.sdeg = sdeg;
  d.art = art;
  return d;
}

// ---- packing on the device: the order, chains and packed CSR that
// decomp_pack (host_decomp.cpp) writes, as steps. Packed BCC i is BCC
// pk_bcc[i]; its local ids follow an exact-order BFS from its max-degree
// vertex (smallest id among equals), plain vertices first, then each chain.
__host__ __device__ inline void amax64u(uint64_t *p, uint64_t v) {
#ifdef __CUDA_ARCH__
  atomicMax((unsigned long long *)p, (unsigned long long)v);
#else
  uint64_t c = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v > c && !__atomic_compare_exchange_n(p, &c, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
#endif
}
// Largest k in [0, m) with a[k] <= v (a ascending, a[0] <= v).
__host__ __device__ inline int64_t floor_index(const int64_t *a, int64_t m, int64_t v) {
  int64_t lo = 0, hi = m - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) / 2;
    if (a[mid] <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Member slots of the packed BCCs, as the packing sees them.
struct Slots {
  const int64_t *mem_off, *sdeg;
  const int32_t *sadj, *slot_b, *pk_of, *members;
  __host__ __device__ int32_t deg(int32_t s) const { return (int32_t)(sdeg[s + 1] - sdeg[s]); }
  // slot of the k-th neighbour of slot s
  __host__ __device__ int32_t nbr(int32_t s, int32_t k) const {
    return (int32_t)(mem_off[slot_b[s]] + sadj[sdeg[s] + k]);
  }
  __host__ __device__ int32_t pk(int32_t s) const { return pk_of[slot_b[s]]; }
  // nbr(s, k) = first(s) + sadj[at(s) + k]
  __host__ __device__ int64_t first(int32_t s) const { return mem_off[slot_b[s]]; }
  __host__ __device__ int64_t at(int32_t s) const { return sdeg[s]; }
  // Far end of the chain that leaves slot x through its neighbour cur (at
  // most nb steps; *len > nb when there is no end).
  __host__ __device__ int32_t walk(int32_t x, int32_t cur, int64_t nb, int64_t *len) const {
    int32_t prev = x;
    int64_t k = 0;
    while (deg(cur) == 2 && k <= nb) {
      const int32_t a0 = nbr(cur, 0), a1 = nbr(cur, 1);
      const int32_t nx = a0 == prev ? a1 : a0;
      prev = cur;
      cur = nx;
      ++k;
    }
    *len = k;
    return cur;
  }
};

struct SlotBcc {
  const int64_t *mem_off;
  int64_t nbcc;
  int32_t *slot_b;
  __host__ __device__ void operator()(int64_t s) const { slot_b[s] = (int32_t)floor_index(mem_off, nbcc, s); }
};
struct RootKey {  // max over a packed BCC's members of (degree, -vertex id); cycle test
  Slots S;
  uint64_t *key;
  int32_t *cyc;
  __host__ __device__ void operator()(int64_t s) const {
    const int32_t i = S.pk((int32_t)s);
    if (i < 0) return;
    const int32_t d = S.deg((int32_t)s);
    if (d != 2) st32(&cyc[i], 0);
    amax64u(&key[i], ((uint64_t)(uint32_t)d << 32) | (uint64_t)(uint32_t)(INT32_MAX - S.members[s]));
  }
};
struct RootSlot {
  Slots S;
  const uint64_t *key;
  int32_t *bq, *seen;
  __host__ __device__ void operator()(int64_t s) const {
    const int32_t i = S.pk((int32_t)s);
    if (i < 0) return;
    if (INT32_MAX - (int32_t)(key[i] & 0xffffffffu) == S.members[s]) {
      bq[i] = (int32_t)s;
      seen[s] = 1;
    }
  }
};
// One level of the BFS of every packed BCC at once, in the sequential
// queue's order: a slot is claimed by the earliest frontier position next to
// it; counts per position, a prefix sum, then each position writes its own.
struct PClaim {
  Slots S;
  const int32_t *bq, *seen;
  int32_t *claim;
  int64_t f0;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t s = bq[f0 + i];
    for (int32_t k = 0; k < S.deg(s); ++k) {
      const int32_t t = S.nbr(s, k);
      if (!seen[t]) min32(&claim[t], (int32_t)i);
    }
  }
  __device__ int64_t len(int64_t i) const { return S.deg(bq[f0 + i]); }
  __device__ void warp(int64_t i, int lane) const {
    const int32_t s = bq[f0 + i], d = S.deg(s);
    const int64_t b = S.first(s), a = S.at(s);
    for (int32_t k = lane; k < d; k += 32) {
      const int32_t t = (int32_t)(b + S.sadj[a + k]);
      if (!seen[t]) min32(&claim[t], (int32_t)i);
    }
  }
};
struct PCount {
  Slots S;
  const int32_t *bq, *seen, *claim;
  int64_t *cnt;
  int64_t f0;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t s = bq[f0 + i];
    int64_t c = 0;
    for (int32_t k = 0; k < S.deg(s); ++k) {
      const int32_t t = S.nbr(s, k);
      c += !seen[t] && ld32(&claim[t]) == (int32_t)i;
    }
    cnt[i] = c;
  }
  __device__ int64_t len(int64_t i) const { return S.deg(bq[f0 + i]); }
  __device__ void warp(int64_t i, int lane) const {
    const int32_t s = bq[f0 + i], d = S.deg(s);
    const int64_t b = S.first(s), a = S.at(s);
    int64_t c = 0;
    for (int32_t k = lane; k < d; k += 32) {
      const int32_t t = (int32_t)(b + S.sadj[a + k]);
      c += !seen[t] && ld32(&claim[t]) == (int32_t)i;
    }
    c = warp_sum64(c);
    if (lane == 0) cnt[i] = c;
  }
};
struct PEmit {
  Slots S;
  const int32_t *seen, *claim;
  const int64_t *at0;  // exclusive prefix of PCount
  int32_t *bq;
  int64_t f0, f1;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t s = bq[f0 + i];
    int64_t at = f1 + at0[i];
    for (int32_t k = 0; k < S.deg(s); ++k) {
      const int32_t t = S.nbr(s, k);
      if (!seen[t] && ld32(&claim[t]) == (int32_t)i) bq[at++] = t;
    }
  }
  __device__ int64_t len(int64_t i) const { return S.deg(bq[f0 + i]); }
  __device__ void warp(int64_t i, int lane) const {  // emitted in arc order, 32 arcs at a time
    const int32_t s = bq[f0 + i], d = S.deg(s);
    const int64_t b = S.first(s), a = S.at(s);
    int64_t at = f1 + at0[i];
    for (int32_t k0 = 0; k0 < d; k0 += 32) {
      const int32_t k = k0 + lane;
      int32_t t = 0;
      bool emit = false;
      if (k < d) {
        t = (int32_t)(b + S.sadj[a + k]);
        emit = !seen[t] && ld32(&claim[t]) == (int32_t)i;
      }
      const unsigned m = __ballot_sync(0xffffffffu, emit);
      if (emit) bq[at + __popc(m & lanes_below())] = t;
      at += __popc(m);
    }
  }
};
struct PMark {
  const int32_t *bq;
  int32_t *seen;
  int64_t f1;
  __host__ __device__ void operator()(int64_t k) const { seen[bq[f1 + k]] = 1; }
};
struct PlainFlag {  // plain = not a chain vertex (every vertex of a cycle BCC is plain)
  Slots S;
  const int32_t *q, *cyc;
  int64_t *flag;
  __host__ __device__ void operator()(int64_t k) const {
    const int32_t s = q[k];
    flag[k] = cyc[S.pk(s)] || S.deg(s) != 2;
  }
};
struct PlainPlace {
  Slots S;
  const int32_t *q, *cyc;
  const int64_t *gidx, *plain_base, *vtx_off;
  int32_t *nid, *pl, *old;
  __host__ __device__ void operator()(int64_t k) const {
    const int32_t s = q[k], i = S.pk(s);
    if (!(cyc[i] || S.deg(s) != 2)) return;
    const int32_t f = (int32_t)(gidx[k] - plain_base[i]);
    nid[s] = f;
    pl[gidx[k]] = s;
    old[vtx_off[i] + f] = s;
  }
};
// Chains, numbered from whichever end comes first in the plain order, their
// vertices from that end: count per plain vertex, then (after prefix sums)
// write.
struct Chains {
  Slots S;
  const int32_t *pl, *cyc, *nid_plain;
  const int64_t *plain_base, *vtx_off;
  int32_t *bad;
  int64_t *cnt, *vcnt;                      // count pass
  const int64_t *cidx, *voff, *voff_base;   // write pass
  const int32_t *n_plain;
  int32_t *ch_start, *ch_len, *ch_l, *ch_r, *nid, *old;
  __host__ __device__ void operator()(int64_t g) const {
    const int32_t x = pl[g], i = S.pk(x);
    if (cnt) cnt[g] = vcnt[g] = 0;
    if (cyc[i]) return;
    const int64_t nb = vtx_off[i + 1] - vtx_off[i];
    const int32_t f = (int32_t)(g - plain_base[i]);
    int64_t c = cnt ? 0 : cidx[g];
    int64_t pos = cnt ? 0 : n_plain[i] + (voff[g] - voff_base[i]);
    int64_t nc = 0, nv = 0;
    for (int32_t k = 0; k < S.deg(x); ++k) {
      const int32_t t = S.nbr(x, k);
      if (S.deg(t) != 2) continue;
      int64_t len;
      const int32_t far = S.walk(x, t, nb, &len);
      if (len > nb || far == x) {
        st32(bad, 1);
        continue;
      }
      if (nid_plain[far] < f) continue;  // numbered from its other end
      if (cnt) {
        ++nc;
        nv += len;
        continue;
      }
      ch_start[c] = (int32_t)pos;
      ch_len[c] = (int32_t)len;
      ch_l[c] = f;
      ch_r[c] = nid_plain[far];
      ++c;
      int32_t prev = x, cur = t;
      for (int64_t j = 0; j < len; ++j) {
        nid[cur] = (int32_t)pos;
        old[vtx_off[i] + pos] = cur;
        ++pos;
        const int32_t a0 = S.nbr(cur, 0), a1 = S.nbr(cur, 1);
        const int32_t nx = a0 == prev ? a1 : a0;
        prev = cur;
        cur = nx;
      }
    }
    if (cnt) {
      cnt[g] = nc;
      vcnt[g] = nv;
    }
  }
  __device__ int64_t len(int64_t g) const { return S.deg(pl[g]); }
  // 32 arcs at a time: each lane walks its arc's chain; chain numbers and
  // vertex positions follow arc order (a warp prefix sum of the lengths)
  __device__ void warp(int64_t g, int lane) const {
    const int32_t x = pl[g], i = S.pk(x);
    if (cyc[i]) {
      if (cnt && lane == 0) cnt[g] = vcnt[g] = 0;
      return;
    }
    const int64_t nb = vtx_off[i + 1] - vtx_off[i];
    const int32_t f = (int32_t)(g - plain_base[i]), d = S.deg(x);
    int64_t c = cnt ? 0 : cidx[g];
    int64_t pos = cnt ? 0 : n_plain[i] + (voff[g] - voff_base[i]);
    for (int32_t k0 = 0; k0 < d; k0 += 32) {
      const int32_t k = k0 + lane;
      int32_t t = 0, far = 0;
      int64_t len = 0;
      bool take = false;
      if (k < d) {
        t = S.nbr(x, k);
        if (S.deg(t) == 2) {
          far = S.walk(x, t, nb, &len);
          if (len > nb || far == x) st32(bad, 1);
          else take = nid_plain[far] >= f;  // else numbered from its other end
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, take);
      const int64_t lv = take ? len : 0, incl = warp_incl64(lv, lane);
      const int64_t tot = __shfl_sync(0xffffffffu, incl, 31);
      if (!cnt && take) {
        const int64_t cc = c + __popc(m & lanes_below());
        int64_t p = pos + incl - lv;
        ch_start[cc] = (int32_t)p;
        ch_len[cc] = (int32_t)len;
        ch_l[cc] = f;
        ch_r[cc] = nid_plain[far];
        int32_t prev = x, cur = t;
        for (int64_t j = 0; j < len; ++j) {
          nid[cur] = (int32_t)p;
          old[vtx_off[i] + p] = cur;
          ++p;
          const int32_t a0 = S.nbr(cur, 0), a1 = S.nbr(cur, 1);
          const int32_t nx = a0 == prev ? a1 : a0;
          prev = cur;
          cur = nx;
        }
      }
      c += __popc(m);
      pos += tot;
    }
    if (cnt && lane == 0) {
      cnt[g] = c;
      vcnt[g] = pos;
    }
  }
};
struct Unset {  // positions no step wrote
  const int32_t *old;
  int32_t *bad;
  __host__ __device__ void operator()(int64_t k) const {
    if (old[k] < 0) st32(bad, 1);
  }
};
struct Inverse {
  const int32_t *old;
  const int64_t *vtx_off;
  int64_t np;
  int32_t *inv;
  __host__ __device__ void operator()(int64_t k) const {
    inv[old[k]] = (int32_t)(k - vtx_off[floor_index(vtx_off, np, k)]);
  }
};
struct RowLen {
  Slots S;
  const int32_t *old;
  int64_t *row;
  __host__ __device__ void operator()(int64_t k) const { row[k] = S.deg(old[k]); }
};
struct ColFill {
  Slots S;
  const int32_t *old, *inv, *head, *comp;
  const int64_t *row, *csize, *below, *hang;
  int32_t *col, *orig, *reach;
  __host__ __device__ void operator()(int64_t k) const {
    const int32_t s = old[k], b = S.slot_b[s], d = S.deg(s);
    int32_t *dst = col + row[k];
    for (int32_t j = 0; j < d; ++j) dst[j] = inv[S.nbr(s, j)];
    if (d <= kSmallRow)
      for (int32_t j = 1; j < d; ++j) {
        const int32_t v = dst[j];
        int32_t t = j;
        for (; t > 0 && dst[t - 1] > v; --t) dst[t] = dst[t - 1];
        dst[t] = v;
      }
    const int32_t x = S.members[s];
    orig[k] = x;
    reach[k] = x == head[b] ? (int32_t)(csize[comp[x]] - 1 - below[b]) : (int32_t)hang[x];
  }
  __device__ int64_t len(int64_t k) const { return S.deg(old[k]); }
  __device__ void warp(int64_t k, int lane) const {
    const int32_t s = old[k], b = S.slot_b[s], d = S.deg(s);
    const int64_t f = S.first(s), a = S.at(s);
    int32_t *dst = col + row[k];
    if (d <= kSmallRow) {  // one neighbour per lane, sorted across the warp
      const int32_t v = warp_sort32(lane < d ? inv[f + S.sadj[a + lane]] : INT32_MAX, lane);
      if (lane < d) dst[lane] = v;
    } else {
      for (int32_t j = lane; j < d; j += 32) dst[j] = inv[f + S.sadj[a + j]];
    }
    if (lane == 0) {
      const int32_t x = S.members[s];
      orig[k] = x;
      reach[k] = x == head[b] ? (int32_t)(csize[comp[x]] - 1 - below[b]) : (int32_t)hang[x];
    }
  }
};

// Rows of more than kSmallRow and at most kSortRow arcs, sorted on the GPU:
// listed (flag, prefix sum, compaction), then one CTA per row sorts it in
// shared memory (bitonic, padded to a power of two). Longer rows are sorted
// on the host.
constexpr int32_t kSortRow = 4096, kSortBlock = 512;
struct LongRowFlag {
  const int64_t *row;
  int64_t *flag;
  __host__ __device__ void operator()(int64_t k) const {
    const int64_t d = row[k + 1] - row[k];
    flag[k] = d > kSmallRow && d <= kSortRow;
  }
};
struct LongRowList {  // flag holds its exclusive prefix sums (npk + 1 entries)
  const int64_t *flag;
  int32_t *list;
  __host__ __device__ void operator()(int64_t k) const {
    if (flag[k + 1] != flag[k]) list[flag[k]] = (int32_t)k;
  }
};
__global__ void __launch_bounds__(kSortBlock) sort_rows_kernel(const int64_t *row, const int32_t *list, int64_t nlist,
                                                                int32_t *col) {
  __shared__ int32_t buf[kSortRow];
  for (int64_t li = blockIdx.x; li < nlist; li += gridDim.x) {
    const int32_t k = list[li];
    const int64_t e0 = row[k];
    const int d = (int)(row[k + 1] - e0);
    int P = 64;
    while (P < d) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) buf[i] = i < d ? col[e0 + i] : INT32_MAX;
    __syncthreads();
    for (int kk = 2; kk <= P; kk <<= 1)
      for (int j = kk >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
          const int o = i ^ j;
          if (o > i) {
            const int32_t x = buf[i], y = buf[o];
            if ((x > y) == ((i & kk) == 0)) {
              buf[i] = y;
              buf[o] = x;
            }
          }
        }
        __syncthreads();
      }
    for (int i = threadIdx.x; i < d; i += blockDim.x) col[e0 + i] = buf[i];
    __syncthreads();
  }
}

inline int64_t DevBackend::sort_rows(const int64_t *row, int32_t *col, int64_t npk) {
  int64_t *flag = alloc<int64_t>((size_t)npk + 1);
  each(npk, LongRowFlag{row, flag});
  each(1, Fill64{flag + npk, 0});
  const int64_t nlist = scan(flag, npk + 1);
  if (nlist > 0) {
    int32_t *list = alloc<int32_t>((size_t)nlist);
    each(npk, LongRowList{flag, list});
    const int64_t blocks = std::min<int64_t>(nlist, (int64_t)grid_cap * 2);
    sort_rows_kernel<<<(unsigned)blocks, kSortBlock, 0, stream>>>(row, list, nlist, col);
    check(cudaGetLastError(), "sort launch");
  }
  return kSortRow;
}

template <class BE>
void pack_steps(BE &be, const DevSplit &d, bc_decomp *D, std::chrono::steady_clock::time_point t0) {
  // packed BCCs: >= 3 members, largest first, equal sizes by BCC id
  std::vector<int64_t> mem_off((size_t)d.nbcc + 1);
  be.download(mem_off.data(), d.mem_off, mem_off.size());
  std::vector<int32_t> pk_bcc, pk_of((size_t)d.nbcc, -1);
  for (int32_t b = 0; b < (int32_t)d.nbcc; ++b)
    if (mem_off[b + 1] - mem_off[b] >= 3) pk_bcc.push_back(b);
  std::stable_sort(pk_bcc.begin(), pk_bcc.end(), [&](int32_t a, int32_t b) {
    return (mem_off[a + 1] - mem_off[a]) > (mem_off[b + 1] - mem_off[b]);
  });
  const int64_t np = (int64_t)pk_bcc.size();
  D->vtx_off.assign((size_t)np + 1, 0);
  for (int64_t i = 0; i < np; ++i) {
    pk_of[pk_bcc[i]] = (int32_t)i;
    D->vtx_off[i + 1] = D->vtx_off[i] + (mem_off[pk_bcc[i] + 1] - mem_off[pk_bcc[i]]);
  }
  const int64_t npk = D->vtx_off[np], ns = d.n_slots;
  int32_t *slot_b = be.template alloc<int32_t>((size_t)ns), *pkof = be.template alloc<int32_t>((size_t)d.nbcc);
  int64_t *vtx_off = be.template alloc<int64_t>((size_t)np + 1);
  be.upload(pkof, pk_of.data(), pk_of.size());
  be.upload(vtx_off, D->vtx_off.data(), D->vtx_off.size());
  be.each(ns, SlotBcc{d.mem_off, d.nbcc, slot_b});
  const Slots S{d.mem_off, d.sdeg, d.sadj, slot_b, pkof, d.members};

  step_mark(be, "d: members+order");
  // roots and the BFS of every packed BCC at once
  uint64_t *key = be.template alloc<uint64_t>((size_t)np);
  int32_t *cyc = be.template alloc<int32_t>((size_t)np), *seen = be.template alloc<int32_t>((size_t)ns);
  int32_t *claim = be.template alloc<int32_t>((size_t)ns), *bq = be.template alloc<int32_t>((size_t)npk);
  int64_t *cnt = be.template alloc<int64_t>((size_t)npk + 1);
  be.each(np, Fill64{(int64_t *)key, 0});
  be.each(np, Fill32{cyc, 1});
  be.each(ns, Fill32{seen, 0});
  be.each(ns, Fill32{claim, INT32_MAX});
  be.each(ns, RootKey{S, key, cyc});
  be.each(ns, RootSlot{S, key, bq, seen});
  int64_t f0 = 0, f1 = np;
  while (f1 > f0) {
    const int64_t fn = f1 - f0;
    be.rows(fn, PClaim{S, bq, seen, claim, f0});
    be.rows(fn, PCount{S, bq, seen, claim, cnt, f0});
    const int64_t add = be.scan(cnt, fn);  // PEmit reads the starts of positions 0..fn-1 only
    if (f1 + add > npk) throw StepError{BCGPU_EINVAL, "packing BFS: inconsistent frontier"};
    be.rows(fn, PEmit{S, seen, claim, cnt, bq, f0, f1});
    be.each(add, PMark{bq, seen, f1});
    f0 = f1;
    f1 += add;
  }
  if (f1 != npk) throw StepError{BCGPU_EINVAL, "a BCC is not connected"};

  step_mark(be, "d: packing bfs");
  // each BCC's queue: its subsequence of the level-major order
  std::vector<int32_t> h_bq((size_t)npk), h_slot_b((size_t)ns), h_q((size_t)npk);
  be.download(h_bq.data(), bq, (size_t)npk);
  be.download(h_slot_b.data(), slot_b, (size_t)ns);
  {
    std::vector<int64_t> at(D->vtx_off.begin(), D->vtx_off.end() - 1);
    for (int64_t k = 0; k < npk; ++k) h_q[at[pk_of[h_slot_b[h_bq[k]]]]++] = h_bq[k];
  }
  int32_t *q = bq;
  be.upload(q, h_q.data(), (size_t)npk);

  step_mark(be, "d: regroup");
  // plain vertices
  int64_t *gidx = cnt;
  be.each(npk, PlainFlag{S, q, cyc, gidx});
  be.each(1, Fill64{gidx + npk, 0});
  const int64_t nplain_all = be.scan(gidx, npk + 1);
  std::vector<int64_t> h_gidx((size_t)npk + 1), plain_base((size_t)np);
  be.download(h_gidx.data(), gidx, (size_t)npk + 1);
  D->n_plain.assign((size_t)np, 0);
  for (int64_t i = 0; i < np; ++i) {
    plain_base[i] = h_gidx[D->vtx_off[i]];
    D->n_plain[i] = (int32_t)(h_gidx[D->vtx_off[i + 1]] - plain_base[i]);
  }
  int64_t *pbase = be.template alloc<int64_t>((size_t)np);
  be.upload(pbase, plain_base.data(), (size_t)np);
  int32_t *nid = claim, *pl = be.template alloc<int32_t>((size_t)nplain_all), *old = seen;
  be.each(ns, Fill32{nid, -1});
  be.each(npk, Fill32{old, -1});
  be.each(npk, PlainPlace{S, q, cyc, gidx, pbase, vtx_off, nid, pl, old});

  step_mark(be, "d: plain");
  // chains: count, prefix sums, write
  int64_t *ccnt = be.template alloc<int64_t>((size_t)nplain_all + 1), *vcnt = be.template alloc<int64_t>((size_t)nplain_all + 1);
  int32_t *bad = be.template alloc<int32_t>(1);
  be.each(1, Fill32{bad, 0});
  be.rows(nplain_all, Chains{S, pl, cyc, nid, pbase, vtx_off, bad, ccnt, vcnt, nullptr, nullptr, nullptr, nullptr,
                             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr});
  int32_t h_bad = 0;
  be.download(&h_bad, bad, 1);
  if (h_bad) throw StepError{BCGPU_EINVAL, "a chain has no end or returns to its start"};
  be.each(1, Fill64{ccnt + nplain_all, 0});
  be.each(1, Fill64{vcnt + nplain_all, 0});
  const int64_t nchains = be.scan(ccnt, nplain_all + 1);
  be.scan(vcnt, nplain_all + 1);
  std::vector<int64_t> h_c((size_t)nplain_all + 1), h_v((size_t)nplain_all + 1), voff_base((size_t)np);
  be.download(h_c.data(), ccnt, h_c.size());
  be.download(h_v.data(), vcnt, h_v.size());
  D->chain_off.assign((size_t)np + 1, 0);
  for (int64_t i = 0; i < np; ++i) {
    D->chain_off[i] = h_c[plain_base[i]];
    voff_base[i] = h_v[plain_base[i]];
  }
  D->chain_off[np] = nchains;
  int64_t *vbase = be.template alloc<int64_t>((size_t)np);
  int32_t *nplain = be.template alloc<int32_t>((size_t)np);
  be.upload(vbase, voff_base.data(), (size_t)np);
  be.upload(nplain, D->n_plain.data(), (size_t)np);
  int32_t *ch = be.template alloc<int32_t>((size_t)nchains * 4);
  be.rows(nplain_all, Chains{S, pl, cyc, nid, pbase, vtx_off, bad, nullptr, nullptr, ccnt, vcnt, vbase, nplain, ch,
                             ch + nchains, ch + 2 * nchains, ch + 3 * nchains, nid, old});
  be.each(npk, Unset{old, bad});
  be.download(&h_bad, bad, 1);
  if (h_bad) throw StepError{BCGPU_EINVAL, "packing left a vertex without a place"};

  step_mark(be, "d: chains");
  // packed CSR in the new local ids, orig, reach
  int32_t *inv = claim;  // nid is no longer needed
  be.each(npk, Inverse{old, vtx_off, np, inv});
  int64_t *row = be.template alloc<int64_t>((size_t)npk + 1);
  be.each(npk, RowLen{S, old, row});
  be.each(1, Fill64{row + npk, 0});
  const int64_t parcs = be.scan(row, npk + 1);
  if (parcs > (int64_t)INT32_MAX * 8) throw StepError{BCGPU_EOVERFLOW, "packed arcs overflow"};
  int32_t *col = be.template alloc<int32_t>((size_t)parcs), *orig = be.template alloc<int32_t>((size_t)npk);
  int32_t *reach = be.template alloc<int32_t>((size_t)npk);
  be.rows(npk, ColFill{S, old, inv, d.head, d.comp, row, d.csize, d.below, d.hang, col, orig, reach});

  const int64_t sorted_max = be.sort_rows(row, col, npk);
  step_mark(be, "d: packed csr");
  // to the host; rows longer than kSmallRow are sorted here
  D->row.resize((size_t)npk + 1);
  D->col.resize((size_t)parcs);
  D->orig.resize((size_t)npk);
  D->reach.resize((size_t)npk);
  D->chain_start.resize((size_t)nchains);
  D->chain_len.resize((size_t)nchains);
  D->chain_l.resize((size_t)nchains);
  D->chain_r.resize((size_t)nchains);
  D->art.resize((size_t)d.n);
  be.download(D->row.data(), row, (size_t)npk + 1);
  be.download(D->col.data(), col, (size_t)parcs);
  be.download(D->orig.data(), orig, (size_t)npk);
  be.download(D->reach.data(), reach, (size_t)npk);
  be.download(D->chain_start.data(), ch, (size_t)nchains);
  be.download(D->chain_len.data(), ch + nchains, (size_t)nchains);
  be.download(D->chain_l.data(), ch + 2 * nchains, (size_t)nchains);
  be.download(D->chain_r.data(), ch + 3 * nchains, (size_t)nchains);
  be.download(D->art.data(), d.art, (size_t)d.n);
  step_mark(be, "d: downloads");
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t k = 0; k < npk; ++k)
    if (D->row[k + 1] - D->row[k] > sorted_max) std::sort(D->col.begin() + D->row[k], D->col.begin() + D->row[k + 1]);
  step_mark(be, "d: sort");
  std::vector<int32_t> h_cyc((size_t)np);
  be.download(h_cyc.data(), cyc, (size_t)np);
  int64_t cycles = 0;
  for (int32_t c : h_cyc) cycles += c;
  int32_t n_art = 0;
  be.download(&n_art, d.n_art, 1);
  decomp_finish(D, d.n, (int32_t)d.nroots, (int32_t)d.nbcc, n_art, cycles, t0);
  step_mark(be, "d: finish");
}

}  // namespace decomp_steps

int decomp_gpu(const bc_graph *g, int device, bc_decomp *D, std::chrono::steady_clock::time_point t0, char *err,
               size_t errlen) {
  auto fail = [&](int code, const std::string &what) {
    if (err && errlen) std::snprintf(err, errlen, "%s", what.c_str());
    return code;
  };
  try {
    if (device < 0) {
      decomp_steps::HostBackend be;
      decomp_steps::pack_steps(be, decomp_steps::run_split(be, g), D, t0);
    } else {
      {
        decomp_steps::DevBackend be(device);
        decomp_steps::pack_steps(be, decomp_steps::run_split(be, g), D, t0);
      }
      HOST_MARK("d: release");
    }
  } catch (const decomp_steps::StepError &e) {
    return fail(e.code, e.what);
  } catch (const std::bad_alloc &) {
    return fail(BCGPU_ENOMEM, "host allocation failed");
  } catch (const std::exception &e) {  // nothing else may cross the C ABI
    return fail(BCGPU_EINVAL, std::string("decomposition steps: ") + e.what());
  }
  return BCGPU_OK;
}

}  // namespace bcg

extern "C" int bc_decompose_gpu(const bc_graph *g, int device, bc_decomp **out, char *err, size_t errlen) {
  if (!g || !out) return BCGPU_EINVAL;
  const auto t0 = std::chrono::steady_clock::now();
  bc_decomp *D = new (std::nothrow) bc_decomp;
  if (!D) return BCGPU_ENOMEM;
  const int rc = bcg::decomp_gpu(g, device, D, t0, err, errlen);
  if (rc != BCGPU_OK) {
    delete D;
    return rc;
  }
  *out = D;
  return BCGPU_OK;
}
