// The BCC split and the arc-to-member pass as data-parallel steps, for the
// GPU (bc_decompose_gpu): Tarjan and Vishkin's method over a BFS forest, the
// same mathematics as the host split in host_decomp.cpp, written as one
// functor per step over vertices, frontier positions or BCCs. A backend runs
// the steps: DevBackend as a grid-stride kernel per step on one GPU,
// HostBackend as OpenMP loops over the very same functors -- a check of the
// GPU steps on a machine without one. Prefix sums (a handful, over vertices,
// roots, BCCs and member slots) are taken on the host in both.
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
//                member's arcs inside the BCC as local ids in arc order.
// The split and reach follow Codes/bicc.cpp:81-161 and
// Codes/modified_apsp.cpp:77-220 in what they compute (not how).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "decomp.h"

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

// ---- the steps; operator()(i) handles item i
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
struct Hook {  // components: one union per edge, from its larger end
  const int64_t *R;
  const int32_t *C;
  int32_t *uf;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = (int32_t)i;
    for (int64_t e = R[x]; e < R[x + 1]; ++e)
      if (C[e] < x) uf_union(uf, x, C[e]);
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
struct LoHiLocal {  // pre range over x and its neighbours other than its parent
  const int64_t *R;
  const int32_t *C, *par, *pre;
  int32_t *lo, *hi;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = (int32_t)i;
    int32_t l = pre[x], h = pre[x];
    for (int64_t e = R[x]; e < R[x + 1]; ++e)
      if (C[e] != par[x]) {
        const int32_t q = pre[C[e]];
        l = q < l ? q : l;
        h = q > h ? q : h;
      }
    lo[x] = l;
    hi[x] = h;
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
struct TreeEdgeUnion {  // tree edges named by their child vertex
  const int64_t *R;
  const int32_t *C, *par, *pre, *lo, *hi;
  const int64_t *nd;
  int32_t *uf;
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t w = (int32_t)i, v = par[w];
    if (v >= 0 && par[v] >= 0 && (lo[w] < pre[v] || (int64_t)hi[w] >= (int64_t)pre[v] + nd[v])) uf_union(uf, v, w);
    for (int64_t e = R[w]; e < R[w + 1]; ++e) {
      const int32_t y = C[e];
      if (y <= w || y == v || w == par[y]) continue;
      const int32_t a = pre[w] < pre[y] ? w : y, b = a == w ? y : w;
      if ((int64_t)pre[b] >= (int64_t)pre[a] + nd[a]) uf_union(uf, w, y);
    }
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
  const int32_t *C, *tbcc, *pre, *head, *locid;
  const int64_t *mem_off;
  int64_t *cnt;           // count pass: arcs per slot
  int64_t *cursor;        // fill pass: next free position per slot
  int32_t *sadj;
  __host__ __device__ int32_t local_of(int32_t x, int32_t b) const {
    return x == head[b] ? (int32_t)(mem_off[b + 1] - mem_off[b] - 1) : locid[x];
  }
  __host__ __device__ void operator()(int64_t i) const {
    const int32_t x = (int32_t)i;
    for (int64_t e = R[x]; e < R[x + 1]; ++e) {
      const int32_t y = C[e];
      const int32_t b = tbcc[pre[x] > pre[y] ? x : y];
      const int64_t s = mem_off[b] + local_of(x, b);
      if (cursor) sadj[cursor[s]++] = local_of(y, b);
      else cnt[s] += 1;
    }
  }
};

template <class F>
__global__ void each_kernel(int64_t n, F f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) f(i);
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
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) f(i);
  }
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
  std::vector<int64_t> tmp;
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
  template <class T>
  void upload(T *dst, const T *src, size_t n) {
    if (n) check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
    check(cudaStreamSynchronize(stream), "upload");
  }
  template <class T>
  void download(T *dst, const T *src, size_t n) {
    if (n) check(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, stream), "download");
    check(cudaStreamSynchronize(stream), "step");
  }
  int64_t scan(int64_t *a, int64_t n) {
    tmp.resize((size_t)n);
    download(tmp.data(), a, (size_t)n);
    const int64_t s = scan_host(tmp.data(), n);
    upload(a, tmp.data(), (size_t)n);
    return s;
  }
};

template <class BE>
void run(BE &be, const bc_graph *g, SplitResult &S) {
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

  // components
  be.each(n, Iota{uf});
  be.each(n, Hook{R, C, uf});
  be.each(n, Compress{uf});
  be.each(n, RootFlag{uf, flag});
  const int64_t nroots = be.scan(flag, n);
  be.each(n, Fill32{par, -2});
  be.each(n, RootScatter{uf, flag, roots, comp, order, par});

  // BFS forest, one launch per level
  std::vector<int64_t> lvl{0, nroots};
  for (int64_t f0 = 0, f1 = nroots; f1 > f0;) {
    be.upload(tail, &f1, 1);
    be.each(f1 - f0, BfsLevel{R, C, order, par, tail, f0});
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

  // subtree sizes, preorder, low/high
  be.each(n, Fill64{nd, 1});
  for (int64_t L = nlev - 1; L >= 1; --L) be.each(lvl[L + 1] - lvl[L], NdUp{order, par, nd, lvl[L]});
  int64_t *csize = be.template alloc<int64_t>((size_t)nroots), *cstart = be.template alloc<int64_t>((size_t)nroots);
  be.each(nroots, RootSizes{roots, nd, csize});
  be.each(nroots, Copy64{cstart, csize});
  be.scan(cstart, nroots);
  be.each(nroots, RootPre{roots, cstart, pre, cur});
  for (int64_t L = 1; L < nlev; ++L) be.each(lvl[L + 1] - lvl[L], PreDown{order, par, nd, pre, cur, lvl[L]});
  be.each(n, LoHiLocal{R, C, par, pre, lo, hi});
  for (int64_t L = nlev - 1; L >= 1; --L) be.each(lvl[L + 1] - lvl[L], LoHiUp{order, par, lo, hi, lvl[L]});

  // BCCs: union-find over tree edges
  be.each(n, Iota{uf});
  be.each(n, TreeEdgeUnion{R, C, par, pre, lo, hi, nd, uf});
  be.each(n, Compress{uf});
  be.each(n, NameFlag{par, uf, flag});
  const int64_t nbcc = be.scan(flag, n);
  be.each(n, BccOf{par, uf, flag, tbcc});

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
  be.each(n, SlotArcs{R, C, tbcc, pre, head, locid, mem_off, sdeg, nullptr, nullptr});
  const int64_t slot_arcs = be.scan(sdeg, n_slots + 1);
  if (slot_arcs != arcs) throw StepError{BCGPU_EINVAL, "member slots do not hold every arc once"};
  int32_t *sadj = be.template alloc<int32_t>((size_t)arcs);
  be.each(n_slots, Copy64{cursor, sdeg});
  be.each(n, SlotArcs{R, C, tbcc, pre, head, locid, mem_off, nullptr, cursor, sadj});

  // results to the host
  S.nbcc = (int32_t)nbcc;
  be.download(&S.n_art, n_art, 1);
  S.comp.resize((size_t)n);
  S.head.resize((size_t)nbcc);
  S.members.resize((size_t)n_slots);
  S.sadj.resize((size_t)arcs);
  S.comp_size.resize((size_t)nroots);
  S.below.resize((size_t)nbcc);
  S.hang.resize((size_t)n);
  S.mem_off.resize((size_t)nbcc + 1);
  S.sdeg.resize((size_t)n_slots + 1);
  S.art.resize((size_t)n);
  be.download(S.comp.data(), comp, (size_t)n);
  be.download(S.head.data(), head, (size_t)nbcc);
  be.download(S.members.data(), members, (size_t)n_slots);
  be.download(S.sadj.data(), sadj, (size_t)arcs);
  be.download(S.comp_size.data(), csize, (size_t)nroots);
  be.download(S.below.data(), below, (size_t)nbcc);
  be.download(S.hang.data(), hang, (size_t)n);
  be.download(S.mem_off.data(), mem_off, (size_t)nbcc + 1);
  be.download(S.sdeg.data(), sdeg, (size_t)n_slots + 1);
  be.download(S.art.data(), art, (size_t)n);
}

}  // namespace decomp_steps

int decomp_split_steps(const bc_graph *g, int device, SplitResult &S, char *err, size_t errlen) {
  auto fail = [&](int code, const std::string &what) {
    if (err && errlen) std::snprintf(err, errlen, "%s", what.c_str());
    return code;
  };
  try {
    if (device < 0) {
      decomp_steps::HostBackend be;
      decomp_steps::run(be, g, S);
    } else {
      decomp_steps::DevBackend be(device);
      decomp_steps::run(be, g, S);
    }
  } catch (const decomp_steps::StepError &e) {
    return fail(e.code, e.what);
  } catch (const std::bad_alloc &) {
    return fail(BCGPU_ENOMEM, "host allocation failed");
  }
  return BCGPU_OK;
}

}  // namespace bcg

extern "C" int bc_decompose_gpu(const bc_graph *g, int device, bc_decomp **out, char *err, size_t errlen) {
  if (!g || !out) return BCGPU_EINVAL;
  const auto t0 = std::chrono::steady_clock::now();
  bc_decomp *D = new (std::nothrow) bc_decomp;
  if (!D) return BCGPU_ENOMEM;
  int rc;
  try {
    bcg::SplitResult S;
    rc = bcg::decomp_split_steps(g, device, S, err, errlen);
    if (rc == BCGPU_OK) {
      rc = bcg::decomp_pack(S, g->n, D, t0);
      if (rc != BCGPU_OK && err && errlen) std::snprintf(err, errlen, "packing failed (status %d)", rc);
    }
  } catch (const std::bad_alloc &) {
    rc = BCGPU_ENOMEM;
    if (err && errlen) std::snprintf(err, errlen, "host allocation failed");
  }
  if (rc != BCGPU_OK) {
    delete D;
    return rc;
  }
  *out = D;
  return BCGPU_OK;
}
