// Host side of libbcgpu: edge-list ingest and the decomposition that feeds the
// GPU kernels (C ABI in include/bchost.h).
//
// What it replaces in the reference and how it differs:
//  * Graph::Graph(char*) (Codes/graph.cpp:38-59) reads with fscanf and keeps
//    duplicates; here the file is parsed from one buffer and the graph is made
//    simple (loops dropped, duplicates merged), the assumption the reference's
//    BFS states (Codes/kernels_free.cu:248).
//  * BiCC::bicc_tarjan (Codes/bicc.cpp:81-161) recurses once per vertex and
//    assumes the DFS root is vertex 0 (:13,:86-87); here Tarjan and
//    Vishkin's method over a BFS forest (split_bccs) finds the BCCs of every
//    component in parallel loops, with no DFS.
//  * fillbccparent/reachfunction (Codes/modified_apsp.cpp:77-220) walk an
//    explicit block-cut tree; here reach and the articulation cross terms come
//    straight from forest subtree sizes: for BCC b with head h (its vertex
//    closest to the component's root) and below(b) the vertices under b's
//    topmost tree edges, reach_b(h) = |comp| - 1 - below(b), and for any
//    other member x, reach_b(x) = the sum of below over the BCCs that x heads
//    (the subtrees split off at x). The cross term of x is
//    S^2 - sum(part^2) over the parts of comp - x (S = |comp| - 1), i.e. the
//    ordered pairs that x separates (Codes/modified_apsp.cpp:209).
//  * bcc_bfs/preSum (Codes/bcc_bfs.cpp:100-236, :247-1330) find ears through a
//    BFS tree, LCAs and "master" edges; the chains they emit are exactly the
//    maximal paths of vertices of degree 2 inside the BCC (a BCC that is one
//    cycle emits none: all its vertices stay free). Here those paths are
//    walked directly from their endpoints in O(n_b + m_b).
#include "bchost.h"
#include "decomp.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <omp.h>
#include <parallel/algorithm>


namespace {

void set_err(char *err, size_t errlen, const std::string &msg) {
  if (err && errlen) {
    std::snprintf(err, errlen, "%s", msg.c_str());
  }
}

int build_csr(int32_t n, int64_t m, const int32_t *u, const int32_t *v, bc_graph *g) {
  g->n = n;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int64_t e = 0; e < m; ++e) bad |= u[e] < 0 || u[e] >= n || v[e] < 0 || v[e] >= n;
  if (bad) return BCGPU_EINVAL;
  // Degrees and the scatter in parallel without atomics: thread t owns the
  // vertices [lo_t, hi_t) and scans every edge, keeping the endpoints it
  // owns, so each adjacency list is filled in edge order by one thread.
  std::vector<int64_t> deg((size_t)n + 1, 0);
  auto owned = [n](int32_t &lo, int32_t &hi) {
    const int T = omp_get_num_threads(), t = omp_get_thread_num();
    lo = (int32_t)((int64_t)n * t / T);
    hi = (int32_t)((int64_t)n * (t + 1) / T);
  };
#pragma omp parallel
  {
    int32_t lo, hi;
    owned(lo, hi);
    for (int64_t e = 0; e < m; ++e) {
      if (u[e] == v[e]) continue;
      if (u[e] >= lo && u[e] < hi) deg[u[e] + 1]++;
      if (v[e] >= lo && v[e] < hi) deg[v[e] + 1]++;
    }
  }
  for (int32_t i = 0; i < n; ++i) deg[i + 1] += deg[i];
  std::vector<int32_t> col((size_t)deg[n]);
#pragma omp parallel
  {
    int32_t lo, hi;
    owned(lo, hi);  // any split works: each vertex is filled by exactly one thread
    std::vector<int64_t> fill(deg.begin() + lo, deg.begin() + hi);
    for (int64_t e = 0; e < m; ++e) {
      if (u[e] == v[e]) continue;
      if (u[e] >= lo && u[e] < hi) col[fill[u[e] - lo]++] = v[e];
      if (v[e] >= lo && v[e] < hi) col[fill[v[e] - lo]++] = u[e];
    }
  }
  // sort + dedup every adjacency list, then compact
  std::vector<int64_t> keep((size_t)n + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t i = 0; i < n; ++i) {
    int32_t *b = col.data() + deg[i], *e = col.data() + deg[i + 1];
    std::sort(b, e);
    keep[i + 1] = std::unique(b, e) - b;
  }
  for (int32_t i = 0; i < n; ++i) keep[i + 1] += keep[i];
  g->row = keep;
  g->col.resize((size_t)keep[n]);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t i = 0; i < n; ++i)
    std::copy(col.data() + deg[i], col.data() + deg[i] + (keep[i + 1] - keep[i]), g->col.data() + keep[i]);
  return BCGPU_OK;
}

// Minimal integer scanner over a memory buffer.
struct Scanner {
  const char *p, *end;
  bool next(int64_t &x) {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    if (p >= end) return false;
    bool neg = false;
    if (*p == '-') { neg = true; ++p; }
    if (p >= end || *p < '0' || *p > '9') return false;
    int64_t v = 0;
    while (p < end && *p >= '0' && *p <= '9') { v = v * 10 + (*p - '0'); ++p; }
    x = neg ? -v : v;
    return true;
  }
};

}  // namespace

extern "C" int bc_graph_from_edges(int32_t n, int64_t m, const int32_t *u, const int32_t *v, bc_graph **out) {
  if (!out || n < 0 || m < 0 || (m > 0 && (!u || !v))) return BCGPU_EINVAL;
  bc_graph *g = new (std::nothrow) bc_graph;
  if (!g) return BCGPU_ENOMEM;
  int rc;
  try {
    rc = build_csr(n, m, u, v, g);
  } catch (const std::bad_alloc &) {
    rc = BCGPU_ENOMEM;
  }
  if (rc != BCGPU_OK) { delete g; return rc; }
  *out = g;
  return BCGPU_OK;
}

namespace {

constexpr char kCsrMagic[8] = {'B', 'C', 'G', 'C', 'S', 'R', '1', '\0'};
constexpr size_t kCsrHeader = 24;  // magic, int32 n, int32 0, int64 arcs

// 64-bit mixing of an ordered vertex pair (splitmix64 finaliser).
inline uint64_t pair_hash(int32_t x, int32_t y) {
  uint64_t z = ((uint64_t)(uint32_t)x << 32 | (uint32_t)y) + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// The binary CSR of bc_graph_save, read straight into the graph and checked
// to be what the text path builds: offsets from 0 to arcs, every list
// strictly increasing (sorted, no duplicates), no loops, and every arc present
// in both directions -- the sums of pair_hash over (x, y) and over (y, x)
// agree exactly when the arc multiset is symmetric, barring a 2^-64 collision.
int load_binary(FILE *fp, long size, bc_graph **out, char *err, size_t errlen) {
  auto bad = [&](const char *why) {
    set_err(err, errlen, std::string("binary CSR: ") + why);
    return BCGPU_EIO;
  };
  char head[kCsrHeader];
  if (size < (long)kCsrHeader || std::fread(head, 1, kCsrHeader, fp) != kCsrHeader) return bad("truncated header");
  int32_t n, pad;
  int64_t arcs;
  std::memcpy(&n, head + 8, 4);
  std::memcpy(&pad, head + 12, 4);
  std::memcpy(&arcs, head + 16, 8);
  if (n < 0 || pad != 0 || arcs < 0 || arcs > (int64_t)size / 4) return bad("bad header");
  const uint64_t want = kCsrHeader + 8ull * ((uint64_t)n + 1) + 4ull * (uint64_t)arcs;
  if (want != (uint64_t)size) return bad("file size does not match its header");
  std::unique_ptr<bc_graph> g(new bc_graph);
  g->n = n;
  g->row.resize((size_t)n + 1);
  g->col.resize((size_t)arcs);
  if (std::fread(g->row.data(), 8, (size_t)n + 1, fp) != (size_t)n + 1 ||
      (arcs && std::fread(g->col.data(), 4, (size_t)arcs, fp) != (size_t)arcs))
    return bad("short read");
  const int64_t *R = g->row.data();
  const int32_t *C = g->col.data();
  int fault = R[0] != 0 || R[n] != arcs;
  uint64_t fwd = 0, rev = 0;
  if (!fault) {
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : fault) reduction(+ : fwd, rev)
    for (int32_t x = 0; x < n; ++x) {
      if (R[x + 1] < R[x] || R[x + 1] > arcs) { fault |= 1; continue; }
      for (int64_t e = R[x]; e < R[x + 1]; ++e) {
        const int32_t y = C[e];
        if (y < 0 || y >= n || y == x || (e > R[x] && C[e - 1] >= y)) { fault |= 2; break; }
        fwd += pair_hash(x, y);
        rev += pair_hash(y, x);
      }
    }
  }
  if (!fault && fwd != rev) fault = 4;
  if (fault)
    return bad(fault & 1 ? "row offsets out of order" : fault & 2 ? "a neighbour list that is not sorted, "
               "repeats a vertex, holds a loop or an id out of range" : "an arc without its reverse");
  *out = g.release();
  return BCGPU_OK;
}

int graph_load(const char *path, bc_graph **out, char *err, size_t errlen) {
  FILE *fp = std::fopen(path, "rb");
  if (!fp) { set_err(err, errlen, std::string("input file cannot be opened: ") + path); return BCGPU_EIO; }
  std::fseek(fp, 0, SEEK_END);
  long size = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  char magic[sizeof kCsrMagic];
  if (size >= (long)sizeof kCsrMagic && std::fread(magic, 1, sizeof magic, fp) == sizeof magic &&
      std::memcmp(magic, kCsrMagic, sizeof magic) == 0) {  // a CSR written by bc_graph_save
    std::fseek(fp, 0, SEEK_SET);
    const int rc = load_binary(fp, size, out, err, errlen);
    std::fclose(fp);
    return rc;
  }
  std::fseek(fp, 0, SEEK_SET);
  std::vector<char> buf(size > 0 ? (size_t)size : 1);
  size_t got = size > 0 ? std::fread(buf.data(), 1, (size_t)size, fp) : 0;
  std::fclose(fp);
  if ((long)got != size) { set_err(err, errlen, "short read"); return BCGPU_EIO; }
  Scanner sc{buf.data(), buf.data() + got};
  int64_t n, m;
  if (!sc.next(n) || !sc.next(m) || n < 0 || m < 0 || n > INT32_MAX) {
    set_err(err, errlen, "bad header: expected 'n m'");
    return BCGPU_EIO;
  }
  // The edge tokens are parsed in parallel: the rest of the buffer is cut
  // into chunks at whitespace (a number never spans a cut), each chunk is
  // scanned twice -- once to count the numbers before its first bad
  // character, once to place number t (global order) as field t % 3 of
  // edge t / 3. Errors are those of a sequential scan: the first edge that
  // is incomplete ("truncated") or, before it, has an id out of range.
  const char *p0 = sc.p, *pend = buf.data() + got;
  const int nchunk = std::max(1, 4 * omp_get_max_threads());
  std::vector<const char *> cut((size_t)nchunk + 1);
  cut[0] = p0;
  for (int k = 1; k < nchunk; ++k) {
    const char *c = std::max(cut[k - 1], p0 + (pend - p0) * k / nchunk);
    while (c < pend && !(*c == ' ' || *c == '\n' || *c == '\r' || *c == '\t')) ++c;
    cut[k] = c;
  }
  cut[nchunk] = pend;
  std::vector<int64_t> cnt((size_t)nchunk + 1, 0);
  std::vector<char> broke((size_t)nchunk, 0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < nchunk; ++k) {
    Scanner s{cut[k], cut[k + 1]};
    int64_t x, c = 0;
    const char *last = s.p;  // where the failing call started
    while (s.next(x)) {
      ++c;
      last = s.p;
    }
    while (last < s.end && (*last == ' ' || *last == '\n' || *last == '\r' || *last == '\t')) ++last;
    cnt[k + 1] = c;
    broke[k] = last < s.end;  // something other than whitespace followed: it starts no number
  }
  int64_t valid = 0;  // numbers before the first bad character
  for (int k = 0; k < nchunk; ++k) {
    valid += cnt[k + 1];
    if (broke[k]) break;
  }
  for (int k = 0; k < nchunk; ++k) cnt[k + 1] += cnt[k];
  const int64_t need = m > INT64_MAX / 3 ? INT64_MAX : 3 * m, have = std::min(valid, need);
  // the edge arrays are sized from the header only once the file holds that
  // many numbers (a header that overstates m is a truncated list, not an allocation)
  const bool complete = have == need;
  std::vector<int32_t> u(complete ? (size_t)m : 0), v(complete ? (size_t)m : 0);
  int64_t first_oob = INT64_MAX;
#pragma omp parallel for schedule(dynamic, 1) reduction(min : first_oob)
  for (int k = 0; k < nchunk; ++k) {
    Scanner s{cut[k], cut[k + 1]};
    int64_t x;
    for (int64_t t = cnt[k]; t < have && s.next(x); ++t) {
      const int64_t e = t / 3;
      const int f = (int)(t % 3);
      if (f == 2) continue;  // the weight: read, not used (as the reference's BFS)
      if (x < 0 || x >= n) {
        first_oob = std::min(first_oob, e);
        x = 0;
      }
      if (complete) (f == 0 ? u : v)[(size_t)e] = (int32_t)x;
    }
  }
  const int64_t trunc_at = have < need ? have / 3 : INT64_MAX;
  if (first_oob < trunc_at) {
    set_err(err, errlen, "vertex id out of range at edge " + std::to_string(first_oob));
    return BCGPU_EIO;
  }
  if (trunc_at != INT64_MAX) {
    set_err(err, errlen, "truncated edge list at edge " + std::to_string(trunc_at) + " of " + std::to_string(m));
    return BCGPU_EIO;
  }
  int rc = bc_graph_from_edges((int32_t)n, m, u.data(), v.data(), out);
  if (rc != BCGPU_OK) set_err(err, errlen, "graph construction failed");
  return rc;
}

}  // namespace

extern "C" int bc_graph_load(const char *path, bc_graph **out, char *err, size_t errlen) {
  if (!path || !out) { set_err(err, errlen, "null argument"); return BCGPU_EINVAL; }
  try {
    return graph_load(path, out, err, errlen);
  } catch (const std::bad_alloc &) {
    set_err(err, errlen, "out of host memory reading the edge list");
    return BCGPU_ENOMEM;
  }
}

extern "C" void bc_graph_free(bc_graph *g) { delete g; }

extern "C" int bc_graph_save(const bc_graph *g, const char *path, char *err, size_t errlen) {
  if (!g || !path) { set_err(err, errlen, "null argument"); return BCGPU_EINVAL; }
  FILE *fp = std::fopen(path, "wb");
  if (!fp) { set_err(err, errlen, std::string("cannot write ") + path); return BCGPU_EIO; }
  const int32_t n = g->n, pad = 0;
  const int64_t arcs = g->row.empty() ? 0 : g->row[(size_t)n];
  bool ok = std::fwrite(kCsrMagic, 1, sizeof kCsrMagic, fp) == sizeof kCsrMagic &&
            std::fwrite(&n, 4, 1, fp) == 1 && std::fwrite(&pad, 4, 1, fp) == 1 && std::fwrite(&arcs, 8, 1, fp) == 1;
  const int64_t zero = 0;
  if (ok && g->row.empty()) ok = std::fwrite(&zero, 8, 1, fp) == 1;  // an empty graph: row = {0}
  else if (ok) ok = std::fwrite(g->row.data(), 8, (size_t)n + 1, fp) == (size_t)n + 1;
  if (ok && arcs) ok = std::fwrite(g->col.data(), 4, (size_t)arcs, fp) == (size_t)arcs;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) { set_err(err, errlen, std::string("short write to ") + path); return BCGPU_EIO; }
  return BCGPU_OK;
}

extern "C" int bc_graph_csr(const bc_graph *g, int32_t *n, int64_t *n_arcs, const int64_t **row, const int32_t **col) {
  if (!g) return BCGPU_EINVAL;
  if (n) *n = g->n;
  if (n_arcs) *n_arcs = g->row.empty() ? 0 : g->row[g->n];
  if (row) *row = g->row.data();
  if (col) *col = g->col.data();
  return BCGPU_OK;
}

namespace {

// ---- data-parallel building blocks. Every loop below is a parallel loop
// over vertices, frontier positions or BCCs whose body touches only its own
// outputs, atomics (GCC builtins, relaxed: each loop ends at an OpenMP
// barrier) or data that no iteration of the same loop writes.
template <class T> inline T ald(const T *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
template <class T> inline void ast(T *p, T v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
template <class T> inline T aadd(T *p, T v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
template <class T> inline bool acas(T *p, T expect, T v) {
  return __atomic_compare_exchange_n(p, &expect, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
}
template <class T> inline void amin(T *p, T v) {
  T c = ald(p);
  while (v < c && !__atomic_compare_exchange_n(p, &c, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
}
template <class T> inline void amax(T *p, T v) {
  T c = ald(p);
  while (v > c && !__atomic_compare_exchange_n(p, &c, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
  }
}

// Union-find whose set roots are the sets' smallest members: a link hangs the
// larger root under the smaller one, so p[x] <= x at all times and concurrent
// finds (with path halving) and links need nothing but compare-and-swap.
int32_t uf_find(int32_t *p, int32_t x) {
  for (;;) {
    const int32_t y = ald(&p[x]);
    if (y == x) return x;
    const int32_t z = ald(&p[y]);
    if (z != y) acas(&p[x], y, z);
    x = z;
  }
}
void uf_union(int32_t *p, int32_t a, int32_t b) {
  for (;;) {
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a == b) return;
    if (a > b) std::swap(a, b);
    if (acas(&p[b], b, a)) return;
  }
}

constexpr int64_t kParFrontier = 2048;  // narrower BFS levels run on one thread

// f(a, b) over chunks [a, b) of [k0, k1): in parallel when the range is
// wide, else as one chunk on this thread (an OpenMP region costs
// microseconds, and deep graphs have thousands of narrow levels).
template <class F>
void for_chunks(int64_t k0, int64_t k1, F &&f) {
  constexpr int64_t kChunk = 1024;
  if (k1 - k0 < kParFrontier) {
    if (k1 > k0) f(k0, k1);
    return;
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c = k0; c < k1; c += kChunk) f(c, std::min(k1, c + kChunk));
}

// Level-synchronous BFS that lists the vertices in exactly the order of the
// sequential queue BFS from src: level by level, the undiscovered neighbours
// of each frontier vertex in adjacency order, frontier vertices in their own
// order. A narrow level is one pass of the sequential queue. A wide level is
// expanded top-down -- a vertex is claimed by the earliest frontier position
// adjacent to it (atomic min), the claims are counted per position and a
// prefix sum places each position's vertices -- or, when the unvisited
// vertices have fewer arcs than the frontier, bottom-up: every unvisited
// vertex finds its earliest adjacent frontier position itself, and the new
// level is sorted by (that position, key). That needs every adjacency list in
// increasing key order, key(y) distinct per vertex.
// adj(x, &ptr) returns the degree of x and points ptr at its neighbours.
// Returns the visit order (the vertices reached).
template <class Adj, class Key>
std::vector<int32_t> bfs_exact_order(int32_t nv, int32_t src, Adj adj, Key key) {
  std::vector<int32_t> order((size_t)nv), claim, lev((size_t)nv, -1), pos((size_t)nv, 0);
  std::vector<int64_t> cnt;
  const int nt = omp_get_max_threads();
  std::vector<std::vector<std::pair<uint64_t, int32_t>>> found((size_t)nt);
  std::vector<std::pair<uint64_t, int32_t>> all;
  int64_t unvisited_arcs = 0;
#pragma omp parallel for schedule(static) reduction(+ : unvisited_arcs)
  for (int32_t x = 0; x < nv; ++x) {
    const int32_t *a;
    unvisited_arcs += adj(x, &a);
  }
  order[0] = src;
  lev[src] = 0;
  int64_t f0 = 0, f1 = 1, frontier_arcs = 0;
  {
    const int32_t *a;
    frontier_arcs = adj(src, &a);
    unvisited_arcs -= frontier_arcs;
  }
  for (int32_t L = 0; f1 > f0; ++L) {
    const int64_t fn = f1 - f0;
    int64_t f2 = f1;
    if (fn < kParFrontier) {
      for (int64_t i = f0; i < f1; ++i) {
        const int32_t *a;
        const int32_t d = adj(order[i], &a);
        for (int32_t j = 0; j < d; ++j)
          if (lev[a[j]] < 0) {
            lev[a[j]] = L + 1;
            order[f2++] = a[j];
          }
      }
    } else if (unvisited_arcs < frontier_arcs) {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < fn; ++i) pos[order[f0 + i]] = (int32_t)i;
#pragma omp parallel
      {
        auto &mine = found[(size_t)omp_get_thread_num()];
        mine.clear();
#pragma omp for schedule(dynamic, 1024)
        for (int32_t y = 0; y < nv; ++y) {
          if (lev[y] >= 0) continue;
          const int32_t *a;
          const int32_t d = adj(y, &a);
          int32_t m = INT32_MAX;
          for (int32_t j = 0; j < d; ++j)
            if (lev[a[j]] == L && pos[a[j]] < m) m = pos[a[j]];
          if (m != INT32_MAX) mine.emplace_back(((uint64_t)(uint32_t)m << 32) | (uint64_t)(uint32_t)key(y), y);
        }
      }
      all.clear();
      for (auto &v : found) all.insert(all.end(), v.begin(), v.end());
      __gnu_parallel::sort(all.begin(), all.end());
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < (int64_t)all.size(); ++k) {
        order[f1 + k] = all[k].second;
        lev[all[k].second] = L + 1;
      }
      f2 = f1 + (int64_t)all.size();
    } else {
      if (claim.empty()) claim.assign((size_t)nv, INT32_MAX);
      int32_t *cl = claim.data();
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t i = 0; i < fn; ++i) {
        const int32_t *a;
        const int32_t d = adj(order[f0 + i], &a);
        for (int32_t j = 0; j < d; ++j)
          if (lev[a[j]] < 0) amin(&cl[a[j]], (int32_t)i);
      }
      cnt.assign((size_t)fn + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t i = 0; i < fn; ++i) {
        const int32_t *a;
        const int32_t d = adj(order[f0 + i], &a);
        int64_t c = 0;
        for (int32_t j = 0; j < d; ++j) c += lev[a[j]] < 0 && ald(&cl[a[j]]) == (int32_t)i;
        cnt[i + 1] = c;
      }
      for (int64_t i = 0; i < fn; ++i) cnt[i + 1] += cnt[i];
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t i = 0; i < fn; ++i) {
        const int32_t *a;
        const int32_t d = adj(order[f0 + i], &a);
        int64_t at = f1 + cnt[i];
        for (int32_t j = 0; j < d; ++j)
          if (lev[a[j]] < 0 && ald(&cl[a[j]]) == (int32_t)i) order[at++] = a[j];
      }
      f2 = f1 + cnt[fn];
#pragma omp parallel for schedule(static)
      for (int64_t k = f1; k < f2; ++k) lev[order[k]] = L + 1;
    }
    frontier_arcs = 0;
#pragma omp parallel for schedule(static) reduction(+ : frontier_arcs) if (f2 - f1 >= kParFrontier)
    for (int64_t k = f1; k < f2; ++k) {
      const int32_t *a;
      frontier_arcs += adj(order[k], &a);
    }
    unvisited_arcs -= frontier_arcs;
    f0 = f1;
    f1 = f2;
  }
  order.resize((size_t)f1);
  return order;
}

// A BFS forest of the CSR graph from the given roots, one level at a time:
// a vertex's parent is whichever adjacent frontier vertex claims it first
// (compare-and-swap), so the forest depends on thread timing -- the callers
// only use properties every BFS forest has. par[x] = -1 for a root; level L
// is order[lvl_off[L], lvl_off[L + 1]).
void bfs_forest(int32_t n, const int64_t *R, const int32_t *C, const std::vector<int32_t> &roots,
                std::vector<int32_t> &par, std::vector<int32_t> &order, std::vector<int64_t> &lvl_off) {
  par.assign((size_t)n, -2);
  order.resize((size_t)n);
  for (size_t i = 0; i < roots.size(); ++i) {
    order[i] = roots[i];
    par[roots[i]] = -1;
  }
  lvl_off.assign({0, (int64_t)roots.size()});
  const int nt = omp_get_max_threads();
  std::vector<std::vector<int32_t>> buf((size_t)nt);
  std::vector<int64_t> boff((size_t)nt + 1);
  int32_t *P = par.data(), *O = order.data();
  int64_t f0 = 0, f1 = (int64_t)roots.size();
  while (f1 > f0) {
    int64_t f2 = f1;
    if (f1 - f0 < kParFrontier) {
      for (int64_t i = f0; i < f1; ++i) {
        const int32_t x = O[i];
        for (int64_t e = R[x]; e < R[x + 1]; ++e)
          if (P[C[e]] == -2) {
            P[C[e]] = x;
            O[f2++] = C[e];
          }
      }
    } else {
#pragma omp parallel
      {
        const int t = omp_get_thread_num();
        std::vector<int32_t> &b = buf[t];
        b.clear();
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = f0; i < f1; ++i) {
          const int32_t x = O[i];
          for (int64_t e = R[x]; e < R[x + 1]; ++e) {
            const int32_t y = C[e];
            if (ald(&P[y]) == -2 && acas(&P[y], -2, x)) b.push_back(y);
          }
        }
#pragma omp single
        {
          boff[0] = f1;
          for (int u = 0; u < nt; ++u) boff[u + 1] = boff[u] + (u < omp_get_num_threads() ? (int64_t)buf[u].size() : 0);
        }
        std::copy(b.begin(), b.end(), O + boff[t]);
      }
      f2 = boff[(size_t)nt];
    }
    f0 = f1;
    f1 = f2;
    lvl_off.push_back(f1);
  }
  lvl_off.pop_back();  // the last, empty level
}

// BCCs of a simple undirected graph by Tarjan and Vishkin's method over a
// BFS spanning forest (any rooted spanning forest serves), every step a
// parallel loop:
//  1. components by union-find over the edges; each is rooted at its
//     smallest vertex;
//  2. one BFS from all roots at once gives the forest (parent, children);
//  3. subtree sizes nd bottom-up, preorder numbers pre top-down, and
//     low/high: the least/greatest pre over a subtree and the non-tree
//     neighbours of its vertices, bottom-up;
//  4. tree edges, named by their child vertex, are joined by union-find
//     (roots again the smallest members) when
//       - a non-tree edge joins two unrelated vertices v, w: tree edges of v
//         and w, or
//       - the subtree of w escapes the subtree of its parent v (low(w) <
//         pre(v) or high(w) >= pre(v) + nd(v)) and v is not a root: tree
//         edges of v and w;
//     the sets are the BCCs; a non-tree edge belongs to the BCC of the tree
//     edge into its endpoint with the larger pre.
// A BCC is named by its smallest non-head member, the root of its set, and
// BCCs are numbered in that order, so the result does not depend on the
// forest or on thread timing. Its head is the parent of its topmost tree
// edges; below(b), the vertices under those edges, gives reach and the
// articulation terms: a member x other than the head reaches the subtrees of
// its children in other BCCs (hang(x), the sum of below over the BCCs x
// heads), the head reaches the rest of its component.
// Replaces the DFS of Codes/bicc.cpp:81-161 and the block-cut tree walk of
// Codes/modified_apsp.cpp:77-220.
struct Split {
  int32_t nbcc = 0;
  std::vector<int32_t> comp, tbcc, pre, head, locid, members;
  std::vector<int64_t> comp_size, below, hang, sq, mem_off;
};

void split_bccs(const bc_graph *g, Split &S) {
  const int32_t n = g->n;
  const int64_t *R = g->row.data();
  const int32_t *C = g->col.data();

  // 1. components
  std::vector<int32_t> uf((size_t)n);
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) uf[x] = x;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t x = 0; x < n; ++x)
    for (int64_t e = R[x]; e < R[x + 1]; ++e)
      if (C[e] < x) uf_union(uf.data(), x, C[e]);
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) uf[x] = uf_find(uf.data(), x);
  std::vector<int32_t> roots;
  S.comp.assign((size_t)n, -1);
  for (int32_t x = 0; x < n; ++x)
    if (uf[x] == x) {
      S.comp[x] = (int32_t)roots.size();
      roots.push_back(x);
    }
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) S.comp[x] = S.comp[uf[x]];

  // 2. BFS forest
  std::vector<int32_t> parv, orderv;
  std::vector<int64_t> lvl_off;
  bfs_forest(n, R, C, roots, parv, orderv, lvl_off);
  const int32_t *par = parv.data(), *order = orderv.data();
  const int64_t nlev = (int64_t)lvl_off.size() - 1;

  // 3. nd bottom-up, pre top-down (siblings in any order: each takes the
  // next range of its parent's interval), low/high bottom-up. A level lists
  // the children of one parent mostly in runs (a claiming thread appends
  // them together), so each run updates its parent with one atomic.
  auto runs = [&](int64_t a, int64_t b, auto &&g) {  // g(parent, run begin, run end)
    for (int64_t k = a; k < b;) {
      const int32_t p = par[order[k]];
      int64_t j = k + 1;
      while (j < b && par[order[j]] == p) ++j;
      g(p, k, j);
      k = j;
    }
  };
  std::vector<int64_t> nd((size_t)n, 1), cur((size_t)n);
  for (int64_t L = nlev - 1; L >= 1; --L)
    for_chunks(lvl_off[L], lvl_off[L + 1], [&](int64_t a, int64_t b) {
      runs(a, b, [&](int32_t p, int64_t k, int64_t j) {
        int64_t s = 0;
        for (int64_t t = k; t < j; ++t) s += nd[order[t]];
        aadd(&nd[p], s);
      });
    });
  S.pre.assign((size_t)n, 0);
  S.comp_size.resize(roots.size());
  int32_t *pre = S.pre.data();
  {
    int64_t q = 0;
    for (size_t i = 0; i < roots.size(); ++i) {
      pre[roots[i]] = (int32_t)q;
      cur[roots[i]] = q + 1;
      S.comp_size[i] = nd[roots[i]];
      q += nd[roots[i]];
    }
  }
  for (int64_t L = 1; L < nlev; ++L)
    for_chunks(lvl_off[L], lvl_off[L + 1], [&](int64_t a, int64_t b) {
      runs(a, b, [&](int32_t p, int64_t k, int64_t j) {
        int64_t s = 0;
        for (int64_t t = k; t < j; ++t) s += nd[order[t]];
        int64_t q = aadd(&cur[p], s);
        for (int64_t t = k; t < j; ++t) {
          const int32_t x = order[t];
          pre[x] = (int32_t)q;
          cur[x] = q + 1;
          q += nd[x];
        }
      });
    });
  std::vector<int32_t> lo((size_t)n), hi((size_t)n);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t x = 0; x < n; ++x) {
    int32_t l = pre[x], h = pre[x];
    for (int64_t e = R[x]; e < R[x + 1]; ++e)
      if (C[e] != par[x]) {
        l = std::min(l, pre[C[e]]);
        h = std::max(h, pre[C[e]]);
      }
    lo[x] = l;
    hi[x] = h;
  }
  for (int64_t L = nlev - 1; L >= 1; --L)
    for_chunks(lvl_off[L], lvl_off[L + 1], [&](int64_t a, int64_t b) {
      runs(a, b, [&](int32_t p, int64_t k, int64_t j) {
        int32_t l = lo[order[k]], h = hi[order[k]];
        for (int64_t t = k + 1; t < j; ++t) {
          l = std::min(l, lo[order[t]]);
          h = std::max(h, hi[order[t]]);
        }
        amin(&lo[p], l);
        amax(&hi[p], h);
      });
    });

  // 4. tree edges joined into BCCs
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) uf[x] = x;
#pragma omp parallel for schedule(dynamic, 1024)
  for (int32_t w = 0; w < n; ++w) {
    const int32_t v = par[w];
    if (v >= 0 && par[v] >= 0 && (lo[w] < pre[v] || (int64_t)hi[w] >= (int64_t)pre[v] + nd[v]))
      uf_union(uf.data(), v, w);
    for (int64_t e = R[w]; e < R[w + 1]; ++e) {
      const int32_t y = C[e];
      if (y <= w || y == par[w] || w == par[y]) continue;
      const int32_t a = pre[w] < pre[y] ? w : y, b = a == w ? y : w;
      if ((int64_t)pre[b] >= (int64_t)pre[a] + nd[a]) uf_union(uf.data(), w, y);
    }
  }
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) uf[x] = uf_find(uf.data(), x);

  // BCC ids in the order of their names; head, below, hang, sq
  S.tbcc.assign((size_t)n, -1);
  int32_t nbcc = 0;
  for (int32_t x = 0; x < n; ++x)
    if (par[x] >= 0 && uf[x] == x) S.tbcc[x] = nbcc++;
  S.nbcc = nbcc;
  int32_t *tbcc = S.tbcc.data();
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x)
    if (par[x] >= 0 && uf[x] != x) tbcc[x] = tbcc[uf[x]];  // uf[x] is a name, only read here
  S.head.assign((size_t)nbcc, -1);
  S.below.assign((size_t)nbcc, 0);
  S.hang.assign((size_t)n, 0);
  S.sq.assign((size_t)n, 0);
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x) {
    const int32_t p = par[x];
    if (p >= 0 && tbcc[p] != tbcc[x]) {  // a topmost tree edge of its BCC (a root's tbcc is -1)
      ast(&S.head[tbcc[x]], p);
      aadd(&S.below[tbcc[x]], nd[x]);
    }
  }
#pragma omp parallel for schedule(static)
  for (int32_t b = 0; b < nbcc; ++b) {
    aadd(&S.hang[S.head[b]], S.below[b]);
    aadd(&S.sq[S.head[b]], S.below[b] * S.below[b]);
  }

  // members: a BCC's non-head members are the child vertices of its tree
  // edges; each chunk of vertices sorts its own by BCC and reserves one range
  // per BCC it touches. Their order inside a BCC is immaterial: everything
  // written out is keyed by vertex ids.
  S.locid.assign((size_t)n, -1);
  std::vector<int64_t> fill((size_t)nbcc, 0);
  constexpr int32_t kChunk = 4096;
#pragma omp parallel
  {
    std::vector<std::pair<int32_t, int32_t>> v;
#pragma omp for schedule(dynamic, 1)
    for (int64_t c0 = 0; c0 < n; c0 += kChunk) {
      v.clear();
      for (int32_t x = (int32_t)c0; x < (int32_t)std::min<int64_t>(n, c0 + kChunk); ++x)
        if (tbcc[x] >= 0) v.emplace_back(tbcc[x], x);
      std::sort(v.begin(), v.end());
      for (size_t i = 0; i < v.size();) {
        size_t j = i;
        while (j < v.size() && v[j].first == v[i].first) ++j;
        int64_t base = aadd(&fill[v[i].first], (int64_t)(j - i));
        for (size_t k = i; k < j; ++k) S.locid[v[k].second] = (int32_t)(base + (int64_t)(k - i));
        i = j;
      }
    }
  }
  S.mem_off.assign((size_t)nbcc + 1, 0);
  for (int32_t b = 0; b < nbcc; ++b) S.mem_off[b + 1] = S.mem_off[b] + fill[b] + 1;
  S.members.assign((size_t)S.mem_off[nbcc], -1);
#pragma omp parallel for schedule(static)
  for (int32_t x = 0; x < n; ++x)
    if (tbcc[x] >= 0) S.members[S.mem_off[tbcc[x]] + S.locid[x]] = x;
#pragma omp parallel for schedule(static)
  for (int32_t b = 0; b < nbcc; ++b) S.members[S.mem_off[b + 1] - 1] = S.head[b];
}

int decompose(const bc_graph *g, bc_decomp *D) {
  auto t0 = std::chrono::steady_clock::now();
  const int32_t n = g->n;
  const int64_t *R = g->row.data();
  const int32_t *C = g->col.data();

  Split SP;
  split_bccs(g, SP);
  const int32_t nbcc = SP.nbcc;
  const std::vector<int32_t> &comp = SP.comp, &tbcc = SP.tbcc, &pre = SP.pre, &head = SP.head,
                             &locid = SP.locid;
  const std::vector<int64_t> &comp_size = SP.comp_size, &hang = SP.hang, &sq = SP.sq, &mem_off = SP.mem_off;
  bcg::SplitResult out;

  // ---- articulation cross terms: S^2 - sum of squared parts of comp - x
  out.art.assign((size_t)n, 0.0);
  int32_t n_art = 0;
#pragma omp parallel for schedule(static) reduction(+ : n_art)
  for (int32_t x = 0; x < n; ++x) {
    const int64_t S = comp_size[comp[x]] - 1, up = S - hang[x];
    const int64_t a = S * S - sq[x] - up * up;
    out.art[x] = (double)a;
    n_art += a > 0;
  }

  // ---- BCC of every arc: the BCC of the tree edge into its endpoint with the larger pre
  const int64_t n_slots = mem_off.back();
  auto local_of = [&](int32_t x, int32_t b) -> int32_t {
    return x == head[b] ? (int32_t)(mem_off[b + 1] - mem_off[b] - 1) : locid[x];
  };
  // A member slot (b, local id of x in b) only receives arcs of x itself, so
  // both passes run in parallel over x with each slot filled in x's arc order.
  std::vector<int64_t> sdeg((size_t)n_slots + 1, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int32_t x = 0; x < n; ++x)
    for (int64_t e = R[x]; e < R[x + 1]; ++e) {
      int32_t y = C[e];
      int32_t b = tbcc[pre[x] > pre[y] ? x : y];
      sdeg[mem_off[b] + local_of(x, b) + 1]++;
    }
  for (int64_t s = 0; s < n_slots; ++s) sdeg[s + 1] += sdeg[s];
  std::vector<int32_t> sadj((size_t)sdeg[n_slots]);
  {
    std::vector<int64_t> fill(sdeg.begin(), sdeg.end() - 1);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t x = 0; x < n; ++x)
      for (int64_t e = R[x]; e < R[x + 1]; ++e) {
        int32_t y = C[e];
        int32_t b = tbcc[pre[x] > pre[y] ? x : y];
        sadj[fill[mem_off[b] + local_of(x, b)]++] = local_of(y, b);
      }
  }
  out.nbcc = nbcc;
  out.n_art = n_art;
  out.comp = std::move(SP.comp);
  out.head = std::move(SP.head);
  out.members = std::move(SP.members);
  out.comp_size = std::move(SP.comp_size);
  out.below = std::move(SP.below);
  out.hang = std::move(SP.hang);
  out.mem_off = std::move(SP.mem_off);
  out.sdeg = std::move(sdeg);
  out.sadj = std::move(sadj);
  return bcg::decomp_pack(out, n, D, t0);
}

}  // namespace

namespace bcg {

int decomp_pack(SplitResult &SR, int32_t n, bc_decomp *D, std::chrono::steady_clock::time_point t0) {
  const int32_t nbcc = SR.nbcc, n_art = SR.n_art;
  const std::vector<int32_t> &comp = SR.comp, &head = SR.head, &members = SR.members, &sadj = SR.sadj;
  const std::vector<int64_t> &comp_size = SR.comp_size, &below = SR.below, &hang = SR.hang, &mem_off = SR.mem_off,
                             &sdeg = SR.sdeg;
  D->art = std::move(SR.art);

  // ---- pack BCCs with >= 3 vertices, largest first
  std::vector<int32_t> order;
  for (int32_t b = 0; b < nbcc; ++b)
    if (mem_off[b + 1] - mem_off[b] >= 3) order.push_back(b);
  std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
    return (mem_off[a + 1] - mem_off[a]) > (mem_off[b + 1] - mem_off[b]);
  });
  const int32_t np_bcc = (int32_t)order.size();
  D->vtx_off.assign((size_t)np_bcc + 1, 0);
  D->chain_off.assign((size_t)np_bcc + 1, 0);
  D->n_plain.assign((size_t)np_bcc, 0);
  for (int32_t i = 0; i < np_bcc; ++i) {
    int32_t b = order[i];
    D->vtx_off[i + 1] = D->vtx_off[i] + (mem_off[b + 1] - mem_off[b]);
  }
  const int64_t n_packed = D->vtx_off[np_bcc];
  D->row.assign((size_t)n_packed + 1, 0);
  D->reach.assign((size_t)n_packed, 0);
  D->orig.assign((size_t)n_packed, 0);
  for (int32_t i = 0; i < np_bcc; ++i) {
    int32_t b = order[i];
    for (int64_t k = mem_off[b]; k < mem_off[b + 1]; ++k) (void)k;
  }
  // arc offsets need the final ids; compute per BCC, in parallel
  std::vector<std::vector<int32_t>> perm((size_t)np_bcc);           // new local -> old local
  std::vector<std::vector<int32_t>> ch_start((size_t)np_bcc), ch_len((size_t)np_bcc), ch_l((size_t)np_bcc),
      ch_r((size_t)np_bcc);
  std::vector<int64_t> n_cycle((size_t)np_bcc, 0);
  // Large BCCs are handled one at a time with their chain walks in parallel,
  // the others one BCC per thread; the result is the same either way.
  constexpr int32_t kBigBcc = 1 << 16;
  auto order_bcc = [&](int32_t i, bool par) -> int {
    int bad = 0;
    const int32_t b = order[i];
    const int32_t nb = (int32_t)(mem_off[b + 1] - mem_off[b]);
    const int64_t *sd = sdeg.data() + mem_off[b];
    auto deg = [&](int32_t k) { return (int32_t)(sd[k + 1] - sd[k]); };
    auto adj = [&](int32_t k) { return sadj.data() + sd[k]; };
    const int32_t *vid = members.data() + mem_off[b];  // local id -> vertex id
    bool cycle = true;
    int32_t root = 0;
    for (int32_t k = 0; k < nb; ++k) {
      if (deg(k) != 2) cycle = false;
      if (deg(k) > deg(root) || (deg(k) == deg(root) && vid[k] < vid[root])) root = k;
    }
    n_cycle[i] = cycle;
    // plain (non-chain) vertices in BFS order from the max-degree vertex (the
    // smallest vertex id among equals); large BCCs level-synchronously, in
    // the same order
    std::vector<int32_t> nid((size_t)nb, -1), old;
    old.reserve((size_t)nb);
    {
      std::vector<int32_t> q;
      if (par) {
        // adjacency lists follow the CSR's arc order, i.e. increasing vertex id
        q = bfs_exact_order(nb, root, [&](int32_t x, const int32_t **a) { *a = adj(x); return deg(x); },
                            [&](int32_t x) { return vid[x]; });
      } else {
        std::vector<char> seen((size_t)nb, 0);
        q.reserve((size_t)nb);
        q.push_back(root);
        seen[root] = 1;
        for (size_t h = 0; h < q.size(); ++h) {
          const int32_t x = q[h];
          const int32_t *a = adj(x);
          for (int32_t j = 0; j < deg(x); ++j)
            if (!seen[a[j]]) { seen[a[j]] = 1; q.push_back(a[j]); }
        }
      }
      for (const int32_t x : q)
        if (cycle || deg(x) != 2) { nid[x] = (int32_t)old.size(); old.push_back(x); }
      if ((int32_t)q.size() != nb) bad = 1;  // a BCC is connected
    }
    const int32_t nplain = (int32_t)old.size();
    if (!cycle && !bad) {
      // Chains, in the order of a scan of the plain vertices (BFS order) and
      // their arcs: a chain is numbered from whichever end comes first, its
      // vertices from that end. Pass 1 finds, per plain vertex, the chains it
      // owns (the far end comes later) and their lengths; prefix sums give
      // every chain's and vertex's position; pass 2 writes them.
      auto walk = [&](int32_t x, int32_t cur, int32_t *len) {  // far end of the chain leaving x through cur
        int32_t prev = x, k = 0;
        while (deg(cur) == 2 && k <= nb) {
          const int32_t *c2 = adj(cur);
          const int32_t nx = c2[0] == prev ? c2[1] : c2[0];
          prev = cur;
          cur = nx;
          ++k;
        }
        *len = k;
        return cur;
      };
      std::vector<int64_t> cnt((size_t)nplain + 1, 0), vcnt((size_t)nplain + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024) if (par) reduction(| : bad)
      for (int32_t f = 0; f < nplain; ++f) {
        const int32_t x = old[f];
        const int32_t *a = adj(x);
        for (int32_t j = 0; j < deg(x); ++j) {
          if (deg(a[j]) != 2) continue;
          int32_t len;
          const int32_t far = walk(x, a[j], &len);
          if (len > nb || far == x) { bad = 1; continue; }  // no end, or a chain back to its start
          if (nid[far] < f) continue;                       // numbered from its other end
          cnt[f + 1] += 1;
          vcnt[f + 1] += len;
        }
      }
      if (!bad) {
        for (int32_t f = 0; f < nplain; ++f) {
          cnt[f + 1] += cnt[f];
          vcnt[f + 1] += vcnt[f];
        }
        old.resize((size_t)(nplain + vcnt[nplain]));
        ch_start[i].resize((size_t)cnt[nplain]);
        ch_len[i].resize((size_t)cnt[nplain]);
        ch_l[i].resize((size_t)cnt[nplain]);
        ch_r[i].resize((size_t)cnt[nplain]);
#pragma omp parallel for schedule(dynamic, 1024) if (par)
        for (int32_t f = 0; f < nplain; ++f) {
          const int32_t x = old[f];
          const int32_t *a = adj(x);
          int64_t c = cnt[f];
          int32_t pos = (int32_t)(nplain + vcnt[f]);
          for (int32_t j = 0; j < deg(x); ++j) {
            if (deg(a[j]) != 2) continue;
            int32_t len;
            const int32_t far = walk(x, a[j], &len);
            if (nid[far] < f) continue;
            ch_start[i][c] = pos;
            ch_len[i][c] = len;
            ch_l[i][c] = f;
            ch_r[i][c] = nid[far];
            ++c;
            int32_t cur = a[j], prev = x;
            for (int32_t k = 0; k < len; ++k) {
              nid[cur] = pos;
              old[pos++] = cur;
              const int32_t *c2 = adj(cur);
              const int32_t nx = c2[0] == prev ? c2[1] : c2[0];
              prev = cur;
              cur = nx;
            }
          }
        }
      }
    }
    if ((int32_t)old.size() != nb) bad = 1;
    perm[i] = std::move(old);
    D->n_plain[i] = nplain;
    return bad;
  };
  int bad = 0;
  for (int32_t i = 0; i < np_bcc; ++i)
    if (mem_off[order[i] + 1] - mem_off[order[i]] >= kBigBcc) bad |= order_bcc(i, true);
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int32_t i = 0; i < np_bcc; ++i)
    if (mem_off[order[i] + 1] - mem_off[order[i]] < kBigBcc) bad |= order_bcc(i, false);
  if (bad) return BCGPU_EINVAL;

  // ---- write packed arrays
  for (int32_t i = 0; i < np_bcc; ++i) {
    const int32_t b = order[i];
    const int64_t base = D->vtx_off[i];
    for (size_t k = 0; k < perm[i].size(); ++k) {
      int32_t o = perm[i][k];
      D->row[base + (int64_t)k + 1] = sdeg[mem_off[b] + o + 1] - sdeg[mem_off[b] + o];
    }
  }
  for (int64_t k = 0; k < n_packed; ++k) D->row[k + 1] += D->row[k];
  if (D->row[n_packed] > (int64_t)INT32_MAX * 8) return BCGPU_EOVERFLOW;
  D->col.assign((size_t)D->row[n_packed], 0);
  // Each BCC writes its own packed range: large BCCs one at a time with their
  // vertices in parallel, the others one BCC per thread.
  auto write_bcc = [&](int32_t i, bool inner_parallel) {
    const int32_t b = order[i];
    const int32_t nb = (int32_t)perm[i].size();
    std::vector<int32_t> inv((size_t)nb);
    for (int32_t k = 0; k < nb; ++k) inv[perm[i][k]] = k;
    const int64_t base = D->vtx_off[i];
#pragma omp parallel for schedule(dynamic, 4096) if (inner_parallel)
    for (int32_t k = 0; k < nb; ++k) {
      int32_t o = perm[i][k];
      int64_t s = mem_off[b] + o;
      int32_t *dst = D->col.data() + D->row[base + k];
      int64_t d = sdeg[s + 1] - sdeg[s];
      for (int64_t j = 0; j < d; ++j) dst[j] = inv[sadj[sdeg[s] + j]];
      std::sort(dst, dst + d);
      int32_t x = members[s];
      D->orig[base + k] = x;
      D->reach[base + k] =
          (x == head[b]) ? (int32_t)(comp_size[comp[x]] - 1 - below[b]) : (int32_t)hang[x];
    }
  };
  for (int32_t i = 0; i < np_bcc; ++i)
    if ((int32_t)perm[i].size() >= kBigBcc) write_bcc(i, true);
#pragma omp parallel for schedule(dynamic, 1)
  for (int32_t i = 0; i < np_bcc; ++i)
    if ((int32_t)perm[i].size() < kBigBcc) write_bcc(i, false);
  for (int32_t i = 0; i < np_bcc; ++i) D->chain_off[i + 1] = D->chain_off[i] + (int64_t)ch_start[i].size();
  for (int32_t i = 0; i < np_bcc; ++i) {
    D->chain_start.insert(D->chain_start.end(), ch_start[i].begin(), ch_start[i].end());
    D->chain_len.insert(D->chain_len.end(), ch_len[i].begin(), ch_len[i].end());
    D->chain_l.insert(D->chain_l.end(), ch_l[i].begin(), ch_l[i].end());
    D->chain_r.insert(D->chain_r.end(), ch_r[i].begin(), ch_r[i].end());
  }

  int64_t cycles = 0;
  for (auto c : n_cycle) cycles += c;
  decomp_finish(D, n, (int32_t)comp_size.size(), nbcc, n_art, cycles, t0);
  return BCGPU_OK;
}

void decomp_finish(bc_decomp *D, int32_t n, int32_t n_components, int32_t nbcc, int32_t n_art, int64_t n_cycle_bccs,
                   std::chrono::steady_clock::time_point t0) {
  const int32_t np_bcc = (int32_t)D->vtx_off.size() - 1;
  const int64_t n_packed = D->vtx_off[np_bcc];
  bc_bccs &V = D->view;
  V.n_bcc = np_bcc;
  V.n_orig = n;
  V.n_packed = n_packed;
  V.n_arcs = D->row[n_packed];
  V.n_chains = D->chain_off[np_bcc];
  V.vtx_off = D->vtx_off.data();
  V.row = D->row.data();
  V.col = D->col.data();
  V.reach = D->reach.data();
  V.orig = D->orig.data();
  V.n_plain = D->n_plain.data();
  V.chain_off = D->chain_off.data();
  V.chain_start = D->chain_start.data();
  V.chain_len = D->chain_len.data();
  V.chain_l = D->chain_l.data();
  V.chain_r = D->chain_r.data();
  V.art = D->art.data();

  bc_decomp_info &I = D->info;
  I.n_components = n_components;
  I.n_bcc_all = nbcc;
  I.n_bcc_packed = np_bcc;
  I.n_articulation = n_art;
  I.n_chains = V.n_chains;
  I.n_chain_vertices = 0;
  for (auto l : D->chain_len) I.n_chain_vertices += l;
  I.n_cycle_bccs = n_cycle_bccs;
  I.host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace bcg

extern "C" int bc_decompose(const bc_graph *g, bc_decomp **out) {
  if (!g || !out) return BCGPU_EINVAL;
  bc_decomp *D = new (std::nothrow) bc_decomp;
  if (!D) return BCGPU_ENOMEM;
  int rc;
  try {
    rc = decompose(g, D);
  } catch (const std::bad_alloc &) {
    rc = BCGPU_ENOMEM;
  }
  if (rc != BCGPU_OK) { delete D; return rc; }
  *out = D;
  return BCGPU_OK;
}

extern "C" void bc_decomp_free(bc_decomp *d) { delete d; }

extern "C" const bc_bccs *bc_decomp_view(const bc_decomp *d) { return d ? &d->view : nullptr; }

extern "C" void bc_decomp_get_info(const bc_decomp *d, bc_decomp_info *info) {
  if (d && info) *info = d->info;
}
