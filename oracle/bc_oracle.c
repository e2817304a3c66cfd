/*
 * ORACLE — test infrastructure only (see bc_oracle.h). CPU restatement of the
 * reference's exact betweenness-centrality method; the product never links it.
 *
 * Reference anchors:
 *   forward BFS (levels, path counts)  Codes/kernels_free.cu:203-362
 *   successor-form dependency sweep    Codes/kernels_free.cu:377-421 (δ update :391,:409)
 *   source weight reach[s]+1           Codes/kernels_free.cu:423-426
 *   chain merge rule                   Codes/postprocesses.cu:329-351
 *   same-chain walk fix                Codes/postprocesses.cu:205-274
 *   articulation cross term            Codes/modified_apsp.cpp:157-220 (:209)
 *   reach vector                       Codes/to_eargraph_construct.cpp:151-160
 *   BCCs of <= 2 vertices skipped      Codes/to_eargraph_construct.cpp:59
 *   pure cycles: every vertex free     (reference's ear decomposition emits no
 *                                       ear for a cycle BCC; see tests/golden)
 */
#include "bc_oracle.h"

#include <stdlib.h>
#include <string.h>
#include <omp.h>

static void *xmalloc(size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (!p) abort();
  return p;
}

/* ---------------------------------------------------------------- rows ---- */

/* BFS from s over CSR (R,C), filling d (-1 = unreached), sigma and the visit
 * order S (returns its length). */
static int32_t bfs_rows(int32_t n, const int64_t *R, const int32_t *C, int32_t s, int32_t *d, double *sigma,
                        int32_t *S) {
  for (int32_t v = 0; v < n; ++v) { d[v] = -1; sigma[v] = 0.0; }
  int32_t head = 0, tail = 0;
  d[s] = 0; sigma[s] = 1.0; S[tail++] = s;
  while (head < tail) {
    int32_t v = S[head++];
    for (int64_t e = R[v]; e < R[v + 1]; ++e) {
      int32_t w = C[e];
      if (d[w] < 0) { d[w] = d[v] + 1; S[tail++] = w; }
      if (d[w] == d[v] + 1) sigma[w] += sigma[v];
    }
  }
  return tail;
}

void orc_bfs_rows(int32_t n, const int64_t *R, const int32_t *C, int32_t s, int32_t *d, double *sigma) {
  int32_t *S = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  bfs_rows(n, R, C, s, d, sigma, S);
  free(S);
}

/* Successor-form dependency sweep over vertices ordered by level (S holds all
 * reached vertices in nondecreasing d). delta[v] = sum over successors w of
 * sigma[v]/sigma[w] * (wt[w] + delta[w]) with wt[w] = reach[w]+1 (1 if reach
 * is NULL). Adds scale*delta[v] into bc for every v != s. */
static void sweep(int32_t n, const int64_t *R, const int32_t *C, const int32_t *reach, const int32_t *d,
                  const double *sigma, const int32_t *S, int32_t nS, double *delta, double scale, double *bc) {
  (void)n;
  for (int32_t i = nS - 1; i >= 0; --i) {
    int32_t v = S[i];
    double acc = 0.0;
    for (int64_t e = R[v]; e < R[v + 1]; ++e) {
      int32_t w = C[e];
      if (d[w] == d[v] + 1) acc += sigma[v] / sigma[w] * ((reach ? (double)reach[w] + 1.0 : 1.0) + delta[w]);
    }
    delta[v] = acc;
  }
  for (int32_t i = 1; i < nS; ++i) bc[S[i]] += scale * delta[S[i]];  /* S[0] is the source */
}

void orc_brandes(int32_t n, const int64_t *R, const int32_t *C, const int32_t *sources, int64_t nsrc, int nthreads,
                 double *bc_out) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  int64_t ns = sources ? nsrc : n;
  double *part = (double *)calloc((size_t)nthreads * (size_t)n, sizeof(double));
  if (!part) abort();
#pragma omp parallel num_threads(nthreads)
  {
    int t = omp_get_thread_num();
    int32_t *d = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    int32_t *S = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
    double *sigma = (double *)xmalloc(sizeof(double) * (size_t)n);
    double *delta = (double *)xmalloc(sizeof(double) * (size_t)n);
    double *mine = part + (size_t)t * (size_t)n;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < ns; ++i) {
      int32_t s = sources ? sources[i] : (int32_t)i;
      int32_t nS = bfs_rows(n, R, C, s, d, sigma, S);
      sweep(n, R, C, NULL, d, sigma, S, nS, delta, 1.0, mine);
    }
    free(d); free(S); free(sigma); free(delta);
  }
  for (int t = 0; t < nthreads; ++t)
    for (int32_t v = 0; v < n; ++v) bc_out[v] += part[(size_t)t * (size_t)n + v];
  free(part);
}

/* ------------------------------------------------- chain (merged) rows ---- */

static int32_t find_chain(int32_t n_chains, const int32_t *chain_start, const int32_t *chain_len, int32_t z) {
  int32_t lo = 0, hi = n_chains - 1;
  while (lo <= hi) {
    int32_t mid = (lo + hi) / 2;
    if (z < chain_start[mid]) hi = mid - 1;
    else if (z >= chain_start[mid] + chain_len[mid]) lo = mid + 1;
    else return mid;
  }
  return -1;
}

/* Rows of source s: BFS unless s lies on a degree-2 chain, in which case the
 * endpoint rows are merged: d = min(dL+ld, dR+rd); sigma from the strictly
 * shorter side, the sum on ties (Codes/postprocesses.cu:334-350); then the
 * chain's own vertices are fixed by walking the chain both ways
 * (Codes/postprocesses.cu:205-274): shorter direct distance -> sigma 1, equal
 * -> sigma + 1. Scratch: dl, sl, dr, sr of length nb. Returns 1 if merged. */
static int source_rows(int32_t nb, const int64_t *R, const int32_t *C, int32_t n_chains, const int32_t *chain_start,
                       const int32_t *chain_len, const int32_t *chain_l, const int32_t *chain_r, int32_t s,
                       int32_t *d, double *sigma, int32_t *dl, double *sl, int32_t *dr, double *sr,
                       int32_t *S) {
  int32_t c = n_chains > 0 ? find_chain(n_chains, chain_start, chain_len, s) : -1;
  if (c < 0) { bfs_rows(nb, R, C, s, d, sigma, S); return 0; }
  int32_t pos = s - chain_start[c];
  int32_t ld = pos + 1, rd = chain_len[c] - pos;
  bfs_rows(nb, R, C, chain_l[c], dl, sl, S);
  bfs_rows(nb, R, C, chain_r[c], dr, sr, S);
  for (int32_t k = 0; k < nb; ++k) {
    int32_t a = dl[k] + ld, b = dr[k] + rd;
    if (a < b) { d[k] = a; sigma[k] = sl[k]; }
    else if (a > b) { d[k] = b; sigma[k] = sr[k]; }
    else { d[k] = b; sigma[k] = sl[k] + sr[k]; }
  }
  for (int32_t j = 0; j < chain_len[c]; ++j) {
    int32_t k = chain_start[c] + j;
    int32_t dist = j > pos ? j - pos : pos - j;
    if (d[k] > dist) { d[k] = dist; sigma[k] = 1.0; }
    else if (d[k] == dist) sigma[k] += 1.0;
  }
  return 1;
}

/* Orders the reached vertices of a row by level (counting sort) into S. */
static int32_t order_by_level(int32_t nb, const int32_t *d, int32_t *S, int32_t *cnt /* nb+1 */) {
  int32_t maxd = 0;
  for (int32_t k = 0; k < nb; ++k) if (d[k] > maxd) maxd = d[k];
  memset(cnt, 0, sizeof(int32_t) * (size_t)(maxd + 2));
  for (int32_t k = 0; k < nb; ++k) if (d[k] >= 0) cnt[d[k] + 1]++;
  for (int32_t l = 0; l <= maxd; ++l) cnt[l + 1] += cnt[l];
  for (int32_t k = 0; k < nb; ++k) if (d[k] >= 0) S[cnt[d[k]]++] = k;
  return cnt[maxd];
}

void orc_bcc_source_rows(int32_t nb, const int64_t *R, const int32_t *C, int32_t n_chains, const int32_t *chain_start,
                         const int32_t *chain_len, const int32_t *chain_l, const int32_t *chain_r, int32_t s,
                         int32_t *d, double *sigma) {
  int32_t *dl = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb), *dr = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
  double *sl = (double *)xmalloc(sizeof(double) * (size_t)nb), *sr = (double *)xmalloc(sizeof(double) * (size_t)nb);
  int32_t *S = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
  source_rows(nb, R, C, n_chains, chain_start, chain_len, chain_l, chain_r, s, d, sigma, dl, sl, dr, sr, S);
  free(dl); free(dr); free(sl); free(sr); free(S);
}

void orc_bcc_sources(int32_t nb, const int64_t *R, const int32_t *C, const int32_t *reach, int32_t n_chains,
                     const int32_t *chain_start, const int32_t *chain_len, const int32_t *chain_l,
                     const int32_t *chain_r, const int32_t *sources, int64_t nsrc, int nthreads, double *bc_local) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  double *part = (double *)calloc((size_t)nthreads * (size_t)nb, sizeof(double));
  if (!part) abort();
#pragma omp parallel num_threads(nthreads)
  {
    int t = omp_get_thread_num();
    int32_t *d = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    int32_t *S = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    int32_t *cnt = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(nb + 2));
    int32_t *dl = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb), *dr = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    double *sigma = (double *)xmalloc(sizeof(double) * (size_t)nb);
    double *delta = (double *)xmalloc(sizeof(double) * (size_t)nb);
    double *sl = (double *)xmalloc(sizeof(double) * (size_t)nb), *sr = (double *)xmalloc(sizeof(double) * (size_t)nb);
    double *mine = part + (size_t)t * (size_t)nb;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < nsrc; ++i) {
      int32_t s = sources[i];
      int merged = source_rows(nb, R, C, n_chains, chain_start, chain_len, chain_l, chain_r, s, d, sigma, dl, sl, dr,
                               sr, S);
      int32_t nS = merged ? order_by_level(nb, d, S, cnt) : 0;
      if (!merged) {  /* BFS order is already level order; recount its length */
        nS = 0;
        for (int32_t k = 0; k < nb; ++k) nS += d[k] >= 0;
      }
      sweep(nb, R, C, reach, d, sigma, S, nS, delta, (double)reach[s] + 1.0, mine);
    }
    free(d); free(S); free(cnt); free(dl); free(dr); free(sigma); free(delta); free(sl); free(sr);
  }
  for (int t = 0; t < nthreads; ++t)
    for (int32_t v = 0; v < nb; ++v) bc_local[v] += part[(size_t)t * (size_t)nb + v];
  free(part);
}

/* ------------------------------------------------ brute-force split ----- */

typedef struct { int32_t *p; } uf_t;
static int32_t uf_find(int32_t *p, int32_t x) {
  while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
  return x;
}
static void uf_union(int32_t *p, int32_t a, int32_t b) {
  a = uf_find(p, a); b = uf_find(p, b);
  if (a == b) return;
  if (a < b) p[b] = a; else p[a] = b;
}

/* CSR over the edge list that remembers the edge index of every arc. */
static void edge_csr(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int64_t **Rp, int32_t **Cp,
                     int64_t **Ep) {
  int64_t *R = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  int32_t *C = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * m));
  int64_t *E = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(2 * m));
  for (int64_t e = 0; e < m; ++e) { R[eu[e] + 1]++; R[ev[e] + 1]++; }
  for (int32_t v = 0; v < n; ++v) R[v + 1] += R[v];
  int64_t *fill = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)n);
  memcpy(fill, R, sizeof(int64_t) * (size_t)n);
  for (int64_t e = 0; e < m; ++e) {
    int64_t a = fill[eu[e]]++, b = fill[ev[e]]++;
    C[a] = ev[e]; E[a] = e; C[b] = eu[e]; E[b] = e;
  }
  free(fill);
  *Rp = R; *Cp = C; *Ep = E;
}

/* Components of G - x: label[v] = component id (x gets -1), returns count. */
static int32_t components_without(int32_t n, const int64_t *R, const int32_t *C, int32_t x, int32_t *label,
                                  int32_t *queue) {
  for (int32_t v = 0; v < n; ++v) label[v] = -2;
  label[x] = -1;
  int32_t ncomp = 0;
  for (int32_t r = 0; r < n; ++r) {
    if (label[r] != -2) continue;
    int32_t head = 0, tail = 0;
    queue[tail++] = r; label[r] = ncomp;
    while (head < tail) {
      int32_t v = queue[head++];
      for (int64_t e = R[v]; e < R[v + 1]; ++e) {
        int32_t w = C[e];
        if (label[w] == -2) { label[w] = ncomp; queue[tail++] = w; }
      }
    }
    ++ncomp;
  }
  return ncomp;
}

int32_t orc_decompose(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int32_t *edge_bcc,
                      double *art_term) {
  int64_t *R, *E; int32_t *C;
  edge_csr(n, m, eu, ev, &R, &C, &E);
  int32_t *p = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  for (int64_t e = 0; e < m; ++e) p[e] = (int32_t)e;
  int32_t *label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int32_t *queue = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int64_t *first = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t *size = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(n + 1));
  for (int32_t x = 0; x < n; ++x) {
    int32_t ncomp = components_without(n, R, C, x, label, queue);
    /* two edges at x lie in one BCC iff their far ends stay connected in G - x */
    for (int32_t k = 0; k < ncomp; ++k) { first[k] = -1; size[k] = 0; }
    for (int64_t e = R[x]; e < R[x + 1]; ++e) {
      int32_t comp = label[C[e]];
      if (first[comp] < 0) first[comp] = E[e];
      else uf_union(p, (int32_t)first[comp], (int32_t)E[e]);
    }
    if (art_term) {
      for (int32_t v = 0; v < n; ++v) if (label[v] >= 0) size[label[v]]++;
      double S = 0.0, sq = 0.0;
      for (int32_t k = 0; k < ncomp; ++k)
        if (first[k] >= 0) { S += (double)size[k]; sq += (double)size[k] * (double)size[k]; }
      art_term[x] = S * S - sq;
    }
  }
  /* number BCCs by their smallest edge index */
  int32_t nb = 0;
  int32_t *id = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  for (int64_t e = 0; e < m; ++e) id[e] = -1;
  for (int64_t e = 0; e < m; ++e) {
    int32_t r = uf_find(p, (int32_t)e);
    if (id[r] < 0) id[r] = nb++;
    edge_bcc[e] = id[r];
  }
  free(id); free(p); free(label); free(queue); free(first); free(size); free(R); free(C); free(E);
  return nb;
}

void orc_reach(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc, int32_t bcc,
               int32_t *reach_out) {
  int64_t *R, *E; int32_t *C;
  edge_csr(n, m, eu, ev, &R, &C, &E);
  char *in = (char *)calloc((size_t)n, 1);
  for (int64_t e = 0; e < m; ++e) if (edge_bcc[e] == bcc) { in[eu[e]] = 1; in[ev[e]] = 1; }
  int32_t *label = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int32_t *queue = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int64_t *size = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(n + 1));
  char *touch = (char *)xmalloc((size_t)n + 1);
  for (int32_t x = 0; x < n; ++x) {
    if (!in[x]) { reach_out[x] = -1; continue; }
    int32_t ncomp = components_without(n, R, C, x, label, queue);
    for (int32_t k = 0; k < ncomp; ++k) { size[k] = 0; touch[k] = 0; }
    for (int32_t v = 0; v < n; ++v) {
      if (label[v] < 0) continue;
      size[label[v]]++;
      if (in[v]) touch[label[v]] = 1;
    }
    /* only components adjacent to x can hang off it */
    char *adj = (char *)calloc((size_t)ncomp + 1, 1);
    for (int64_t e = R[x]; e < R[x + 1]; ++e) adj[label[C[e]]] = 1;
    int64_t r = 0;
    for (int32_t k = 0; k < ncomp; ++k) if (adj[k] && !touch[k]) r += size[k];
    free(adj);
    reach_out[x] = (int32_t)r;
  }
  free(in); free(label); free(queue); free(size); free(touch); free(R); free(C); free(E);
}

/* ------------------------------------------------------ whole method ---- */

int32_t orc_method_bc(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int nthreads, double *bc_out) {
  int32_t *edge_bcc = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  double *art = (double *)calloc((size_t)n, sizeof(double));
  int32_t nbcc = orc_decompose(n, m, eu, ev, edge_bcc, art);
  for (int32_t v = 0; v < n; ++v) bc_out[v] = art[v];
  int32_t *reach = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int32_t *loc = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  int32_t *deg = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)n);
  for (int32_t b = 0; b < nbcc; ++b) {
    /* vertex set and induced degrees of BCC b */
    for (int32_t v = 0; v < n; ++v) { loc[v] = -1; deg[v] = 0; }
    int32_t nb = 0;
    int64_t mb = 0;
    for (int64_t e = 0; e < m; ++e) {
      if (edge_bcc[e] != b) continue;
      ++mb; deg[eu[e]]++; deg[ev[e]]++;
      if (loc[eu[e]] < 0) loc[eu[e]] = nb++;
      if (loc[ev[e]] < 0) loc[ev[e]] = nb++;
    }
    if (nb <= 2) continue;
    int32_t *vert = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    for (int32_t v = 0; v < n; ++v) if (loc[v] >= 0) vert[loc[v]] = v;
    int is_cycle = 1;
    for (int32_t i = 0; i < nb; ++i) if (deg[vert[i]] != 2) { is_cycle = 0; break; }
    /* adjacency in first-seen local ids */
    int64_t *R0 = (int64_t *)calloc((size_t)nb + 1, sizeof(int64_t));
    int32_t *C0 = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * mb));
    for (int32_t i = 0; i < nb; ++i) R0[i + 1] = R0[i] + deg[vert[i]];
    int64_t *fill = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)nb);
    memcpy(fill, R0, sizeof(int64_t) * (size_t)nb);
    for (int64_t e = 0; e < m; ++e) {
      if (edge_bcc[e] != b) continue;
      int32_t a = loc[eu[e]], c = loc[ev[e]];
      C0[fill[a]++] = c; C0[fill[c]++] = a;
    }
    /* new ids: non-chain vertices first, then each degree-2 chain contiguous from
     * its endpoint chain_l to chain_r */
    int32_t *nid = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    int32_t *old = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    for (int32_t i = 0; i < nb; ++i) nid[i] = -1;
    int32_t next = 0;
    for (int32_t i = 0; i < nb; ++i)
      if (is_cycle || deg[vert[i]] != 2) { nid[i] = next; old[next] = i; ++next; }
    int32_t maxch = nb;
    int32_t *cs = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)maxch), *cl = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)maxch);
    int32_t *cL = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)maxch), *cR = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)maxch);
    int32_t nch = 0;
    if (!is_cycle) {
      for (int32_t i = 0; i < nb; ++i) {
        if (deg[vert[i]] == 2) continue;
        for (int64_t e = R0[i]; e < R0[i + 1]; ++e) {
          int32_t prev = i, cur = C0[e];
          if (deg[vert[cur]] != 2 || nid[cur] >= 0) continue;
          int32_t start = next;
          while (deg[vert[cur]] == 2) {
            nid[cur] = next; old[next] = cur; ++next;
            int32_t a = C0[R0[cur]], c = C0[R0[cur] + 1];
            int32_t nx = (a == prev) ? c : a;
            prev = cur; cur = nx;
          }
          cs[nch] = start; cl[nch] = next - start; cL[nch] = nid[i]; cR[nch] = cur; /* cur: old id, fixed below */
          ++nch;
        }
      }
      for (int32_t c = 0; c < nch; ++c) cR[c] = nid[cR[c]];
    }
    int64_t *R = (int64_t *)calloc((size_t)nb + 1, sizeof(int64_t));
    int32_t *C = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * mb));
    for (int32_t k = 0; k < nb; ++k) R[k + 1] = R[k] + (R0[old[k] + 1] - R0[old[k]]);
    for (int32_t k = 0; k < nb; ++k) {
      int64_t o = R[k];
      for (int64_t e = R0[old[k]]; e < R0[old[k] + 1]; ++e) C[o++] = nid[C0[e]];
    }
    /* reach per new local id */
    orc_reach(n, m, eu, ev, edge_bcc, b, reach);
    int32_t *rl = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    int32_t *src = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)nb);
    for (int32_t k = 0; k < nb; ++k) { rl[k] = reach[vert[old[k]]]; src[k] = k; }
    double *bcl = (double *)calloc((size_t)nb, sizeof(double));
    orc_bcc_sources(nb, R, C, rl, nch, cs, cl, cL, cR, src, nb, nthreads, bcl);
    for (int32_t k = 0; k < nb; ++k) bc_out[vert[old[k]]] += bcl[k];
    free(bcl); free(src); free(rl); free(R); free(C); free(R0); free(C0); free(fill); free(nid); free(old);
    free(cs); free(cl); free(cL); free(cR); free(vert);
  }
  free(edge_bcc); free(art); free(reach); free(loc); free(deg);
  return nbcc;
}

/* ------------------------------------------------- linear decomposition --- */

/* Depth-first search state of the whole graph (iterative, explicit stacks). */
typedef struct {
  int32_t n, nbcc;
  int64_t *R;          /* adjacency CSR with edge ids */
  int32_t *C, *E;
  int32_t *disc, *low, *parent, *pe, *sub, *root;
  int64_t *sep, *sep_sq; /* per vertex: sum (and sum of squares) of the subtree sizes of its separating children */
} Dfs;

static void dfs_free(Dfs *g) {
  free(g->R); free(g->C); free(g->E); free(g->disc); free(g->low); free(g->parent); free(g->pe); free(g->sub);
  free(g->root); free(g->sep); free(g->sep_sq);
}

/* Hopcroft-Tarjan: edge_bcc[e] gets a BCC id in order of discovery. */
static void dfs_run(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, Dfs *g, int32_t *edge_bcc) {
  g->n = n;
  g->R = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
  g->C = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * m + 1));
  g->E = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * m + 1));
  for (int64_t e = 0; e < m; ++e) { g->R[eu[e] + 1]++; g->R[ev[e] + 1]++; }
  for (int32_t v = 0; v < n; ++v) g->R[v + 1] += g->R[v];
  int64_t *fill = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(n + 1));
  memcpy(fill, g->R, sizeof(int64_t) * (size_t)(n + 1));
  for (int64_t e = 0; e < m; ++e) {
    g->C[fill[eu[e]]] = ev[e]; g->E[fill[eu[e]]++] = (int32_t)e;
    g->C[fill[ev[e]]] = eu[e]; g->E[fill[ev[e]]++] = (int32_t)e;
  }
  size_t nn = (size_t)(n > 0 ? n : 1);
  g->disc = (int32_t *)xmalloc(sizeof(int32_t) * nn); g->low = (int32_t *)xmalloc(sizeof(int32_t) * nn);
  g->parent = (int32_t *)xmalloc(sizeof(int32_t) * nn); g->pe = (int32_t *)xmalloc(sizeof(int32_t) * nn);
  g->sub = (int32_t *)xmalloc(sizeof(int32_t) * nn); g->root = (int32_t *)xmalloc(sizeof(int32_t) * nn);
  g->sep = (int64_t *)calloc(nn, sizeof(int64_t)); g->sep_sq = (int64_t *)calloc(nn, sizeof(int64_t));
  int64_t *it = fill; /* reused as the per-vertex adjacency cursor */
  int32_t *vs = (int32_t *)xmalloc(sizeof(int32_t) * nn);
  int32_t *es = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  for (int32_t v = 0; v < n; ++v) { g->disc[v] = -1; it[v] = g->R[v]; }
  int32_t t = 0, nbcc = 0;
  for (int32_t r = 0; r < n; ++r) {
    if (g->disc[r] >= 0) continue;
    int32_t top = 0;
    int64_t etop = 0;
    vs[top++] = r;
    g->disc[r] = g->low[r] = t++; g->parent[r] = -1; g->pe[r] = -1; g->sub[r] = 1; g->root[r] = r;
    while (top > 0) {
      const int32_t v = vs[top - 1];
      if (it[v] < g->R[v + 1]) {
        const int32_t w = g->C[it[v]], e = g->E[it[v]];
        ++it[v];
        if (e == g->pe[v]) continue;
        if (g->disc[w] < 0) {
          es[etop++] = e;
          g->parent[w] = v; g->pe[w] = e; g->disc[w] = g->low[w] = t++; g->sub[w] = 1; g->root[w] = r;
          vs[top++] = w;
        } else if (g->disc[w] < g->disc[v]) { /* back edge to an ancestor */
          es[etop++] = e;
          if (g->disc[w] < g->low[v]) g->low[v] = g->disc[w];
        }
      } else {
        --top;
        const int32_t p = g->parent[v];
        if (p < 0) continue;
        if (g->low[v] < g->low[p]) g->low[p] = g->low[v];
        g->sub[p] += g->sub[v];
        if (g->low[v] >= g->disc[p]) { /* p separates v's subtree: the edges above it on the stack form a BCC */
          g->sep[p] += g->sub[v];
          g->sep_sq[p] += (int64_t)g->sub[v] * g->sub[v];
          int32_t e;
          do { e = es[--etop]; edge_bcc[e] = nbcc; } while (e != g->pe[v]);
          ++nbcc;
        }
      }
    }
  }
  g->nbcc = nbcc;
  free(fill); free(vs); free(es);
}

int32_t orc_decompose_linear(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int32_t *edge_bcc,
                             double *art_term) {
  Dfs g;
  dfs_run(n, m, eu, ev, &g, edge_bcc);
  /* renumber by smallest edge index (orc_decompose's numbering) */
  int32_t *first = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(g.nbcc > 0 ? g.nbcc : 1));
  int32_t *map = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(g.nbcc > 0 ? g.nbcc : 1));
  for (int32_t b = 0; b < g.nbcc; ++b) first[b] = -1;
  int32_t next = 0;
  for (int64_t e = 0; e < m; ++e)
    if (first[edge_bcc[e]] < 0) { first[edge_bcc[e]] = (int32_t)e; map[edge_bcc[e]] = next++; }
  for (int64_t e = 0; e < m; ++e) edge_bcc[e] = map[edge_bcc[e]];
  /* articulation cross terms: S^2 - sum of squared part sizes, the parts being
   * the separating children's subtrees and (below the root) the rest of the
   * component (Codes/modified_apsp.cpp:157-220) */
  for (int32_t v = 0; v < n; ++v) {
    const int64_t S = (int64_t)g.sub[g.root[v]] - 1;
    int64_t sq = g.sep_sq[v];
    if (g.parent[v] >= 0) {
      const int64_t rest = S - g.sep[v];
      sq += rest * rest;
    }
    art_term[v] = (double)(S * S - sq);
  }
  const int32_t nb = g.nbcc;
  free(first); free(map); dfs_free(&g);
  return nb;
}

/* Vertex count and edge count of BCC b. */
void orc_bcc_size(int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc, int32_t n, int32_t b,
                  int32_t *nb_out, int64_t *mb_out) {
  char *in = (char *)calloc((size_t)(n > 0 ? n : 1), 1);
  int32_t nb = 0;
  int64_t mb = 0;
  for (int64_t e = 0; e < m; ++e) {
    if (edge_bcc[e] != b) continue;
    ++mb;
    if (!in[eu[e]]) { in[eu[e]] = 1; ++nb; }
    if (!in[ev[e]]) { in[ev[e]] = 1; ++nb; }
  }
  free(in);
  *nb_out = nb;
  *mb_out = mb;
}

int32_t orc_pack_bcc(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc, int32_t b,
                     int32_t *vert_out, int64_t *R, int32_t *C, int32_t *reach_out, int32_t *chain_start,
                     int32_t *chain_len, int32_t *chain_l, int32_t *chain_r) {
  /* a fresh DFS for subtree sizes (the BCC partition does not depend on the DFS) */
  int32_t *eb2 = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
  Dfs g;
  dfs_run(n, m, eu, ev, &g, eb2);
  free(eb2);
  int32_t *loc = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  int32_t *deg = (int32_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
  for (int32_t v = 0; v < n; ++v) loc[v] = -1;
  int32_t nb = 0;
  int64_t mb = 0;
  for (int64_t e = 0; e < m; ++e) {
    if (edge_bcc[e] != b) continue;
    ++mb; deg[eu[e]]++; deg[ev[e]]++;
    if (loc[eu[e]] < 0) loc[eu[e]] = nb++;
    if (loc[ev[e]] < 0) loc[ev[e]] = nb++;
  }
  int32_t *vert = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(nb > 0 ? nb : 1));
  for (int32_t v = 0; v < n; ++v) if (loc[v] >= 0) vert[loc[v]] = v;
  /* reach: the head (smallest discovery time) loses everything but the
   * subtree of its child in this BCC; any other vertex keeps exactly the
   * subtrees of its separating children */
  int32_t head = vert[0];
  for (int32_t i = 1; i < nb; ++i) if (g.disc[vert[i]] < g.disc[head]) head = vert[i];
  int32_t cb = -1;
  for (int64_t e = g.R[head]; e < g.R[head + 1]; ++e)
    if (edge_bcc[g.E[e]] == b && g.parent[g.C[e]] == head && g.pe[g.C[e]] == g.E[e]) cb = g.C[e];
  int is_cycle = 1;
  for (int32_t i = 0; i < nb; ++i) if (deg[vert[i]] != 2) { is_cycle = 0; break; }
  int64_t *R0 = (int64_t *)calloc((size_t)nb + 1, sizeof(int64_t));
  int32_t *C0 = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(2 * mb + 1));
  for (int32_t i = 0; i < nb; ++i) R0[i + 1] = R0[i] + deg[vert[i]];
  int64_t *fill = (int64_t *)xmalloc(sizeof(int64_t) * (size_t)(nb > 0 ? nb : 1));
  memcpy(fill, R0, sizeof(int64_t) * (size_t)nb);
  for (int64_t e = 0; e < m; ++e) {
    if (edge_bcc[e] != b) continue;
    const int32_t a = loc[eu[e]], c = loc[ev[e]];
    C0[fill[a]++] = c; C0[fill[c]++] = a;
  }
  /* new ids: non-chain vertices first, then each maximal degree-2 path
   * contiguous from chain_l to chain_r (a cycle BCC has none) */
  int32_t *nid = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(nb > 0 ? nb : 1));
  int32_t *old = (int32_t *)xmalloc(sizeof(int32_t) * (size_t)(nb > 0 ? nb : 1));
  for (int32_t i = 0; i < nb; ++i) nid[i] = -1;
  int32_t next = 0, nch = 0;
  for (int32_t i = 0; i < nb; ++i)
    if (is_cycle || deg[vert[i]] != 2) { nid[i] = next; old[next] = i; ++next; }
  if (!is_cycle) {
    for (int32_t i = 0; i < nb; ++i) {
      if (deg[vert[i]] == 2) continue;
      for (int64_t e = R0[i]; e < R0[i + 1]; ++e) {
        int32_t prev = i, cur = C0[e];
        if (deg[vert[cur]] != 2 || nid[cur] >= 0) continue;
        const int32_t start = next;
        while (deg[vert[cur]] == 2) {
          nid[cur] = next; old[next] = cur; ++next;
          const int32_t a = C0[R0[cur]], c = C0[R0[cur] + 1];
          const int32_t nx = (a == prev) ? c : a;
          prev = cur; cur = nx;
        }
        chain_start[nch] = start; chain_len[nch] = next - start; chain_l[nch] = nid[i]; chain_r[nch] = cur;
        ++nch;
      }
    }
    for (int32_t c = 0; c < nch; ++c) chain_r[c] = nid[chain_r[c]];
  }
  R[0] = 0;
  for (int32_t k = 0; k < nb; ++k) R[k + 1] = R[k] + (R0[old[k] + 1] - R0[old[k]]);
  for (int32_t k = 0; k < nb; ++k) {
    int64_t o = R[k];
    for (int64_t e = R0[old[k]]; e < R0[old[k] + 1]; ++e) C[o++] = nid[C0[e]];
    const int32_t x = vert[old[k]];
    vert_out[k] = x;
    reach_out[k] = x == head ? (cb >= 0 ? g.sub[g.root[x]] - 1 - g.sub[cb] : 0) : (int32_t)g.sep[x];
  }
  free(loc); free(deg); free(vert); free(R0); free(C0); free(fill); free(nid); free(old);
  dfs_free(&g);
  return nch;
}
