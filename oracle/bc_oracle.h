/*
 * ORACLE — test infrastructure only. CPU restatement of the reference's exact
 * betweenness-centrality method, used by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg as the CHECKER. Never linked into, or called by,
 * the product library (centrality-gpu_b200/), which has no CPU fallback.
 *
 * Conventions (reference): undirected simple graph, ordered-pair BC (both
 * directions counted, Codes/modified_apsp.cpp:209 "To Match with baders results").
 *
 * Parity status: the decomposition parts (BCC split, reach, articulation cross
 * terms, degree-2 chains with ld/rd) are pinned against the reference's own host
 * pipeline run here (oracle/ref and the tests/golden ref dumps); BC values are pinned
 * against networkx's independent Brandes (the tests/golden bc fixtures).
 */
#ifndef BC_ORACLE_H
#define BC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Ground truth: plain Brandes on the whole graph (CSR with int64 row offsets),
 * FP64 dependencies and path counts. Accumulates
 * bc_out[v] += sum over listed sources s of delta_s(v)   (ordered pairs).
 * sources == NULL means all vertices. OpenMP over sources, static schedule,
 * per-thread partials reduced in thread order (deterministic). */
void orc_brandes(int32_t n, const int64_t *R, const int32_t *C, const int32_t *sources, int64_t nsrc,
                 int nthreads, double *bc_out);

/* BFS rows from s: d[v] (-1 unreachable) and sigma[v] (FP64, exact below 2^53).
 * Follows the level/sigma definition of the reference's forward phase
 * (Codes/kernels_free.cu:245-362). */
void orc_bfs_rows(int32_t n, const int64_t *R, const int32_t *C, int32_t s, int32_t *d, double *sigma);

/* Brute-force decomposition of an edge list (duplicates / self loops must be
 * removed by the caller). Independent of the product's DFS-based split:
 *   edge_bcc[e]  BCC id of edge e (ids numbered by smallest edge index)
 *   art_term[v]  ordered pairs separated by v: S^2 - sum(part_i^2) over the
 *                components of G - v adjacent to v (Codes/modified_apsp.cpp:157-220)
 * Returns the number of BCCs. O(n*m). */
int32_t orc_decompose(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int32_t *edge_bcc,
                      double *art_term);

/* reach_out[v] for BCC `bcc` (after orc_decompose): number of vertices outside
 * the BCC that hang off v, i.e. lie in components of G - v holding no other
 * vertex of the BCC; -1 for vertices not in the BCC
 * (Codes/modified_apsp.cpp:157-220, Codes/to_eargraph_construct.cpp:151-160). */
void orc_reach(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc,
               int32_t bcc, int32_t *reach_out);

/* The whole reference method on a small graph, restated: BCC split, reach,
 * articulation cross terms, per-BCC sources — free and chain-endpoint sources
 * by BFS, degree-2 chain sources by merging their endpoints' rows
 * (Codes/postprocesses.cu:276-363 incl. the chain walk :205-274) — and the
 * reach-weighted backward sweep (Codes/kernels_free.cu:377-426). Writes BC
 * (ordered pairs) into bc_out (overwritten). Returns number of BCCs. */
int32_t orc_method_bc(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int nthreads, double *bc_out);

/* Per-BCC kernel restatement on the packed format the GPU library consumes:
 * one BCC with local CSR (R has nb+1 entries, C local ids), reach per local
 * vertex, and degree-2 chains as contiguous local-id ranges
 * [chain_start[c], chain_start[c]+chain_len[c]) running from endpoint
 * chain_l[c] to chain_r[c]. For each listed source: chain vertices take the
 * merged rows of their endpoints, all others a BFS; then the backward sweep.
 * bc_local[v] += (reach[s]+1) * delta_s(v). Used as the timed CPU baseline. */
void orc_bcc_sources(int32_t nb, const int64_t *R, const int32_t *C, const int32_t *reach, int32_t n_chains,
                     const int32_t *chain_start, const int32_t *chain_len, const int32_t *chain_l,
                     const int32_t *chain_r, const int32_t *sources, int64_t nsrc, int nthreads, double *bc_local);

/* Rows of one source as the method defines them (merge for chain vertices,
 * BFS otherwise) on the packed per-BCC format above. */
void orc_bcc_source_rows(int32_t nb, const int64_t *R, const int32_t *C, int32_t n_chains,
                         const int32_t *chain_start, const int32_t *chain_len, const int32_t *chain_l,
                         const int32_t *chain_r, int32_t s, int32_t *d, double *sigma);

/* The same decomposition in linear time (iterative Hopcroft-Tarjan over an
 * explicit edge stack; articulation terms from the DFS subtree sizes), with
 * orc_decompose's outputs and numbering. For graphs beyond the brute force's
 * reach (the RMAT workloads); pinned against orc_decompose by the tests. */
int32_t orc_decompose_linear(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, int32_t *edge_bcc,
                             double *art_term);

/* Vertices and edges of BCC b (edge_bcc from either decomposition). */
void orc_bcc_size(int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc, int32_t n, int32_t b,
                  int32_t *nb_out, int64_t *mb_out);

/* BCC b in the packed per-BCC format of orc_bcc_sources, built by the
 * oracle alone: vert_out[k] original id of local vertex k (non-chain vertices
 * first, then each maximal degree-2 path from chain_l to chain_r), R [nb+1],
 * C [2 mb] local ids, reach_out [nb] (vertices outside the BCC hanging off
 * the vertex, from DFS subtree sizes), chains (arrays of nb entries).
 * Returns the number of chains. */
int32_t orc_pack_bcc(int32_t n, int64_t m, const int32_t *eu, const int32_t *ev, const int32_t *edge_bcc, int32_t b,
                     int32_t *vert_out, int64_t *R, int32_t *C, int32_t *reach_out, int32_t *chain_start,
                     int32_t *chain_len, int32_t *chain_l, int32_t *chain_r);

#ifdef __cplusplus
}
#endif
#endif
