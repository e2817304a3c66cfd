/*
 * libbcgpu host side — graph ingest and the decomposition that feeds the GPU.
 * Same C ABI conventions as bcgpu.h (status codes, no exit()).
 *
 * Replaces the reference's host pipeline ahead of begin_gpu:
 *   Graph::Graph(char*)                Codes/graph.cpp:38-59     -> bc_graph_load / bc_graph_from_edges
 *   BiCC::run_bicc / bicc_tarjan       Codes/bicc.cpp:39,81-161  -> bc_decompose (parallel, no recursion)
 *   per-BCC relabel                    Codes/modified_apsp.cpp:273-363
 *   fillbccparent / reachfunction      Codes/modified_apsp.cpp:77-220 (reach, articulation terms)
 *   bcc_bfs + preSum (ear chains)      Codes/bcc_bfs.cpp:247-1330, :100-236
 *   parse_active_nodes / read_ear_info Codes/make_ear_graph.cpp:119-218, Codes/readeardata.cpp:117-192
 */
#ifndef BCHOST_H
#define BCHOST_H
#include "bcgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Simple undirected graph in CSR (self loops dropped, duplicate edges merged). */
typedef struct bc_graph bc_graph;

/* Reads the reference's edge-list file: "n m" then m lines "u v w" (0-based,
 * w ignored as in the reference's BFS). Writes a message to err on failure.
 * A file written by bc_graph_save (it starts with the bytes "BCGCSR1\0") is
 * read as that CSR instead, with no parsing: it must describe a simple
 * undirected graph (sorted adjacency, no loops or duplicates, every arc
 * mirrored), else BCGPU_EIO with the reason. */
int bc_graph_load(const char *path, bc_graph **out, char *err, size_t errlen);
/* Writes g's CSR in the binary form bc_graph_load reads back: the 8 bytes
 * "BCGCSR1\0", int32 n, int32 0, int64 arcs, int64 row[n+1], int32 col[arcs]
 * (host byte order). A cache of a large edge list: reloading it skips the
 * text parse, the deduplication and the sort. No reference counterpart (the
 * reference re-reads the text file every run, Codes/graph.cpp:38-59). */
int bc_graph_save(const bc_graph *g, const char *path, char *err, size_t errlen);
int bc_graph_from_edges(int32_t n, int64_t m, const int32_t *u, const int32_t *v, bc_graph **out);
void bc_graph_free(bc_graph *g);
/* Borrowed views of the CSR: row[n+1] (int64), col[row[n]] (int32). */
int bc_graph_csr(const bc_graph *g, int32_t *n, int64_t *n_arcs, const int64_t **row, const int32_t **col);

typedef struct bc_decomp bc_decomp;
typedef struct bc_decomp_info {
  int32_t n_components;   /* connected components (isolated vertices included) */
  int32_t n_bcc_all;      /* all BCCs incl. bridges */
  int32_t n_bcc_packed;   /* BCCs of >= 3 vertices (those with BFS work) */
  int32_t n_articulation;
  int64_t n_chain_vertices;
  int64_t n_chains;
  int64_t n_cycle_bccs;   /* BCCs that are a single cycle: all their vertices are free sources */
  double host_ms;         /* wall time of bc_decompose */
} bc_decomp_info;

/* Splits g into BCCs, computes reach and articulation terms, finds degree-2
 * chains and packs every BCC of >= 3 vertices (largest first; equal sizes in
 * the order of their smallest vertex other than the head, the member closest
 * to the smallest vertex of the component). The result depends only on g,
 * not on the host thread count. */
int bc_decompose(const bc_graph *g, bc_decomp **out);
/* bc_decompose as data-parallel steps on GPU `device`: the BCC split, the
 * arc-to-member pass and the packing (BFS order, chains, packed CSR); prefix
 * sums, the regrouping of the BFS order by BCC and the sort of rows longer
 * than 32 arcs run on the host. The result is the same as bc_decompose's.
 * device < 0 runs the same steps as host loops instead: a check of the GPU
 * steps on a machine without one, slower than bc_decompose. Writes a message
 * to err on failure (BCGPU_ECUDA without a usable device). */
int bc_decompose_gpu(const bc_graph *g, int device, bc_decomp **out, char *err, size_t errlen);
void bc_decomp_free(bc_decomp *d);
/* Borrowed view, valid until bc_decomp_free. */
const bc_bccs *bc_decomp_view(const bc_decomp *d);
void bc_decomp_get_info(const bc_decomp *d, bc_decomp_info *info);

#ifdef __cplusplus
}
#endif
#endif /* BCHOST_H */
