/*
 * libbcgpu — exact betweenness centrality on one NVIDIA B200 (sm_100a).
 *
 * C ABI: plain pointers and sizes, status codes, no C++ or torch types.
 * Every entry point returns BCGPU_OK (0) or an error code; the text of the
 * last error is available from bc_last_error(). Nothing here calls exit().
 * There is no CPU fallback: without a usable CUDA device bc_create fails.
 *
 * Method (the reference's, Goutam363/centrality-GPU): the graph is split into
 * biconnected components (BCCs); every BCC of >= 3 vertices runs exact Brandes
 * from each of its vertices, weighting sources and targets by reach + 1 (the
 * number of vertices hanging off that vertex outside the BCC, itself
 * included); sources on degree-2 chains take the merged rows of the chain's
 * endpoints instead of a BFS; articulation points add the pairs they separate.
 * BC counts ordered pairs (both directions).
 */
#ifndef BCGPU_H
#define BCGPU_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status ---- */
enum {
  BCGPU_OK = 0,
  BCGPU_EINVAL = 1,   /* bad argument or malformed input */
  BCGPU_ECUDA = 2,    /* CUDA runtime error (no device, launch failure, ...) */
  BCGPU_ENOMEM = 3,   /* device or host allocation failed / over the workspace limit */
  BCGPU_ETIMEOUT = 4, /* a device-side wait ran out of its iteration limit */
  BCGPU_EIO = 5,      /* file could not be read or parsed */
  BCGPU_EOVERFLOW = 6 /* a size exceeds what the kernels index (e.g. > 2^31-1 arcs per BCC) */
};

/* Computation schedule. PLAIN: one source per CTA at a time, FP64 path
 * counts and dependencies, FP64 atomics into BC. BATCHED: many sources per
 * pass as a bitmask multi-source BFS, FP64 path counts with per-level
 * power-of-two scaling, deterministic FP64 per-block BC partials. */
enum { BCGPU_MODE_PLAIN = 0, BCGPU_MODE_BATCHED = 1 };
/* Dependency (delta) arithmetic for the BATCHED mode. */
enum { BCGPU_DELTA_FP64 = 0, BCGPU_DELTA_FP32C = 1 /* FP32 with two-sum compensated accumulation */ };

typedef struct bc_opts {
  int32_t device;        /* CUDA device ordinal; -1 = highest compute capability (reference choose_device) */
  int32_t mode;          /* BCGPU_MODE_* */
  int32_t delta;         /* BCGPU_DELTA_* (BATCHED only) */
  int32_t batch_width;   /* sources per batched pass: multiple of 32, <= 1024; 0 = 512
                            (bc_autotune_width measures the best width for a graph) */
  void *stream;          /* cudaStream_t to launch on; NULL = a stream owned by the context */
  int64_t workspace_limit; /* device bytes the context may hold; 0 = 80% of free memory */
  int32_t rescale_exp;   /* BATCHED: rescale a level's path counts above 2^rescale_exp; 0 = 900.
                            Lower values only exercise the scaling path (tests). */
  int32_t plain_core;    /* BATCHED: BCCs whose core (the vertices off degree-2 chains) has fewer
                            vertices than this, or whose levels run deeper than 96, use the
                            per-source schedule inside the same plan (small or deep BCCs
                            gain nothing from multi-source passes); 0 = 8192, negative =
                            every BCC in multi-source passes */
  int32_t graph;         /* nonzero: bc_plan_run replays a CUDA graph of each unit range's device
                            work (counter resets + the persistent kernels), recorded by stream
                            capture on bc_plan_record or on the range's first run; 0 = enqueue
                            the work directly on every run. The stream must be capturable
                            (not the legacy NULL stream). */
  int32_t plain_ctas_per_sm; /* per-source schedule: CTAs (sources in flight) per SM; 0 = four
                            256-thread CTAs, fewer and larger when their rows do not fit the
                            workspace budget; 8 or 16 = that many CTAs of 128 or 64 threads
                            (more sources in flight for deep, narrow BCCs), with the same
                            fallback; other values are rejected */
  int32_t lazy_tables;   /* 1 (default): a one-shot bc_run_bccs_units call builds the multi-source
                            slot, seed and arming tables of the passes it runs only (and the
                            source order up to the last of them); 0 = of every pass (the same
                            BC, bit for bit) */
  int32_t tile_max;      /* BATCHED: BCCs routed away from multi-source passes run on the
                            small-BCC schedule (a CTA per range of sources of one BCC, its CSR
                            slice staged in shared memory by a bulk copy, one warp per source)
                            when they have at most tile_max vertices, fit shared memory and
                            cannot overflow FP64 path counts; the others use the per-source
                            schedule. 0 = as large as shared memory allows, -1 = off.
                            No reference counterpart (one source per CTA for every BCC,
                            Codes/begin_gpupgm.cu:52-65). */
  int32_t wait_limit_ms; /* limit of one device-side wait (the multi-source kernel's grid
                            barrier), in milliseconds of device time; a wait that runs out
                            records an error and the run returns BCGPU_ETIMEOUT. 0 = 60000.
                            No reference counterpart: the reference has no device-side
                            waits and exit()s on any CUDA error (Codes/kernels.cuh:25-32). */
} bc_opts;

typedef struct bc_ctx bc_ctx;

/* Fills opts with defaults (device -1, BATCHED, FP32C, width 0 = 512, lazy tables on, graph off). */
void bc_default_opts(bc_opts *opts);
int bc_create(const bc_opts *opts, bc_ctx **out);
/* Releases the context, every plan still alive on it and its device-memory
 * pool (plans allocate from a pool of the context's; memory a destroyed plan
 * held stays reserved for the context's next plans until bc_destroy). */
void bc_destroy(bc_ctx *ctx);
/* Message of the last failing call on ctx (or of bc_create when ctx is NULL). */
const char *bc_last_error(const bc_ctx *ctx);

/* -------------------------------------------------- packed BCC input ---- */
/* All BCCs with >= 3 vertices, each a contiguous range of "packed" vertex ids.
 * Within BCC b (n_b = vtx_off[b+1]-vtx_off[b] vertices) local ids run 0..n_b-1;
 * local ids < n_plain[b] are free vertices or chain endpoints, the rest are
 * degree-2 chain vertices, each chain contiguous from its left endpoint to its
 * right endpoint. Arc lists use LOCAL neighbour ids; row[] holds global arc
 * offsets. */
typedef struct bc_bccs {
  int32_t n_bcc;          /* BCCs listed (>= 3 vertices each) */
  int32_t n_orig;         /* vertices of the original graph: length of BC output */
  int64_t n_packed;       /* total packed vertices = vtx_off[n_bcc] */
  int64_t n_arcs;         /* total arcs = row[n_packed] */
  int64_t n_chains;       /* total chains = chain_off[n_bcc] */
  const int64_t *vtx_off; /* [n_bcc+1] */
  const int64_t *row;     /* [n_packed+1] global arc offsets */
  const int32_t *col;     /* [n_arcs] local neighbour ids */
  const int32_t *reach;   /* [n_packed] vertices hanging off the vertex outside its BCC */
  const int32_t *orig;    /* [n_packed] original vertex id */
  const int32_t *n_plain; /* [n_bcc] */
  const int64_t *chain_off;   /* [n_bcc+1] chain-table range of each BCC */
  const int32_t *chain_start; /* [n_chains] local id of the chain's first vertex (next to chain_l) */
  const int32_t *chain_len;   /* [n_chains] degree-2 vertices on the chain */
  const int32_t *chain_l;     /* [n_chains] local id of the left endpoint */
  const int32_t *chain_r;     /* [n_chains] local id of the right endpoint */
  const double *art;      /* [n_orig] articulation cross terms added to BC; may be NULL */
} bc_bccs;

typedef struct bc_stats {
  int64_t sources;        /* sources whose dependencies were accumulated */
  int64_t bfs_sources;    /* of which ran a forward BFS (the others were merged from chain endpoints) */
  int64_t aux_bfs;        /* extra forward-only BFS runs for chain endpoints */
  int64_t teps_edges;     /* sum over sources of the arcs of the source's BCC (TEPS numerator) */
  double kernel_ms;       /* device time of the BC kernels (CUDA events) */
  double total_ms;        /* device time of the whole call incl. copies */
  int32_t kernel_launches;/* kernels this library launched */
  int32_t batch_width;    /* width used (BATCHED) */
  int64_t h2d_bytes;      /* bytes the call copied host -> device (the packed BCCs and the tables built from them) */
  int64_t d2h_bytes;      /* bytes the call copied device -> host (BC and status words) */
} bc_stats;

/* Whole computation, host buffers in and out: uploads the packed BCCs, runs
 * every source of every BCC, adds the articulation terms and writes the BC of
 * every original vertex (FP64, ordered pairs) to bc_out[n_orig] (overwritten).
 * Replaces the per-BCC pair of begin_gpu calls in the reference's
 * BiCC::to_eargraph loop (Codes/to_eargraph_construct.cpp:54-200). */
int bc_run_bccs(bc_ctx *ctx, const bc_bccs *bccs, double *bc_out, bc_stats *stats);

/* Same, for a subset of the work: units [unit_begin, unit_end) of the plan
 * bc_plan_create would build with this context's options (see below), e.g. a
 * sampled estimate or one shard of a multi-GPU run. bc_out gets the
 * contributions of those units (plus the articulation terms when
 * with_art != 0). Host buffers in and out, uploads included. */
int bc_run_bccs_units(bc_ctx *ctx, const bc_bccs *bccs, int64_t unit_begin, int64_t unit_end, int32_t with_art,
                      double *bc_out, bc_stats *stats);

/* ---------------------------------------------- mirrors of begin_gpu ---- */
/* One BCC, free sources. Mirrors begin_gpu(R,C,F,n,m,ear_info,self_ear,
 * req_nodes,artnodes,bc,time) (reference Codes/ear_graph.h:45-46,
 * Codes/begin_gpupgm.cu:42-71): R[n+1], C[m] with m = number of ARCS (the
 * reference passes 2x edges); sources req_nodes[n_req]; reach = artnodes[n].
 * bc[n] is OVERWRITTEN with this call's contributions (FP64 computed, rounded
 * to float as the reference's buffer type); *time_s is INCREASED by the device
 * seconds spent. The reference's row-of-arc array F is not needed. */
int bc_begin_free(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *req_nodes,
                  int32_t n_req, const int32_t *reach, float *bc, double *time_s);

/* Variant of bc_begin_free that allocates nothing (no reference counterpart).
 * BC is accumulated like the per-source schedule's (fixed-point counters
 * folded to FP64: the same result on every call, whatever the order in which
 * the CTAs finish their sources); the first call on a device clears the
 * array's rows and counters, later calls reuse what the previous call left.
 * For callers that cannot create device allocations of their own -- their
 * device memory belongs to another allocator (a framework's caching pool, an
 * arena budgeted up front), so a cudaMalloc/cudaFree here would break that
 * accounting or stall the device. Inputs and the output are the CALLER's
 * DEVICE buffers: R[n+1], C[m] (m = arcs), req_nodes[n_req], reach[n], and
 * bc[n] (FP64, overwritten). All other working memory is one file-scope
 * __device__ array of about 20 MiB that every GPU loading this library holds
 * until the process exits. Limits: n <= 16384 and n_req <= 16384
 * (BCGPU_EOVERFLOW beyond, with the reason in bc_last_error).
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call reuses the same array and clears what it needs at start; calls
 * that overlap on the GPU (several threads or streams at once) race on it,
 * so serialise them. Runs on the context's stream and returns when done;
 * *time_s (may be NULL) is increased by the device seconds spent. */
int bc_begin_free_noalloc(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m,
                          const int32_t *req_nodes, int32_t n_req, const int32_t *reach, double *bc, double *time_s);

/* One BCC, chain endpoints ("active" vertices) and their chains ("ears").
 * Mirrors the second begin_gpu overload (reference Codes/ear_graph.h:48-49,
 * Codes/begin_gpupgm.cu:73-89, Codes/kernels_active.cu:18-223 with
 * postprocess Codes/postprocesses.cu:8-203). Ears are flattened: ear e runs
 * from lnode[e] to rnode[e] through cnt[e] degree-2 vertices
 * nodes[off[e] .. off[e]+cnt[e]) with path distances ld/rd to the two ends
 * (ear_premble, Codes/ear_graph.h:3-32). Every active vertex and every ear
 * vertex is a source. bc[n] is READ and the contributions ADDED (the
 * reference seeds its device buffer from bc, Codes/kernels_active.cu:78);
 * *time_s is increased. */
int bc_begin_active(bc_ctx *ctx, const int32_t *R, const int32_t *C, int32_t n, int32_t m, const int32_t *active,
                    int32_t n_active, int32_t n_ears, const int32_t *lnode, const int32_t *rnode, const int32_t *cnt,
                    const int32_t *off, const int32_t *nodes, const int32_t *ld, const int32_t *rd,
                    const int32_t *reach, float *bc, double *time_s);

/* Self-check of the bounded device-side wait (no reference counterpart): runs
 * a one-CTA kernel whose thread 0 waits, with the same wait primitive as the
 * multi-source kernel's grid barrier, on a device flag that nothing sets,
 * with a limit of limit_ms (> 0) milliseconds. The wait runs out, so the call
 * returns BCGPU_ETIMEOUT (the status a plan run returns when one of its waits
 * runs out) and the context stays usable. *waited_ms (may be NULL) receives
 * the device time the kernel took. */
int bc_wait_probe(bc_ctx *ctx, int32_t limit_ms, double *waited_ms);

/* ------------------------------------ device-resident plans (benchmark) -- */
/* A plan uploads the packed BCCs once and keeps the BC accumulator on the
 * device. Work is split into units (PLAIN: one free/endpoint source plus the
 * chains it owns; BATCHED: one multi-source pass); running a range of units
 * accumulates their contributions. */
typedef struct bc_plan bc_plan;
int bc_plan_create(bc_ctx *ctx, const bc_bccs *bccs, bc_plan **out);
/* Must not be called after bc_destroy of the plan's context (which already
 * released it). The plan's device memory returns to the context's pool,
 * ordered on its stream: a later plan of the context reuses it without a new
 * device allocation (the workspace limit counts it as free). */
void bc_plan_destroy(bc_plan *plan);
int64_t bc_plan_num_units(const bc_plan *plan);
/* Work covered by units [begin, end): sources, TEPS arcs (sum over sources of
 * their BCC's arcs) and vertex visits (sum over sources of their BCC's
 * vertices); any output may be NULL. */
int bc_plan_unit_work(const bc_plan *plan, int64_t begin, int64_t end, int64_t *sources, int64_t *teps_edges,
                      int64_t *vertex_visits);
/* Packed ids of the sources whose dependencies units [begin, end) accumulate
 * (forward-only helper BFS runs excluded). Writes up to cap ids to out and
 * returns the total count (negative error code on failure). */
int64_t bc_plan_unit_sources(const bc_plan *plan, int64_t begin, int64_t end, int64_t *out, int64_t cap);
/* Device buffers the plan consumes (for roofline accounting). */
int64_t bc_plan_device_bytes(const bc_plan *plan);
/* The small-BCC schedule's launches, in launch order: each one's CTA class
 * (0 warp per source; 1, 2, 3: one source per 256-, 512-, 1024-thread CTA;
 * 4, 5: a 1024-thread CTA of two / four source groups) and grid size. Writes
 * up to cap entries; returns the number of launches (negative error code on
 * failure). Introspection for tests and tools; no reference counterpart. */
int bc_plan_tile_launches(const bc_plan *plan, int32_t *cls, int32_t *grid, int32_t cap);
/* Work units that run at once: PLAIN, the resident CTAs (one item each);
 * BATCHED, 1 (one pass at a time over the whole GPU). No reference
 * counterpart: the reference launches one source at a time. */
int bc_plan_concurrency(const bc_plan *plan);

/* Batch-width autotuner (no reference counterpart: the reference has one
 * source per launch). For each candidate width 128, 256, 512, 1024 it builds a
 * BATCHED plan of these BCCs with ctx's other options, times up to
 * `passes` multi-source passes from the middle of the source order (after one
 * warm-up pass) and writes the fastest width to *width; gteps_out (4 entries,
 * may be NULL) receives each candidate's TEPS / 1e9 (0 if it did not fit). A
 * plan without multi-source passes (every BCC routed per-source) leaves
 * *width = 0. Pass the width back as bc_opts.batch_width. */
int bc_autotune_width(bc_ctx *ctx, const bc_bccs *bccs, int32_t passes, int32_t *width, double *gteps_out);
int bc_plan_reset(bc_plan *plan);
/* Enqueues units [begin, end) on the context's stream; asynchronous unless
 * stats is non-NULL (then synchronises and fills it). With bc_opts.graph set
 * the work is one cudaGraphLaunch of the range's recorded graph. */
int bc_plan_run(bc_plan *plan, int64_t begin, int64_t end, bc_stats *stats);
/* Graph mode (bc_opts.graph != 0) only: records the device work of units
 * [begin, end) into a CUDA graph by stream capture and instantiates it,
 * WITHOUT running it, so that later bc_plan_run calls of that exact range are
 * single graph launches (recording again replaces the graph). Each recorded
 * range keeps its instantiated graph until the plan is destroyed. No reference
 * counterpart: the reference launches kernels one source batch at a time
 * from host loops (Codes/kernels_active.cu:98-180). */
int bc_plan_record(bc_plan *plan, int64_t begin, int64_t end);
/* Synchronises, copies BC to the host and adds the articulation terms. */
int bc_plan_read(bc_plan *plan, double *bc_out);
/* Levels and path counts of one source (packed id) as the GPU computes them
 * (BFS, or the chain merge for chain vertices); d_out/sigma_out have the
 * source's BCC size. For parity tests. */
int bc_plan_source_rows(bc_plan *plan, int64_t packed_source, int32_t *d_out, double *sigma_out);
/* Multi-source pass `unit` (a unit below the plan's pass count): with null
 * outputs, its slot count and its BCC's core vertex count only; else the pass
 * is run (its BC contributions are added like any run's) and read back:
 * src_out[b] = slot b's source (local id in the BCC), and for each slot b and
 * core vertex v, d_out[b * ncore + v] its level and sigma_out[b * ncore + v]
 * its path count with the per-level power-of-two bases applied. For parity
 * tests of the multi-source form against per-source BFS (the reference keeps
 * its per-source levels and counts in d_d / sigma_d, Codes/kernels_free.cu:55-62). */
int bc_plan_pass_rows(bc_plan *plan, int64_t unit, int32_t *nslots, int32_t *ncore, int32_t *src_out, int32_t *d_out,
                      double *sigma_out);

#ifdef __cplusplus
}
#endif
#endif /* BCGPU_H */
