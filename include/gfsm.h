/*
 * gfsm.h -- C ABI of the B200 GFSM subgraph matcher (libgfsm.so).
 *
 * The reference has no FFI layer: its boundary is the `./GFSM <query> <data>`
 * CLI (main.cu:56-65) and the HnSetup C++ namespace (HnGPU.cuh:60-80), with
 * global device buffers and exit() on every error.  This header is the
 * replacement boundary: opaque handles, plain pointers and sizes, a status
 * code on every call, 64-bit counts.  The GFSM CLI, the Python package and
 * the batched / served drivers all call through it.
 *
 * Semantics (the reference's, kept bit-exact): non-induced, injective,
 * edge-label-checked subgraph matching where each query vertex is placed in
 * the reference's matching order and checked against the reference's
 * requirement table; every automorphic image counts (on symmetric inputs the
 * matcher enumerates one embedding per orbit of the query's automorphism
 * group and multiplies, see gfsm_plan_symmetry -- the count is the same);
 * vertex labels are ignored unless gfsm_limits.vertex_labels is set.
 */
#ifndef GFSM_H
#define GFSM_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The non-zero values below 256 are the reference's process
 * exit codes for the same failure (HnHelper.cuh:16-19, ccsr.cpp:127,195,
 * HnGPU.cu:811,918), so the CLI can exit with them unchanged. */
typedef enum {
    GFSM_OK = 0,
    GFSM_ERR_QUERY = 1,          /* disconnected / unplannable query (ccsr.cpp:126-128, 192-196) */
    GFSM_ERR_MISSING_FILE = 232, /* HnHelper.cuh:16 */
    GFSM_ERR_INVALID_DATA = 233, /* HnHelper.cuh:17 */
    GFSM_ERR_MISSING_DATA = 234, /* HnHelper.cuh:18 */
    GFSM_ERR_ARG = 300,          /* bad argument / handle */
    GFSM_ERR_CUDA = 301,         /* a CUDA runtime call failed */
    GFSM_ERR_NOMEM = 302,        /* MEMLIMIT too small for the graph or one frontier step */
    GFSM_ERR_TOO_LARGE = 303,    /* graph or query beyond the supported sizes */
    GFSM_ERR_DEVICE_WAIT = 304,  /* reserved: a bounded device-side wait ran out (no kernel waits today) */
    GFSM_ERR_NO_EXTENSION = 305, /* no CUDA device / kernels unavailable */
    GFSM_ERR_BUSY = 306,         /* server queue full */
    GFSM_ERR_STOPPED = 307       /* server stopped */
} gfsm_status;

/* Environment.h knobs (Environment.h:6-11).  Defaults are the reference's;
 * gfsm_limits_default() also applies GFSM_<NAME> environment overrides. */
typedef struct {
    uint32_t ccsr_rel_size;    /* CCSRRelSize: edge-label bits kept (1..8), default 8          */
    uint64_t max_soln_size;    /* MAXSOLNSIZE: max partial mappings held per frontier level   */
    uint64_t max_scan_size;    /* MAXSCANSIZE: max candidates examined by one frontier step   */
    uint64_t mem_limit;        /* MEMLIMIT: device bytes the matcher may hold (graph+frontier) */
    uint64_t upper_mem_limit;  /* UPPERMEMLIMIT: cap on any mem_limit override                */
    int32_t  vertex_labels;    /* 0 = reference semantics (labels ignored), 1 = must match    */
    int32_t  degree_filter;    /* 1 = skip candidates whose degree is below the query degree
                                  (count-preserving; applied only to symmetric graphs)       */
    uint64_t max_candidates;   /* stop a call with GFSM_ERR_TOO_LARGE once this many
                                  candidates were examined; 0 = no cap                        */
} gfsm_limits;

typedef struct gfsm_ctx gfsm_ctx;
typedef struct gfsm_graph gfsm_graph;
typedef struct gfsm_plan gfsm_plan;
typedef struct gfsm_server gfsm_server;

typedef struct {
    uint32_t n;            /* vertices (header count)                          */
    uint64_t m;            /* directed adjacency entries                       */
    uint32_t rows;         /* vertices with at least one entry                 */
    uint32_t max_degree;
    int32_t  symmetric;    /* every entry u->v has a v->u entry                */
    int32_t  multi_edges;  /* some (u,v) pair appears more than once           */
    int32_t  n_edge_labels;/* distinct edge labels (after CCSRRelSize masking) */
    int32_t  on_device;    /* device CCSR built                                */
    uint64_t device_bytes;
    /* device CCSR build (0 until built): allocation, host-to-device copies,
     * device passes, copies back (CUDA events), and host wall time, ms */
    double   build_alloc_ms, build_h2d_ms, build_kernel_ms, build_d2h_ms, build_wall_ms;
} gfsm_graph_info;

typedef struct {
    uint64_t count;              /* embeddings (the reference's "Function Count") */
    uint64_t expansions;         /* partial mappings produced, all levels          */
    uint64_t candidates;         /* candidates examined, all levels                */
    uint64_t alg_bytes;          /* algorithmic bytes (parent tuples + backward-neighbour rows + child tuples) */
    uint64_t steps;              /* frontier steps launched                        */
    uint64_t retries;            /* steps re-run with a smaller chunk              */
    uint64_t peak_frontier_bytes;/* most device bytes of partial mappings held at once
                                    (measured: the live depth buffers after each step) */
    double   kernel_ms;          /* device time of the level-step kernels (sum)    */
    double   device_ms;          /* device timeline of the call: first step to last */
    double   wall_ms;            /* host wall time of the call                     */
    uint64_t h2d_bytes;          /* host->device bytes copied by the call          */
    uint64_t d2h_bytes;          /* device->host bytes copied by the call          */
    int32_t  tile_variant;       /* tile geometry the autotuner chose (0..3)        */
    uint32_t launches;           /* kernels the call launched (graph nodes included) */
    int32_t  driver;             /* 1: the whole schedule ran as one CUDA graph launch;
                                    0: the host-driven step loop                   */
    int32_t  graph_error;        /* a graph was wanted but could not be built (cudaError_t) */
} gfsm_stats;

typedef struct {
    uint64_t req_id;
    uint64_t count;
    int32_t  status;
    double   submit_ms;          /* times relative to gfsm_serve_start */
    double   start_ms;
    double   done_ms;
} gfsm_result;

typedef struct {
    int32_t  slots;              /* concurrent device batches (streams), default 2   */
    int32_t  max_batch;          /* queries per device batch, default 256            */
    int32_t  queue_capacity;     /* pending requests, default 65536                  */
    uint64_t frontier_bytes;     /* admission budget per slot (sum of the batch's predicted
                                    frontier bytes); 0 = 8 x mem_limit / slots */
} gfsm_serve_config;

/* --- context ----------------------------------------------------------- */
void        gfsm_limits_default(gfsm_limits *lim);
/* replaces HnSetup::preinit (HnGPU.cu:847-862): binds a device, records the
 * knobs; frontier memory is allocated lazily and bounded by mem_limit.
 * device == -1 gives a host-only context (parsing and planning only; every
 * matching call then returns GFSM_ERR_NO_EXTENSION). */
gfsm_status gfsm_init(gfsm_ctx **ctx, const gfsm_limits *lim, int device);
void        gfsm_destroy(gfsm_ctx *ctx);
const char *gfsm_status_str(gfsm_status s);
const char *gfsm_last_error(gfsm_ctx *ctx);

/* --- graphs ------------------------------------------------------------ */
/* replaces fileParse (HnHelper.cuh:283-499): parses `t # / v / e` text on the
 * host (multi-threaded) and, for data graphs, builds the CCSR on the device.
 * A regular file is mapped read-only while it is parsed, not copied: another
 * process truncating it meanwhile faults this one (SIGBUS), as with any
 * mapping. */
gfsm_status gfsm_graph_load_text(gfsm_ctx *ctx, const char *path, gfsm_graph **out);
gfsm_status gfsm_graph_load_buffer(gfsm_ctx *ctx, const char *buf, uint64_t len, gfsm_graph **out);
/* Directed edge list (give both directions for an undirected graph).
 * elabel may be NULL (all labels 1), vlabel may be NULL (all 0). */
gfsm_status gfsm_graph_from_edges(gfsm_ctx *ctx, uint32_t n, uint64_t m,
                                  const uint32_t *src, const uint32_t *dst,
                                  const uint32_t *elabel, const uint32_t *vlabel,
                                  gfsm_graph **out);
/* Builds the device CCSR now (otherwise done on first use as a data graph). */
gfsm_status gfsm_graph_to_device(gfsm_ctx *ctx, gfsm_graph *g);
gfsm_status gfsm_graph_info_get(const gfsm_graph *g, gfsm_graph_info *info);
/* Copies of the device CCSR in the reference's row order: rowptr[n+1],
 * adj[m] (row index of the target), elab[m], order[n] (row -> original id).
 * Any pointer may be NULL. */
gfsm_status gfsm_graph_download(gfsm_ctx *ctx, const gfsm_graph *g, uint32_t *rowptr,
                                uint32_t *adj, uint8_t *elab, uint32_t *order);
void        gfsm_graph_destroy(gfsm_graph *g);

/* --- query planning ---------------------------------------------------- */
/* replaces HnSetup::preProcessQuery (HnGPU.cu:749-816) and
 * CCSR::genereateCCSRRequirements (ccsr.cpp:98-204): the reference's
 * matching order and requirement table. */
gfsm_status gfsm_query_prepare(gfsm_ctx *ctx, const gfsm_graph *query, gfsm_plan **out);
/* Plans a query for one data graph: where the embedding count cannot depend
 * on the matching order (query and data symmetric with equal labels both
 * ways, no repeated edge), a data-aware order -- root with the fewest data
 * candidates per query edge, then the seen vertex with the most placed
 * neighbours, then the fewest candidates; otherwise the reference's order.
 * No counterpart in the reference (its order is fixed, ccsr.cpp:114-123).
 * The plan counts the same embeddings; matching it against another data
 * graph is allowed but may be slower. */
gfsm_status gfsm_query_prepare_for(gfsm_ctx *ctx, const gfsm_graph *query, const gfsm_graph *data,
                                   gfsm_plan **out);
/* planner: 0 the reference's order, 1 data-aware; order_invariant: 1 if the
 * query's count cannot depend on the order.  Either pointer may be NULL. */
gfsm_status gfsm_plan_info(const gfsm_plan *p, uint32_t *planner, uint32_t *order_invariant);
/* Symmetry breaking of an order-invariant query: its automorphism group has
 * *aut elements (keeping vertex labels when the context matches them), and
 * counting only embeddings f with f(cond[2i]) < f(cond[2i+1]) for every
 * i < *n_cond (query vertex ids, any fixed order of data vertices) and
 * multiplying by *aut gives the full count -- which the matcher does for
 * symmetric, single-edge-label data without repeated edges (not for mapping
 * rows; GFSM_SYMMETRY=0 disables it).  No counterpart in the reference,
 * which enumerates every automorphic image.  cond holds 2*(k-1)*k entries at
 * most; any pointer may be NULL. */
gfsm_status gfsm_plan_symmetry(const gfsm_plan *p, uint64_t *aut, uint32_t *n_cond, uint32_t *cond);
/* gfsm_graph_from_edges + gfsm_query_prepare (data == NULL) or
 * gfsm_query_prepare_for (data given) for nq queries in one call, spread
 * over the host's threads.  No counterpart in the reference, which plans one
 * query per process (main.cu:56-65); for the batched and served forms.
 * Query i has nv[i] vertices and the directed edges [eoff[i], eoff[i+1]) of
 * src/dst/elabel (ids local to the query); its vertex labels are the next
 * nv[i] entries of vlabel (query after query).  elabel / vlabel may be NULL.
 * On success out[i] is query i's plan; on failure every out[i] is NULL,
 * *failed (if given) is the first failing query and that query's status is
 * returned. */
gfsm_status gfsm_query_prepare_batch(gfsm_ctx *ctx, int nq, const uint32_t *nv, const uint64_t *eoff,
                                     const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                     const uint32_t *vlabel, const gfsm_graph *data, gfsm_plan **out,
                                     int *failed);
/* The plan in the reference's buffer layout: order[k] (query row index per
 * depth), header[3k] {numReqs, reqOffset, firstQ}, reqs[2*maxValency*k]
 * {distance delta, relation bits}.  Any output pointer may be NULL. */
gfsm_status gfsm_plan_tables(const gfsm_plan *p, uint32_t *k, uint32_t *max_valency,
                             uint32_t *order, uint32_t *header, uint32_t *reqs);
/* Query vertex id (as in the query file) placed at each depth. */
gfsm_status gfsm_plan_columns(const gfsm_plan *p, uint32_t *qvid);
void        gfsm_plan_destroy(gfsm_plan *p);
/* gfsm_plan_destroy for n plans at once (NULL entries are skipped), e.g. the
 * output of gfsm_query_prepare_batch.  No counterpart in the reference. */
void        gfsm_plan_destroy_array(gfsm_plan *const *plans, int n);

/* --- matching ---------------------------------------------------------- */
/* replaces HnSetup::solve / gpuLaunch (HnGPU.cu:710-1063): one query. */
gfsm_status gfsm_match_count(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data,
                             uint64_t *count, gfsm_stats *stats);
/* Full mappings (hnWrite, HnGPU.cu:674-699, with the query-column mapping
 * done right): rows[i*k + c] = data vertex id matched to query vertex c.
 * Writes min(count, max_rows) rows; *count is the exact total. */
gfsm_status gfsm_match_mappings(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data,
                                uint32_t *rows, uint64_t max_rows, uint64_t *n_rows,
                                uint64_t *count, gfsm_stats *stats);
/* No counterpart in the reference.  Counts one query like gfsm_match_count
 * but allocates no device memory: no cudaMalloc / cudaFree / cudaMallocHost /
 * cudaMallocAsync and no stream or event creation.  It is meant for callers
 * that may not allocate during a match -- a fixed device-memory budget or
 * pool, a latency-critical path that cannot take cudaMalloc/cudaFree's
 * implicit synchronisation.  All scratch lives in one fixed 64 MiB device
 * array inside libgfsm.so (held on each device that loads the library until
 * the process exits); data's device CCSR must already exist
 * (gfsm_graph_to_device), and the work runs on `stream` (a cudaStream_t,
 * NULL = the default stream).  Every call looks up the array's device
 * address; the first call on a device may load the module: make it before
 * any stream capture.  Every call shares the array, so calls that overlap on
 * the GPU (other streams, other host threads) race and must be serialised;
 * a call that fails waits for its own queued work before it returns.  A
 * query that cannot fit one tile of frontier per level in the array returns
 * GFSM_ERR_TOO_LARGE, as does one that passes the candidate cap
 * (max_candidates) of data's context. */
gfsm_status gfsm_match_count_noalloc(const gfsm_plan *plan, const gfsm_graph *data, void *stream,
                                     uint64_t *count);
/* Many queries against one resident data graph in one device pass (at most
 * 4,194,303 queries per call; more return GFSM_ERR_TOO_LARGE). */
gfsm_status gfsm_batch_count(gfsm_ctx *ctx, const gfsm_plan *const *plans, int nq,
                             const gfsm_graph *data, uint64_t *counts, gfsm_stats *stats);

/* --- root partition across GPUs ---------------------------------------- */
/* No counterpart in the reference (its FFS runs on one GPU).  FFS subtrees
 * under different root candidates are independent, so a query's count is
 * the sum of counts over disjoint parts of its root window -- the data
 * vertices its first query vertex may map to, in the order the first level
 * step takes them.  One process per GPU, each with the data graph on its
 * device, counts its own part; the parts' counts are summed (one 8-byte
 * value per query: an all-reduce or a host sum).
 *
 * gfsm_partition_rows: the cut itself, host only.  [lo, hi) is a window of
 * CCSR rows, rowptr the CCSR row pointer (rowptr[hi] valid); writes
 * bounds[0..nparts], offsets into the window, so that part k =
 * [lo + bounds[k], lo + bounds[k+1]) holds about 1/nparts of the window's
 * entries (a root's entries are its first expansion). */
gfsm_status gfsm_partition_rows(const uint32_t *rowptr, uint32_t lo, uint32_t hi, uint32_t nparts,
                                uint64_t *bounds);
/* The cut of plan's root window against data (built on the device first);
 * *window_lo receives the window's first internal id. */
gfsm_status gfsm_root_partition(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data, uint32_t nparts,
                                uint32_t *window_lo, uint64_t *bounds);
/* gfsm_batch_count restricted to part `part` (0 <= part < nparts) of every
 * query's root window: summed over the nparts parts, the counts equal
 * gfsm_batch_count's. */
gfsm_status gfsm_batch_count_part(gfsm_ctx *ctx, const gfsm_plan *const *plans, int nq,
                                  const gfsm_graph *data, uint32_t part, uint32_t nparts, uint64_t *counts,
                                  gfsm_stats *stats);

/* --- serving ------------------------------------------------------------ */
gfsm_status gfsm_serve_start(gfsm_ctx *ctx, const gfsm_graph *data, const gfsm_serve_config *cfg,
                             gfsm_server **out);
/* The served form's admission estimate of a query's peak frontier bytes on
 * `data` (no counterpart in the reference): level counts grown by each
 * level's expected candidate slice and halved per extra requirement; the
 * measured peak of a call is gfsm_stats.peak_frontier_bytes. */
gfsm_status gfsm_predict_frontier_bytes(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data,
                                        double *bytes);
/* The plan is copied; the caller may destroy it after the call. */
gfsm_status gfsm_serve_submit(gfsm_server *s, const gfsm_plan *plan, uint64_t req_id);
/* Non-blocking; returns up to max finished results. */
gfsm_status gfsm_serve_poll(gfsm_server *s, gfsm_result *out, int max, int *n);
/* Blocks until every submitted request has finished (or timeout_ms passes). */
gfsm_status gfsm_serve_drain(gfsm_server *s, double timeout_ms);
gfsm_status gfsm_serve_stop(gfsm_server *s);

#ifdef __cplusplus
}
#endif
#endif
