/*
 * gfsm_oracle.h -- CPU oracle for the GFSM forest-based subgraph matching path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (libgfsm, the GFSM CLI,
 * the gfsm_b200 package) links, loads or calls this code.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg use it,
 * and only as the checker or as the timed CPU baseline.
 *
 * Three independent pieces:
 *   1. orc_parse_*   : restatement of the reference text parser / CCSR builder
 *                      (HnHelper.cuh:283-499 fileParse, parseValues :191-266),
 *                      kept "wide" (separate target offset and label arrays)
 *                      so it also works past the reference's 24-bit field.
 *   2. orc_plan      : restatement of the reference planner
 *                      (HnGPU.cu:749-816 preProcessQuery,
 *                       ccsr.cpp:98-204 genereateCCSRRequirements,
 *                       ccsr.cpp:206-219 getMaxValency).
 *   3. orc_ffs_count : restatement of the FFS count semantics
 *                      (HnGPU.cu:76-109 hnInit, :114-185 hnGen,
 *                       :190-262 hnCheck, :34-52 reqExists, :455-669 hnSolve),
 *                      evaluated depth-first with 64-bit counts.
 *   4. orc_bt_count  : an independent backtracking enumerator working on the
 *                      raw edge lists (no CCSR, no planner): label-preserving
 *                      subgraph monomorphism, optional vertex labels.
 *
 * Parity is pinned (a) against the reference's own parser and planner
 * compiled from its sources into oracle/_ref (see oracle/Makefile), and
 * (b) by agreement of 3 and 4 plus closed-form counts.
 */
#ifndef GFSM_ORACLE_H
#define GFSM_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Wide CCSR as produced by the reference parser.  seg_val[i] is the row
 * degree at a row header and the target value of an edge entry otherwise
 * (the target's row offset when the label bits are non-zero, the raw vertex
 * id otherwise -- exactly HnHelper.cuh:452-460).  seg_lab[i] is the label
 * field of entry i (0 at row headers). */
typedef struct {
    uint32_t n;          /* vertex count from the header line              */
    uint64_t size;       /* number of CCSR segments (rows + entries)       */
    uint32_t rows;       /* number of rows (vertices of degree >= 1)       */
    uint32_t *seg_val;   /* [size]                                         */
    uint32_t *seg_lab;   /* [size]                                         */
    uint32_t *vlocs;     /* verticeLocs[n]   vertex id -> row offset       */
    uint32_t *inv;       /* invVerticeLocs[n] sorted position -> vertex id */
    uint32_t maxlen;     /* stagger size (max degree)                      */
    uint32_t *staggers;  /* [maxlen]                                       */
    uint32_t *sinfo;     /* [2*maxlen] StaggerInfo {offset, normOffset}    */
    uint32_t *vlabel;    /* [n] vertex label per vertex id (v lines)       */
    uint32_t n_edges;    /* edge lines seen                                */
    uint32_t *e_src, *e_dst, *e_lab; /* raw edge lines [n_edges] (label = value as parsed) */
    int32_t err;         /* 0, or the reference's exit code (232/233/234/1) */
} orc_graph;

/* Planner output: identical layout to the reference's buffers. */
typedef struct {
    uint32_t k;          /* query vertex count                             */
    uint32_t max_valency;
    uint32_t rel_bits;   /* relations are stored as label << (32-rel_bits) */
    uint32_t *reqs;      /* [2*max_valency*k] (dist delta, relation bits)  */
    uint32_t *header;    /* [3*k] (numReqs, reqOffset, firstQ)             */
    uint32_t *order;     /* [k] query row index mapped at each depth       */
    int32_t err;         /* 0 or 1 (the reference exits with 1)            */
} orc_plan_t;

int  orc_parse_file(const char *path, uint32_t rel_bits, orc_graph *g);
int  orc_parse_buffer(const char *buf, uint64_t len, uint32_t rel_bits, orc_graph *g);
void orc_graph_free(orc_graph *g);

int  orc_plan(const orc_graph *q, uint32_t rel_bits, orc_plan_t *p);
void orc_plan_free(orc_plan_t *p);

/* Pack the wide CCSR into the reference's 32-bit segments (only meaningful
 * while every offset fits in 32-rel_bits bits). */
void orc_pack_segments(const orc_graph *g, uint32_t rel_bits, uint32_t *out);

/* Reference-semantics count (64-bit).  vlabel_mode adds the constraint
 * vlabel(data) == vlabel(query) (off reproduces the reference).  Returns 0 on
 * success.  If rows_out is non-NULL and max_rows > 0, up to max_rows full
 * mappings are written as original vertex ids, columns ordered by original
 * query vertex id; *n_rows receives the number written. */
int orc_ffs_count(const orc_graph *q, const orc_plan_t *p, const orc_graph *d,
                  int vlabel_mode, int threads, uint64_t *count,
                  uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows);
/* orc_ffs_count over the roots in CCSR rows [root_begin, root_end) only (the
 * rows the reference's hnInit takes in that order): the counts of
 * consecutive row ranges add up to the whole count. */
int orc_ffs_count_rows(const orc_graph *q, const orc_plan_t *p, const orc_graph *d,
                       int vlabel_mode, int threads, uint32_t root_begin, uint32_t root_end, uint64_t *count,
                       uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows);

/* Independent backtracking enumerator over raw edge lists. */
int orc_bt_count(uint32_t qn, uint32_t qm, const uint32_t *qs, const uint32_t *qd,
                 const uint32_t *ql, const uint32_t *qvl,
                 uint32_t dn, uint64_t dm, const uint32_t *ds, const uint32_t *dd,
                 const uint32_t *dl, const uint32_t *dvl,
                 uint32_t rel_bits, int vlabel_mode, int threads, uint64_t *count,
                 uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows);

/* Triangles of an undirected simple graph given as edges (u < v). */
int orc_triangles(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, int threads,
                  uint64_t *count);
/* The same enumeration, histogrammed by vertex labels: hist[(a*nl + b)*nl + c]
 * = embeddings of the 3-vertex triangle query whose vertices carry labels
 * (a, b, c) in query order (each triangle counts once per ordering of its
 * vertices); *count = triangles.  vlabel[v] < nl <= 64. */
int orc_triangle_label_hist(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                            const uint32_t *vlabel, uint32_t nl, int threads, uint64_t *hist, uint64_t *count);

#ifdef __cplusplus
}
#endif
#endif
