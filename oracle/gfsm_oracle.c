/*
 * gfsm_oracle.c -- CPU oracle for the GFSM forest-based subgraph matching path.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU legs of bench.py as the checker / timed CPU baseline.  The product never
 * links or calls it.  See gfsm_oracle.h for the map from each function to the
 * reference file:line it restates.
 */
#define _GNU_SOURCE
#include "gfsm_oracle.h"
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ERR_MISSING_FILE 232 /* HnHelper.cuh:16 */
#define ERR_INVALID_DATA 233 /* HnHelper.cuh:17 */
#define ERR_MISSING_DATA 234 /* HnHelper.cuh:18 */

/* ------------------------------------------------------------------------- */
/* 1. Parser + CCSR builder (HnHelper.cuh:191-266 parseValues,               */
/*    HnHelper.cuh:283-499 fileParse)                                        */
/* ------------------------------------------------------------------------- */

enum { P_COMPLETE, P_FAIL, P_EDGES, P_END };
enum { M_HEADER, M_VERTEX, M_EDGE };

/* One line of the `t # / v / e` format, tokenised the way parseValues does:
 * maximal digit runs are values, every other byte advances to the next value
 * slot, '\n' ends the line (HnHelper.cuh:233-263).  Digits accumulate with
 * 32-bit wrap-around like the reference's uint32_t arithmetic. */
static int parse_values(const char **s, const char *end, uint32_t *values, int mode)
{
    if (*s >= end) return P_END; /* the reference reads past the buffer here */
    char ch = **s;
    if (ch == 't') { /* HnHelper.cuh:196-201 */
        if (end - *s < 6 || strncmp(*s, "t # -1", 6)) return P_FAIL;
        return P_END;
    }
    switch (mode) {
    case M_HEADER: *s -= 2; break;                 /* HnHelper.cuh:206-210 */
    case M_VERTEX:
        if (ch == 'e') return P_EDGES;             /* :213-215 */
        if (ch != 'v') return P_FAIL;              /* :216-218 */
        break;
    default:
        if (ch != 'e') return P_FAIL;              /* :224-226 */
        break;
    }
    uint32_t cur = 0;
    for (*s += 2; *s < end; (*s)++) {
        ch = **s;
        if (ch >= '0' && ch <= '9') {
            if (cur < 4) values[cur] = values[cur] * 10u + (uint32_t)(ch - '0');
        } else {
            cur++;
            if (ch == '\n') { (*s)++; break; }
        }
    }
    return P_COMPLETE;
}

typedef struct { uint32_t id, size; } ord_pair;

/* HnHelper.cuh:26-31: degree descending, then vertex id ascending. */
static int ord_cmp(const void *a, const void *b)
{
    const ord_pair *x = a, *y = b;
    if (x->size != y->size) return x->size > y->size ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

/* A row's entries by target alone, entries of equal target in their input
 * order (pos): what the reference's std::sort with nodeCompare
 * (ccsr.cpp:13-16) leaves them in for rows of up to 16 entries (libstdc++
 * insertion-sorts such ranges) and for rows already in target order, which
 * it does not sort (HnHelper.cuh:469-478).  A longer unsorted row with a
 * repeated target may come out of std::sort in another tie order. */
typedef struct { uint32_t val, lab, pos; } seg_pair;
static int seg_cmp(const void *a, const void *b)
{
    const seg_pair *x = a, *y = b;
    if (x->val != y->val) return x->val < y->val ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

void orc_graph_free(orc_graph *g)
{
    free(g->seg_val); free(g->seg_lab); free(g->vlocs); free(g->inv);
    free(g->staggers); free(g->sinfo); free(g->vlabel);
    free(g->e_src); free(g->e_dst); free(g->e_lab);
    memset(g, 0, sizeof(*g));
}

int orc_parse_buffer(const char *buf, uint64_t len, uint32_t rel_bits, orc_graph *g)
{
    memset(g, 0, sizeof(*g));
    const uint32_t vert_bits = 32u - rel_bits;
    const uint32_t lab_mask = rel_bits >= 32 ? 0xffffffffu : ((1u << rel_bits) - 1u);
    const char *end = buf + len, *s = buf;
    if (len < 6 || strncmp(buf, "t # 0\n", 6)) { g->err = ERR_INVALID_DATA; return g->err; } /* :312-314 */
    s += 6;
    uint32_t values[4] = {0, 0, 0, 0};
    int st = parse_values(&s, end, values, M_HEADER);                       /* :322-325 */
    if (st == P_FAIL) { g->err = ERR_INVALID_DATA; return g->err; }
    const uint32_t n = values[0], ecount = values[1];
    g->n = n;
    g->vlabel = calloc(n ? n : 1, sizeof(uint32_t));

    uint32_t vseen = 0;                                                      /* :333-349 */
    for (st = P_COMPLETE; st == P_COMPLETE;) {
        values[0] = values[1] = 0;
        st = parse_values(&s, end, values, M_VERTEX);
        if (st == P_FAIL) { g->err = ERR_INVALID_DATA; return g->err; }
        if (st == P_END) break;
        if (st == P_COMPLETE && values[0] < n) g->vlabel[values[0]] = values[1];
        vseen++; /* counted for the 'e' line that ends the section too (:344) */
    }
    if (vseen < n) { g->err = ERR_MISSING_DATA; return g->err; }

    uint64_t cap = 1024;
    uint32_t *es = malloc(cap * 4), *ed = malloc(cap * 4), *el = malloc(cap * 4);
    uint32_t eseen = 0;                                                      /* :364-381 */
    for (st = P_COMPLETE; st == P_COMPLETE; eseen++) {
        values[0] = values[1] = values[2] = 0;
        st = parse_values(&s, end, values, M_EDGE);
        if (st == P_FAIL) { g->err = ERR_INVALID_DATA; goto fail_edges; }
        if (st == P_END) break;
        if (values[0] >= n) { g->err = ERR_INVALID_DATA; goto fail_edges; } /* reference: out of bounds */
        if (eseen == cap) {
            cap *= 2;
            es = realloc(es, cap * 4); ed = realloc(ed, cap * 4); el = realloc(el, cap * 4);
        }
        es[eseen] = values[0]; ed[eseen] = values[1]; el[eseen] = values[2];
    }
    if (eseen < ecount) { g->err = ERR_MISSING_DATA; goto fail_edges; }
    g->n_edges = eseen; g->e_src = es; g->e_dst = ed; g->e_lab = el;

    /* Row sizes (insertion order is kept inside each row: Dynamic2D::put). */
    uint32_t *deg = calloc(n ? n : 1, 4);
    for (uint32_t i = 0; i < eseen; i++) deg[es[i]]++;
    uint64_t alloc = 0; uint32_t maxlen = 0, rows = 0;
    ord_pair *ord = malloc(sizeof(ord_pair) * (n ? n : 1));
    for (uint32_t i = 0; i < n; i++) {                                        /* :384-393 */
        if (deg[i]) { alloc += deg[i] + 1; rows++; }
        if (deg[i] > maxlen) maxlen = deg[i];
        ord[i].id = i; ord[i].size = deg[i];
    }
    /* bucket the edges per source row, keeping input order */
    uint64_t *rstart = calloc((uint64_t)n + 1, 8);
    for (uint32_t i = 0; i < n; i++) rstart[i + 1] = rstart[i] + deg[i];
    uint32_t *fill = calloc(n ? n : 1, 4);
    uint32_t *rowv = malloc(((uint64_t)eseen + 1) * 4), *rowl = malloc(((uint64_t)eseen + 1) * 4);
    for (uint32_t i = 0; i < eseen; i++) {
        uint64_t pos = rstart[es[i]] + fill[es[i]]++;
        /* (values[1] & vertMask) | (values[2] << CCSRVertSize)  (:375-376) --
         * the wide form keeps the whole id; the label keeps only the bits
         * that survive the shift. */
        rowv[pos] = ed[i];
        rowl[pos] = vert_bits >= 32 ? 0u : ((uint32_t)(el[i] << vert_bits) >> vert_bits) & lab_mask;
    }
    qsort(ord, n, sizeof(ord_pair), ord_cmp);                                /* :413 */

    g->size = alloc; g->rows = rows; g->maxlen = maxlen;
    g->seg_val = malloc((alloc + 1) * 4); g->seg_lab = calloc(alloc + 1, 4);
    g->vlocs = calloc(n ? n : 1, 4); g->inv = calloc(n ? n : 1, 4);
    g->staggers = calloc(maxlen ? maxlen : 1, 4);
    g->sinfo = calloc(2 * (maxlen ? maxlen : 1), 4);
    uint32_t *dcounts = calloc(maxlen ? maxlen : 1, 4);
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; i++) {                                        /* :417-436 */
        uint32_t v = ord[i].id, sz = ord[i].size;
        g->vlocs[v] = (uint32_t)w;
        g->inv[i] = v;
        if (sz) {
            g->seg_val[w] = sz; g->seg_lab[w] = 0;
            memcpy(&g->seg_val[w + 1], &rowv[rstart[v]], (uint64_t)sz * 4);
            memcpy(&g->seg_lab[w + 1], &rowl[rstart[v]], (uint64_t)sz * 4);
            g->staggers[sz - 1] += sz + 1;
            dcounts[sz - 1]++;
            w += sz + 1;
        }
    }
    if (maxlen) {                                                             /* :443-448 */
        g->sinfo[2 * (maxlen - 1)] = 0; g->sinfo[2 * (maxlen - 1) + 1] = 0;
        for (int64_t i = (int64_t)maxlen - 2; i >= 0; i--) {
            g->sinfo[2 * i] = g->sinfo[2 * (i + 1)] + g->staggers[i + 1];
            g->sinfo[2 * i + 1] = g->sinfo[2 * (i + 1) + 1] + dcounts[i + 1];
        }
    }
    /* Remap targets to row offsets where the label field is non-zero (:452-460). */
    for (uint64_t i = 0; i < alloc;) {
        uint32_t sz = g->seg_val[i];
        for (uint32_t j = 1; j <= sz; j++) {
            if (g->seg_lab[i + j]) {
                uint32_t t = g->seg_val[i + j];
                if (t >= n) { g->err = ERR_INVALID_DATA; break; } /* reference: out of bounds */
                g->seg_val[i + j] = g->vlocs[t];
            }
        }
        i += sz + 1;
    }
    /* Sort every row by target (:469-478). */
    seg_pair *tmp = malloc(sizeof(seg_pair) * (maxlen ? maxlen : 1));
    for (uint64_t i = 0; i < alloc;) {
        uint32_t sz = g->seg_val[i];
        for (uint32_t j = 0; j < sz; j++) { tmp[j].val = g->seg_val[i + 1 + j]; tmp[j].lab = g->seg_lab[i + 1 + j]; tmp[j].pos = j; }
        qsort(tmp, sz, sizeof(seg_pair), seg_cmp);
        for (uint32_t j = 0; j < sz; j++) { g->seg_val[i + 1 + j] = tmp[j].val; g->seg_lab[i + 1 + j] = tmp[j].lab; }
        i += sz + 1;
    }
    free(tmp); free(dcounts); free(rowv); free(rowl); free(fill); free(rstart); free(ord); free(deg);
    return g->err;

fail_edges:
    free(es); free(ed); free(el);
    return g->err;
}

int orc_parse_file(const char *path, uint32_t rel_bits, orc_graph *g)
{
    memset(g, 0, sizeof(*g));
    FILE *f = fopen(path, "rb");
    if (!f) { g->err = ERR_MISSING_FILE; return g->err; }                    /* :289-294 */
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    rewind(f);
    char *buf = malloc(sz > 0 ? sz : 1);
    size_t got = fread(buf, 1, sz > 0 ? (size_t)sz : 0, f);
    fclose(f);
    int r = orc_parse_buffer(buf, got, rel_bits, g);
    free(buf);
    return r;
}

void orc_pack_segments(const orc_graph *g, uint32_t rel_bits, uint32_t *out)
{
    const uint32_t vert_bits = 32u - rel_bits;
    const uint32_t vmask = vert_bits >= 32 ? 0xffffffffu : ((1u << vert_bits) - 1u);
    for (uint64_t i = 0; i < g->size; i++)
        out[i] = (g->seg_val[i] & vmask) | (vert_bits >= 32 ? 0u : (g->seg_lab[i] << vert_bits));
}

/* ------------------------------------------------------------------------- */
/* 2. Planner (HnGPU.cu:749-816, ccsr.cpp:98-219)                            */
/* ------------------------------------------------------------------------- */

/* Requirements by distance alone (ccsr.cpp:82-84, 170), equal distances in
 * the order they were found (pos), as std::sort leaves up to 16 of them. */
typedef struct { uint32_t req, rel, pos; } req_rel;
static int req_cmp(const void *a, const void *b)
{
    const req_rel *x = a, *y = b;
    if (x->req != y->req) return x->req < y->req ? -1 : 1;
    return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

static uint32_t max_valency(const orc_graph *g) /* ccsr.cpp:206-219 */
{
    uint32_t m = 0;
    for (uint64_t i = 0; i < g->size; i += (uint64_t)g->seg_val[i] + 1)
        if (g->seg_val[i] > m) m = g->seg_val[i];
    return m;
}

void orc_plan_free(orc_plan_t *p)
{
    free(p->reqs); free(p->header); free(p->order);
    memset(p, 0, sizeof(*p));
}

/* ccsr.cpp:98-204, one depth.  rowoff[i] is the offset of row i (the
 * reference's localVerticeLocs).  Returns 0, or 1 where the reference exits. */
static int gen_reqs(const orc_graph *q, const uint32_t *rowoff, uint32_t maxv, uint32_t depth,
                    int32_t *mapping, uint32_t *reqs, uint32_t *header, uint32_t *order, uint32_t vert_bits)
{
    const uint32_t count = q->n;
    uint32_t rel_depth = 0; int found = 0;
    for (uint32_t i = 0; i < count; i++) {                                   /* :114-123 */
        if (mapping[i] == 0 && !found) { mapping[i] = 1; rel_depth = i; found = 1; }
        else if (mapping[i] > 0) mapping[i]++;
    }
    if (!found) return 1;                                                    /* :126-128 */
    order[depth] = rel_depth;
    uint64_t row = rowoff[rel_depth];
    uint32_t deg = q->seg_val[row];
    uint32_t nreq = 0, req_off = depth * maxv * 2;
    req_rel *rr = calloc(maxv ? maxv : 1, sizeof(req_rel));
    for (uint32_t e = 0; e < deg; e++) {                                     /* :142-167 */
        uint32_t tgt = q->seg_val[row + 1 + e];
        uint32_t idx = count; /* getIndex: linear find of the row offset */
        for (uint32_t i = 0; i < count; i++) if (rowoff[i] == tgt) { idx = i; break; }
        if (idx >= count) { free(rr); return 1; } /* reference: out of bounds */
        if (mapping[idx] < 0) mapping[idx] = 0;
        if (mapping[idx] > 0) {
            uint32_t rel = q->seg_lab[row + 1 + e];
            uint64_t refl = tgt;
            uint32_t rdeg = q->seg_val[refl];
            for (uint32_t j = 0; j < rdeg; j++) {
                if (q->seg_val[refl + 1 + j] == (uint32_t)row) { rel = q->seg_lab[refl + 1 + j]; break; }
            }
            rr[nreq].req = (uint32_t)(mapping[idx] - 1);
            rr[nreq].rel = vert_bits >= 32 ? 0u : rel << vert_bits; /* relation bits, as packed */
            rr[nreq].pos = nreq;
            nreq++;
        }
    }
    uint32_t firstq = 0;
    if (nreq) {                                                              /* :169-187 */
        qsort(rr, nreq, sizeof(req_rel), req_cmp);
        reqs[req_off] = rr[0].req; reqs[req_off + 1] = rr[0].rel;
        for (uint32_t i = 1; i < nreq; i++) {
            reqs[req_off + 2 * i] = rr[i].req - rr[i - 1].req;
            reqs[req_off + 2 * i + 1] = rr[i].rel;
        }
        firstq = reqs[req_off];
        for (uint32_t i = 0; i < nreq; i++) { firstq = reqs[req_off + 2 * i]; if (firstq) break; }
    }
    free(rr);
    if ((firstq > depth && depth) || (depth && !firstq)) return 1;           /* :192-196 */
    header[depth * 3 + 0] = nreq;
    header[depth * 3 + 1] = req_off;
    header[depth * 3 + 2] = firstq;
    return 0;
}

int orc_plan(const orc_graph *q, uint32_t rel_bits, orc_plan_t *p)
{
    memset(p, 0, sizeof(*p));
    p->rel_bits = rel_bits;
    const uint32_t k = q->n;
    p->k = k;
    if (q->err) { p->err = q->err; return p->err; }
    if (k == 0 || q->rows != k) { p->err = 1; return 1; } /* reference: undefined (walks past the CCSR) */
    uint32_t maxv = max_valency(q);
    p->max_valency = maxv;
    p->reqs = calloc(2 * (uint64_t)maxv * k + 1, 4);
    p->header = calloc(3 * (uint64_t)k, 4);
    p->order = calloc(k, 4);
    int32_t *mapping = malloc(sizeof(int32_t) * k);
    for (uint32_t i = 0; i < k; i++) mapping[i] = -1;
    uint32_t *rowoff = malloc(sizeof(uint32_t) * k);
    uint64_t off = 0;
    for (uint32_t i = 0; i < k; i++) { rowoff[i] = (uint32_t)off; off += q->seg_val[off] + 1; }
    /* HnGPU.cu:759-769: root = the first row of maximal degree (row 0 of a
     * degree-sorted CCSR); mappingData is indexed by that segment offset. */
    uint32_t degval = q->seg_val[0]; uint64_t loc = 0;
    for (uint64_t i = 0; i < q->size; i += (uint64_t)q->seg_val[i] + 1)
        if (degval < q->seg_val[i]) { degval = q->seg_val[i]; loc = i; }
    if (loc >= k) { p->err = 1; goto out; }
    mapping[loc] = 0;
    for (uint32_t d = 0; d < k; d++) {                                        /* :771-773 */
        if (gen_reqs(q, rowoff, maxv, d, mapping, p->reqs, p->header, p->order, 32u - rel_bits)) { p->err = 1; goto out; }
    }
    for (uint64_t i = 0; i < (uint64_t)maxv * k; i++)                        /* :807-813 */
        if (p->reqs[i * 2] > k) { p->err = 1; goto out; }
out:
    free(mapping); free(rowoff);
    return p->err;
}

/* ------------------------------------------------------------------------- */
/* 3. FFS count semantics (HnGPU.cu:34-52, 76-109, 114-262, 455-669),         */
/*    evaluated depth-first: identical candidate order, injectivity and     */
/*    requirement checks, 64-bit count.                                      */
/* ------------------------------------------------------------------------- */

typedef struct {
    const orc_graph *q, *d;
    const orc_plan_t *p;
    int vlabel_mode;
    uint32_t *row_list;      /* data row offsets in CCSR order */
    uint32_t *row_vid;       /* row offset -> original vertex id (via a map) */
    uint32_t nrows;
    uint32_t root_begin, root_end; /* roots taken: CCSR rows [root_begin, root_end) */
    uint32_t *qcol;          /* depth -> original query vertex id */
    uint32_t *qlab;          /* depth -> query vertex label */
    _Atomic uint64_t next_root;
    _Atomic uint64_t total;
    /* mapping capture (single-threaded) */
    uint32_t *rows_out; uint64_t max_rows, n_rows;
    pthread_mutex_t mu;
} ffs_ctx;

/* reqExists (HnGPU.cu:34-52): linear scan for (relation, vertex). */
static int req_exists(const orc_graph *d, uint64_t row, uint32_t rel, uint32_t v, uint32_t vert_bits)
{
    uint32_t deg = d->seg_val[row];
    for (uint32_t i = 0; i < deg; i++)
        if ((vert_bits >= 32 ? 0u : d->seg_lab[row + 1 + i] << vert_bits) == rel && d->seg_val[row + 1 + i] == v)
            return 1;
    return 0;
}

static uint32_t vid_of_offset(const ffs_ctx *c, uint32_t off)
{
    /* binary search over the sorted row list */
    uint32_t lo = 0, hi = c->nrows;
    while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (c->row_list[mid] < off) lo = mid + 1; else hi = mid; }
    if (lo < c->nrows && c->row_list[lo] == off) return c->row_vid[lo];
    return 0xffffffffu;
}

static uint64_t ffs_dfs(ffs_ctx *c, uint32_t depth, uint32_t *m)
{
    const orc_plan_t *p = c->p;
    const orc_graph *d = c->d;
    if (depth == p->k) {
        if (c->rows_out) {
            pthread_mutex_lock(&c->mu);
            if (c->n_rows < c->max_rows) {
                uint32_t *row = c->rows_out + c->n_rows * p->k;
                for (uint32_t i = 0; i < p->k; i++) row[c->qcol[i]] = vid_of_offset(c, m[i]);
                c->n_rows++;
            }
            pthread_mutex_unlock(&c->mu);
        }
        return 1;
    }
    const uint32_t *h = &p->header[depth * 3];
    const uint32_t nreq = h[0], roff = h[1], firstq = h[2];
    uint32_t anchor = m[depth - firstq];
    uint32_t deg = d->seg_val[anchor];
    uint64_t total = 0;
    for (uint32_t e = 0; e < deg; e++) {
        uint32_t v = d->seg_val[anchor + 1 + e];
        int ok = 1;
        for (uint32_t i = 0; i < depth && ok; i++) if (m[i] == v) ok = 0;    /* ISOSOLVE :223-236 */
        uint32_t dist = 0;
        for (uint32_t r = 0; r < nreq && ok; r++) {                          /* :243-252 */
            dist += p->reqs[roff + 2 * r];
            uint32_t u = dist == 0 ? v : m[depth - dist];
            if (!req_exists(d, u, p->reqs[roff + 2 * r + 1], v, 32u - p->rel_bits)) ok = 0;
        }
        if (ok && c->vlabel_mode) {
            uint32_t vid = vid_of_offset(c, v);
            if (vid == 0xffffffffu || d->vlabel[vid] != c->qlab[depth]) ok = 0;
        }
        if (!ok) continue;
        m[depth] = v;
        total += ffs_dfs(c, depth + 1, m);
    }
    return total;
}

static void *ffs_worker(void *arg)
{
    ffs_ctx *c = arg;
    const orc_plan_t *p = c->p;
    uint32_t m[64];
    uint64_t local = 0;
    for (;;) {
        uint64_t i = c->root_begin + atomic_fetch_add(&c->next_root, 1);
        if (i >= c->root_end) break;
        uint32_t r = c->row_list[i];
        int ok = 1;
        for (uint32_t j = 0; j < p->header[0] && ok; j++)                      /* hnInit :95-102 */
            if (!req_exists(c->d, r, p->reqs[j * 2 + 1], r, 32u - p->rel_bits)) ok = 0;
        if (ok && c->vlabel_mode && c->d->vlabel[c->row_vid[i]] != c->qlab[0]) ok = 0;
        if (!ok) continue;
        m[0] = r;
        local += ffs_dfs(c, 1, m);
    }
    atomic_fetch_add(&c->total, local);
    return NULL;
}

int orc_ffs_count(const orc_graph *q, const orc_plan_t *p, const orc_graph *d,
                  int vlabel_mode, int threads, uint64_t *count,
                  uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows)
{
    return orc_ffs_count_rows(q, p, d, vlabel_mode, threads, 0, 0xffffffffu, count, rows_out, max_rows, n_rows);
}

int orc_ffs_count_rows(const orc_graph *q, const orc_plan_t *p, const orc_graph *d,
                       int vlabel_mode, int threads, uint32_t root_begin, uint32_t root_end, uint64_t *count,
                       uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows)
{
    if (p->err || q->err || d->err) return -1;
    if (p->k > 64) return -2;
    ffs_ctx c;
    memset(&c, 0, sizeof(c));
    c.q = q; c.d = d; c.p = p; c.vlabel_mode = vlabel_mode;
    c.nrows = d->rows;
    c.root_end = root_end < d->rows ? root_end : d->rows;
    c.root_begin = root_begin < c.root_end ? root_begin : c.root_end;
    c.row_list = malloc(sizeof(uint32_t) * (d->rows + 1));
    c.row_vid = malloc(sizeof(uint32_t) * (d->rows + 1));
    uint64_t off = 0;
    for (uint32_t i = 0; i < d->rows; i++) {
        c.row_list[i] = (uint32_t)off; c.row_vid[i] = d->inv[i];
        off += d->seg_val[off] + 1;
    }
    c.qcol = malloc(sizeof(uint32_t) * p->k);
    c.qlab = malloc(sizeof(uint32_t) * p->k);
    for (uint32_t i = 0; i < p->k; i++) {
        c.qcol[i] = q->inv[p->order[i]];
        c.qlab[i] = q->vlabel[c.qcol[i]];
    }
    c.rows_out = rows_out; c.max_rows = rows_out ? max_rows : 0;
    pthread_mutex_init(&c.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, ffs_worker, &c);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    *count = atomic_load(&c.total);
    if (n_rows) *n_rows = c.n_rows;
    pthread_mutex_destroy(&c.mu);
    free(th); free(c.row_list); free(c.row_vid); free(c.qcol); free(c.qlab);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* 4. Independent backtracking enumerator (no CCSR, no reference planner).   */
/*    Counts injective f: Vq -> Vd such that every query edge (a->b, l) has a */
/*    data edge (f(a)->f(b), l); optional vertex-label equality.  Edge sets  */
/*    are de-duplicated (set semantics).                                     */
/* ------------------------------------------------------------------------- */

typedef struct { uint32_t n; uint64_t *off; uint64_t *key; } adjset; /* key = nbr<<32 | label */

static int u32_cmp(const void *a, const void *b)
{
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : (x > y);
}

static int u64_cmp(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y);
}

static void adj_build(adjset *a, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                      const uint32_t *lab, uint32_t lmask)
{
    a->n = n;
    a->off = calloc((uint64_t)n + 1, 8);
    uint64_t *tmp = malloc(sizeof(uint64_t) * (m + 1));
    for (uint64_t i = 0; i < m; i++) a->off[src[i] + 1]++;
    for (uint32_t i = 0; i < n; i++) a->off[i + 1] += a->off[i];
    uint64_t *fill = calloc((uint64_t)n + 1, 8);
    for (uint64_t i = 0; i < m; i++)
        tmp[a->off[src[i]] + fill[src[i]]++] = ((uint64_t)dst[i] << 32) | (lab[i] & lmask);
    /* sort + dedupe each row */
    uint64_t w = 0;
    uint64_t *newoff = calloc((uint64_t)n + 1, 8);
    for (uint32_t v = 0; v < n; v++) {
        uint64_t b = a->off[v], e = a->off[v + 1];
        qsort(tmp + b, e - b, 8, u64_cmp);
        newoff[v] = w;
        for (uint64_t i = b; i < e; i++)
            if (i == b || tmp[i] != tmp[i - 1]) tmp[w++] = tmp[i];
    }
    newoff[n] = w;
    free(a->off); free(fill);
    a->off = newoff; a->key = tmp;
}

static int adj_has(const adjset *a, uint32_t u, uint32_t v, uint32_t l)
{
    uint64_t key = ((uint64_t)v << 32) | l;
    uint64_t lo = a->off[u], hi = a->off[u + 1];
    while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (a->key[mid] < key) lo = mid + 1; else hi = mid; }
    return lo < a->off[u + 1] && a->key[lo] == key;
}

typedef struct { uint32_t other; uint32_t lab; int out; } qcon; /* out: edge order[i]->other */

typedef struct {
    uint32_t qn, dn;
    adjset dout, din;
    const uint32_t *qvl, *dvl;
    int vlabel_mode;
    uint32_t order[64];
    /* per depth: candidate source (a matched depth + direction) and checks */
    int32_t gen_depth[64]; int gen_out[64];
    uint32_t ncheck[64]; qcon *checks[64]; /* other = depth index of matched vertex, or self (== depth) */
    _Atomic uint64_t next_root, total;
    uint32_t *rows_out; uint64_t max_rows, n_rows;
    pthread_mutex_t mu;
} bt_ctx;

static uint64_t bt_dfs(bt_ctx *c, uint32_t depth, uint32_t *m, uint8_t *used)
{
    if (depth == c->qn) {
        if (c->rows_out) {
            pthread_mutex_lock(&c->mu);
            if (c->n_rows < c->max_rows) {
                uint32_t *row = c->rows_out + c->n_rows * c->qn;
                for (uint32_t i = 0; i < c->qn; i++) row[c->order[i]] = m[i];
                c->n_rows++;
            }
            pthread_mutex_unlock(&c->mu);
        }
        return 1;
    }
    uint32_t qv = c->order[depth];
    uint64_t total = 0;
    uint64_t b, e; const adjset *src;
    if (c->gen_depth[depth] >= 0) {
        uint32_t fu = m[c->gen_depth[depth]];
        src = c->gen_out[depth] ? &c->dout : &c->din;
        b = src->off[fu]; e = src->off[fu + 1];
    } else { src = NULL; b = 0; e = c->dn; }
    uint32_t prev = 0xffffffffu;
    for (uint64_t i = b; i < e; i++) {
        uint32_t v = src ? (uint32_t)(src->key[i] >> 32) : (uint32_t)i;
        if (src && v == prev) continue; /* several labels to the same neighbour */
        prev = v;
        if (used[v]) continue;
        if (c->vlabel_mode && c->dvl[v] != c->qvl[qv]) continue;
        int ok = 1;
        for (uint32_t j = 0; j < c->ncheck[depth] && ok; j++) {
            const qcon *k = &c->checks[depth][j];
            uint32_t fo = k->other == depth ? v : m[k->other];
            ok = k->out ? adj_has(&c->dout, v, fo, k->lab) : adj_has(&c->dout, fo, v, k->lab);
        }
        if (!ok) continue;
        m[depth] = v; used[v] = 1;
        total += bt_dfs(c, depth + 1, m, used);
        used[v] = 0;
    }
    return total;
}

static void *bt_worker(void *arg)
{
    bt_ctx *c = arg;
    uint32_t m[64];
    uint8_t *used = calloc(c->dn ? c->dn : 1, 1);
    uint64_t local = 0;
    uint32_t qv = c->order[0];
    for (;;) {
        uint64_t r = atomic_fetch_add(&c->next_root, 1);
        if (r >= c->dn) break;
        uint32_t v = (uint32_t)r;
        if (c->vlabel_mode && c->dvl[v] != c->qvl[qv]) continue;
        int ok = 1;
        for (uint32_t j = 0; j < c->ncheck[0] && ok; j++)
            ok = adj_has(&c->dout, v, v, c->checks[0][j].lab);
        if (!ok) continue;
        m[0] = v; used[v] = 1;
        local += bt_dfs(c, 1, m, used);
        used[v] = 0;
    }
    free(used);
    atomic_fetch_add(&c->total, local);
    return NULL;
}

int orc_bt_count(uint32_t qn, uint32_t qm, const uint32_t *qs, const uint32_t *qd,
                 const uint32_t *ql, const uint32_t *qvl,
                 uint32_t dn, uint64_t dm, const uint32_t *ds, const uint32_t *dd,
                 const uint32_t *dl, const uint32_t *dvl,
                 uint32_t rel_bits, int vlabel_mode, int threads, uint64_t *count,
                 uint32_t *rows_out, uint64_t max_rows, uint64_t *n_rows)
{
    if (qn == 0 || qn > 64) return -2;
    const uint32_t lmask = rel_bits >= 32 ? 0xffffffffu : ((1u << rel_bits) - 1u);
    for (uint64_t i = 0; i < dm; i++) if (ds[i] >= dn || dd[i] >= dn) return -3;
    for (uint32_t i = 0; i < qm; i++) if (qs[i] >= qn || qd[i] >= qn) return -3;
    bt_ctx c;
    memset(&c, 0, sizeof(c));
    c.qn = qn; c.dn = dn; c.qvl = qvl; c.dvl = dvl; c.vlabel_mode = vlabel_mode;
    adj_build(&c.dout, dn, dm, ds, dd, dl, lmask);
    adj_build(&c.din, dn, dm, dd, ds, dl, lmask);
    /* de-duplicated query edge set */
    adjset qa;
    adj_build(&qa, qn, qm, qs, qd, ql, lmask);
    /* matching order: highest query degree first (lowest id on ties), then the
     * vertex with most edges into the matched set, ties by degree then id. */
    uint32_t *qdeg = calloc(qn, 4);
    for (uint32_t v = 0; v < qn; v++)
        for (uint64_t i = qa.off[v]; i < qa.off[v + 1]; i++) {
            uint32_t o = (uint32_t)(qa.key[i] >> 32);
            qdeg[v]++; if (o != v) qdeg[o]++;
        }
    uint8_t inord[64] = {0};
    int32_t depth_of[64];
    for (uint32_t i = 0; i < qn; i++) depth_of[i] = -1;
    for (uint32_t dpt = 0; dpt < qn; dpt++) {
        int best = -1; uint32_t bconn = 0;
        for (uint32_t v = 0; v < qn; v++) {
            if (inord[v]) continue;
            uint32_t conn = 0;
            for (uint32_t u = 0; u < qn; u++) {
                if (!inord[u]) continue;
                for (uint64_t i = qa.off[u]; i < qa.off[u + 1]; i++) if ((uint32_t)(qa.key[i] >> 32) == v) conn++;
                for (uint64_t i = qa.off[v]; i < qa.off[v + 1]; i++) if ((uint32_t)(qa.key[i] >> 32) == u) conn++;
            }
            if (best < 0 || conn > bconn || (conn == bconn && qdeg[v] > qdeg[best])) { best = (int)v; bconn = conn; }
        }
        inord[best] = 1; c.order[dpt] = (uint32_t)best; depth_of[best] = (int32_t)dpt;
    }
    for (uint32_t dpt = 0; dpt < qn; dpt++) {
        uint32_t v = c.order[dpt];
        c.gen_depth[dpt] = -1;
        qcon *chk = malloc(sizeof(qcon) * (2 * qm + 2));
        uint32_t nc = 0;
        /* edges v -> u (u matched earlier or v itself) */
        for (uint64_t i = qa.off[v]; i < qa.off[v + 1]; i++) {
            uint32_t u = (uint32_t)(qa.key[i] >> 32), l = (uint32_t)qa.key[i];
            if (depth_of[u] <= (int32_t)dpt) {
                chk[nc].other = (uint32_t)depth_of[u]; chk[nc].lab = l; chk[nc].out = 1; nc++;
                if (u != v && c.gen_depth[dpt] < 0) { c.gen_depth[dpt] = depth_of[u]; c.gen_out[dpt] = 0; }
            }
        }
        /* edges u -> v, u matched earlier */
        for (uint32_t u = 0; u < qn; u++) {
            if (u == v || depth_of[u] >= (int32_t)dpt) continue;
            for (uint64_t i = qa.off[u]; i < qa.off[u + 1]; i++) {
                if ((uint32_t)(qa.key[i] >> 32) != v) continue;
                chk[nc].other = (uint32_t)depth_of[u]; chk[nc].lab = (uint32_t)qa.key[i]; chk[nc].out = 0; nc++;
                if (c.gen_depth[dpt] < 0 || c.gen_out[dpt] == 0) { c.gen_depth[dpt] = depth_of[u]; c.gen_out[dpt] = 1; }
            }
        }
        c.ncheck[dpt] = nc; c.checks[dpt] = chk;
    }
    /* candidate generation through v's in-neighbours (edge f(v)->f(u) means f(v) is an
     * in-neighbour of f(u)) -- gen_out=0 reads din of f(u). */
    c.rows_out = rows_out; c.max_rows = rows_out ? max_rows : 0;
    pthread_mutex_init(&c.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, bt_worker, &c);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    *count = atomic_load(&c.total);
    if (n_rows) *n_rows = c.n_rows;
    pthread_mutex_destroy(&c.mu);
    free(th);
    for (uint32_t dpt = 0; dpt < qn; dpt++) free(c.checks[dpt]);
    free(qdeg);
    free(qa.off); free(qa.key);
    free(c.dout.off); free(c.dout.key); free(c.din.off); free(c.din.key);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* 5. Triangle count of an undirected simple graph (edges u < v), by the     */
/*    degree-ordered orientation + sorted-list intersection method; an        */
/*    independent check of the triangle query at sizes the enumerators       */
/*    cannot reach (each triangle is 6 embeddings of the triangle query).    */
/* ------------------------------------------------------------------------- */
typedef struct {
    uint32_t n; const uint64_t *ptr; const uint32_t *adj;
    const uint32_t *vl; uint32_t nl;          /* vertex labels (NULL: no histogram) */
    uint64_t *hist; pthread_mutex_t mu;       /* [nl^3] ordered label triples */
    _Atomic uint64_t next, total;
} tri_ctx;

static void tri_label_add(uint64_t *h, uint32_t nl, uint32_t a, uint32_t b, uint32_t c)
{
    /* the 6 orderings of the triangle's vertices (a 3-vertex triangle query
     * maps onto every ordering once) */
    h[(a * nl + b) * nl + c]++; h[(a * nl + c) * nl + b]++;
    h[(b * nl + a) * nl + c]++; h[(b * nl + c) * nl + a]++;
    h[(c * nl + a) * nl + b]++; h[(c * nl + b) * nl + a]++;
}

static void *tri_worker(void *arg)
{
    tri_ctx *c = arg;
    uint64_t local = 0;
    uint64_t *lh = c->vl ? calloc((uint64_t)c->nl * c->nl * c->nl, 8) : NULL;
    for (;;) {
        uint64_t x = atomic_fetch_add(&c->next, 64);
        if (x >= c->n) break;
        uint64_t xe = x + 64 < c->n ? x + 64 : c->n;
        for (; x < xe; x++) {
            for (uint64_t i = c->ptr[x]; i < c->ptr[x + 1]; i++) {
                uint32_t y = c->adj[i];
                uint64_t a = c->ptr[x], ae = c->ptr[x + 1], b = c->ptr[y], be = c->ptr[y + 1];
                while (a < ae && b < be) {
                    if (c->adj[a] < c->adj[b]) a++;
                    else if (c->adj[a] > c->adj[b]) b++;
                    else {
                        local++;
                        if (lh) tri_label_add(lh, c->nl, c->vl[x], c->vl[y], c->vl[c->adj[a]]);
                        a++; b++;
                    }
                }
            }
        }
    }
    atomic_fetch_add(&c->total, local);
    if (lh) {
        pthread_mutex_lock(&c->mu);
        for (uint64_t i = 0; i < (uint64_t)c->nl * c->nl * c->nl; i++) c->hist[i] += lh[i];
        pthread_mutex_unlock(&c->mu);
        free(lh);
    }
    return NULL;
}

static int triangles_impl(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                          const uint32_t *vl, uint32_t nl, uint64_t *hist, int threads, uint64_t *count);

int orc_triangles(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, int threads, uint64_t *count)
{
    return triangles_impl(n, m, src, dst, NULL, 0, NULL, threads, count);
}

int orc_triangle_label_hist(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                            const uint32_t *vlabel, uint32_t nl, int threads, uint64_t *hist, uint64_t *count)
{
    if (!vlabel || nl == 0 || nl > 64) return -1;
    for (uint32_t v = 0; v < n; v++) if (vlabel[v] >= nl) return -2;
    memset(hist, 0, 8ull * nl * nl * nl);
    return triangles_impl(n, m, src, dst, vlabel, nl, hist, threads, count);
}

static int triangles_impl(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                          const uint32_t *vl, uint32_t nl, uint64_t *hist, int threads, uint64_t *count)
{
    uint64_t *deg = calloc((uint64_t)n + 1, 8);
    for (uint64_t i = 0; i < m; i++) { deg[src[i]]++; deg[dst[i]]++; }
    uint64_t *ptr = calloc((uint64_t)n + 2, 8);
    /* orient each edge from the lower (degree, id) endpoint to the higher */
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u = src[i], v = dst[i];
        int swap = deg[u] > deg[v] || (deg[u] == deg[v] && u > v);
        ptr[(swap ? v : u) + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) ptr[i + 1] += ptr[i];
    uint32_t *adj = malloc(sizeof(uint32_t) * (m + 1));
    uint64_t *fill = malloc(8 * ((uint64_t)n + 1));
    memcpy(fill, ptr, 8 * ((uint64_t)n + 1));
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u = src[i], v = dst[i];
        int swap = deg[u] > deg[v] || (deg[u] == deg[v] && u > v);
        if (swap) { uint32_t t = u; u = v; v = t; }
        adj[fill[u]++] = v;
    }
    for (uint32_t x = 0; x < n; x++) {
        uint64_t b = ptr[x], e = ptr[x + 1];
        /* insertion sort is fine for short rows, qsort otherwise */
        if (e - b > 32) qsort(adj + b, e - b, 4, u32_cmp);
        else for (uint64_t i = b + 1; i < e; i++) { uint32_t t = adj[i]; uint64_t j = i; while (j > b && adj[j - 1] > t) { adj[j] = adj[j - 1]; j--; } adj[j] = t; }
    }
    tri_ctx c; memset(&c, 0, sizeof(c));
    c.n = n; c.ptr = ptr; c.adj = adj;
    c.vl = vl; c.nl = nl; c.hist = hist;
    pthread_mutex_init(&c.mu, NULL);
    if (threads < 1) threads = 1;
    pthread_t *th = malloc(sizeof(pthread_t) * threads);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, tri_worker, &c);
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    *count = atomic_load(&c.total);
    pthread_mutex_destroy(&c.mu);
    free(th); free(adj); free(fill); free(ptr); free(deg);
    return 0;
}
