/*
 * synth.c -- seeded synthetic workloads for the GFSM matcher.
 *
 * The reference benchmarks on SNAP / RDF graphs that are not available here;
 * these generators stand in for them with the shapes the workload configs
 * name: Erdos-Renyi, R-MAT, Barabasi-Albert, a perturbed 2D grid, vertex
 * labels (uniform or Zipf), and random-walk query extraction.  All output is
 * undirected (u < v) edge lists; the text writer emits both directions in the
 * reference's `t # / v / e` format (HnHelper.cuh:283-381).
 *
 * Deterministic: every generator is driven by splitmix64 from its seed.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint64_t s; } rng_t;
static inline uint64_t rng_next(rng_t *r)
{
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static inline double rng_unif(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline uint64_t rng_below(rng_t *r, uint64_t n) { return n ? rng_next(r) % n : 0; }

void syn_free(void *p) { free(p); }

/* --- open-addressing set of undirected edge keys, insertion ordered ------- */
typedef struct { uint64_t *slot; uint64_t mask, count; } eset;
static void eset_init(eset *s, uint64_t expect)
{
    uint64_t cap = 16;
    while (cap < expect * 2) cap <<= 1;
    s->slot = malloc(cap * 8);
    memset(s->slot, 0xff, cap * 8);
    s->mask = cap - 1; s->count = 0;
}
static inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
    return x;
}
/* returns 1 if newly inserted */
static inline int eset_add(eset *s, uint64_t key)
{
    uint64_t h = mix64(key) & s->mask;
    for (;;) {
        if (s->slot[h] == ~0ull) { s->slot[h] = key; s->count++; return 1; }
        if (s->slot[h] == key) return 0;
        h = (h + 1) & s->mask;
    }
}

typedef struct { uint32_t *src, *dst; uint64_t m, cap; } elist;
static void el_push(elist *e, uint32_t u, uint32_t v)
{
    if (e->m == e->cap) {
        e->cap = e->cap ? e->cap * 2 : 1024;
        e->src = realloc(e->src, e->cap * 4); e->dst = realloc(e->dst, e->cap * 4);
    }
    e->src[e->m] = u; e->dst[e->m] = v; e->m++;
}
static int el_add_undirected(elist *e, eset *s, uint32_t u, uint32_t v)
{
    if (u == v) return 0;
    if (u > v) { uint32_t t = u; u = v; v = t; }
    if (!eset_add(s, ((uint64_t)u << 32) | v)) return 0;
    el_push(e, u, v);
    return 1;
}

/* Erdos-Renyi G(n, p) with p = avg_deg / (n-1), via geometric skipping over
 * the pairs (i < j) in row-major order. */
int syn_er(uint32_t n, double avg_deg, uint64_t seed, uint64_t *m, uint32_t **src, uint32_t **dst)
{
    rng_t r = {seed};
    elist e = {0};
    double p = n > 1 ? avg_deg / (double)(n - 1) : 0.0;
    if (p > 1.0) p = 1.0;
    if (p > 0.0) {
        double lq = log(1.0 - p);
        int64_t v = 1, w = -1;
        while (v < (int64_t)n) {
            double u = 1.0 - rng_unif(&r);
            w = w + 1 + (p >= 1.0 ? 0 : (int64_t)floor(log(u) / lq));
            while (w >= v && v < (int64_t)n) { w -= v; v++; }
            if (v < (int64_t)n) el_push(&e, (uint32_t)w, (uint32_t)v);
        }
    }
    *m = e.m; *src = e.src; *dst = e.dst;
    return 0;
}

/* R-MAT(a, b, c, 1-a-b-c) on 2^scale vertices.  Samples edges until `target`
 * distinct undirected non-loop edges exist (kept in generation order), then
 * relabels vertices through a seeded random permutation so that vertex id
 * carries no degree information. */
int syn_rmat(uint32_t scale, uint64_t target, double a, double b, double c, uint64_t seed,
             uint64_t *m, uint32_t **src, uint32_t **dst)
{
    rng_t r = {seed};
    const uint32_t n = 1u << scale;
    elist e = {0};
    eset s; eset_init(&s, target + 16);
    e.cap = target; e.src = malloc(target * 4 + 4); e.dst = malloc(target * 4 + 4);
    const double ab = a + b, abc = a + b + c;
    uint64_t tries = 0, max_tries = target * 64 + 1024;
    while (e.m < target && tries < max_tries) {
        tries++;
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            double x = rng_unif(&r);
            uint32_t bu = 0, bv = 0;
            if (x < a) {} else if (x < ab) bv = 1; else if (x < abc) bu = 1; else { bu = 1; bv = 1; }
            u = (u << 1) | bu; v = (v << 1) | bv;
        }
        el_add_undirected(&e, &s, u, v);
    }
    free(s.slot);
    uint32_t *perm = malloc((uint64_t)n * 4);
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    for (uint32_t i = n - 1; i > 0; i--) { uint32_t j = (uint32_t)rng_below(&r, (uint64_t)i + 1); uint32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t; }
    for (uint64_t i = 0; i < e.m; i++) {
        uint32_t u = perm[e.src[i]], v = perm[e.dst[i]];
        if (u > v) { uint32_t t = u; u = v; v = t; }
        e.src[i] = u; e.dst[i] = v;
    }
    free(perm);
    *m = e.m; *src = e.src; *dst = e.dst;
    return 0;
}

/* Barabasi-Albert: start from a clique on m0 = m+1 vertices; every new vertex
 * attaches to m distinct earlier vertices chosen proportionally to degree
 * (uniform draw from the endpoint list). */
int syn_ba(uint32_t n, uint32_t mm, uint64_t seed, uint64_t *m, uint32_t **src, uint32_t **dst)
{
    rng_t r = {seed};
    elist e = {0};
    uint32_t m0 = mm + 1;
    if (n < m0) m0 = n;
    uint64_t total = (uint64_t)m0 * (m0 - 1) / 2 + (uint64_t)(n > m0 ? n - m0 : 0) * mm;
    e.cap = total + 1; e.src = malloc(e.cap * 4); e.dst = malloc(e.cap * 4);
    uint32_t *ends = malloc((2 * total + 2) * 4);
    uint64_t ne = 0;
    for (uint32_t i = 0; i < m0; i++)
        for (uint32_t j = i + 1; j < m0; j++) { el_push(&e, i, j); ends[ne++] = i; ends[ne++] = j; }
    uint32_t *pick = malloc((mm + 1) * 4);
    for (uint32_t v = m0; v < n; v++) {
        uint32_t k = 0;
        while (k < mm) {
            uint32_t t = ends[rng_below(&r, ne)];
            int dup = 0;
            for (uint32_t i = 0; i < k; i++) if (pick[i] == t) { dup = 1; break; }
            if (!dup) pick[k++] = t;
        }
        for (uint32_t i = 0; i < mm; i++) { el_push(&e, pick[i], v); ends[ne++] = pick[i]; ends[ne++] = v; }
    }
    free(pick); free(ends);
    *m = e.m; *src = e.src; *dst = e.dst;
    return 0;
}

/* side x side grid (4-neighbour), a seeded fraction of grid edges removed and
 * shortcut_frac * |grid edges| uniformly random long-range shortcuts added. */
int syn_grid(uint32_t side, double remove_frac, double shortcut_frac, uint64_t seed,
             uint64_t *m, uint32_t **src, uint32_t **dst)
{
    rng_t r = {seed};
    const uint64_t n = (uint64_t)side * side;
    uint64_t grid_edges = 2ull * side * (side - 1);
    elist e = {0};
    eset s; eset_init(&s, grid_edges + (uint64_t)(shortcut_frac * grid_edges) + 16);
    for (uint32_t y = 0; y < side; y++)
        for (uint32_t x = 0; x < side; x++) {
            uint32_t v = y * side + x;
            if (x + 1 < side && rng_unif(&r) >= remove_frac) el_add_undirected(&e, &s, v, v + 1);
            if (y + 1 < side && rng_unif(&r) >= remove_frac) el_add_undirected(&e, &s, v, v + side);
        }
    uint64_t want = (uint64_t)(shortcut_frac * (double)grid_edges), added = 0, tries = 0;
    while (added < want && tries < want * 16 + 16) {
        tries++;
        added += el_add_undirected(&e, &s, (uint32_t)rng_below(&r, n), (uint32_t)rng_below(&r, n));
    }
    free(s.slot);
    *m = e.m; *src = e.src; *dst = e.dst;
    return 0;
}

/* Vertex labels: uniform over [0, nl) when zipf_s <= 0, else Zipf(s) over
 * ranks 1..nl mapped to labels 0..nl-1. */
int syn_vlabels(uint32_t n, uint32_t nl, double zipf_s, uint64_t seed, uint32_t *out)
{
    rng_t r = {seed};
    if (nl == 0) nl = 1;
    if (zipf_s <= 0.0) {
        for (uint32_t i = 0; i < n; i++) out[i] = (uint32_t)rng_below(&r, nl);
        return 0;
    }
    double *cdf = malloc(sizeof(double) * nl), acc = 0.0;
    for (uint32_t i = 0; i < nl; i++) { acc += 1.0 / pow((double)(i + 1), zipf_s); cdf[i] = acc; }
    for (uint32_t i = 0; i < n; i++) {
        double x = rng_unif(&r) * acc;
        uint32_t lo = 0, hi = nl - 1;
        while (lo < hi) { uint32_t mid = (lo + hi) / 2; if (cdf[mid] < x) lo = mid + 1; else hi = mid; }
        out[i] = lo;
    }
    free(cdf);
    return 0;
}

/* Undirected CSR (both directions, rows sorted by neighbour id). */
int syn_csr(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst, uint64_t *rowptr, uint32_t *adj)
{
    memset(rowptr, 0, ((uint64_t)n + 1) * 8);
    for (uint64_t i = 0; i < m; i++) { rowptr[src[i] + 1]++; rowptr[dst[i] + 1]++; }
    for (uint32_t i = 0; i < n; i++) rowptr[i + 1] += rowptr[i];
    uint64_t *fill = malloc(((uint64_t)n + 1) * 8);
    memcpy(fill, rowptr, ((uint64_t)n + 1) * 8);
    for (uint64_t i = 0; i < m; i++) { adj[fill[src[i]]++] = dst[i]; adj[fill[dst[i]]++] = src[i]; }
    free(fill);
    return 0;
}

/* Random-walk query extraction.  Starts at a uniformly random vertex of
 * degree >= 1 and walks to uniformly random neighbours until k distinct
 * vertices are visited (restarting after 64*k steps without progress).
 * tree != 0 keeps only the discovery edges (a spanning tree); otherwise all
 * induced edges among the visited vertices are kept.  Query vertex ids are the
 * visit order.  Outputs undirected query edges (u < v) as query ids, and the
 * visited data vertex ids.  Returns 0, or -1 if no walk reached k vertices. */
int syn_rw_query(uint32_t n, const uint64_t *rowptr, const uint32_t *adj, uint32_t k, int tree,
                 uint64_t seed, uint32_t *visited, uint32_t *qm, uint32_t *qsrc, uint32_t *qdst)
{
    rng_t r = {seed};
    if (k == 0 || k > 64) return -1;
    for (int attempt = 0; attempt < 1000; attempt++) {
        uint32_t start = 0; int ok = 0;
        for (int t = 0; t < 1000; t++) {
            start = (uint32_t)rng_below(&r, n);
            if (rowptr[start + 1] > rowptr[start]) { ok = 1; break; }
        }
        if (!ok) return -1;
        uint32_t nv = 1, ne = 0, cur = start, stall = 0;
        visited[0] = start;
        while (nv < k && stall < 64 * k) {
            uint64_t d = rowptr[cur + 1] - rowptr[cur];
            if (!d) break;
            uint32_t nxt = adj[rowptr[cur] + rng_below(&r, d)];
            int seen = -1;
            for (uint32_t i = 0; i < nv; i++) if (visited[i] == nxt) { seen = (int)i; break; }
            if (seen < 0) {
                if (tree) {
                    uint32_t a = 0;
                    for (uint32_t i = 0; i < nv; i++) if (visited[i] == cur) { a = i; break; }
                    qsrc[ne] = a; qdst[ne] = nv; ne++;
                }
                visited[nv++] = nxt;
                stall = 0;
            } else {
                stall++;
            }
            cur = nxt;
        }
        if (nv < k) continue;
        if (!tree) {
            ne = 0;
            for (uint32_t i = 0; i < k; i++) {
                uint32_t u = visited[i];
                for (uint32_t j = i + 1; j < k; j++) {
                    uint32_t v = visited[j];
                    uint64_t lo = rowptr[u], hi = rowptr[u + 1];
                    /* rows are sorted */
                    while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (adj[mid] < v) lo = mid + 1; else hi = mid; }
                    if (lo < rowptr[u + 1] && adj[lo] == v) { qsrc[ne] = i; qdst[ne] = j; ne++; }
                }
            }
        }
        *qm = ne;
        return 0;
    }
    return -1;
}

/* Writes a graph in the `t # / v / e` format with both directions of every
 * undirected edge (label elab[i], or 1 when elab is NULL). */
int syn_write_text(const char *path, uint32_t n, const uint32_t *vlabels, uint64_t m,
                   const uint32_t *src, const uint32_t *dst, const uint32_t *elab)
{
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    static char buf[1 << 20];
    setvbuf(f, buf, _IOFBF, sizeof(buf));
    fprintf(f, "t # 0\n%u %llu 1 1\n", n, (unsigned long long)(2 * m));
    for (uint32_t i = 0; i < n; i++) fprintf(f, "v %u %u\n", i, vlabels ? vlabels[i] : 1u);
    for (uint64_t i = 0; i < m; i++) {
        uint32_t l = elab ? elab[i] : 1u;
        fprintf(f, "e %u %u %u\ne %u %u %u\n", src[i], dst[i], l, dst[i], src[i], l);
    }
    fputs("t # -1", f);
    fclose(f);
    return 0;
}
