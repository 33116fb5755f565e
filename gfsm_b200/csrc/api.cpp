// api.cpp -- the C ABI (include/gfsm.h) over the host parser/planner, the
// device CCSR builder and the matching engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <thread>

#include "engine.h"
#include "gfsm_internal.h"

using namespace gfsm;

namespace {

uint64_t env_u64(const char *name, uint64_t dflt) {
    const char *s = getenv(name);
    if (!s || !*s) return dflt;
    char *end = nullptr;
    double v = strtod(s, &end);
    if (end == s || v < 0) return dflt;
    return (uint64_t)v;
}

gfsm_status set_err(gfsm_ctx *ctx, gfsm_status rc, const std::string &msg) {
    if (ctx && rc != GFSM_OK) ctx->last_error = msg.empty() ? gfsm_status_str(rc) : msg;
    return rc;
}

Engine *ctx_engine(gfsm_ctx *ctx, const DeviceGraph &g, gfsm_status &rc, std::string &err) {
    Engine *e = static_cast<Engine *>(ctx->engine);
    if (!e) {
        e = new (std::nothrow) Engine();
        if (!e) { rc = GFSM_ERR_NOMEM; return nullptr; }
        rc = e->init(ctx->device, 0, ctx->lim.max_scan_size, err);
        if (rc != GFSM_OK) { delete e; return nullptr; }
        ctx->engine = e;
    }
    // MEMLIMIT covers the data graph, the engine's fixed buffers and the arena.
    const uint64_t used = g.bytes + e->small_bytes;
    const uint64_t lim_cap = ctx->lim.mem_limit > used ? ctx->lim.mem_limit - used : 0;
    uint64_t cap = lim_cap;
    // Free device memory is read when the arena is first sized and then every
    // 1024th call (a chance to grow): the query goes through the driver,
    // which other processes on the machine share, and it sometimes stalls
    // for milliseconds -- too long for every call of a sub-millisecond query.
    const bool probe = !e->arena || e->arena_bytes > lim_cap || (ctx->calls++ & 1023u) == 0;
    size_t free_b = 0, total_b = 0;
    if (probe && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        uint64_t avail = (uint64_t)free_b + e->arena_bytes;
        avail = avail > (1ull << 30) ? avail - (1ull << 30) : avail / 2;
        cap = std::min(cap, avail);
    }
    // Keep an arena that MEMLIMIT still allows: free-memory readings move a
    // little between calls, and re-allocating a multi-GB arena for that costs
    // tens of milliseconds.  Grow it only for 25% more room.
    if (e->arena && e->arena_bytes <= lim_cap && (!probe || cap < e->arena_bytes + e->arena_bytes / 4))
        cap = e->arena_bytes;
    if (e->arena && e->arena_bytes > cap) {
        cudaFree(e->arena);
        e->arena = nullptr;
        e->arena_bytes = 0;
    }
    e->arena_cap = cap;
    rc = GFSM_OK;
    return e;
}

gfsm_status ensure_device(gfsm_ctx *ctx, gfsm_graph *g) {
    if (g->dev) return GFSM_OK;
    if (ctx->device < 0) return set_err(ctx, GFSM_ERR_NO_EXTENSION, "host-only context: no CUDA device bound");
    auto *dg = new (std::nothrow) DeviceGraph();
    if (!dg) return GFSM_ERR_NOMEM;
    std::string err;
    gfsm_status rc = build_device_graph(g->h, ctx->device, g->vl_mode, *dg, err);
    if (rc != GFSM_OK) {
        delete dg;
        return set_err(ctx, rc, "device CCSR build: " + err);
    }
    g->dev = dg;
    return GFSM_OK;
}

}  // namespace

extern "C" {

void gfsm_limits_default(gfsm_limits *lim) {
    if (!lim) return;
    lim->ccsr_rel_size = (uint32_t)env_u64("GFSM_CCSRRELSIZE", kCCSRRelSize);
    lim->max_soln_size = env_u64("GFSM_MAXSOLNSIZE", kMaxSolnSize);
    lim->max_scan_size = env_u64("GFSM_MAXSCANSIZE", kMaxScanSize);
    lim->upper_mem_limit = env_u64("GFSM_UPPERMEMLIMIT", kUpperMemLimit);
    lim->mem_limit = env_u64("GFSM_MEMLIMIT", kMemLimit);
    lim->vertex_labels = (int32_t)env_u64("GFSM_VERTEX_LABELS", 0);
    lim->degree_filter = (int32_t)env_u64("GFSM_DEGREE_FILTER", 1);
    lim->max_candidates = env_u64("GFSM_MAXCANDIDATES", 0);
}

const char *gfsm_status_str(gfsm_status s) {
    switch (s) {
    case GFSM_OK: return "ok";
    case GFSM_ERR_QUERY: return "query cannot be planned (disconnected or unsupported)";
    case GFSM_ERR_MISSING_FILE: return "missing file";
    case GFSM_ERR_INVALID_DATA: return "invalid graph data";
    case GFSM_ERR_MISSING_DATA: return "missing graph data";
    case GFSM_ERR_ARG: return "invalid argument";
    case GFSM_ERR_CUDA: return "CUDA error";
    case GFSM_ERR_NOMEM: return "MEMLIMIT too small";
    case GFSM_ERR_TOO_LARGE: return "graph or query too large";
    case GFSM_ERR_DEVICE_WAIT: return "bounded device wait ran out";
    case GFSM_ERR_NO_EXTENSION: return "no CUDA device";
    case GFSM_ERR_BUSY: return "queue full";
    case GFSM_ERR_STOPPED: return "server stopped";
    }
    return "unknown status";
}

const char *gfsm_last_error(gfsm_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

gfsm_status gfsm_init(gfsm_ctx **out, const gfsm_limits *lim, int device) {
    if (!out) return GFSM_ERR_ARG;
    *out = nullptr;
    gfsm_limits l;
    if (lim) l = *lim;
    else gfsm_limits_default(&l);
    if (l.ccsr_rel_size < 1 || l.ccsr_rel_size > 8) return GFSM_ERR_ARG;
    if (l.mem_limit > l.upper_mem_limit) return GFSM_ERR_ARG;
    if (l.max_soln_size < 1024 || l.max_scan_size < 1024) return GFSM_ERR_ARG;
    if (device == -1) {  // host-only context: parsing and planning, no matching
        auto *ctx = new (std::nothrow) gfsm_ctx();
        if (!ctx) return GFSM_ERR_NOMEM;
        ctx->lim = l;
        ctx->device = -1;
        *out = ctx;
        return GFSM_OK;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return GFSM_ERR_NO_EXTENSION;
    }
    if (device < 0 || device >= n) return GFSM_ERR_ARG;
    auto *ctx = new (std::nothrow) gfsm_ctx();
    if (!ctx) return GFSM_ERR_NOMEM;
    ctx->lim = l;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return GFSM_ERR_CUDA;
    }
    *out = ctx;
    return GFSM_OK;
}

void gfsm_destroy(gfsm_ctx *ctx) {
    if (!ctx) return;
    delete static_cast<Engine *>(ctx->engine);
    delete ctx;
}

gfsm_status gfsm_graph_load_buffer(gfsm_ctx *ctx, const char *buf, uint64_t len, gfsm_graph **out) {
    if (!ctx || !out || (!buf && len)) return GFSM_ERR_ARG;
    *out = nullptr;
    auto g = std::make_unique<gfsm_graph>();
    g->ctx = ctx;
    g->rel_bits = ctx->lim.ccsr_rel_size;
    g->vl_mode = ctx->lim.vertex_labels != 0;
    gfsm_status rc = parse_text(buf, len, g->rel_bits, g->h);
    if (rc != GFSM_OK) return set_err(ctx, rc, "");
    *out = g.release();
    return GFSM_OK;
}

gfsm_status gfsm_graph_load_text(gfsm_ctx *ctx, const char *path, gfsm_graph **out) {
    if (!ctx || !path || !out) return GFSM_ERR_ARG;
    *out = nullptr;
    FileBytes text;
    gfsm_status rc = text.open(path);
    if (rc != GFSM_OK) return set_err(ctx, rc, std::string("missing file ") + path);
    return gfsm_graph_load_buffer(ctx, text.data(), text.size(), out);
}

// An edge list as a host graph; edge labels keep the relation bits the
// reference's packed CCSR keeps (CCSRRelSize).
static gfsm_status edges_to_host(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                                 const uint32_t *elabel, const uint32_t *vlabel, uint32_t rel_bits, HostGraph &h) {
    h.n = n;
    h.src.assign(src, src + m);
    h.dst.assign(dst, dst + m);
    h.lab.resize(m);
    const uint32_t vb = 32u - rel_bits;
    for (uint64_t i = 0; i < m; ++i) {
        if (src[i] >= n || dst[i] >= n) return GFSM_ERR_INVALID_DATA;
        const uint32_t l = elabel ? elabel[i] : 1u;
        h.lab[i] = (uint8_t)(((uint32_t)(l << vb)) >> vb);
    }
    h.vlabel.assign(n, 0);
    if (vlabel) std::memcpy(h.vlabel.data(), vlabel, (uint64_t)n * 4);
    return GFSM_OK;
}

gfsm_status gfsm_graph_from_edges(gfsm_ctx *ctx, uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                                  const uint32_t *elabel, const uint32_t *vlabel, gfsm_graph **out) {
    if (!ctx || !out || (m && (!src || !dst))) return GFSM_ERR_ARG;
    *out = nullptr;
    if (m >= (1ull << 32)) return GFSM_ERR_TOO_LARGE;
    auto g = std::make_unique<gfsm_graph>();
    g->ctx = ctx;
    g->rel_bits = ctx->lim.ccsr_rel_size;
    g->vl_mode = ctx->lim.vertex_labels != 0;
    if (edges_to_host(n, m, src, dst, elabel, vlabel, g->rel_bits, g->h) != GFSM_OK)
        return set_err(ctx, GFSM_ERR_INVALID_DATA, "edge endpoint out of range");
    *out = g.release();
    return GFSM_OK;
}

gfsm_status gfsm_graph_to_device(gfsm_ctx *ctx, gfsm_graph *g) {
    if (!ctx || !g) return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    return ensure_device(ctx, g);
}

gfsm_status gfsm_graph_info_get(const gfsm_graph *g, gfsm_graph_info *info) {
    if (!g || !info) return GFSM_ERR_ARG;
    std::memset(info, 0, sizeof(*info));
    info->n = g->h.n;
    info->m = g->h.src.size();
    if (g->dev) {
        const DeviceGraph &d = *g->dev;
        info->rows = d.rows;
        info->max_degree = d.max_degree;
        info->symmetric = d.symmetric;
        info->multi_edges = d.multi;
        info->n_edge_labels = d.n_edge_labels;
        info->on_device = 1;
        info->device_bytes = d.bytes;
        info->build_alloc_ms = d.build_ms[0];
        info->build_h2d_ms = d.build_ms[1];
        info->build_kernel_ms = d.build_ms[2];
        info->build_d2h_ms = d.build_ms[3];
        info->build_wall_ms = d.build_wall_ms;
    } else {
        std::vector<uint32_t> deg(g->h.n, 0);
        for (uint32_t s : g->h.src) deg[s]++;
        for (uint32_t x : deg) {
            info->rows += x ? 1 : 0;
            info->max_degree = std::max(info->max_degree, x);
        }
    }
    return GFSM_OK;
}

gfsm_status gfsm_graph_download(gfsm_ctx *ctx, const gfsm_graph *g, uint32_t *rowptr, uint32_t *adj, uint8_t *elab,
                                uint32_t *order) {
    if (!ctx || !g) return GFSM_ERR_ARG;
    if (!g->dev) return GFSM_ERR_ARG;
    const DeviceGraph &d = *g->dev;
    cudaSetDevice(d.device);
    if (rowptr) std::memcpy(rowptr, d.h_rowptr.data(), ((uint64_t)d.n + 1) * 4);
    if (order) std::memcpy(order, d.h_order.data(), (uint64_t)d.n * 4);
    if (adj && d.m && cudaMemcpy(adj, d.adj, d.m * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return GFSM_ERR_CUDA;
    if (elab && d.m) {
        if (d.elab) {
            if (cudaMemcpy(elab, d.elab, d.m, cudaMemcpyDeviceToHost) != cudaSuccess) return GFSM_ERR_CUDA;
        } else {
            std::memset(elab, (int)d.single_label, d.m);
        }
    }
    return GFSM_OK;
}

void gfsm_graph_destroy(gfsm_graph *g) {
    if (!g) return;
    if (g->dev) {
        cudaSetDevice(g->dev->device);
        free_device_graph(*g->dev);
        delete g->dev;
    }
    delete g;
}

gfsm_status gfsm_query_prepare(gfsm_ctx *ctx, const gfsm_graph *q, gfsm_plan **out) {
    if (!ctx || !q || !out) return GFSM_ERR_ARG;
    *out = nullptr;
    auto p = std::make_unique<gfsm_plan>();
    gfsm_status rc = plan_query(q->h, q->rel_bits, p->p);
    if (rc != GFSM_OK) return set_err(ctx, rc, "");
    plan_symmetry(q->h, p->p, ctx->lim.vertex_labels != 0);
    *out = p.release();
    return GFSM_OK;
}

// The data graph's planner statistics, built on first use: vertex labels
// with their out-degrees, and whether embedding counts are independent of the
// matching order (every edge has its reverse with the same label and no
// edge repeats -- what FFS counts with a different anchor edge then equals).
static const PlanStats &plan_stats(const gfsm_graph *data) {
    gfsm_graph *g = const_cast<gfsm_graph *>(data);
    std::lock_guard<std::mutex> lk(g->stats_mu);
    if (g->stats) return *g->stats;
    auto st = std::make_unique<PlanStats>();
    const HostGraph &h = g->h;
    const uint64_t m = h.src.size();
    std::vector<uint32_t> outdeg(h.n, 0);
    for (uint64_t i = 0; i < m; ++i) outdeg[h.src[i]]++;
    // edges as (src, dst, label) and reversed; equal sorted lists <=> symmetric
    std::vector<std::pair<uint64_t, uint8_t>> fwd(m), rev(m);
    for (uint64_t i = 0; i < m; ++i) {
        fwd[i] = {((uint64_t)h.src[i] << 32) | h.dst[i], h.lab[i]};
        rev[i] = {((uint64_t)h.dst[i] << 32) | h.src[i], h.lab[i]};
    }
    std::sort(fwd.begin(), fwd.end());
    std::sort(rev.begin(), rev.end());
    bool inv = fwd == rev;
    for (uint64_t i = 1; i < m && inv; ++i)
        if (fwd[i].first == fwd[i - 1].first) inv = false;
    st->order_invariant = inv;
    std::vector<uint32_t> lab(h.n, 0);
    if (g->vl_mode) lab = h.vlabel;
    st->labels = lab;
    std::sort(st->labels.begin(), st->labels.end());
    st->labels.erase(std::unique(st->labels.begin(), st->labels.end()), st->labels.end());
    st->deg.resize(st->labels.size());
    for (uint32_t v = 0; v < h.n; ++v) {
        const size_t li = std::lower_bound(st->labels.begin(), st->labels.end(), lab[v]) - st->labels.begin();
        st->deg[li].push_back(outdeg[v]);
    }
    for (auto &d : st->deg) std::sort(d.begin(), d.end(), std::greater<uint32_t>());
    g->stats = std::move(st);
    return *g->stats;
}

// Data candidates of every query vertex: data vertices with its label (when
// labels are matched) and, under the degree filter, at least its degree --
// the sizes of the windows the level steps search.
static std::vector<double> candidate_weights(const HostGraph &q, const Plan &p, const PlanStats &st, bool vl,
                                             bool degree_filter) {
    std::vector<double> w(q.n, 0.0);
    for (uint32_t d = 0; d < p.k; ++d) {
        const uint32_t v = p.qvid[d];
        const uint32_t l = vl ? p.qlabel[d] : 0u;
        const auto it = std::lower_bound(st.labels.begin(), st.labels.end(), l);
        if (it == st.labels.end() || *it != l) continue;  // no such label: no candidates
        const std::vector<uint32_t> &dg = st.deg[it - st.labels.begin()];
        const uint32_t need = std::max<uint32_t>(degree_filter ? p.qdeg[d] : 0u, 1u);
        // degrees are descending: count those >= need
        const size_t c = std::partition_point(dg.begin(), dg.end(), [&](uint32_t x) { return x >= need; }) - dg.begin();
        w[v] = (double)c;
    }
    return w;
}

// Plans q for data: the data-aware order where the count cannot depend on
// the order, otherwise the reference's.
static gfsm_status plan_for(const HostGraph &q, uint32_t rel_bits, const PlanStats *st, const gfsm_limits &lim,
                            bool vl, Plan &out) {
    gfsm_status rc = plan_query(q, rel_bits, out);
    if (rc == GFSM_OK && st && st->order_invariant && out.order_invariant) {
        const std::vector<double> w = candidate_weights(q, out, *st, vl, lim.degree_filter != 0);
        Plan alt;
        if (plan_query(q, rel_bits, alt, &w) == GFSM_OK) out = std::move(alt);
    }
    if (rc == GFSM_OK) plan_symmetry(q, out, lim.vertex_labels != 0);
    return rc;
}

gfsm_status gfsm_query_prepare_for(gfsm_ctx *ctx, const gfsm_graph *q, const gfsm_graph *data, gfsm_plan **out) {
    if (!ctx || !q || !data || !out) return GFSM_ERR_ARG;
    *out = nullptr;
    const PlanStats &st = plan_stats(data);
    auto p = std::make_unique<gfsm_plan>();
    gfsm_status rc = plan_for(q->h, q->rel_bits, &st, ctx->lim, data->vl_mode, p->p);
    if (rc != GFSM_OK) return set_err(ctx, rc, "");
    *out = p.release();
    return GFSM_OK;
}

gfsm_status gfsm_plan_info(const gfsm_plan *p, uint32_t *planner, uint32_t *order_invariant) {
    if (!p) return GFSM_ERR_ARG;
    if (planner) *planner = p->p.planner;
    if (order_invariant) *order_invariant = p->p.order_invariant ? 1u : 0u;
    return GFSM_OK;
}

gfsm_status gfsm_plan_symmetry(const gfsm_plan *p, uint64_t *aut, uint32_t *n_cond, uint32_t *cond) {
    if (!p) return GFSM_ERR_ARG;
    if (aut) *aut = p->p.aut;
    if (n_cond) *n_cond = (uint32_t)p->p.sym_cond.size();
    if (cond)
        for (size_t i = 0; i < p->p.sym_cond.size(); ++i) {
            cond[2 * i] = p->p.sym_cond[i].first;
            cond[2 * i + 1] = p->p.sym_cond[i].second;
        }
    return GFSM_OK;
}

gfsm_status gfsm_query_prepare_batch(gfsm_ctx *ctx, int nq, const uint32_t *nv, const uint64_t *eoff,
                                     const uint32_t *src, const uint32_t *dst, const uint32_t *elabel,
                                     const uint32_t *vlabel, const gfsm_graph *data, gfsm_plan **out,
                                     int *failed) {
    if (failed) *failed = -1;
    if (!ctx || nq < 0 || (nq && (!nv || !eoff || !out))) return GFSM_ERR_ARG;
    if (nq == 0) return GFSM_OK;
    if (eoff[nq] && (!src || !dst)) return GFSM_ERR_ARG;
    for (int i = 0; i < nq; ++i) {
        out[i] = nullptr;
        if (eoff[i + 1] < eoff[i] || eoff[i + 1] - eoff[i] >= (1ull << 32)) return GFSM_ERR_ARG;
    }
    std::vector<uint64_t> voff(nq + 1, 0);
    for (int i = 0; i < nq; ++i) voff[i + 1] = voff[i] + nv[i];
    const uint32_t rel_bits = ctx->lim.ccsr_rel_size;
    const PlanStats *st = data ? &plan_stats(data) : nullptr;
    const bool vl = data ? data->vl_mode : false;
    std::vector<gfsm_status> rc(nq, GFSM_OK);
    // queries are tiny: one worker per ~64 of them, up to the host's threads
    const int hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min(hw, (nq + 63) / 64));
    auto work = [&](int t) {
        HostGraph h;  // reused: every field is reassigned per query, its capacity kept
        for (int i = t; i < nq; i += nt) {
            const uint64_t e0 = eoff[i], m = eoff[i + 1] - e0;
            rc[i] = edges_to_host(nv[i], m, src + e0, dst + e0, elabel ? elabel + e0 : nullptr,
                                  vlabel ? vlabel + voff[i] : nullptr, rel_bits, h);
            if (rc[i] != GFSM_OK) continue;
            auto p = std::unique_ptr<gfsm_plan>(new (std::nothrow) gfsm_plan());
            if (!p) { rc[i] = GFSM_ERR_NOMEM; continue; }
            rc[i] = plan_for(h, rel_bits, st, ctx->lim, vl, p->p);
            if (rc[i] == GFSM_OK) out[i] = p.release();
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    for (int i = 0; i < nq; ++i)
        if (rc[i] != GFSM_OK) {
            for (int j = 0; j < nq; ++j) {
                delete out[j];
                out[j] = nullptr;
            }
            if (failed) *failed = i;
            return set_err(ctx, rc[i], "query " + std::to_string(i) + " of the batch");
        }
    return GFSM_OK;
}

gfsm_status gfsm_plan_tables(const gfsm_plan *p, uint32_t *k, uint32_t *max_valency, uint32_t *order,
                             uint32_t *header, uint32_t *reqs) {
    if (!p) return GFSM_ERR_ARG;
    const Plan &x = p->p;
    if (k) *k = x.k;
    if (max_valency) *max_valency = x.max_valency;
    if (order) std::copy(x.order.begin(), x.order.end(), order);
    if (header) std::copy(x.header.begin(), x.header.end(), header);
    if (reqs) {
        // relation fields in the reference's packed form: label << CCSRVertSize
        const uint32_t vb = 32u - x.rel_bits;
        for (size_t i = 0; i < x.reqs.size(); ++i) reqs[i] = (i & 1) ? (x.reqs[i] << vb) : x.reqs[i];
    }
    return GFSM_OK;
}

gfsm_status gfsm_plan_columns(const gfsm_plan *p, uint32_t *qvid) {
    if (!p || !qvid) return GFSM_ERR_ARG;
    std::copy(p->p.qvid.begin(), p->p.qvid.end(), qvid);
    return GFSM_OK;
}

void gfsm_plan_destroy(gfsm_plan *p) { delete p; }

void gfsm_plan_destroy_array(gfsm_plan *const *plans, int n) {
    if (!plans) return;
    // a plan is a dozen small vectors: large batches free on a few host
    // threads (a worker that cannot be started runs on this thread)
    const int hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::max(1, std::min(hw, n / 256));
    auto work = [&](int t) {
        for (int i = t; i < n; i += nt) delete plans[i];
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) {
        try {
            pool.emplace_back(work, t);
        } catch (...) {
            work(t);
        }
    }
    work(0);
    for (auto &th : pool) th.join();
}

gfsm_status gfsm_batch_count(gfsm_ctx *ctx, const gfsm_plan *const *plans, int nq, const gfsm_graph *data,
                             uint64_t *counts, gfsm_stats *stats) {
    if (!ctx || !data || nq < 0 || (nq && (!plans || !counts))) return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    gfsm_status rc = ensure_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    std::string err;
    Engine *e = ctx_engine(ctx, *data->dev, rc, err);
    if (!e) return set_err(ctx, rc, err);
    std::vector<const Plan *> ps(nq);
    for (int i = 0; i < nq; ++i) {
        if (!plans[i]) return GFSM_ERR_ARG;
        ps[i] = &plans[i]->p;
    }
    rc = e->run(ps, *data->dev, ctx->lim, counts, stats, nullptr, 0, nullptr, err);
    return set_err(ctx, rc, err);
}

gfsm_status gfsm_batch_count_part(gfsm_ctx *ctx, const gfsm_plan *const *plans, int nq, const gfsm_graph *data,
                                  uint32_t part, uint32_t nparts, uint64_t *counts, gfsm_stats *stats) {
    if (!ctx || !data || nq < 0 || (nq && (!plans || !counts)) || nparts == 0 || part >= nparts)
        return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    gfsm_status rc = ensure_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    std::string err;
    Engine *e = ctx_engine(ctx, *data->dev, rc, err);
    if (!e) return set_err(ctx, rc, err);
    std::vector<const Plan *> ps(nq);
    for (int i = 0; i < nq; ++i) {
        if (!plans[i]) return GFSM_ERR_ARG;
        ps[i] = &plans[i]->p;
    }
    rc = e->run(ps, *data->dev, ctx->lim, counts, stats, nullptr, 0, nullptr, err, -1, part, nparts);
    return set_err(ctx, rc, err);
}

gfsm_status gfsm_partition_rows(const uint32_t *rowptr, uint32_t lo, uint32_t hi, uint32_t nparts,
                                uint64_t *bounds) {
    if (!rowptr || !bounds || nparts == 0 || hi < lo) return GFSM_ERR_ARG;
    root_partition(rowptr, lo, hi, nparts, bounds);
    return GFSM_OK;
}

gfsm_status gfsm_root_partition(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data, uint32_t nparts,
                                uint32_t *window_lo, uint64_t *bounds) {
    if (!ctx || !plan || !data || !bounds || !window_lo || nparts == 0) return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    gfsm_status rc = ensure_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    DQuery dq;
    uint32_t lo = 0, hi = 0;
    bool never = false;
    rc = build_dquery(plan->p, *data->dev, ctx->lim, dq, lo, hi, never);
    if (rc != GFSM_OK) return set_err(ctx, rc, "query cannot be planned against this graph");
    if (never) hi = lo;  // no root can match: an empty window
    *window_lo = lo;
    root_partition(data->dev->h_rowptr.data(), lo, hi, nparts, bounds);
    return GFSM_OK;
}

gfsm_status gfsm_match_count(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data, uint64_t *count,
                             gfsm_stats *stats) {
    if (!plan || !count) return GFSM_ERR_ARG;
    return gfsm_batch_count(ctx, &plan, 1, data, count, stats);
}

gfsm_status gfsm_match_mappings(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data, uint32_t *rows,
                                uint64_t max_rows, uint64_t *n_rows, uint64_t *count, gfsm_stats *stats) {
    if (!ctx || !plan || !data || !count || (max_rows && !rows)) return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    gfsm_status rc = ensure_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    std::string err;
    Engine *e = ctx_engine(ctx, *data->dev, rc, err);
    if (!e) return set_err(ctx, rc, err);
    std::vector<const Plan *> ps{&plan->p};
    uint64_t c = 0;
    rc = e->run(ps, *data->dev, ctx->lim, &c, stats, rows, max_rows, n_rows, err);
    *count = c;
    return set_err(ctx, rc, err);
}

}  // extern "C"
