// serve.cpp -- served form: a request loop over a resident data graph.
//
// Requests are admitted into per-slot device batches.  Each slot is its own
// Engine (CUDA stream + frontier arena holding an equal share of MEMLIMIT),
// so a batch can start while other slots' batches are still on the GPU and
// their work overlaps on the device.  A slot admits pending requests in
// arrival order while their predicted frontier bytes fit its budget (the
// first request is always admitted; the engine's chunking keeps its memory
// bounded either way), up to max_batch.  The reference has no serving path;
// its only unit of work is one query per process (main.cu:56-65).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>

#include "engine.h"
#include "gfsm_internal.h"

using namespace gfsm;

namespace {

using Clock = std::chrono::steady_clock;

constexpr uint64_t kAdmitArenas = 8;  // default admission budget, in slot arenas

struct Req {
    uint64_t id;
    Plan plan;
    double submit_ms;
    double pred_bytes;
};

}  // namespace

namespace gfsm {

// Prefix sums of squared row lengths over internal ids (deg2[i] = sum of
// deg(v)^2 for v < i), built once per data graph on first use.
const std::vector<double> &graph_deg2(const gfsm_graph *data) {
    gfsm_graph *g = const_cast<gfsm_graph *>(data);
    std::lock_guard<std::mutex> lk(g->stats_mu);
    if (g->deg2.empty()) {
        const DeviceGraph &d = *data->dev;
        g->deg2.resize((size_t)d.n + 1);
        g->deg2[0] = 0.0;
        for (uint32_t v = 0; v < d.n; ++v) {
            const double x = (double)(d.h_rowptr[v + 1] - d.h_rowptr[v]);
            g->deg2[v + 1] = g->deg2[v] + x * x;
        }
    }
    return g->deg2;
}

// Predicted peak frontier bytes of one query: the partial mappings of every
// non-final depth held at once, each level's count the previous one's times
// its expected candidate slice times 1/2 per extra requirement.  The
// expected slice of a parent is the anchor's expected row length -- the
// size-biased mean deg^2 / deg over the anchor's window, since the anchor
// was itself reached along an edge (the plain mean for the root) -- times
// the share of all CCSR entries that land in the new vertex's window.
double predict_bytes(const Plan &p, const DeviceGraph &g, const std::vector<double> &deg2, const gfsm_limits &lim) {
    DQuery dq;
    uint32_t lo = 0, hi = 0;
    bool never = false;
    if (build_dquery(p, g, lim, dq, lo, hi, never) != GFSM_OK || never || g.m == 0) return 0.0;
    const double vol_all = (double)g.m;
    auto vol = [&](uint32_t a, uint32_t b) { return (double)(g.h_rowptr[b] - g.h_rowptr[a]); };
    std::vector<double> f(p.k, 0.0);
    f[0] = (double)(hi - lo);
    double peak = 0.0, live = 0.0;
    for (uint32_t d = 1; d < p.k; ++d) {
        const DLevel &L = dq.lv[d];
        const uint32_t a = L.anchor;  // tuple position of the anchor
        const DLevel &A = dq.lv[a];
        const double va = vol(A.lo, A.hi);
        const double row = va <= 0.0 ? 0.0
                           : a == 0 ? va / std::max(1.0, (double)(A.hi - A.lo))
                                    : (deg2[A.hi] - deg2[A.lo]) / va;
        double grow = row * vol(L.lo, L.hi) / vol_all;
        for (uint32_t r = 0; r < L.nreq; ++r) grow *= 0.5;
        f[d] = f[d - 1] * grow;
        if (d + 1 < p.k) {
            live += f[d] * (double)tuple_bytes(d);
            peak = std::max(peak, live);
        }
        if (peak > 1e18) break;
    }
    return peak;
}

}  // namespace gfsm

struct gfsm_server {
    gfsm_ctx *ctx = nullptr;
    const gfsm_graph *data = nullptr;
    gfsm_serve_config cfg{};
    uint64_t slot_budget = 0;
    std::vector<std::unique_ptr<Engine>> engines;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<Req> pending;
    std::vector<gfsm_result> done;
    uint64_t submitted = 0, finished = 0;
    bool stop = false;
    Clock::time_point t0;
    std::string err;

    double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }

    void worker(int slot) {
        Engine *e = engines[slot].get();
        for (;;) {
            std::vector<Req> batch;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !pending.empty(); });
                if (stop && pending.empty()) return;
                double budget = (double)slot_budget, used = 0.0;
                while (!pending.empty() && (int)batch.size() < cfg.max_batch) {
                    const double b = pending.front().pred_bytes;
                    if (!batch.empty() && used + b > budget) break;
                    used += b;
                    batch.push_back(std::move(pending.front()));
                    pending.pop_front();
                }
            }
            const double start = now_ms();
            std::vector<const Plan *> ps(batch.size());
            for (size_t i = 0; i < batch.size(); ++i) ps[i] = &batch[i].plan;
            std::vector<uint64_t> counts(batch.size(), 0);
            std::string err_local;
            gfsm_status rc = e->run(ps, *data->dev, ctx->lim, counts.data(), nullptr, nullptr, 0, nullptr, err_local);
            const double end = now_ms();
            {
                std::lock_guard<std::mutex> lk(mu);
                for (size_t i = 0; i < batch.size(); ++i) {
                    gfsm_result r{};
                    r.req_id = batch[i].id;
                    r.count = counts[i];
                    r.status = rc;
                    r.submit_ms = batch[i].submit_ms;
                    r.start_ms = start;
                    r.done_ms = end;
                    done.push_back(r);
                }
                finished += batch.size();
                if (rc != GFSM_OK) err = err_local;
            }
            cv_done.notify_all();
        }
    }
};

extern "C" {

gfsm_status gfsm_serve_start(gfsm_ctx *ctx, const gfsm_graph *data, const gfsm_serve_config *cfg,
                             gfsm_server **out) {
    if (!ctx || !data || !out) return GFSM_ERR_ARG;
    *out = nullptr;
    gfsm_status rc = gfsm_graph_to_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    auto s = std::make_unique<gfsm_server>();
    s->ctx = ctx;
    s->data = data;
    gfsm_serve_config c{};
    if (cfg) c = *cfg;
    if (c.slots <= 0) c.slots = 2;
    if (c.max_batch <= 0) c.max_batch = 256;
    if (c.queue_capacity <= 0) c.queue_capacity = 65536;
    s->cfg = c;
    const DeviceGraph &g = *data->dev;
    const uint64_t avail = ctx->lim.mem_limit > g.bytes ? ctx->lim.mem_limit - g.bytes : 0;
    uint64_t per_slot = avail / (uint64_t)c.slots;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        uint64_t f = free_b > (2ull << 30) ? free_b - (2ull << 30) : free_b / 2;
        per_slot = std::min<uint64_t>(per_slot, f / (uint64_t)c.slots);
    }
    for (int i = 0; i < c.slots; ++i) {
        auto e = std::make_unique<Engine>();
        std::string err;
        const uint64_t scan = std::min<uint64_t>(ctx->lim.max_scan_size, 1ull << 28);
        rc = e->init(ctx->device, 0, scan, err);
        if (rc != GFSM_OK) return rc;
        e->arena_cap = per_slot > e->small_bytes ? per_slot - e->small_bytes : 0;
        e->autotune = false;  // a request never waits for tuning runs ...
        // ... but a slot uses the tile geometries the context's own engine
        // has already chosen (batched calls on the same context)
        if (ctx->engine) e->tuned = static_cast<Engine *>(ctx->engine)->tuned;
        // pinned staging for a full batch's plans, so no request allocates it
        const uint64_t stage = std::max<uint64_t>(1ull << 20, (uint64_t)c.max_batch * sizeof(DQuery) * 2);
        if (cudaMallocHost(&e->h_stage, stage) != cudaSuccess) return GFSM_ERR_NOMEM;
        e->h_stage_bytes = stage;
        // the graph a single-query batch runs is built now, not on a request
        // (if no argument slot is left, the slot runs the host-driven loop)
        std::string gerr;
        e->build_graph(0, gerr);
        // and the slot's frontier arena: a first request must not pay a
        // multi-GB cudaMalloc
        rc = e->ensure_arena(e->arena_cap, err);
        if (rc != GFSM_OK) return rc;
        s->engines.push_back(std::move(e));
    }
    // default admission budget: 8 arenas' worth of predicted (unchunked)
    // frontier -- the engine's depth-first chunking runs such a batch in its
    // own arena with a few more steps, while a budget of one arena split
    // saturated batches into a few hundred queries and lost the shared
    // prefixes (40k offered queries/s on the road grid: 28k -> see the bench)
    s->slot_budget = c.frontier_bytes ? c.frontier_bytes : kAdmitArenas * per_slot;
    s->t0 = Clock::now();
    gfsm_server *raw = s.get();
    for (int i = 0; i < c.slots; ++i) s->workers.emplace_back([raw, i] { raw->worker(i); });
    *out = s.release();
    return GFSM_OK;
}

gfsm_status gfsm_predict_frontier_bytes(gfsm_ctx *ctx, const gfsm_plan *plan, const gfsm_graph *data,
                                        double *bytes) {
    if (!ctx || !plan || !data || !bytes) return GFSM_ERR_ARG;
    gfsm_status rc = gfsm_graph_to_device(ctx, const_cast<gfsm_graph *>(data));
    if (rc != GFSM_OK) return rc;
    *bytes = predict_bytes(plan->p, *data->dev, graph_deg2(data), ctx->lim);
    return GFSM_OK;
}

gfsm_status gfsm_serve_submit(gfsm_server *s, const gfsm_plan *plan, uint64_t req_id) {
    if (!s || !plan) return GFSM_ERR_ARG;
    Req r;
    r.id = req_id;
    r.plan = plan->p;
    r.pred_bytes = predict_bytes(r.plan, *s->data->dev, graph_deg2(s->data), s->ctx->lim);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return GFSM_ERR_STOPPED;
        if ((int)s->pending.size() >= s->cfg.queue_capacity) return GFSM_ERR_BUSY;
        r.submit_ms = s->now_ms();
        s->pending.push_back(std::move(r));
        s->submitted++;
    }
    s->cv.notify_one();
    return GFSM_OK;
}

gfsm_status gfsm_serve_poll(gfsm_server *s, gfsm_result *out, int max, int *n) {
    if (!s || !n || (max > 0 && !out)) return GFSM_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    int k = std::min<int>(max, (int)s->done.size());
    for (int i = 0; i < k; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return GFSM_OK;
}

gfsm_status gfsm_serve_drain(gfsm_server *s, double timeout_ms) {
    if (!s) return GFSM_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto pred = [&] { return s->finished >= s->submitted; };
    if (timeout_ms <= 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred))
        return GFSM_ERR_BUSY;
    return GFSM_OK;
}

gfsm_status gfsm_serve_stop(gfsm_server *s) {
    if (!s) return GFSM_ERR_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto &t : s->workers) t.join();
    delete s;
    return GFSM_OK;
}

}  // extern "C"
