// engine.h -- one matching engine = one CUDA stream + one frontier arena.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "gfsm_internal.h"

namespace gfsm {

struct Engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_begin = nullptr, ev_end = nullptr;
    void *arena = nullptr;         // frontier buffers + per-call plans/counts
    uint64_t arena_bytes = 0;
    uint64_t arena_cap = 0;        // bytes the arena may use (MEMLIMIT share)
    void *small = nullptr;         // step result, counters, tile directory, control block
    uint64_t small_bytes = 0;
    uint32_t dir_tiles = 0;        // tile directory capacity (tiles per step)
    StepResult *d_result = nullptr;
    StepResult *h_result = nullptr;  // pinned
    void *h_stage = nullptr;         // pinned staging of a call's arena head (plans, root tables, ...)
    uint64_t h_stage_bytes = 0;
    uint32_t *rows_ctr = nullptr;
    uint32_t *tile_parent = nullptr;
    uint64_t max_scan = 0;
    // graph-driven schedule (one graph launch per call; built once per engine)
    int arg_slot = -1;             // constant-memory slot for this engine's step arguments
    void *ctl = nullptr;           // device control block (inside the small region)
    // one graph per tile geometry the schedule is instantiated for (two)
    int step_blocks[2] = {0, 0};   // fixed grid of the graph's step kernel
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t graph_exec[2] = {nullptr, nullptr};
    bool graph_failed[2] = {false, false};
    int last_graph_error = 0;      // why the last graph could not be built (cudaError_t, or -2: no slot)

    Engine() = default;
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;
    ~Engine();
    void release();
    gfsm_status init(int dev, uint64_t arena_limit, uint64_t scan_limit, std::string &err);
    gfsm_status ensure_arena(uint64_t bytes, std::string &err);
    // The graph-driven schedule for tile geometry `variant` (built once,
    // relaunched by every call); GFSM_ERR_CUDA where there is none.
    gfsm_status build_graph(int variant, std::string &err);
    // Counts every plan against g; counts_out[i] for plans[i].  With rows_out
    // (single plan only) also writes up to max_rows full mappings.
    // variant < 0: tile geometry chosen by the autotuner.
    // part / nparts: count only the embeddings whose root lies in part
    // `part` of each query's root window cut by root_partition (counts of
    // the nparts parts add up to the whole count).
    gfsm_status run(const std::vector<const Plan *> &plans, const DeviceGraph &g, const gfsm_limits &lim,
                    uint64_t *counts_out, gfsm_stats *stats, uint32_t *rows_out, uint64_t max_rows,
                    uint64_t *n_rows, std::string &err, int variant = -1, uint32_t part = 0, uint32_t nparts = 1);
    int pick_variant(const std::vector<const Plan *> &plans, const DeviceGraph &g, const gfsm_limits &lim,
                     std::string &err);
    std::map<uint64_t, int> tuned;  // autotuner: workload class -> tile geometry
    // per workload class, the next-level candidates per candidate each depth
    // saw in the last call: the next call sizes a depth's first step from it
    // instead of the conservative first-step cap
    std::map<uint64_t, std::vector<double>> nxt_seen;
    bool autotune = true;           // off for served slots: tuning runs would sit on the request path
    // the driver tuning runs take (that of the call being tuned): 0 host
    // loop, 1 graph; -1 outside tuning (chosen by the call's size)
    int tune_driver = -1;
};

}  // namespace gfsm
