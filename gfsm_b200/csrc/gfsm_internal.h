// gfsm_internal.h -- host/device structures shared inside libgfsm.
#pragma once
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gfsm.h"

namespace gfsm {

constexpr int MAXQ = 16;              // query vertices supported by the device plan
constexpr uint8_t REQ_SELF = 0xFF;    // requirement on the candidate's own row (query self-loop)

// Environment.h:6-11 defaults.
constexpr uint32_t kCCSRRelSize = 8;
constexpr uint64_t kMaxSolnSize = 500'000'000ull;
constexpr uint64_t kMaxScanSize = 500'000'000ull;
constexpr uint64_t kMemLimit = 22'000'000'000ull;
constexpr uint64_t kUpperMemLimit = 44'000'000'000ull;

// Allocator whose resize() leaves new elements uninitialised: the code that
// resizes the edge arrays below writes every element, on several threads,
// which then also take the first-touch page faults instead of one thread
// zeroing tens of MB first.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <class U>
    void construct(U *p) noexcept {
        ::new (static_cast<void *>(p)) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a) {
        ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
    }
};
template <class T>
using RawVec = std::vector<T, NoInitAlloc<T>>;

// ---------------------------------------------------------------------------
// Host-side graph: the parsed edge lines, labels masked to CCSRRelSize bits.
// ---------------------------------------------------------------------------
struct HostGraph {
    uint32_t n = 0;
    RawVec<uint32_t> src, dst;        // directed entries, input order
    RawVec<uint8_t> lab;              // edge label & ((1<<CCSRRelSize)-1)
    std::vector<uint32_t> vlabel;     // per vertex id (v lines), 0 if absent
};

// Device CCSR.  Internal vertex ids are the reference's CCSR row order
// (degree descending, then id ascending; HnHelper.cuh:26-31, 413), grouped by
// vertex label first when vertex labels are matched.  Rows list neighbour
// internal ids ascending (HnHelper.cuh:470-478).
struct DeviceGraph {
    int device = 0;
    uint32_t n = 0, rows = 0, max_degree = 0;
    uint64_t m = 0;
    uint32_t *rowptr = nullptr;       // [n+1]
    uint32_t *adj = nullptr;          // [m]
    uint8_t *elab = nullptr;          // [m], null when every entry has the same label
    uint32_t single_label = 0;        // the label when elab == null
    uint32_t *order = nullptr;        // [n] internal id -> original id
    void *block = nullptr;            // the one allocation rowptr, adj, order and elab live in
    bool symmetric = false, multi = false;
    int n_edge_labels = 0;
    bool vl_grouped = false;
    // host copies used by the planner (degree windows) and for output
    std::vector<uint32_t> h_rowptr;   // [n+1]
    std::vector<uint32_t> h_order;    // [n]
    std::vector<uint32_t> group_value;// sorted distinct vertex label values (grouped mode)
    std::vector<uint32_t> group_start;// [groups+1]
    // degree windows: deg_cut[g * kCutDeltas + delta] = the first id of
    // group g whose degree is below delta (ids in a group are
    // degree-descending), for delta < kCutDeltas
    static constexpr uint32_t kCutDeltas = 17;
    std::vector<uint32_t> deg_cut;
    uint64_t bytes = 0;
    // build time: allocation, host-to-device copies, device passes, copies
    // back (CUDA events on the build stream), and the host wall time
    double build_ms[4] = {0, 0, 0, 0};
    double build_wall_ms = 0;
    uint32_t degree(uint32_t v) const { return h_rowptr[v + 1] - h_rowptr[v]; }
};

// ---------------------------------------------------------------------------
// Query plan (host).  The reference tables plus what the device plan needs.
// ---------------------------------------------------------------------------
struct Plan {
    uint32_t k = 0, max_valency = 0;
    uint32_t rel_bits = 8;           // CCSRRelSize the query was parsed with
    std::vector<uint32_t> order;     // depth -> query CCSR row index
    std::vector<uint32_t> header;    // [3k]
    std::vector<uint32_t> reqs;      // [2*maxv*k] (distance delta, label value)
    std::vector<uint32_t> qvid;      // depth -> query vertex id
    std::vector<uint32_t> qlabel;    // depth -> query vertex label value
    std::vector<uint32_t> qdeg;      // depth -> distinct non-self neighbours
    bool symmetric = false;          // query structure is symmetric
    bool order_invariant = false;    // symmetric with equal labels both ways, no repeated edge
    uint32_t planner = 0;            // 0: the reference's order; 1: data-aware order
    // Symmetry breaking (order-invariant queries only): the query's
    // automorphism group has `aut` elements; counting only the embeddings f
    // with f(a) < f(b) for every (a, b) in sym_cond (query vertex ids) and
    // multiplying by `aut` gives the full count.  sym_vl: automorphisms were
    // required to keep vertex labels (vertex-label matching).
    uint64_t aut = 1;
    bool sym_vl = false;
    std::vector<std::pair<uint32_t, uint32_t>> sym_cond;
};

// Per-depth device plan of one query against one data graph.
struct alignas(16) DLevel {
    uint32_t lo, hi;           // candidate id window of this depth
    uint32_t next_lo, next_hi; // window of depth+1
    uint8_t anchor;            // tuple position of the anchor (depth index)
    uint8_t next_anchor;       // anchor position for depth+1
    uint8_t nreq;              // extra requirement checks
    uint8_t anchor_lab;        // label of the anchor requirement
    uint8_t final_;            // depth == k-1
    uint8_t anchor_check;      // bit 0: the anchor requirement needs a row search (multi-edge
                               // data); bit 1 (a branching trie node's representative): every
                               // child node's depth+1 is a last vertex counted at its parent
    uint16_t next_ub;          // symmetry breaking: depth+1's candidate < tuple[pos] for these positions
    uint8_t req_pos[MAXQ];     // tuple position, or REQ_SELF
    uint8_t req_lab[MAXQ];
    // shared-prefix trie (set on a node's representative): the node's child
    // nodes at depth+1 are fan_list[fan_start, fan_start + fan_count) when it
    // has more than one
    uint16_t fan_count;
    uint16_t next_lb;          // symmetry breaking: depth+1's candidate > tuple[pos] for these positions
    uint32_t fan_start;
};
static_assert(sizeof(DLevel) == 64, "DLevel layout");

struct alignas(16) DQuery {
    DLevel lv[MAXQ];
    uint8_t col[MAXQ];         // depth -> output column (query vertex id)
    uint32_t k;
    uint32_t pad[3];
};

// Totals of one level step.  `alloc` hands out child slots: every tile adds
// (its children << kAllocShift) + (their next-level candidates) with one
// atomic, so slot order and the candidate prefix advance together; once the
// step has finished the word holds the step's totals, which the host copies
// into n_children / total_next.
struct StepResult {
    unsigned long long n_children;
    unsigned long long total_next;
    unsigned long long alg_bytes;
    unsigned long long alloc;
    unsigned int err;          // error bits a kernel may raise (none does today; the host checks them)
    unsigned int rows;         // mapping rows claimed (mapping mode)
    unsigned int tile_ctr;     // graph-driven steps: tiles handed out so far (tickets)
    unsigned int next_ovf;     // the step's next-level candidates exceed the allocator's field
};

constexpr int kAllocShift = 34;                                  // child count: bits 34..63
constexpr unsigned long long kAllocMask = (1ull << kAllocShift) - 1;  // candidates: bits 0..33
// An emitting step takes fewer candidates than the child-count field holds,
// so the count never wraps (every candidate yields at most one child); a
// step whose children's next-level candidates pass 2^34 raises next_ovf and
// is re-run smaller.  The schedule sizes a depth's steps so that the next
// level's candidates, at the rate observed there, fill at most half the
// field; a depth's first step (rate not yet seen) takes at most
// kFirstEmitChunk candidates.
constexpr unsigned long long kMaxEmitChunk = (1ull << (64 - kAllocShift)) - 1024;
constexpr unsigned long long kFirstEmitChunk = 1ull << 26;

// Error bits of a schedule (the graph-driven controller sets them; the
// host-driven loop checks the same conditions on the host).
enum : uint32_t {
    KERR_CAP = 16u,            // the candidate cap (max_candidates) was reached, or one tile overflowed
};

}  // namespace gfsm

// ---------------------------------------------------------------------------
// Opaque C handles
// ---------------------------------------------------------------------------
struct gfsm_ctx {
    gfsm_limits lim{};
    int device = 0;
    std::string last_error;
    std::mutex mu;
    void *engine = nullptr;   // default gfsm::Engine (stream + frontier arena)
    uint64_t calls = 0;       // matching calls on the default engine
};

namespace gfsm {
// What the data-aware planner needs of a data graph (built once, on demand).
struct PlanStats {
    bool order_invariant = false;            // symmetric with equal labels both ways, no repeated edge
    std::vector<uint32_t> labels;            // distinct vertex labels, ascending
    std::vector<std::vector<uint32_t>> deg;  // per label: out-degrees, descending
};
}  // namespace gfsm

struct gfsm_graph {
    gfsm_ctx *ctx = nullptr;
    gfsm::HostGraph h;
    gfsm::DeviceGraph *dev = nullptr;
    uint32_t rel_bits = 8;
    bool vl_mode = false;
    std::mutex stats_mu;
    std::unique_ptr<gfsm::PlanStats> stats;
    std::vector<double> deg2;  // prefix sums of squared row lengths (served form's predictor)
};

struct gfsm_plan {
    gfsm::Plan p;
};

namespace gfsm {
// host_graph.cpp
gfsm_status parse_text(const char *buf, uint64_t len, uint32_t rel_bits, HostGraph &g);
// A file's bytes: mapped read-only where it can be (no copy; the parse
// threads fault their own chunks in), else read whole into memory.
class FileBytes {
public:
    FileBytes() = default;
    FileBytes(const FileBytes &) = delete;
    FileBytes &operator=(const FileBytes &) = delete;
    ~FileBytes() { close(); }
    gfsm_status open(const char *path);
    void close();
    const char *data() const { return map_ ? static_cast<const char *>(map_) : buf_.data(); }
    uint64_t size() const { return len_; }

private:
    void *map_ = nullptr;
    uint64_t len_ = 0;
    std::string buf_;
};
// weight == nullptr: the reference's matching order.  Otherwise weight[v]
// estimates query vertex v's data candidates and the order is data-aware
// (only valid where the count cannot depend on the order).
gfsm_status plan_query(const HostGraph &q, uint32_t rel_bits, Plan &p, const std::vector<double> *weight = nullptr);
// Fills p.aut / p.sym_cond for an order-invariant query (labels kept when
// vl).  Base points follow the matching order, so conditions bound later
// depths by earlier ones.  Leaves aut = 1 if the search grows too large.
void plan_symmetry(const HostGraph &q, Plan &p, bool vl);
// builder.cu
gfsm_status build_device_graph(const HostGraph &h, int device, bool vl_mode, DeviceGraph &out,
                               std::string &err);
void free_device_graph(DeviceGraph &g);
// engine.cu
// sym: also encode the plan's symmetry-breaking conditions (the caller then
// multiplies the count by p.aut).
gfsm_status build_dquery(const Plan &p, const DeviceGraph &g, const gfsm_limits &lim,
                         DQuery &dq, uint32_t &root_lo, uint32_t &root_hi, bool &never, bool sym = false);
// Device bytes one partial mapping of depth d's buffer takes: query id and
// d+1 tuple columns, its next-level slice start and candidate prefix.
#ifdef __CUDACC__
__host__ __device__
#endif
constexpr unsigned long long tuple_bytes(uint32_t d) { return 4ull * (d + 2) + 4 + 8; }
// Degree-balanced cut of a root window [lo, hi) of internal ids into nparts
// consecutive ranges: bounds[0..nparts] are offsets into the window, part k
// is [lo + bounds[k], lo + bounds[k+1]), and each part's rows hold about
// 1/nparts of the window's CCSR entries (a root's entries are its first
// expansion).  rowptr is the CCSR row pointer over internal ids.
void root_partition(const uint32_t *rowptr, uint32_t lo, uint32_t hi, uint32_t nparts, uint64_t *bounds);
}  // namespace gfsm
