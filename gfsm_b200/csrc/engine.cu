// engine.cu -- the FFS level expansion on sm_100a (the hot path).
//
// Reference: HnGPU.cu:455-669 hnSolve drives, per level, hnGen (:114-185:
// copy the anchor's row as candidates), hnCheck (:190-262: injectivity +
// requirement rows), two CUB scans (:339-349) and hnRemove (:309-334:
// compaction), with CDP launches and device-side syncs.
//
// Here one kernel, k_step, does a whole level step over a range of the
// candidate space:
//   * candidate space = for every parent partial mapping, the part of its
//     anchor's row that passes the degree/label window of the new query
//     vertex (rows are sorted by a degree-descending, label-grouped id, so
//     the window is one contiguous slice found by two binary searches when
//     the parent was produced);
//   * tiles of 512-1024 candidates (autotuned geometry), so hub rows are
//     split across tiles and every thread does the same amount of row work --
//     the load balance the reference's thread-per-parent hnGen lacks;
//   * per candidate: injectivity against the parent tuple, the anchor's edge
//     label, and a search in each other backward neighbour's row for the
//     remaining requirements;
//   * survivors are ranked with __ballot_sync/__popc into shared memory, and
//     the tile's output offset (child count and next-level candidate count)
//     comes from one 64-bit atomic on the step's allocator word -- no tile
//     waits for another;
//   * a batch shares query prefixes through a trie of its plans: a tuple
//     stands for every query of its trie node, and a branching node's
//     candidates run over (child node, row offset);
//   * children are written as full tuples (SoA columns) together with their
//     own next-level candidate slice, so the next step needs no scan, no
//     pointer chasing up a forest, and no separate compaction;
//   * at the last query vertex nothing is written: survivors are counted.
// The host drives the steps depth-first over candidate chunks so that the
// frontier never exceeds MEMLIMIT (the reference restarts at 2x memory).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <type_traits>

#include "engine.h"

namespace gfsm {

namespace {

constexpr int T = 256;
constexpr int CPT = 4;
constexpr int TILE = T * CPT;

// First index in a[0, n) whose value is >= key (branch-free halving).
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t n, uint32_t key) {
    if (n == 0) return 0;
    const uint32_t *base = a;
    while (n > 1) {
        uint32_t half = n >> 1;
        base = (__ldg(base + half) < key) ? base + half : base;
        n -= half;
    }
    return (uint32_t)(base - a) + (__ldg(base) < key ? 1u : 0u);
}

struct GraphView {
    const uint32_t *__restrict__ rowptr;
    const uint32_t *__restrict__ adj;
    const uint8_t *__restrict__ elab;
    const uint32_t *__restrict__ order;
    uint32_t single_label;
    uint32_t n;
};

// Rows of at most SHORT_ROW entries (most rows of road-like and sparse
// graphs) are read with independent loads -- one memory round trip -- and
// searched in registers instead of by a chain of dependent probes.
constexpr uint32_t SHORT_ROW = 8;

// reqExists (HnGPU.cu:34-52) as a search: does the row adj[rs, re) hold
// (v, lab)?
__device__ __forceinline__ bool row_holds(const GraphView &g, uint32_t rs, uint32_t re, uint32_t v, uint32_t lab) {
    if (!g.elab && lab != g.single_label) return false;
    if (!g.elab && re - rs <= SHORT_ROW) {
        bool f = false;
#pragma unroll
        for (uint32_t i = 0; i < SHORT_ROW; ++i)
            if (rs + i < re && __ldg(g.adj + rs + i) == v) f = true;
        return f;
    }
    uint32_t p = rs + lower_bound_u32(g.adj + rs, re - rs, v);
    if (!g.elab) return p < re && __ldg(g.adj + p) == v;
    for (; p < re && __ldg(g.adj + p) == v; ++p)
        if (__ldg(g.elab + p) == lab) return true;
    return false;
}

// Does u's row hold (v, lab)?
__device__ __forceinline__ bool has_edge(const GraphView &g, uint32_t u, uint32_t v, uint32_t lab) {
    return row_holds(g, __ldg(g.rowptr + u), __ldg(g.rowptr + u + 1), v, lab);
}

struct StepArgs {
    GraphView g;
    const DQuery *__restrict__ plans;
    uint32_t depth;
    // parents: SoA columns (qid, m_0 .. m_{depth-1}), column c at ptup + c*pstride
    const uint32_t *__restrict__ ptup;
    uint64_t pstride;
    const uint32_t *__restrict__ pcstart;
    unsigned long long *pcoff;                      // [np+1]; pcoff[np] = pcoff_end, written by the partition
    unsigned long long pcoff_end;
    uint64_t np;
    const uint32_t *__restrict__ tile_parent;       // [ntiles+1]
    unsigned long long c0, cend;
    uint32_t ntiles;
    // children: SoA columns (qid, m_0 .. m_depth)
    uint32_t *ctup;
    uint64_t cstride, ccap;
    uint32_t *ccstart;
    unsigned long long *ccoff;                      // [ccap+1]
    // results
    unsigned long long *counts;                     // per query
    StepResult *result;
    // mapping capture at the final depth (optional)
    uint32_t *rows_out;
    uint64_t max_rows;
    uint32_t *rows_ctr;
    // shared query prefixes: root parent i is the trie node of query
    // root_rep[i]; a tuple's query id is its node's representative, with
    // kBranch set when the node has several child nodes (fan_list)
    const uint32_t *__restrict__ root_rep;
    const uint32_t *__restrict__ fan_list;
    // count a last query vertex when its parent is written, where nothing is
    // left to check (next_slice); only where the step's counts are committed
    // after the step is accepted (a re-run step must not count twice)
    uint32_t leaf_count;
};

// A tuple's column 0: its trie node (bits 0-21) with flags.  kBranch: the
// node has several child nodes (fan_list).  Bits 22-29: entries of the
// tuple's next-level slice (bit i = entry i) that are vertices of the tuple
// itself -- they would fail injectivity, so they are not candidates.
// kInjDone: that set is complete (the slice came from a short row), so the
// next level need not compare its candidates with the tuple again.
constexpr uint32_t kBranch = 1u << 31;
constexpr uint32_t kInjDone = 1u << 30;
constexpr uint32_t kExclShift = 22;
constexpr uint32_t kNodeMask = (1u << kExclShift) - 1u;

// Also zeroes the step's per-query count scratch: final-level counts of a
// step are added to the totals only once the host accepts the step, so a step
// re-run after a frontier overflow never counts twice.
//
// The parents' candidate prefix gets its closing entry here (coff[np] =
// coff_end, the total the host took from the step that wrote the parents):
// no tile of that step had to wait for the others to publish it.
__global__ void k_partition(unsigned long long *coff, uint64_t np, unsigned long long coff_end,
                            unsigned long long c0, unsigned long long ncand, uint32_t ntiles, uint32_t tile_size,
                            uint32_t *__restrict__ tile_parent, StepResult *result,
                            unsigned long long *step_counts, uint32_t nq) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t i = t; i < nq; i += gridDim.x * blockDim.x) step_counts[i] = 0;
    if (t == 0) {
        *result = StepResult{};
        coff[np] = coff_end;  // the searches below read coff[0, np) only
    }
    if (t > ntiles) return;
    const unsigned long long c = c0 + (t < ntiles ? (unsigned long long)t * tile_size : ncand - 1);
    uint64_t lo = 0, hi = np;  // largest p with coff[p] <= c
    while (hi - lo > 1) {
        uint64_t mid = lo + ((hi - lo) >> 1);
        if (coff[mid] <= c) lo = mid; else hi = mid;
    }
    tile_parent[t] = (uint32_t)lo;
}

// Adds an accepted step's final-level counts to the per-query totals.
__global__ void k_commit(unsigned long long *__restrict__ counts, const unsigned long long *__restrict__ step_counts,
                         uint32_t nq) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x)
        counts[i] += step_counts[i];
}

template <typename V>
__device__ __forceinline__ V warp_incl_scan(V x, uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        V y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    return x;
}
template <typename V>
__device__ __forceinline__ V warp_sum(V x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// One survivor staged in shared memory between the candidate pass and the
// coalesced write pass: parent index, candidate, and the child's own
// next-level candidate slice (start, then its exclusive prefix in the tile).
struct Stage {
    uint32_t p, v, cs, cnt, q;
};

// First index in a[0, n) with a[i] >= key, searched by a whole warp: 32
// probes per round narrow the range 32x, so a hub row of 10^5 entries takes
// four dependent loads instead of seventeen.  All 32 lanes must call it with
// the same arguments.
__device__ __forceinline__ uint32_t warp_lower_bound(const uint32_t *__restrict__ a, uint32_t n, uint32_t key,
                                                     uint32_t lane) {
    uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi]
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) >> 5;
        const uint32_t probe = lo + step * (lane + 1) - 1;  // last index of this lane's segment
        const bool less = probe < hi && __ldg(a + probe) < key;
        const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, less));
        const uint32_t nhi = min(hi, lo + (cnt + 1) * step - 1);
        lo = lo + cnt * step;
        hi = nhi;
    }
    const bool less = lo + lane < hi && __ldg(a + lo + lane) < key;
    return lo + __popc(__ballot_sync(0xffffffffu, less));
}

// Branch-free lower bound over a shared-memory array.
__device__ __forceinline__ uint32_t smem_lower_bound(const uint32_t *a, uint32_t n, uint32_t key) {
    if (n == 0) return 0;
    const uint32_t *base = a;
    while (n > 1) {
        const uint32_t half = n >> 1;
        base = (base[half] < key) ? base + half : base;
        n -= half;
    }
    return (uint32_t)(base - a) + (*base < key ? 1u : 0u);
}

constexpr int NSTAGE = 2;           // requirement rows a single-parent tile stages

// Tile geometry of a level-step instantiation: threads per CTA, candidates
// per thread, the CTAs per SM its register budget is fitted to, the entries
// of each requirement row a single-parent tile stages in shared memory, and
// whether the tile's parent window is kept as 16-bit offsets.  Shared memory
// and L1 share one 256 KiB array per SM, and the driver picks the smallest
// shared-memory carve-out that holds the CTAs the registers allow (196 KiB
// for 8 CTAs of 21.9 KB), leaving L1 the rest -- so shared bytes are L1
// bytes.  (256,2) stages only 64 entries per row (longer row parts are
// searched in global memory over the staged bounds): its 8 CTAs fit 132 KiB,
// 124 KiB of L1 instead of 60 KiB (grid batch level step 96.1 -> 92.3 ms);
// its 32-register kernel keeps the whole 64-bit window, which measured
// faster there.  The 40-register geometries take the 16-bit window: (256,4)
// fits 196 KiB instead of 228 KiB, 60 KiB of L1 instead of 28 KiB (R-MAT
// triangle 91.1 -> 80.9 ms).
template <int T_, int CPT_, int MINB_, int REQ_ = 768, bool W16_ = true>
struct Geo {
    static constexpr int T = T_, CPT = CPT_, TILE = T_ * CPT_, WIN = T_ * CPT_ + 2, NWARP = T_ / 32,
                         WC = 32 * CPT_, MINB = MINB_, REQ = REQ_;
    static constexpr bool W16 = W16_;
    using WinT = std::conditional_t<W16_, uint16_t, unsigned long long>;
};
using Geo0 = Geo<256, 4, 6>;               // 1024-candidate tiles, 8 warps (the default)
using Geo1 = Geo<128, 4, 11>;              // 512-candidate tiles, 4 warps
using Geo2 = Geo<256, 2, 7, 64, false>;    // 512-candidate tiles, 8 warps
using Geo3 = Geo<512, 2, 3>;               // 1024-candidate tiles, 16 warps
// Survivors one warp stages per tile, at most; their slice counts are
// summed in 32 bits (see the trie fan-out cap in Engine::run).
constexpr uint64_t kWarpStage = 128;
static_assert(Geo0::WC <= kWarpStage && Geo1::WC <= kWarpStage && Geo2::WC <= kWarpStage && Geo3::WC <= kWarpStage,
              "a warp stages at most kWarpStage survivors");
constexpr int kVariants = 4;
constexpr uint32_t kMinTile = 512;   // the tile directory is sized for this tile
__host__ __device__ constexpr uint32_t variant_tile(int v) {
    return v == 0 ? Geo0::TILE : v == 1 ? Geo1::TILE : v == 2 ? Geo2::TILE : Geo3::TILE;
}

// Shared memory of one tile of a level step.
template <class G>
struct StepSmem {
    static_assert(!G::W16 || G::TILE < 65536, "16-bit window offsets");
    // the parents' candidate prefix over the tile, win[i] for parent plo+i:
    // whole (64-bit), or (W16) as the offset from the tile's first candidate
    // for the parents that start inside the tile (0 < i < nwin-1), with the
    // first parent's start and the last one's end, which lie outside it,
    // kept whole in win_ends
    typename G::WinT win[G::WIN];
    unsigned long long win_ends[2];
    Stage stage[G::TILE];
    uint32_t req[NSTAGE][G::REQ];
    uint32_t rlo[NSTAGE], rhi[NSTAGE], rmode[NSTAGE];  // mode 0 none, 1 shared, 2 global range
    uint32_t wcnt[G::NWARP], wofs[G::NWARP + 1];
    unsigned long long wdeg[G::NWARP], wdofs[G::NWARP], wbytes[G::NWARP];
    uint32_t q0, vfirst, vlast;
    unsigned long long excl_cnt, excl_deg, fcount;
};

// Child slots of one tile (called by one thread): a single atomic on the
// step's allocator takes agg_cnt consecutive slots and the matching range of
// the next level's candidate prefix, so no tile waits for another.  Slot
// order across tiles is the order of their atomics.  The step's totals are
// the allocator word itself once the step has finished (the host, or the
// schedule controller, reads them from there).
__device__ __forceinline__ void tile_alloc(const StepArgs &a, const unsigned long long agg_cnt,
                                           const unsigned long long agg_deg, unsigned long long &ex_cnt,
                                           unsigned long long &ex_deg) {
    StepResult *r = a.result;
    const bool big = agg_deg > kAllocMask;
    const unsigned long long old =
        agg_cnt ? atomicAdd(&r->alloc, (agg_cnt << kAllocShift) + (big ? 0ull : agg_deg)) : 0ull;
    ex_cnt = old >> kAllocShift;
    ex_deg = old & kAllocMask;
    if (big || ex_deg + agg_deg > kAllocMask) atomicOr(&r->next_ovf, 1u);  // the host redoes a smaller chunk
}

// Per-tile context of the candidate check: the parents' candidate prefix
// window (shared memory, or null to search global memory), and for a tile
// inside one parent's slice the staged requirement-row slices.
template <class W>
struct CandCtx {
    const W *win;
    const unsigned long long *win_ends;
    uint32_t nwin, plo;
    bool single;
    const uint32_t *req;
    uint32_t req_stride;
    const uint32_t *rlo, *rhi, *rmode;
};

// The child a surviving candidate becomes: its own candidate slice for
// depth+1 (r.cs, r.cnt; r.q gains kBranch when its trie node branches).
// False when the slice is empty -- such a child cannot be extended and is
// not written.
__device__ __forceinline__ bool next_slice(const StepArgs &a, const uint32_t d, Stage &r,
                                           unsigned long long &my_bytes, uint32_t &fq, unsigned long long &fc) {
    const uint32_t p = r.p, v = r.v, q = r.q;
    const DLevel *L = &a.plans[q].lv[d];
    const uint32_t na = L->next_anchor;
    const uint32_t w = na == d ? v : __ldg(a.ptup + (uint64_t)(1 + na) * a.pstride + p);
    const uint32_t rs = __ldg(a.g.rowptr + w), re = __ldg(a.g.rowptr + w + 1);
    // depth+1's window, narrowed by symmetry breaking: its candidate
    // must exceed the vertices of next_lb and stay below those of next_ub
    uint32_t klo = L->next_lo, khi = L->next_hi;
    for (uint32_t m = L->next_lb; m; m &= m - 1u) {
        const uint32_t pos = __ffs(m) - 1;
        const uint32_t x = pos == d ? v : __ldg(a.ptup + (uint64_t)(1 + pos) * a.pstride + p);
        klo = max(klo, x + 1);
    }
    for (uint32_t m = L->next_ub; m; m &= m - 1u) {
        const uint32_t pos = __ffs(m) - 1;
        const uint32_t x = pos == d ? v : __ldg(a.ptup + (uint64_t)(1 + pos) * a.pstride + p);
        khi = min(khi, x);
    }
    uint32_t s = rs, e = re;  // the part of w's row inside that window
    uint32_t excl = 0, flags = 0;
    if (klo >= khi) {
        e = s;
    } else if (re - rs <= SHORT_ROW) {
        // the row in registers: the window's bounds in one pass, and the
        // slice entries that are vertices of the child's tuple (v and the
        // parent's positions): they would fail injectivity at depth+1
        // (HnGPU.cu:223-236) and are left out of its candidates
        const uint32_t n = re - rs;
        uint32_t b1 = 0, b2 = 0;
#pragma unroll
        for (uint32_t i = 0; i < SHORT_ROW; ++i)
            if (i < n) {
                const uint32_t x = __ldg(a.g.adj + rs + i);
                b1 += x < klo;
                b2 += x < khi;
            }
        s = rs + b1;
        e = rs + b2;
        for (uint32_t i = 0; i < b2 - b1; ++i) {
            const uint32_t x = __ldg(a.g.adj + s + i);
            bool in = x == v;
            for (uint32_t t = 0; t < d && !in; ++t) in = __ldg(a.ptup + (uint64_t)(1 + t) * a.pstride + p) == x;
            excl |= (in ? 1u : 0u) << i;
        }
        flags = kInjDone;
    } else {
        if (klo) s = rs + lower_bound_u32(a.g.adj + rs, re - rs, klo);
        if (khi < a.g.n) e = rs + lower_bound_u32(a.g.adj + rs, re - rs, khi);
    }
    if (e <= s) return false;
    const uint32_t len = (e - s) - __popc(excl);
    if (!len) return false;  // every entry of the slice is a vertex of the tuple
    // a branching node's child offers its slice to every child node
    const uint32_t nf = L->fan_count;
    const uint32_t mult = nf > 1 ? nf : 1u;
    // the child's tuple and anchor row, read once per (member) parent
    my_bytes += (4ull * (d + 1) + 4ull * (re - rs + 1)) * mult;
    if (a.leaf_count && flags && !a.g.elab) {
        // depth+1 is the last query vertex with nothing to check beyond the
        // anchor edge (no requirement, no row search for the anchor): every
        // entry left in the slice is an embedding -- count them here and
        // write no child.  A branching node whose child nodes all end so
        // (anchor_check bit 1) counts the slice once for each of them.
        if (nf <= 1) {
            const DLevel *N = &a.plans[q].lv[d + 1];
            if (N->final_ && N->nreq == 0 && !(N->anchor_check & 1u)) {
                if (fc && q != fq) {
                    atomicAdd(&a.counts[fq], fc);
                    fc = 0;
                }
                fq = q;
                fc += len;
                return false;
            }
        } else if (L->anchor_check & 2u) {
            for (uint32_t j = 0; j < nf; ++j) {
                const uint32_t qj = __ldg(a.fan_list + L->fan_start + j);
                if (fc && qj != fq) {
                    atomicAdd(&a.counts[fq], fc);
                    fc = 0;
                }
                fq = qj;
                fc += len;
            }
            return false;
        }
    }
    r.cs = s;
    r.cnt = len * mult;
    r.q = q | (excl << kExclShift) | flags | (nf > 1 ? kBranch : 0u);
    return true;
}

// One candidate c (offset off in its tile) of a level step: find its
// parent, check it (injectivity, anchor label, remaining requirements), and
// either count it (last query vertex) or describe the child it becomes
// (emit, rec).
template <bool ROOT, class W>
__device__ __forceinline__ void check_candidate(const StepArgs &a, const uint32_t d, const unsigned long long c,
                                                const uint32_t off, const CandCtx<W> &t, bool &emit, Stage &rec,
                                                unsigned long long &my_bytes, uint32_t &fq, unsigned long long &fc) {
    constexpr bool W16 = sizeof(W) == 2;
    // parent = largest p in [plo, phi] with coff[p] <= c; local = c - coff[p]
    uint32_t lo = 0, hi = t.nwin - 1, local;
    if (t.win) {  // (W16: the probes only reach parents that start inside the tile)
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            const bool le = W16 ? (uint32_t)t.win[mid] <= off : (unsigned long long)t.win[mid] <= c;
            if (le) lo = mid; else hi = mid;
        }
        if constexpr (W16)
            local = lo == 0 ? (uint32_t)(c - t.win_ends[0]) : off - (uint32_t)t.win[lo];
        else
            local = (uint32_t)(c - t.win[lo]);
    } else {
        while (hi - lo > 1) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if (__ldg(a.pcoff + t.plo + mid) <= c) lo = mid; else hi = mid;
        }
        local = (uint32_t)(c - __ldg(a.pcoff + t.plo + lo));
    }
    const uint32_t p = t.plo + lo;
    uint32_t q = ROOT ? __ldg(a.root_rep + p) : __ldg(a.ptup + p);
    const uint32_t excl = ROOT ? 0u : (q >> kExclShift) & 0xffu;
    const bool inj_done = !ROOT && (q & kInjDone);
    if (!ROOT && (q & kBranch)) {
        // the parent's trie node branches: its candidates run over (child
        // node, row offset), one copy of its slice per child node
        q &= kNodeMask;
        const DLevel *P = &a.plans[q].lv[d - 1];
        // the parent's candidates: local + (its end - c), below 2^32 by the
        // fan-out cap
        uint32_t span;
        if (!t.win)
            span = local + (uint32_t)(__ldg(a.pcoff + p + 1) - c);
        else if constexpr (W16)
            span = local + (lo + 2 == t.nwin ? (uint32_t)(t.win_ends[1] - c) : (uint32_t)t.win[lo + 1] - off);
        else
            span = (uint32_t)(t.win[lo + 1] - t.win[lo]);
        const uint32_t slen = span / P->fan_count;
        const uint32_t j = local / slen;
        local -= j * slen;
        q = __ldg(a.fan_list + P->fan_start + j);
    } else if (!ROOT) {
        q &= kNodeMask;
    }
    // the parent's first candidate (of each child node) does the parent's
    // byte accounting below
    const bool acct = !ROOT && local == 0;
    // row offset of the local-th slice entry that is not left out (excl,
    // ascending positions)
    for (uint32_t m = excl; m; m &= m - 1u)
        if ((uint32_t)(__ffs(m) - 1) <= local) ++local;
    const DLevel *L = &a.plans[q].lv[d];
    uint32_t v;
    bool pass = true;
    if (ROOT) {
        v = __ldg(a.pcstart + p) + local;
        my_bytes += 4;  // degree/label read of a data vertex
    } else {
        const uint32_t idx = __ldg(a.pcstart + p) + local;
        v = __ldg(a.g.adj + idx);
        if (L->anchor_check & 1u)
            pass = has_edge(a.g, __ldg(a.ptup + (uint64_t)(1 + L->anchor) * a.pstride + p), v, L->anchor_lab);
        else if (a.g.elab)
            pass = __ldg(a.g.elab + idx) == L->anchor_lab;
        // injectivity (HnGPU.cu:223-236), unless the parent's slice already
        // left out every vertex of its tuple
        if (!inj_done)
            for (uint32_t i = 0; i < d; ++i)
                if (__ldg(a.ptup + (uint64_t)(1 + i) * a.pstride + p) == v) pass = false;
    }
    // Algorithmic bytes of a parent (its tuple, its anchor row and every
    // requirement row, each read once): the tuple and anchor-row terms were
    // added when the parent was written (below, where the anchor row's bounds
    // are at hand); the parent's first candidate adds its requirement rows
    // here, from the same row bounds the requirement checks load.
    // remaining requirements (HnGPU.cu:243-252)
    for (uint32_t r = 0; r < L->nreq && (pass || acct); ++r) {
        const uint32_t mode = (t.single && r < (uint32_t)NSTAGE) ? t.rmode[r] : 0u;
        const uint32_t pos = L->req_pos[r];
        if (mode == 0u) {
            const uint32_t u = pos == REQ_SELF ? v : __ldg(a.ptup + (uint64_t)(1 + pos) * a.pstride + p);
            const uint32_t rs = __ldg(a.g.rowptr + u), re = __ldg(a.g.rowptr + u + 1);
            if (acct && pos != REQ_SELF) my_bytes += 4ull * (re - rs + 1);
            if (pass) pass = row_holds(a.g, rs, re, v, L->req_lab[r]);
            continue;
        }
        if (acct) {  // a staged row (pos is never REQ_SELF there)
            const uint32_t u = __ldg(a.ptup + (uint64_t)(1 + pos) * a.pstride + p);
            my_bytes += 4ull * (__ldg(a.g.rowptr + u + 1) - __ldg(a.g.rowptr + u) + 1);
        }
        if (!pass) continue;
        const uint32_t n = t.rhi[r] - t.rlo[r];
        if (mode == 1u) {
            const uint32_t k = smem_lower_bound(t.req + r * t.req_stride, n, v);
            pass = k < n && t.req[r * t.req_stride + k] == v && L->req_lab[r] == a.g.single_label;
        } else {
            const uint32_t k = lower_bound_u32(a.g.adj + t.rlo[r], n, v);
            pass = k < n && __ldg(a.g.adj + t.rlo[r] + k) == v && L->req_lab[r] == a.g.single_label;
        }
    }
    if (pass) {
        if (L->final_) {
            if (a.rows_out) {
                const uint32_t slot = atomicAdd(a.rows_ctr, 1u);
                if (slot < a.max_rows) {
                    const DQuery *Q = &a.plans[q];
                    uint32_t *row = a.rows_out + (uint64_t)slot * Q->k;
                    for (uint32_t i = 0; i < d; ++i)
                        row[Q->col[i]] =
                            __ldg(a.g.order + __ldg(a.ptup + (uint64_t)(1 + i) * a.pstride + p));
                    row[Q->col[d]] = __ldg(a.g.order + v);
                }
            }
            if (fc && q != fq) {
                atomicAdd(&a.counts[fq], fc);
                fc = 0;
            }
            fq = q;
            ++fc;
        } else {
            // the child's next-level slice is found in the tile's second
            // pass, over the warp's survivors packed together
            rec = Stage{p, v, 0, 0, q};
            emit = true;
        }
    }
}

// One tile of a level step: candidates [c0 + tile*TILE, ...) of the step.
template <bool ROOT, class G>
__device__ __forceinline__ void step_tile(const StepArgs &a, const uint32_t tile, StepSmem<G> &sm) {
    constexpr int T = G::T, CPT = G::CPT, TILE = G::TILE, WIN = G::WIN, NWARP = G::NWARP, WC = G::WC;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sm.fcount = 0;
    if (tid < NSTAGE) sm.rmode[tid] = 0;
    __syncthreads();
    const unsigned long long base = a.c0 + (unsigned long long)tile * TILE;
    const unsigned long long tend = min(base + (unsigned long long)TILE, a.cend);
    const uint32_t plo = __ldg(a.tile_parent + tile), phi = __ldg(a.tile_parent + tile + 1);
    const uint32_t nwin = phi - plo + 2;  // coff[plo .. phi+1]
    const bool win_smem = nwin <= (uint32_t)WIN;
    if (win_smem)
        for (uint32_t i = tid; i < nwin; i += T) {
            const unsigned long long x = __ldg(a.pcoff + plo + i);
            if constexpr (G::W16) {
                if (i == 0) sm.win_ends[0] = x;
                if (i == nwin - 1) sm.win_ends[1] = x;
                sm.win[i] = (i == 0 || i == nwin - 1) ? (uint16_t)0 : (uint16_t)(x - base);
            } else {
                sm.win[i] = x;
            }
        }
    const uint32_t d = a.depth;
    const bool emits = a.ctup != nullptr;

    // ---- a tile inside one parent's slice (hub rows): stage the part of each
    // requirement row that can hold this tile's candidates
    const bool single = !ROOT && plo == phi && a.g.elab == nullptr &&
                        !(__ldg(a.ptup + plo) & (kBranch | (0xffu << kExclShift)));
    if (single) {
        const uint32_t q0 = __ldg(a.ptup + plo) & kNodeMask;
        const DLevel *L0 = &a.plans[q0].lv[d];
        if (tid == 0) {
            const uint32_t cs0 = __ldg(a.pcstart + plo);
            const unsigned long long c00 = __ldg(a.pcoff + plo);
            sm.vfirst = __ldg(a.g.adj + cs0 + (uint32_t)(base - c00));
            sm.vlast = __ldg(a.g.adj + cs0 + (uint32_t)(tend - 1 - c00));
        }
        __syncthreads();
        if (warp < 2 * NSTAGE) {
            const uint32_t r = warp >> 1;
            if (r < L0->nreq && L0->req_pos[r] != REQ_SELF) {
                const uint32_t u = __ldg(a.ptup + (uint64_t)(1 + L0->req_pos[r]) * a.pstride + plo);
                const uint32_t rs = __ldg(a.g.rowptr + u), re = __ldg(a.g.rowptr + u + 1);
                const uint32_t key = (warp & 1) ? sm.vlast + 1 : sm.vfirst;
                const uint32_t b = rs + warp_lower_bound(a.g.adj + rs, re - rs, key, lane);
                if (lane == 0) {
                    if (warp & 1) sm.rhi[r] = b; else sm.rlo[r] = b;
                }
            }
        }
        __syncthreads();
        for (uint32_t r = 0; r < (uint32_t)NSTAGE; ++r) {
            if (r >= L0->nreq || L0->req_pos[r] == REQ_SELF) continue;
            const uint32_t lo = sm.rlo[r], n = sm.rhi[r] - sm.rlo[r];
            if (n <= (uint32_t)G::REQ)
                for (uint32_t i = tid; i < n; i += T) sm.req[r][i] = __ldg(a.g.adj + lo + i);
            if (tid == 0) sm.rmode[r] = n <= (uint32_t)G::REQ ? 1u : 2u;
        }
    }
    if (tid == 0) sm.q0 = ROOT ? __ldg(a.root_rep + plo) : (__ldg(a.ptup + plo) & kNodeMask);
    __syncthreads();

    unsigned long long my_bytes = 0, fc = 0, my_deg = 0;
    uint32_t fq = 0xffffffffu, wcnt = 0;
    Stage *wstage = sm.stage + warp * WC;
    const CandCtx<typename G::WinT> tctx{win_smem ? sm.win : nullptr, sm.win_ends, nwin, plo, single, &sm.req[0][0], (uint32_t)G::REQ,
                       sm.rlo, sm.rhi, sm.rmode};

#pragma unroll 1
    for (int j = 0; j < CPT; ++j) {
        const uint32_t off = warp * WC + j * 32 + lane;
        const unsigned long long c = base + off;
        bool emit = false;
        Stage rec{0, 0, 0, 0, 0};
        if (c < tend) check_candidate<ROOT>(a, d, c, off, tctx, emit, rec, my_bytes, fq, fc);
        if (emits) {
            const uint32_t bal = __ballot_sync(0xffffffffu, emit);
            if (emit) wstage[wcnt + __popc(bal & ((1u << lane) - 1u))] = rec;
            wcnt += __popc(bal);
        }
    }
    if (emits) {
        // second pass over this warp's survivors, packed: each becomes a
        // child with its next-level slice, or is dropped (empty slice); the
        // kept ones move down in place (a round reads its entries before
        // any is overwritten, and writes only at or below them).  Packed
        // survivors keep all 32 lanes busy on the slice searches, and the
        // first pass's state is dead by then (fewer live registers).
        __syncwarp();
        uint32_t kept = 0;
        for (uint32_t e0 = 0; e0 < wcnt; e0 += 32) {
            const uint32_t e = e0 + lane;
            Stage r{0, 0, 0, 0, 0};
            bool keep = false;
            if (e < wcnt) {
                r = wstage[e];
                keep = next_slice(a, d, r, my_bytes, fq, fc);
            }
            const uint32_t bal = __ballot_sync(0xffffffffu, keep);
            if (keep) wstage[kept + __popc(bal & ((1u << lane) - 1u))] = r;
            kept += __popc(bal);
            my_deg += keep ? r.cnt : 0u;
            __syncwarp();
        }
        wcnt = kept;
    }

    // ---- final-depth counts: one shared add per warp in the common case
    {
        const bool uniform = __all_sync(0xffffffffu, fc == 0 || fq == sm.q0);
        if (uniform) {
            const unsigned long long sum = warp_sum(fc);
            if (lane == 0 && sum) atomicAdd(&sm.fcount, sum);
        } else if (fc) {
            atomicAdd(&a.counts[fq], fc);
        }
        const unsigned long long wb = warp_sum(my_bytes);
        if (lane == 0) sm.wbytes[warp] = wb;
    }
    if (!emits) {
        __syncthreads();
        if (tid == 0) {
            unsigned long long bb = 0;
            for (int w = 0; w < NWARP; ++w) bb += sm.wbytes[w];
            if (bb) atomicAdd(&a.result->alg_bytes, bb);
            if (sm.fcount) atomicAdd(&a.counts[sm.q0], sm.fcount);
        }
        return;
    }
    // ---- per-warp exclusive prefix of the staged slice lengths
    __syncwarp();  // the segment was written by every lane of this warp
    {
        const unsigned long long wd = warp_sum(my_deg);
        // lane l scans entries [4l, 4l+4) of this warp's segment
        uint32_t loc[CPT];
        unsigned long long sum = 0;
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            const uint32_t e = lane * CPT + i;
            loc[i] = e < wcnt ? wstage[e].cnt : 0u;
            sum += loc[i];
        }
        const unsigned long long incl = warp_incl_scan<unsigned long long>(sum, lane);
        unsigned long long run = incl - sum;
#pragma unroll
        for (int i = 0; i < CPT; ++i) {
            const uint32_t e = lane * CPT + i;
            if (e < wcnt) wstage[e].cnt = (uint32_t)run;  // warp-local exclusive prefix (< 2^32)
            run += loc[i];
        }
        if (lane == 0) {
            sm.wcnt[warp] = wcnt;
            sm.wdeg[warp] = wd;
        }
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long cc = 0, dd = 0, bb = 0;
        for (int w = 0; w < NWARP; ++w) {
            sm.wofs[w] = (uint32_t)cc;
            sm.wdofs[w] = dd;
            cc += sm.wcnt[w];
            dd += sm.wdeg[w];
            bb += sm.wbytes[w];
        }
        sm.wofs[NWARP] = (uint32_t)cc;
        unsigned long long ex_cnt = 0, ex_deg = 0;
        tile_alloc(a, cc, dd, ex_cnt, ex_deg);
        sm.excl_cnt = ex_cnt;
        sm.excl_deg = ex_deg;
        if (bb) atomicAdd(&a.result->alg_bytes, bb);
        if (sm.fcount) atomicAdd(&a.counts[sm.q0], sm.fcount);
    }
    __syncthreads();
    // ---- write the tile's children: every warp writes its own packed
    // survivors to its consecutive range of the tile's slots
    const unsigned long long ex_cnt = sm.excl_cnt + sm.wofs[warp], ex_deg = sm.excl_deg + sm.wdofs[warp];
    for (uint32_t i = lane; i < wcnt; i += 32) {
        const Stage r = wstage[i];
        const uint64_t slot = ex_cnt + i;
        if (slot >= a.ccap) continue;  // overflow: the host retries with a smaller chunk
        a.ctup[slot] = r.q;
        for (uint32_t k = 0; k < d; ++k)
            a.ctup[(uint64_t)(1 + k) * a.cstride + slot] = __ldg(a.ptup + (uint64_t)(1 + k) * a.pstride + r.p);
        a.ctup[(uint64_t)(1 + d) * a.cstride + slot] = r.v;
        a.ccstart[slot] = r.cs;
        a.ccoff[slot] = ex_deg + r.cnt;
    }
}

template <bool ROOT, class G>
__global__ void __launch_bounds__(G::T, G::MINB) k_step(const StepArgs a) {
    __shared__ StepSmem<G> sm;
    step_tile<ROOT, G>(a, blockIdx.x, sm);
}



// Launches one level step with the given tile geometry.
void launch_step(int variant, bool root, const StepArgs &a, uint32_t ntiles, cudaStream_t st) {
    switch (variant) {
    case 1:
        if (root) k_step<true, Geo1><<<ntiles, Geo1::T, 0, st>>>(a);
        else k_step<false, Geo1><<<ntiles, Geo1::T, 0, st>>>(a);
        break;
    case 2:
        if (root) k_step<true, Geo2><<<ntiles, Geo2::T, 0, st>>>(a);
        else k_step<false, Geo2><<<ntiles, Geo2::T, 0, st>>>(a);
        break;
    case 3:
        if (root) k_step<true, Geo3><<<ntiles, Geo3::T, 0, st>>>(a);
        else k_step<false, Geo3><<<ntiles, Geo3::T, 0, st>>>(a);
        break;
    default:
        if (root) k_step<true, Geo0><<<ntiles, Geo0::T, 0, st>>>(a);
        else k_step<false, Geo0><<<ntiles, Geo0::T, 0, st>>>(a);
        break;
    }
}

// ---------------------------------------------------------------------------
// Device-driven schedule: a CUDA graph whose WHILE node repeats (controller ->
// tile directory -> level step).  The controller kernel makes the host loop's
// decisions (chunk size, retry on overflow, descend / return) on the device,
// so no step returns to the host.
// ---------------------------------------------------------------------------
static_assert(sizeof(StepArgs) % 4 == 0, "StepArgs is copied as 32-bit words");

// The most candidates an emitting step may take so that its children's
// next-level candidates, at nxt per candidate (the largest rate seen at this
// depth; 0: none seen yet), fill at most half the allocator's field.
__host__ __device__ inline unsigned long long emit_chunk_cap(const double nxt) {
    if (nxt <= 0.0) return kFirstEmitChunk;
    const double lim = (double)(kAllocMask / 2) / nxt;
    return lim < (double)kMaxEmitChunk ? (unsigned long long)(lim > 1.0 ? lim : 1.0) : kMaxEmitChunk;
}

struct Ctl {
    unsigned long long total[MAXQ + 1], pos[MAXQ + 1], np[MAXQ + 1];
    float ratio[MAXQ + 1];
    float nxt[MAXQ + 1];         // next-level candidates per candidate seen at each depth (emit_chunk_cap)
    uint32_t *tup[MAXQ];
    unsigned long long cap[MAXQ];
    uint32_t *cstart[MAXQ];
    unsigned long long *coff[MAXQ];
    StepArgs args;               // the step in flight (static fields preset by the host)
    unsigned long long *root_coff;
    const uint32_t *root_cstart;
    unsigned long long *counts;        // per-entity totals (args.counts is the step scratch)
    uint32_t nq, accepted;
    uint32_t tile;                     // candidates per tile of the graph's step kernel
    unsigned long long chunk, max_scan, max_candidates;
    unsigned long long steps, retries, candidates, expansions, alg_bytes;
    unsigned long long held[MAXQ], peak;  // tuples each depth's buffer holds; largest bytes held at once
    uint32_t d, dmax, emits, done, err;
};


// Chooses the next step (the host loop's logic); sets done when none is left.
__device__ void ctl_plan(Ctl &c) {
    for (;;) {
        if (c.pos[c.d] < c.total[c.d]) break;
        if (c.d == 0) {
            c.done = 1;
            return;
        }
        --c.d;
    }
    const uint32_t d = c.d;
    const bool emits = d < c.dmax;
    unsigned long long chunk = c.total[d] - c.pos[d];
    if (chunk > c.max_scan) chunk = c.max_scan;
    if (emits) {
        const double allowed = (double)c.cap[d] / fmax((double)c.ratio[d], 1.0 / 8192.0);
        const unsigned long long lim = (unsigned long long)fmax(allowed, (double)c.tile);
        if (chunk > lim) chunk = lim;
        const unsigned long long ncap = emit_chunk_cap((double)c.nxt[d]);
        if (chunk > ncap) chunk = ncap;
    }
    StepArgs &a = c.args;
    a.depth = d;
    if (d == 0) {
        a.ptup = nullptr;
        a.pstride = 0;
        a.pcstart = c.root_cstart;
        a.pcoff = c.root_coff;
    } else {
        a.ptup = c.tup[d - 1];
        a.pstride = c.cap[d - 1];
        a.pcstart = c.cstart[d - 1];
        a.pcoff = c.coff[d - 1];
    }
    a.np = c.np[d];
    a.pcoff_end = c.total[d];
    a.c0 = c.pos[d];
    a.cend = c.pos[d] + chunk;
    a.ntiles = (uint32_t)((chunk + c.tile - 1) / c.tile);
    if (emits) {
        a.ctup = c.tup[d];
        a.cstride = c.cap[d];
        a.ccap = c.cap[d];
        a.ccstart = c.cstart[d];
        a.ccoff = c.coff[d];
    } else {
        a.ctup = nullptr;
        a.cstride = a.ccap = 0;
        a.ccstart = nullptr;
        a.ccoff = nullptr;
    }
    c.chunk = chunk;
    c.emits = emits;
    *a.result = StepResult{};
}

// Accounts the finished step (the host loop's logic).
__device__ void ctl_after(Ctl &c) {
    const StepResult *rp = c.args.result;
    const unsigned long long alloc = __ldcg(&rp->alloc);
    const unsigned long long n = alloc >> kAllocShift, next = alloc & kAllocMask;
    const unsigned long long ab = __ldcg(&rp->alg_bytes);
    uint32_t e = __ldcg(&rp->err);
    const uint32_t ovf = __ldcg(&rp->next_ovf);
    const uint32_t d = c.d;
    c.steps++;
    c.accepted = 0;
    if (c.emits && ovf && c.chunk <= c.tile) e |= KERR_CAP;  // one tile's children alone overflow
    if (e) {
        c.err |= e;
        c.done = 1;
        return;
    }
    if (c.emits && (n > c.cap[d] || ovf)) {
        c.retries++;
        c.ratio[d] = (float)fmax((double)c.ratio[d] * 4.0, 2.0 * (double)n / (double)c.chunk);
        if (ovf)  // the next level's candidates overflowed the field: at most half this chunk next
            c.nxt[d] = (float)fmax((double)c.nxt[d] * 4.0, (double)kAllocMask / (double)c.chunk);
        return;
    }
    c.accepted = 1;
    c.candidates += c.chunk;
    c.expansions += n;
    c.alg_bytes += ab + (c.emits ? n * 4ull * (d + 1) : 0ull);
    if (c.max_candidates && c.candidates > c.max_candidates) {
        c.err |= KERR_CAP;
        c.done = 1;
        return;
    }
    c.pos[d] += c.chunk;
    if (c.emits) {
        c.held[d] = n;
        unsigned long long live = 0;  // the buffers of depths <= d are live now
        for (uint32_t i = 0; i <= d; ++i) live += c.held[i] * tuple_bytes(i);
        if (live > c.peak) c.peak = live;
        c.ratio[d] = (float)fmax(2.0 * (double)n / (double)c.chunk, (double)c.ratio[d] * 0.5);
        c.nxt[d] = (float)fmax((double)next / (double)c.chunk, (double)c.nxt[d] * 0.5);
        if (n > 0 && next > 0) {
            c.np[d + 1] = n;
            c.total[d + 1] = next;
            c.pos[d + 1] = 0;
            c.d = d + 1;
        }
    }
}

// Per-engine step arguments for the graph-driven schedule: the graph's copy
// node moves the controller's next StepArgs here, so the step kernels read
// them from the constant bank like kernel parameters.
constexpr int kArgSlots = 8;
__constant__ StepArgs c_args[kArgSlots];

// Graph node: the schedule controller (first: plan the first step; else
// account the finished step and plan the next) and the loop condition.
__global__ void k_ctl(Ctl *ctl, cudaGraphConditionalHandle h, int first) {
    Ctl &c = *ctl;
    __shared__ uint32_t s_accept;
    if (!first) {
        if (threadIdx.x == 0) {
            ctl_after(c);
            s_accept = c.accepted;
        }
        __syncthreads();
        if (s_accept)  // an accepted step's final-level counts join the totals
            for (uint32_t i = threadIdx.x; i < c.nq; i += blockDim.x) c.counts[i] += c.args.counts[i];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (first || !c.done) ctl_plan(c);
        cudaGraphSetConditional(h, c.done ? 0u : 1u);
    }
}

// Graph node: first parent of every tile of the step (strided fixed grid).
// The graph kernels are instantiated per argument slot, so the slot's
// fields are compile-time constant-bank operands like kernel parameters (a
// runtime slot index turns every field read into a load: the R-MAT triangle
// ran 10% slower that way).
template <int SLOT, uint32_t TILE_SIZE>
__global__ void k_part_g(const Ctl *ctl) {
    const StepArgs &a = c_args[SLOT];
    const unsigned long long ncand = a.cend - a.c0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ctl->nq; i += gridDim.x * blockDim.x)
        a.counts[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.pcoff[a.np] = a.pcoff_end;  // see k_partition
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= a.ntiles; t += gridDim.x * blockDim.x) {
        const unsigned long long c = a.c0 + (t < a.ntiles ? (unsigned long long)t * TILE_SIZE : ncand - 1);
        uint64_t lo = 0, hi = a.np;
        while (hi - lo > 1) {
            const uint64_t mid = lo + ((hi - lo) >> 1);
            if (a.pcoff[mid] <= c) lo = mid; else hi = mid;
        }
        const_cast<uint32_t *>(a.tile_parent)[t] = (uint32_t)lo;
    }
}

// Graph nodes: the level step on a fixed grid.  A step with no more tiles
// than CTAs gives each CTA its own tile; otherwise every CTA takes tiles from
// the step's tile counter (StepResult::tile_ctr, zeroed with the result by
// the tile directory), so tiles go to whichever CTA frees first, as they
// would with one CTA per tile.  The ticket for a CTA's next tile is taken
// when its current tile starts and read when it ends, so the atomic's round
// trip hides behind the tile.  One instantiation per argument slot, tile
// geometry and step kind: the root step and the deeper levels are separate
// nodes, and the one whose kind the step is not returns at once (one kernel
// holding both had twice the code and spilled).
template <int SLOT, class G, bool ROOT>
__global__ void __launch_bounds__(G::T, G::MINB) k_step_g() {
    __shared__ StepSmem<G> sm;
    __shared__ uint32_t s_tile;
    const StepArgs &a = c_args[SLOT];
    if ((a.depth == 0) != ROOT || blockIdx.x >= a.ntiles) return;
    if (a.ntiles <= gridDim.x) {  // a step that fits the grid: one tile per CTA, no tickets
        step_tile<ROOT, G>(a, blockIdx.x, sm);
        return;
    }
    if (threadIdx.x == 0) s_tile = atomicAdd(&a.result->tile_ctr, 1u);
    __syncthreads();
    for (;;) {
        // (256,4) tiles: values derived from the step's arguments are read
        // again each tile instead of held across the loop -- that geometry
        // otherwise spills 88 bytes per thread here, and none with this
        if constexpr (G::CPT == 4) asm volatile("" ::: "memory");
        const uint32_t tile = s_tile;
        if (tile >= a.ntiles) break;
        uint32_t next = 0;
        if (threadIdx.x == 0) next = atomicAdd(&a.result->tile_ctr, 1u);
        step_tile<ROOT, G>(a, tile, sm);  // its barriers order every thread's read of s_tile before the write
        if (threadIdx.x == 0) s_tile = next;
        __syncthreads();
    }
}

// Tile geometries the graph-driven schedule is instantiated for (the others
// run the host-driven loop): graph_geo(variant) is the index into them, or
// -1.
constexpr int kGraphGeos = 2;
// First-level candidates (CCSR entries of the root windows) up to which a
// call runs on the graph by default.
constexpr uint64_t kGraphRootEntries = 1ull << 22;
constexpr int graph_geo(int variant) { return variant == 0 ? 0 : variant == 2 ? 1 : -1; }

// Graph node kernels of argument slot s and graph geometry ggeo: kind 0 the
// tile directory, 1 the root step, 2 the deeper levels' step.
template <int... S>
const void *slot_kernel(int s, int ggeo, int kind) {
    static const void *part[kGraphGeos][sizeof...(S)] = {{(const void *)k_part_g<S, Geo0::TILE>...},
                                                          {(const void *)k_part_g<S, Geo2::TILE>...}};
    static const void *root[kGraphGeos][sizeof...(S)] = {{(const void *)k_step_g<S, Geo0, true>...},
                                                          {(const void *)k_step_g<S, Geo2, true>...}};
    static const void *stepk[kGraphGeos][sizeof...(S)] = {{(const void *)k_step_g<S, Geo0, false>...},
                                                           {(const void *)k_step_g<S, Geo2, false>...}};
    return kind == 0 ? part[ggeo][s] : kind == 1 ? root[ggeo][s] : stepk[ggeo][s];
}

inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

}  // namespace

// ---------------------------------------------------------------------------
// Device plan of one query against one data graph
// ---------------------------------------------------------------------------
gfsm_status build_dquery(const Plan &p, const DeviceGraph &g, const gfsm_limits &lim, DQuery &dq,
                         uint32_t &root_lo, uint32_t &root_hi, bool &never, bool sym) {
    std::memset(&dq, 0, sizeof(dq));
    never = false;
    const uint32_t k = p.k;
    if (k == 0 || k > (uint32_t)MAXQ) return GFSM_ERR_TOO_LARGE;
    dq.k = k;
    const bool use_deg = lim.degree_filter && g.symmetric && p.symmetric;
    std::vector<uint32_t> lo(k), hi(k);
    for (uint32_t d = 0; d < k; ++d) {
        uint32_t glo = 0, ghi = g.n;
        size_t gsel = 0;  // the depth's vertex-label group (group 0: labels not matched)
        if (g.vl_grouped) {
            auto it = std::lower_bound(g.group_value.begin(), g.group_value.end(), p.qlabel[d]);
            if (it == g.group_value.end() || *it != p.qlabel[d]) { never = true; glo = ghi = 0; }
            else {
                gsel = (size_t)(it - g.group_value.begin());
                glo = g.group_start[gsel];
                ghi = g.group_start[gsel + 1];
            }
        }
        // degree window: ids in a group are degree-descending, so
        // "degree >= delta" is a prefix of the group.
        uint32_t delta = use_deg ? p.qdeg[d] : 0;
        if (d == 0) delta = std::max<uint32_t>(delta, 1);  // a root needs a CCSR row (HnGPU.cu:475-495)
        uint32_t cut = ghi;
        if (delta > 0 && glo < ghi) {
            if (delta < DeviceGraph::kCutDeltas && !g.deg_cut.empty()) {
                cut = g.deg_cut[gsel * DeviceGraph::kCutDeltas + delta];
            } else {
                uint32_t a = glo, b = ghi;
                while (a < b) {
                    uint32_t mid = a + (b - a) / 2;
                    if (g.degree(mid) >= delta) a = mid + 1; else b = mid;
                }
                cut = a;
            }
        }
        lo[d] = glo;
        hi[d] = cut;
        if (lo[d] >= hi[d]) never = true;
    }
    for (uint32_t d = 0; d < k; ++d) {
        DLevel &L = dq.lv[d];
        L.lo = lo[d];
        L.hi = hi[d];
        L.final_ = d + 1 == k;
        dq.col[d] = (uint8_t)p.qvid[d];
        const uint32_t nreq = p.header[3 * d], roff = p.header[3 * d + 1], firstq = p.header[3 * d + 2];
        uint32_t dist = 0, nr = 0;
        bool anchor_done = false;
        for (uint32_t r = 0; r < nreq; ++r) {
            dist += p.reqs[roff + 2 * r];
            const uint32_t rel = p.reqs[roff + 2 * r + 1];
            if (!g.elab && g.m && rel != g.single_label) never = true;  // no such edge label in the data
            if (d > 0 && !anchor_done && dist == firstq) {
                anchor_done = true;
                L.anchor = (uint8_t)(d - firstq);
                L.anchor_lab = (uint8_t)rel;
                L.anchor_check = g.multi ? 1 : 0;
                continue;
            }
            if (nr >= (uint32_t)MAXQ) return GFSM_ERR_TOO_LARGE;
            L.req_pos[nr] = dist == 0 ? REQ_SELF : (uint8_t)(d - dist);
            L.req_lab[nr] = (uint8_t)rel;
            ++nr;
        }
        if (d > 0 && !anchor_done) return GFSM_ERR_QUERY;
        L.nreq = (uint8_t)nr;
    }
    for (uint32_t d = 0; d + 1 < k; ++d) {
        DLevel &L = dq.lv[d];
        const DLevel &N = dq.lv[d + 1];
        L.next_anchor = N.anchor;
        L.next_lo = N.lo;
        L.next_hi = N.hi;
    }
    if (sym) {
        // f(a) < f(b): a bound on whichever of the two is placed later, taken
        // from the earlier one's tuple position when its parent is written
        std::vector<uint32_t> depth(k, 0);
        for (uint32_t d = 0; d < k; ++d) depth[p.qvid[d]] = d;
        for (const auto &c : p.sym_cond) {
            const uint32_t da = depth[c.first], db = depth[c.second];
            if (da < db) dq.lv[db - 1].next_lb |= (uint16_t)(1u << da);
            else dq.lv[da - 1].next_ub |= (uint16_t)(1u << db);
        }
    }
    root_lo = lo[0];
    root_hi = hi[0];
    return GFSM_OK;
}

void root_partition(const uint32_t *rowptr, uint32_t lo, uint32_t hi, uint32_t nparts, uint64_t *bounds) {
    const uint64_t n = hi > lo ? hi - lo : 0;
    const uint64_t w = n ? (uint64_t)rowptr[hi] - rowptr[lo] : 0;
    bounds[0] = 0;
    for (uint32_t k = 1; k < nparts; ++k) {
        if (w == 0) {  // no entries to balance: equal numbers of rows
            bounds[k] = n * k / nparts;
            continue;
        }
        // smallest x with rowptr[lo + x] - rowptr[lo] >= ceil(k * w / nparts)
        const uint64_t target = (k * w + nparts - 1) / nparts;
        uint64_t a = bounds[k - 1], b = n;
        while (a < b) {
            const uint64_t mid = a + (b - a) / 2;
            if ((uint64_t)rowptr[lo + mid] - rowptr[lo] >= target) b = mid; else a = mid + 1;
        }
        bounds[k] = a;
    }
    bounds[nparts] = n;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
#define ECHECK(x)                                                               \
    do {                                                                        \
        cudaError_t e_ = (x);                                                   \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#x) + ": " + cudaGetErrorString(e_);              \
            return e_ == cudaErrorMemoryAllocation ? GFSM_ERR_NOMEM : GFSM_ERR_CUDA; \
        }                                                                       \
    } while (0)

Engine::~Engine() { release(); }

namespace {
std::mutex g_slot_mu;
uint32_t g_slot_used = 0;

int acquire_arg_slot() {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    for (int i = 0; i < kArgSlots; ++i)
        if (!(g_slot_used & (1u << i))) {
            g_slot_used |= 1u << i;
            return i;
        }
    return -1;
}

void release_arg_slot(int s) {
    if (s < 0) return;
    std::lock_guard<std::mutex> lk(g_slot_mu);
    g_slot_used &= ~(1u << s);
}
}  // namespace

static_assert(kGraphGeos == 2, "Engine keeps one graph per graph geometry");

void Engine::release() {
    for (int i = 0; i < kGraphGeos; ++i) {
        if (graph_exec[i]) cudaGraphExecDestroy(graph_exec[i]);
        if (graph[i]) cudaGraphDestroy(graph[i]);
        graph_exec[i] = nullptr;
        graph[i] = nullptr;
    }
    release_arg_slot(arg_slot);
    arg_slot = -1;
    if (arena) cudaFree(arena);
    if (small) cudaFree(small);
    if (h_result) cudaFreeHost(h_result);
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    h_stage_bytes = 0;
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_begin) cudaEventDestroy(ev_begin);
    if (ev_end) cudaEventDestroy(ev_end);
    if (stream) cudaStreamDestroy(stream);
    arena = nullptr;
    small = nullptr;
    h_result = nullptr;
    ev0 = ev1 = ev_begin = ev_end = nullptr;
    stream = nullptr;
}

gfsm_status Engine::init(int dev, uint64_t arena_limit, uint64_t scan_limit, std::string &err) {
    device = dev;
    ECHECK(cudaSetDevice(dev));
    ECHECK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    ECHECK(cudaEventCreate(&ev0));
    ECHECK(cudaEventCreate(&ev1));
    ECHECK(cudaEventCreate(&ev_begin));
    ECHECK(cudaEventCreate(&ev_end));
    ECHECK(cudaMallocHost(&h_result, sizeof(StepResult)));
    max_scan = std::min<uint64_t>(std::max<uint64_t>(scan_limit, TILE), 1ull << 31);
    dir_tiles = (uint32_t)div_up(max_scan, kMinTile);
    // small region: result, mapping-row counter, tile directory, schedule control block
    small_bytes = 512 + ((((uint64_t)dir_tiles + 2) * 4 + 255) & ~255ull) + ((sizeof(Ctl) + 255) & ~255ull);
    ECHECK(cudaMalloc(&small, small_bytes));
    ECHECK(cudaMemsetAsync(small, 0, small_bytes, stream));
    char *p = static_cast<char *>(small);
    static_assert(sizeof(StepResult) <= 64, "StepResult fits its slot");
    d_result = reinterpret_cast<StepResult *>(p);
    p += 128;
    rows_ctr = reinterpret_cast<uint32_t *>(p);
    p += 64;
    tile_parent = reinterpret_cast<uint32_t *>(p);
    p += (((uint64_t)dir_tiles + 2) * 4 + 255) & ~255ull;
    ctl = p;
    arena_cap = arena_limit;
    {
        int sms = 0, per_sm0 = 0, per_sm2 = 0;
        ECHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        ECHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm0, k_step_g<0, Geo0, false>, Geo0::T, 0));
        ECHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_step_g<0, Geo2, false>, Geo2::T, 0));
        step_blocks[graph_geo(0)] = sms * std::max(per_sm0, 1);
        step_blocks[graph_geo(2)] = sms * std::max(per_sm2, 1);
    }
    arg_slot = acquire_arg_slot();
    ECHECK(cudaStreamSynchronize(stream));
    return GFSM_OK;
}

gfsm_status Engine::ensure_arena(uint64_t bytes, std::string &err) {
    if (arena && arena_bytes >= bytes) return GFSM_OK;
    if (arena) cudaFree(arena);
    arena = nullptr;
    arena_bytes = 0;
    ECHECK(cudaMalloc(&arena, bytes));
    arena_bytes = bytes;
    return GFSM_OK;
}

// The schedule as a CUDA graph: k_ctl(first) -> WHILE(cond) { copy the step's
// arguments to this engine's constant slot -> tile directory -> level step ->
// k_ctl(next step, cond) }.  Every pointer the nodes take is fixed for the
// engine's lifetime (control block, constant slot), so the graph is built and
// instantiated once and relaunched by every call.
gfsm_status Engine::build_graph(int variant, std::string &err) {
    const int gg = graph_geo(variant);
    if (gg < 0) return GFSM_ERR_CUDA;
    if (graph_exec[gg]) return GFSM_OK;
    if (arg_slot < 0) {
        last_graph_error = -2;  // every constant-memory argument slot is taken
        return GFSM_ERR_CUDA;
    }
    if (graph_failed[gg]) return GFSM_ERR_CUDA;
    cudaGraph_t g = nullptr;
    auto fail = [&](cudaError_t e, const char *what) {
        if (g) cudaGraphDestroy(g);
        graph_failed[gg] = true;
        last_graph_error = (int)e;
        cudaGetLastError();
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return GFSM_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return fail(e, "cudaGraphCreate");
    cudaGraphConditionalHandle h;
    if ((e = cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault)) != cudaSuccess)
        return fail(e, "cudaGraphConditionalHandleCreate");
    Ctl *cp = static_cast<Ctl *>(ctl);
    int first = 1, next = 0, slot = arg_slot;
    void *a_first[] = {&cp, &h, &first};
    void *a_next[] = {&cp, &h, &next};
    void *a_part[] = {&cp};
    cudaKernelNodeParams kp{};
    kp.func = (void *)k_ctl;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(256);
    kp.kernelParams = a_first;
    cudaGraphNode_t n0, n1;
    if ((e = cudaGraphAddKernelNode(&n0, g, nullptr, 0, &kp)) != cudaSuccess) return fail(e, "ctl node");
    cudaGraphNodeParams cnp{};
    cnp.type = cudaGraphNodeTypeConditional;
    cnp.conditional.handle = h;
    cnp.conditional.type = cudaGraphCondTypeWhile;
    cnp.conditional.size = 1;
    if ((e = cudaGraphAddNode(&n1, g, &n0, 1, &cnp)) != cudaSuccess) return fail(e, "while node");
    cudaGraph_t body = cnp.conditional.phGraph_out[0];
    cudaGraphNode_t b0, b1, b2, b3;
    if ((e = cudaGraphAddMemcpyNodeToSymbol(&b0, body, nullptr, 0, c_args, &cp->args, sizeof(StepArgs),
                                            (size_t)slot * sizeof(StepArgs), cudaMemcpyDeviceToDevice)) != cudaSuccess)
        return fail(e, "args copy node");
    kp.func = const_cast<void *>(slot_kernel<0, 1, 2, 3, 4, 5, 6, 7>(slot, gg, 0));
    kp.gridDim = dim3((unsigned)step_blocks[gg]);
    kp.blockDim = dim3(256);
    kp.kernelParams = a_part;
    if ((e = cudaGraphAddKernelNode(&b1, body, &b0, 1, &kp)) != cudaSuccess) return fail(e, "partition node");
    kp.func = const_cast<void *>(slot_kernel<0, 1, 2, 3, 4, 5, 6, 7>(slot, gg, 1));
    kp.blockDim = dim3(gg == 0 ? Geo0::T : Geo2::T);
    kp.kernelParams = nullptr;
    cudaGraphNode_t b1r;
    if ((e = cudaGraphAddKernelNode(&b1r, body, &b1, 1, &kp)) != cudaSuccess) return fail(e, "root step node");
    kp.func = const_cast<void *>(slot_kernel<0, 1, 2, 3, 4, 5, 6, 7>(slot, gg, 2));
    if ((e = cudaGraphAddKernelNode(&b2, body, &b1r, 1, &kp)) != cudaSuccess) return fail(e, "step node");
    kp.func = (void *)k_ctl;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(256);
    kp.kernelParams = a_next;
    if ((e = cudaGraphAddKernelNode(&b3, body, &b2, 1, &kp)) != cudaSuccess) return fail(e, "ctl node");
    if ((e = cudaGraphInstantiate(&graph_exec[gg], g, 0)) != cudaSuccess) {
        graph_exec[gg] = nullptr;
        return fail(e, "cudaGraphInstantiate");
    }
    cudaGraphUpload(graph_exec[gg], stream);  // its first launch does not pay the upload
    graph[gg] = g;
    return GFSM_OK;
}

// Autotuner: the tile geometry (threads per CTA x candidates per thread) is
// picked per workload class -- (deepest level, log2 average degree, log2
// batch size) -- by timing every geometry on a sample of the call's queries
// the first time a class is seen.  GFSM_TILE=<0..3> forces a geometry and
// GFSM_AUTOTUNE=0 keeps the default.
// Workload class of a call (the autotuner's and the step sizer's memory key):
// the largest query size, log2 of the data graph's average degree and log2
// of the number of queries.
static uint64_t workload_class(const std::vector<const Plan *> &plans, const DeviceGraph &g) {
    uint32_t kmax = 0;
    for (const Plan *p : plans) kmax = std::max(kmax, p->k);
    const double avg = g.n ? (double)g.m / (double)g.n : 0.0;
    return ((uint64_t)kmax << 16) | ((uint64_t)std::lround(std::log2(avg + 1.0)) << 8) |
           (uint64_t)std::lround(std::log2((double)plans.size() + 1.0));
}

int Engine::pick_variant(const std::vector<const Plan *> &plans, const DeviceGraph &g, const gfsm_limits &lim,
                         std::string &err) {
    const char *force = getenv("GFSM_TILE");
    if (force && *force) {
        const int v = atoi(force);
        return v >= 0 && v < kVariants ? v : 0;
    }
    const char *at = getenv("GFSM_AUTOTUNE");
    if (at && *at == '0') return 0;
    const uint64_t key = workload_class(plans, g);
    auto it = tuned.find(key);
    if (it != tuned.end()) return it->second;
    if (!autotune) {
        // no tuning runs here (served slots): the choice already made for the
        // nearest batch size of the same workload class, else the default
        int best = 0;
        long dist = -1;
        for (const auto &kv : tuned)
            if ((kv.first >> 8) == (key >> 8)) {
                const long dd = std::labs((long)(kv.first & 0xff) - (long)(key & 0xff));
                if (dist < 0 || dd < dist) {
                    dist = dd;
                    best = kv.second;
                }
            }
        return best;
    }
    // The samples run on the driver the whole call takes -- the graph for a
    // light call (first level of at most kGraphRootEntries candidates), else
    // the host loop -- since a geometry's graph kernel and its one-CTA-per-
    // tile kernel rank differently (the grid batch: (256,2) did not beat
    // (256,4) by 2% on a 128-query sample on the graph, and takes the whole
    // batch 7% faster on the host loop).  Geometries are compared on
    // level-step time, which the host loop's round trips do not dilute.
    uint64_t first_level = 0;
    for (size_t i = 0; i < plans.size() && first_level <= kGraphRootEntries; ++i) {
        DQuery dq;
        uint32_t lo = 0, hi = 0;
        bool never = false;
        if (build_dquery(*plans[i], g, lim, dq, lo, hi, never) == GFSM_OK && !never)
            first_level += (uint64_t)g.h_rowptr[hi] - g.h_rowptr[lo];
    }
    const bool heavy = first_level > kGraphRootEntries;
    struct DriverScope {
        int &d;
        ~DriverScope() { d = -1; }
    } scope{tune_driver};
    tune_driver = heavy ? 0 : 1;
    // The sample is the call's first 32 queries, grown fourfold (up to 2,048)
    // while the default geometry takes under 2 ms on it (8 ms for a host-loop
    // call, whose steps at full size are many waves long): shorter samples
    // are launch-bound and their timings mostly noise.  Another geometry
    // must beat the default by 2% to be chosen (repeat timings of a sample
    // agree within ~0.5%).
    const double min_ms = heavy ? 8.0 : 2.0;
    int best = 0;
    for (size_t ns = std::min<size_t>(plans.size(), 32);; ns = std::min<size_t>(plans.size(), ns * 4)) {
        std::vector<const Plan *> sample(plans.begin(), plans.begin() + ns);
        std::vector<uint64_t> cnt(ns);
        gfsm_stats s0{};
        if (run(sample, g, lim, cnt.data(), &s0, nullptr, 0, nullptr, err, 0) != GFSM_OK) return 0;
        if (s0.device_ms < min_ms) {
            if (ns < plans.size() && ns < 2048) continue;
            break;  // the whole call is short: keep the default
        }
        const double base_ms = s0.kernel_ms;
        double best_ms = base_ms;
        for (int v = 1; v < kVariants; ++v) {
            gfsm_stats sv{};
            if (run(sample, g, lim, cnt.data(), &sv, nullptr, 0, nullptr, err, v) != GFSM_OK) return 0;
            if (sv.kernel_ms < best_ms && sv.kernel_ms < 0.98 * base_ms) {
                best_ms = sv.kernel_ms;
                best = v;
            }
        }
        break;
    }
    tuned[key] = best;
    return best;
}

gfsm_status Engine::run(const std::vector<const Plan *> &plans, const DeviceGraph &g, const gfsm_limits &lim,
                        uint64_t *counts_out, gfsm_stats *stats, uint32_t *rows_out, uint64_t max_rows,
                        uint64_t *n_rows, std::string &err, int variant, uint32_t part, uint32_t nparts) {
    if (nparts == 0 || part >= nparts || (nparts > 1 && rows_out)) return GFSM_ERR_ARG;
    // GFSM_TRACE=1: one line per step on stderr (depth, candidates, survivors,
    // kernel ms) -- the per-level frontier statistics of the reference's
    // pcsv_printf HnStep / HnPred lines (HnGPU.cu:431, 525)
    static const bool trace = [] {
        const char *t = getenv("GFSM_TRACE");
        return t && *t && *t != '0';
    }();
    // Driver: GFSM_DRIVER=graph|host forces one.  By default a light call --
    // first level of at most kGraphRootEntries candidates over all its
    // queries -- runs its whole schedule as one CUDA graph launch (no host
    // round trip per step: plain p50 0.41 -> 0.33 ms on the grid workload);
    // heavier calls run the host-driven loop, whose steps launch one CTA per
    // tile (the graph's fixed persistent grid runs a large step ~10% slower:
    // it spills more at the 32-register budget).  A single query takes the
    // default geometry, a batch the autotuned one.
    const char *drv = getenv("GFSM_DRIVER");
    const bool env_drv = drv && *drv;
    const bool force_graph = !trace && ((env_drv && !strcmp(drv, "graph")) || (!env_drv && tune_driver == 1));
    const bool force_host = trace || (env_drv && strcmp(drv, "graph")) || (!env_drv && tune_driver == 0);
    if (variant < 0) variant = (plans.size() <= 1) ? 0 : pick_variant(plans, g, lim, err);
    auto t_start = std::chrono::steady_clock::now();
    const int nq = (int)plans.size();
    gfsm_stats st{};
    for (int i = 0; i < nq; ++i) counts_out[i] = 0;
    if (n_rows) *n_rows = 0;
    ECHECK(cudaSetDevice(device));

    // device plans for the queries that can match at all
    std::vector<DQuery> dq;
    std::vector<int> active;
    std::vector<uint32_t> rlo, rhi;
    uint32_t dmax = 0;
    // Symmetry breaking (a plan's aut > 1): exact where the count is the
    // automorphism group's order times the count of one embedding per orbit
    // -- symmetric data with one edge label and no repeated edge, counts
    // only (mapping rows list every embedding); GFSM_SYMMETRY=0 turns it off.
    const char *symv = getenv("GFSM_SYMMETRY");
    const bool sym_ok = !rows_out && g.symmetric && !g.multi && g.elab == nullptr && !(symv && *symv == '0');
    const bool vl_on = lim.vertex_labels != 0;
    {
        // independent per query: large batches use a few host threads; the
        // plans are built in place and the active ones compacted below
        dq.resize(nq);
        std::vector<DQuery> &all = dq;
        std::vector<uint32_t> lo(nq), hi(nq);
        std::vector<char> never(nq, 0);
        std::vector<gfsm_status> qrc(nq, GFSM_OK);
        const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), nq / 512));
        auto work = [&](int t) {
            for (int i = t; i < nq; i += nt) {
                bool nv = false;
                qrc[i] = build_dquery(*plans[i], g, lim, all[i], lo[i], hi[i], nv, sym_ok && plans[i]->aut > 1 &&
                                                                                         plans[i]->sym_vl == vl_on);
                never[i] = nv;
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto &th : pool) th.join();
        std::vector<uint64_t> cut(nparts + 1);
        size_t w = 0;
        for (int i = 0; i < nq; ++i) {
            if (qrc[i] != GFSM_OK) return qrc[i];
            if (never[i]) continue;
            if (nparts > 1) {  // this part's share of the root window
                root_partition(g.h_rowptr.data(), lo[i], hi[i], nparts, cut.data());
                const uint32_t base = lo[i];
                lo[i] = base + (uint32_t)cut[part];
                hi[i] = base + (uint32_t)cut[part + 1];
            }
            if (w != (size_t)i) all[w] = all[i];
            ++w;
            active.push_back(i);
            rlo.push_back(lo[i]);
            rhi.push_back(hi[i]);
            dmax = std::max(dmax, all[w - 1].k - 1);
        }
        dq.resize(w);
    }
    const uint32_t na = (uint32_t)active.size();
    const auto t_plans = std::chrono::steady_clock::now();
    if (na > kNodeMask) {  // a tuple's trie node id has 22 bits
        err = "a call takes at most " + std::to_string(kNodeMask) + " queries";
        return GFSM_ERR_TOO_LARGE;
    }
    if (na == 0) {
        if (stats) {
            st.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
            *stats = st;
        }
        return GFSM_OK;
    }
    const uint64_t rows_bytes = rows_out ? max_rows * (uint64_t)dq[0].k * 4 : 0;

    // Shared prefixes: a trie of the queries' device plans.  A node at depth
    // d is a set of queries whose plans for depths 0..d are byte-identical
    // (windows, requirements, final flags and the depth-(d+1) slice), so one
    // tuple stands for all of them.  A node is named by its smallest member
    // (its representative); a node with several child nodes lists their
    // representatives in fan_list, recorded in the representative's lv[d]
    // (fan_start, fan_count), and the step at depth d+1 runs such a parent's
    // candidates over (child node, row offset).  Final-level counts go to the
    // final node's representative and are copied to its members here.
    const char *shr = getenv("GFSM_SHARE");
    bool share = !rows_out && na >= 2 && !(shr && *shr == '0');
    // A tuple's next-level candidate count (its row slice, times its node's
    // child nodes) and a warp's running sum of up to kWarpStage of them are
    // 32-bit: the data graph's largest row bounds both, and caps the fan-out.
    const uint64_t row_max = std::max<uint64_t>(g.max_degree, 1);
    if (row_max * kWarpStage > 0xffffffffull) {
        err = "a data row of " + std::to_string(g.max_degree) + " entries exceeds the level step's 32-bit slice sums";
        return GFSM_ERR_TOO_LARGE;
    }
    const uint64_t fan_cap = 0xffffffffull / (row_max * kWarpStage);
    std::vector<uint32_t> root_rep, fan_list, final_rep(na);
    for (uint32_t i = 0; i < na; ++i) final_rep[i] = i;
    if (share) {
        // members of a node grouped by their plan at depth d (hash of the
        // 64 plan bytes, equality checked bytewise), each group's members
        // ascending, groups ordered by representative (smallest member)
        auto lv_hash = [&](uint32_t i, uint32_t d) {
            uint64_t w[sizeof(DLevel) / 8];
            std::memcpy(w, &dq[i].lv[d], sizeof(DLevel));
            uint64_t h = 0x9e3779b97f4a7c15ull;
            for (uint64_t x : w) h = (h ^ x) * 0xff51afd7ed558ccdull, h ^= h >> 32;
            return h;
        };
        auto split = [&](const std::vector<uint32_t> &mem, uint32_t d) {
            std::vector<std::vector<uint32_t>> out;
            if (mem.size() == 1) {
                out.push_back(mem);
                return out;
            }
            // members sorted by (plan hash, id): a run of equal hashes holds
            // one group per distinct plan (compared bytewise), each group's
            // members ascending; then the groups by representative
            std::vector<std::pair<uint64_t, uint32_t>> hv(mem.size());
            for (size_t i = 0; i < mem.size(); ++i) hv[i] = {lv_hash(mem[i], d), mem[i]};
            std::sort(hv.begin(), hv.end());
            for (size_t i = 0; i < hv.size();) {
                size_t j = i;
                while (j < hv.size() && hv[j].first == hv[i].first) ++j;
                const size_t run0 = out.size();
                for (size_t t = i; t < j; ++t) {
                    const uint32_t m = hv[t].second;
                    size_t gi = out.size();
                    for (size_t g2 = run0; g2 < out.size(); ++g2)
                        if (!std::memcmp(&dq[out[g2][0]].lv[d], &dq[m].lv[d], sizeof(DLevel))) {
                            gi = g2;
                            break;
                        }
                    if (gi == out.size()) out.emplace_back();
                    out[gi].push_back(m);
                }
                i = j;
            }
            std::sort(out.begin(), out.end(),
                      [](const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) { return a[0] < b[0]; });
            return out;
        };
        std::vector<uint32_t> all(na);
        for (uint32_t i = 0; i < na; ++i) all[i] = i;
        std::vector<std::vector<uint32_t>> level = split(all, 0);
        for (const auto &n : level) root_rep.push_back(n[0]);
        for (uint32_t d = 0; !level.empty() && share; ++d) {
            std::vector<std::vector<uint32_t>> next;
            for (auto &n : level) {
                const uint32_t r = n[0];
                if (dq[r].lv[d].final_) {
                    for (uint32_t m : n) final_rep[m] = r;
                    continue;
                }
                auto kids = split(n, d + 1);
                if (kids.size() > fan_cap || kids.size() > 0xffffu) {  // too wide for the 32-bit slice sums
                    share = false;
                    break;
                }
                if (kids.size() > 1) {
                    dq[r].lv[d].fan_count = (uint16_t)kids.size();
                    dq[r].lv[d].fan_start = (uint32_t)fan_list.size();
                    bool leaves = true;  // every child node's depth d+1 is counted at its parent
                    for (const auto &k : kids) {
                        fan_list.push_back(k[0]);
                        const DLevel &N = dq[k[0]].lv[d + 1];
                        leaves = leaves && N.final_ && N.nreq == 0 && !(N.anchor_check & 1u);
                    }
                    if (leaves) dq[r].lv[d].anchor_check |= 2u;
                }
                // a node of one query has no fan-out below it and counts to
                // itself: it is not carried to deeper levels
                for (auto &k : kids)
                    if (k.size() > 1) next.push_back(std::move(k));
            }
            level.swap(next);
        }
        if (!share) {
            for (DQuery &q : dq)
                for (DLevel &l : q.lv) l.fan_count = 0, l.fan_start = 0, l.anchor_check &= 1u;
            fan_list.clear();
            root_rep.clear();
            for (uint32_t i = 0; i < na; ++i) final_rep[i] = i;
        }
    }
    if (!share)
        for (uint32_t i = 0; i < na; ++i) root_rep.push_back(i);
    const uint32_t ne = na;                        // count slots: one per query (representatives)
    const uint32_t nr = (uint32_t)root_rep.size();  // root-level parents
    const auto t_trie = std::chrono::steady_clock::now();
    if (fan_list.empty()) fan_list.push_back(0);

    // arena layout: plans | counts | step counts | root coff | root cstart |
    //               root representatives | fan list | mapping rows | depth buffers
    auto al = [](uint64_t b) { return (b + 255) & ~255ull; };
    const uint64_t plans_bytes = (uint64_t)ne * sizeof(DQuery);
    const uint64_t head = al(plans_bytes) + 2 * al((uint64_t)ne * 8) + al(((uint64_t)nr + 1) * 8) +
                          2 * al((uint64_t)nr * 4) + al((uint64_t)fan_list.size() * 4) + al(rows_bytes);
    uint64_t budget = arena_cap;
    if (budget <= head + (1ull << 20) * dmax) return GFSM_ERR_NOMEM;
    gfsm_status rc = ensure_arena(budget, err);
    if (rc != GFSM_OK) return rc;
    char *p = static_cast<char *>(arena);
    DQuery *d_plans = reinterpret_cast<DQuery *>(p);
    p += al(plans_bytes);
    unsigned long long *d_counts = reinterpret_cast<unsigned long long *>(p);
    p += al((uint64_t)ne * 8);
    unsigned long long *d_step_counts = reinterpret_cast<unsigned long long *>(p);
    p += al((uint64_t)ne * 8);
    unsigned long long *d_rcoff = reinterpret_cast<unsigned long long *>(p);
    p += al(((uint64_t)nr + 1) * 8);
    uint32_t *d_rcstart = reinterpret_cast<uint32_t *>(p);
    p += al((uint64_t)nr * 4);
    uint32_t *d_root_rep = reinterpret_cast<uint32_t *>(p);
    p += al((uint64_t)nr * 4);
    uint32_t *d_fan_list = reinterpret_cast<uint32_t *>(p);
    p += al((uint64_t)fan_list.size() * 4);
    uint32_t *d_rows = rows_out ? reinterpret_cast<uint32_t *>(p) : nullptr;
    const uint64_t head_used = (uint64_t)(p - static_cast<char *>(arena));  // everything the call sends
    p += al(rows_bytes);

    // The head (plans, zeroed counts, root tables, fan list) is laid out in a
    // pinned staging buffer exactly as in the arena and sent with one copy.
    // A copy of an earlier call (one that returned early) may still read it.
    ECHECK(cudaStreamSynchronize(stream));
    if (h_stage_bytes < head_used) {
        // grown geometrically: freeing pinned memory synchronises the device,
        // and served slots see batches of every size
        const uint64_t want = std::max<uint64_t>({head_used, 2 * h_stage_bytes, 1ull << 20});
        if (h_stage) cudaFreeHost(h_stage);
        h_stage = nullptr;
        h_stage_bytes = 0;
        ECHECK(cudaMallocHost(&h_stage, want));
        h_stage_bytes = want;
    }
    char *hs = static_cast<char *>(h_stage);
    auto host_of = [&](const void *dev) { return hs + (static_cast<const char *>(dev) - static_cast<char *>(arena)); };
    std::memcpy(host_of(d_plans), dq.data(), plans_bytes);
    std::memset(host_of(d_counts), 0, 2 * al((uint64_t)ne * 8));  // counts and step counts
    {
        unsigned long long *rcoff = reinterpret_cast<unsigned long long *>(host_of(d_rcoff));
        uint32_t *rcstart = reinterpret_cast<uint32_t *>(host_of(d_rcstart));
        rcoff[0] = 0;
        for (uint32_t i = 0; i < nr; ++i) {
            rcstart[i] = rlo[root_rep[i]];
            rcoff[i + 1] = rcoff[i] + (rhi[root_rep[i]] - rlo[root_rep[i]]);
        }
    }
    std::memcpy(host_of(d_root_rep), root_rep.data(), (uint64_t)nr * 4);
    std::memcpy(host_of(d_fan_list), fan_list.data(), (uint64_t)fan_list.size() * 4);
    const unsigned long long root_total =
        reinterpret_cast<const unsigned long long *>(host_of(d_rcoff))[nr];
    ECHECK(cudaMemcpyAsync(arena, h_stage, head_used, cudaMemcpyHostToDevice, stream));
    ECHECK(cudaMemsetAsync(rows_ctr, 0, 4, stream));
    st.h2d_bytes += head_used;
    // per-query totals: every member of a final node gets its representative's count
    // (times the automorphism group's order where symmetry breaking ran)
    auto gather_counts = [&](const std::vector<unsigned long long> &cnt) {
        std::vector<unsigned long long> out(na);
        for (uint32_t i = 0; i < na; ++i) {
            const Plan &pl = *plans[active[i]];
            const bool sb = sym_ok && pl.aut > 1 && pl.sym_vl == vl_on;
            out[i] = cnt[final_rep[i]] * (sb ? pl.aut : 1ull);
        }
        return out;
    };
    if (trace) {
        auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        fprintf(stderr, "gfsm-host plans=%.3f trie=%.3f staging=%.3f ms (queries %u, root nodes %u)\n",
                ms(t_start, t_plans), ms(t_plans, t_trie), ms(t_trie, std::chrono::steady_clock::now()), na, nr);
    }
    ECHECK(cudaEventRecord(ev_begin, stream));

    // depth buffers 0 .. dmax-1 (depth dmax is count-only)
    const uint64_t rest = budget - (uint64_t)(p - static_cast<char *>(arena));
    struct Buf {
        uint32_t *tup;
        uint64_t cap;
        uint32_t *cstart;
        unsigned long long *coff;
    };
    std::vector<Buf> buf(dmax);
    {
        // every depth buffer starts on a 256-byte boundary (u64 coff arrays)
        const uint64_t share = dmax ? (rest / dmax) & ~255ull : 0;
        for (uint32_t d = 0; d < dmax; ++d) {
            const uint64_t per = tuple_bytes(d);
            uint64_t cap = share > 1024 ? (share - 1024) / per : 0;
            cap = std::min<uint64_t>(cap, lim.max_soln_size);
            cap = std::min<uint64_t>(cap, 0xffffffffull);
            if (cap < TILE) return GFSM_ERR_NOMEM;
            Buf &b = buf[d];
            b.cap = cap;
            char *q = p + share * d;
            b.coff = reinterpret_cast<unsigned long long *>(q);
            q += ((cap + 1) * 8 + 255) & ~255ull;
            b.tup = reinterpret_cast<uint32_t *>(q);
            q += (cap * 4 * (d + 2) + 255) & ~255ull;
            b.cstart = reinterpret_cast<uint32_t *>(q);
            if ((reinterpret_cast<uintptr_t>(b.coff) | reinterpret_cast<uintptr_t>(b.tup) |
                 reinterpret_cast<uintptr_t>(b.cstart)) & 255u) {
                err = "frontier buffer not 256-byte aligned";
                return GFSM_ERR_CUDA;
            }
        }
    }

    GraphView gv{g.rowptr, g.adj, g.elab, g.order, g.single_label, g.n};
    // GFSM_SURVIVOR_GUESS: the survivor ratio assumed for a depth's first
    // chunk (default 1: a first chunk never overflows).  A smaller guess takes
    // larger first chunks -- fewer steps where survival is low, re-runs where
    // it is not.  Later chunks follow the observed ratio either way.
    // last query vertices counted when their parents are written (next_slice):
    // not when mappings are captured (such a vertex gets no row)
    const bool leaf_ok = !rows_out;
    const double ratio_init = [] {  // read per call: cheap, and tests change it
        const char *v = getenv("GFSM_SURVIVOR_GUESS");
        const double x = v && *v ? atof(v) : 1.0;
        return x > 0.0 ? std::min(1.0, std::max(x, 1.0 / 8192.0)) : 1.0;
    }();
    // the graph-driven schedule (falls back to the host loop if the graph
    // cannot be built, e.g. when every constant-memory argument slot is taken)
    uint64_t first_level = 0;  // CCSR entries of the root windows: the first level's candidates, at most
    for (uint32_t i = 0; i < na && first_level <= kGraphRootEntries; ++i)
        first_level += (uint64_t)g.h_rowptr[rhi[i]] - g.h_rowptr[rlo[i]];
    const bool want_graph = !force_host && (force_graph || first_level <= kGraphRootEntries);
    bool graph_driver = false;
    if (want_graph && graph_geo(variant) >= 0) {
        std::string gerr;
        graph_driver = build_graph(variant, gerr) == GFSM_OK;
        if (!graph_driver) st.graph_error = last_graph_error ? last_graph_error : -1;
    }
    // next-level candidates per candidate each depth saw in this workload
    // class's last call: the first step of a depth is sized from it
    std::vector<double> &seen = nxt_seen[workload_class(plans, g)];
    if (seen.size() < (size_t)dmax + 1) seen.resize((size_t)dmax + 1, 0.0);
    if (graph_driver) {
        Ctl c;
        std::memset(&c, 0, sizeof(c));
        c.total[0] = root_total;
        for (uint32_t i = 0; i <= dmax; ++i) c.nxt[i] = (float)seen[i];
        c.np[0] = nr;
        for (int i = 0; i <= MAXQ; ++i) c.ratio[i] = (float)ratio_init;
        for (uint32_t i = 0; i < dmax; ++i) {
            c.tup[i] = buf[i].tup;
            c.cap[i] = buf[i].cap;
            c.cstart[i] = buf[i].cstart;
            c.coff[i] = buf[i].coff;
        }
        c.root_coff = d_rcoff;
        c.root_cstart = d_rcstart;
        c.counts = d_counts;
        c.nq = ne;
        c.max_scan = max_scan;
        c.max_candidates = lim.max_candidates;
        c.dmax = dmax;
        c.tile = variant_tile(variant);
        StepArgs &a = c.args;
        a.g = gv;
        a.plans = d_plans;
        a.tile_parent = tile_parent;
        a.counts = d_step_counts;
        a.result = d_result;
        a.rows_out = d_rows;
        a.max_rows = max_rows;
        a.rows_ctr = rows_ctr;
        a.root_rep = d_root_rep;
        a.fan_list = d_fan_list;
        a.leaf_count = leaf_ok ? 1u : 0u;
        Ctl *d_ctl = static_cast<Ctl *>(ctl);
        ECHECK(cudaMemcpyAsync(d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
        st.h2d_bytes += sizeof(Ctl);
        ECHECK(cudaEventRecord(ev0, stream));
        ECHECK(cudaGraphLaunch(graph_exec[graph_geo(variant)], stream));
        ECHECK(cudaEventRecord(ev1, stream));
        ECHECK(cudaMemcpyAsync(&c, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        std::vector<unsigned long long> ecnt(ne);
        ECHECK(cudaMemcpyAsync(ecnt.data(), d_counts, (uint64_t)ne * 8, cudaMemcpyDeviceToHost, stream));
        ECHECK(cudaStreamSynchronize(stream));
        st.d2h_bytes += sizeof(Ctl) + (uint64_t)ne * 8;
        const std::vector<unsigned long long> cnt = gather_counts(ecnt);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        st.steps = c.steps;
        for (uint32_t i = 0; i <= dmax; ++i) seen[i] = c.nxt[i];
        st.peak_frontier_bytes = c.peak;
        st.launches = (uint32_t)(1 + 4 * c.steps);  // first controller, then partition, root step, step, controller
        st.retries = c.retries;
        st.candidates = c.candidates;
        st.expansions = c.expansions;
        st.alg_bytes = c.alg_bytes;
        st.kernel_ms = ms;
        st.device_ms = ms;
        st.tile_variant = variant;
        st.driver = 1;
        if (c.err) {
            err = "device schedule error bits " + std::to_string(c.err);
            if (stats) *stats = st;
            return (c.err & KERR_CAP) ? GFSM_ERR_TOO_LARGE : GFSM_ERR_CUDA;
        }
        for (uint32_t i = 0; i < na; ++i) counts_out[active[i]] = cnt[i];
        if (rows_out) {
            uint32_t claimed = 0;
            ECHECK(cudaMemcpy(&claimed, rows_ctr, 4, cudaMemcpyDeviceToHost));
            const uint64_t nr = std::min<uint64_t>(claimed, max_rows);
            if (nr) ECHECK(cudaMemcpy(rows_out, d_rows, nr * dq[0].k * 4, cudaMemcpyDeviceToHost));
            st.d2h_bytes += nr * dq[0].k * 4;
            if (n_rows) *n_rows = nr;
        }
        for (uint32_t i = 0; i < na; ++i) st.count += cnt[i];
        st.wall_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        if (stats) *stats = st;
        return GFSM_OK;
    }
    std::vector<unsigned long long> total(dmax + 1, 0), pos(dmax + 1, 0), np(dmax + 1, 0), held(dmax + 1, 0);
    std::vector<double> ratio(dmax + 1, ratio_init);
    std::vector<double> nxt(seen.begin(), seen.begin() + dmax + 1);  // emit_chunk_cap's rates
    std::vector<char> has_final(dmax + 1, 0);  // some query ends at this depth
    for (const DQuery &q : dq) {
        has_final[q.k - 1] = 1;
        if (leaf_ok && q.k >= 2) has_final[q.k - 2] = 1;  // last vertices counted when their parents are written
    }
    total[0] = root_total;
    np[0] = nr;
    uint32_t d = 0;
    float kms = 0.f;
    for (;;) {
        if (pos[d] >= total[d]) {
            if (d == 0) break;
            --d;
            continue;
        }
        const bool emits = d < dmax;
        unsigned long long chunk = std::min<unsigned long long>(total[d] - pos[d], (unsigned long long)max_scan);
        if (emits) {
            const double allowed = (double)buf[d].cap / std::max(ratio[d], 1.0 / 8192.0);
            chunk = std::min<unsigned long long>(chunk, (unsigned long long)std::max<double>(allowed, TILE));
            chunk = std::min<unsigned long long>(chunk, emit_chunk_cap(nxt[d]));
        }
        const uint32_t vtile = variant_tile(variant);
        chunk = std::min<unsigned long long>(chunk, (unsigned long long)dir_tiles * vtile);
        const uint32_t ntiles = (uint32_t)div_up(chunk, vtile);
        StepArgs a{};
        a.g = gv;
        a.plans = d_plans;
        a.depth = d;
        if (d == 0) {
            a.ptup = nullptr;
            a.pstride = 0;
            a.pcstart = d_rcstart;
            a.pcoff = d_rcoff;
        } else {
            a.ptup = buf[d - 1].tup;
            a.pstride = buf[d - 1].cap;
            a.pcstart = buf[d - 1].cstart;
            a.pcoff = buf[d - 1].coff;
        }
        a.np = np[d];
        a.tile_parent = tile_parent;
        a.c0 = pos[d];
        a.cend = pos[d] + chunk;
        a.ntiles = ntiles;
        if (emits) {
            a.ctup = buf[d].tup;
            a.cstride = buf[d].cap;
            a.ccap = buf[d].cap;
            a.ccstart = buf[d].cstart;
            a.ccoff = buf[d].coff;
        }
        a.counts = d_step_counts;
        a.result = d_result;
        a.rows_out = d_rows;
        a.max_rows = max_rows;
        a.rows_ctr = rows_ctr;
        a.root_rep = d_root_rep;
        a.fan_list = d_fan_list;
        a.leaf_count = leaf_ok ? 1u : 0u;
        a.pcoff_end = total[d];
        k_partition<<<(unsigned)div_up((uint64_t)std::max<uint32_t>(ntiles + 1, ne), 256), 256, 0, stream>>>(
            a.pcoff, a.np, a.pcoff_end, a.c0, chunk, ntiles, vtile, tile_parent, d_result, d_step_counts, ne);
        ECHECK(cudaEventRecord(ev0, stream));
        launch_step(variant, d == 0, a, ntiles, stream);
        ECHECK(cudaGetLastError());
        st.launches += 2;  // partition + level step
        ECHECK(cudaEventRecord(ev1, stream));
        ECHECK(cudaMemcpyAsync(h_result, d_result, sizeof(StepResult), cudaMemcpyDeviceToHost, stream));
        ECHECK(cudaStreamSynchronize(stream));
        st.d2h_bytes += sizeof(StepResult);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        kms += ms;
        st.steps++;
        StepResult r = *h_result;
        r.n_children = r.alloc >> kAllocShift;  // the step's totals are its allocator word
        r.total_next = r.alloc & kAllocMask;
        if (r.err) {
            err = "device step error bits " + std::to_string(r.err);
            return GFSM_ERR_CUDA;
        }
        if (emits && r.next_ovf && chunk <= vtile) {
            err = "one tile's children have more next-level candidates than a step can index";
            return GFSM_ERR_TOO_LARGE;
        }
        if (emits && (r.n_children > buf[d].cap || r.next_ovf)) {
            // more survivors than the level buffer holds (or more next-level
            // candidates than the allocator indexes): redo a smaller chunk
            st.retries++;
            ratio[d] = std::max(ratio[d] * 4.0, 2.0 * (double)r.n_children / (double)chunk);
            if (r.next_ovf)  // the next level's candidates overflowed the field: at most half this chunk next
                nxt[d] = std::max(nxt[d] * 4.0, (double)kAllocMask / (double)chunk);
            continue;
        }
        if (trace)
            fprintf(stderr, "gfsm-step depth=%u cand=%llu children=%llu next=%llu tiles=%u ms=%.4f\n", d, chunk,
                    emits ? r.n_children : 0ull, emits ? r.total_next : 0ull, ntiles, ms);
        if (has_final[d]) {
            k_commit<<<(unsigned)div_up(ne, 256), 256, 0, stream>>>(d_counts, d_step_counts, ne);
            st.launches += 1;
        }
        st.candidates += chunk;
        st.expansions += r.n_children;
        if (lim.max_candidates && st.candidates > lim.max_candidates) {
            err = "candidate cap (max_candidates) reached";
            if (stats) *stats = st;
            return GFSM_ERR_TOO_LARGE;
        }
        st.alg_bytes += r.alg_bytes + (emits ? r.n_children * 4ull * (d + 1) : 0ull);
        pos[d] += chunk;
        if (emits) {
            held[d] = r.n_children;
            unsigned long long live = 0;  // the buffers of depths <= d are live now
            for (uint32_t i = 0; i <= d; ++i) live += held[i] * tuple_bytes(i);
            st.peak_frontier_bytes = std::max<uint64_t>(st.peak_frontier_bytes, live);
            const double obs = (double)r.n_children / (double)chunk;
            ratio[d] = std::max(2.0 * obs, ratio[d] * 0.5);
            nxt[d] = std::max((double)r.total_next / (double)chunk, nxt[d] * 0.5);
            if (r.n_children > 0 && r.total_next > 0) {
                np[d + 1] = r.n_children;
                total[d + 1] = r.total_next;
                pos[d + 1] = 0;
                ++d;
            }
        }
    }
    ECHECK(cudaEventRecord(ev_end, stream));
    for (uint32_t i = 0; i <= dmax; ++i) seen[i] = nxt[i];
    std::vector<unsigned long long> ecnt(ne);
    ECHECK(cudaMemcpyAsync(ecnt.data(), d_counts, (uint64_t)ne * 8, cudaMemcpyDeviceToHost, stream));
    st.d2h_bytes += (uint64_t)ne * 8;
    if (rows_out) ECHECK(cudaMemcpyAsync(h_result, d_result, sizeof(StepResult), cudaMemcpyDeviceToHost, stream));
    ECHECK(cudaStreamSynchronize(stream));
    const std::vector<unsigned long long> cnt = gather_counts(ecnt);
    for (uint32_t i = 0; i < na; ++i) counts_out[active[i]] = cnt[i];
    if (rows_out) {
        uint64_t total_rows = 0;
        for (uint32_t i = 0; i < na; ++i) total_rows += cnt[i];
        const uint64_t nr = std::min<uint64_t>(total_rows, max_rows);
        if (nr) ECHECK(cudaMemcpy(rows_out, d_rows, nr * dq[0].k * 4, cudaMemcpyDeviceToHost));
        st.d2h_bytes += nr * dq[0].k * 4;
        if (n_rows) *n_rows = nr;
    }
    for (uint32_t i = 0; i < na; ++i) st.count += cnt[i];
    st.kernel_ms = kms;
    st.tile_variant = variant;
    {
        float dms = 0.f;
        cudaEventElapsedTime(&dms, ev_begin, ev_end);
        st.device_ms = dms;
    }
    st.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    if (stats) *stats = st;
    return GFSM_OK;
}

}  // namespace gfsm

// ---------------------------------------------------------------------------
// gfsm_match_count_noalloc: the level steps above, run entirely out of one
// fixed, file-scope device array instead of memory the library allocates.
//
// Who needs it: callers that must not allocate device memory during a
// match -- code that owns a fixed device-memory budget (or its own pool) and
// cannot let a library take more, code on a latency-critical path where
// cudaMalloc/cudaFree's implicit device synchronisation is not acceptable,
// and code that issues its work into a stream it does not want the library to
// synchronise with other streams.  They build the data graph's device CCSR
// once at set-up (gfsm_graph_to_device) and prepare plans on the host; each
// match then allocates nothing: no cudaMalloc / cudaFree / cudaMallocHost /
// cudaMallocAsync, no stream or event creation.
//
// Limit: the scratch is kNoAllocScratchBytes (64 MiB) per device -- the
// tile directory for steps of up to kNoAllocTiles * 1024 candidates plus a
// frontier arena shared by the query's levels.  Queries always fit because the
// depth-first chunking shrinks steps to the arena; a query whose plan cannot
// get even one tile of frontier per level is rejected with
// GFSM_ERR_TOO_LARGE.  Every process that loads libgfsm.so holds this array
// on every device where the module is loaded, until it exits.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoAllocScratchBytes = 64ull << 20;
constexpr uint32_t kNoAllocTiles = 65536;  // 64M candidates per step

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;  // serialises host threads; the array itself is one per device

}  // namespace

extern "C" gfsm_status gfsm_match_count_noalloc(const gfsm_plan *plan, const gfsm_graph *data, void *stream,
                                                uint64_t *count) {
    using namespace gfsm;
    if (!plan || !data || !count) return GFSM_ERR_ARG;
    if (!data->dev || !data->ctx) return GFSM_ERR_ARG;  // build the device CCSR first (gfsm_graph_to_device)
    const DeviceGraph &g = *data->dev;
    const gfsm_limits &lim = data->ctx->lim;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    *count = 0;
    if (cudaSetDevice(g.device) != cudaSuccess) return GFSM_ERR_CUDA;

    // The host only knows the array by a stand-in symbol: its device address
    // is looked up on every call, with the data graph's device current (cheap
    // once the module is loaded, and still right after a device reset has
    // reloaded the module elsewhere).  The first call on a device may load
    // the module, so it belongs before any stream capture.
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    unsigned char *scratch = nullptr;
    {
        void *addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return GFSM_ERR_CUDA;
        scratch = static_cast<unsigned char *>(addr);
    }
    // Once work is queued, a failing call waits for it before returning, so
    // no copy or kernel of a failed call still touches the shared array when
    // the next call starts.
    bool queued = false;
    auto fail = [&](gfsm_status s) {
        if (queued) cudaStreamSynchronize(st);
        cudaGetLastError();
        return s;
    };
    const bool trace = [] {
        const char *t = getenv("GFSM_TRACE");
        return t && *t && *t != '0';
    }();

    DQuery dq;
    uint32_t rlo = 0, rhi = 0;
    bool never = false;
    gfsm_status rc = build_dquery(plan->p, g, lim, dq, rlo, rhi, never);
    if (rc != GFSM_OK) return rc;
    if (never) return GFSM_OK;
    const uint32_t dmax = dq.k - 1;

    // scratch layout: result | counters | tile directory |
    //                 plan | count | root coff | root slice start | depth buffers
    unsigned char *p = scratch;
    StepResult *d_result = reinterpret_cast<StepResult *>(p);
    p += 256;
    uint32_t *rows_ctr = reinterpret_cast<uint32_t *>(p);
    p += 256;
    uint32_t *tile_parent = reinterpret_cast<uint32_t *>(p);
    p += (((uint64_t)kNoAllocTiles + 2) * 4 + 255) & ~255ull;
    DQuery *d_plan = reinterpret_cast<DQuery *>(p);
    p += (sizeof(DQuery) + 255) & ~255ull;
    unsigned long long *d_count = reinterpret_cast<unsigned long long *>(p);
    unsigned long long *d_rcoff = d_count + 4;
    uint32_t *d_rcstart = reinterpret_cast<uint32_t *>(d_count + 8);
    uint32_t *d_root_rep = d_rcstart + 4;  // the single root parent is query 0 of the plan array
    p += 256;
    const uint64_t used = (uint64_t)(p - scratch);
    const uint64_t share = dmax ? ((kNoAllocScratchBytes - used) / dmax) & ~255ull : 0;
    struct Buf {
        uint32_t *tup;
        uint64_t cap;
        uint32_t *cstart;
        unsigned long long *coff;
    } buf[MAXQ];
    for (uint32_t d = 0; d < dmax; ++d) {
        const uint64_t per = 4ull * (d + 2) + 4 + 8;
        uint64_t cap = share > 1024 ? (share - 1024) / per : 0;
        cap = std::min<uint64_t>(cap, lim.max_soln_size);
        if (cap < (uint64_t)TILE) return GFSM_ERR_TOO_LARGE;  // needs more than the fixed scratch
        unsigned char *q = p + share * d;
        buf[d].cap = cap;
        buf[d].coff = reinterpret_cast<unsigned long long *>(q);
        q += ((cap + 1) * 8 + 255) & ~255ull;
        buf[d].tup = reinterpret_cast<uint32_t *>(q);
        q += (cap * 4 * (d + 2) + 255) & ~255ull;
        buf[d].cstart = reinterpret_cast<uint32_t *>(q);
    }

    // per-call inputs into the scratch; the count must start at zero
    const unsigned long long rc2[2] = {0ull, (unsigned long long)(rhi - rlo)};
    queued = true;
    if (cudaMemcpyAsync(d_plan, &dq, sizeof(DQuery), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_rcoff, rc2, sizeof(rc2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_rcstart, &rlo, 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(d_count, 0, 8, st) != cudaSuccess || cudaMemsetAsync(d_root_rep, 0, 4, st) != cudaSuccess ||
        cudaMemsetAsync(rows_ctr, 0, 4, st) != cudaSuccess)
        return fail(GFSM_ERR_CUDA);

    const uint64_t max_scan = std::min<uint64_t>(lim.max_scan_size, (uint64_t)kNoAllocTiles * TILE);
    GraphView gv{g.rowptr, g.adj, g.elab, g.order, g.single_label, g.n};
    unsigned long long total[MAXQ + 1] = {}, pos[MAXQ + 1] = {}, np[MAXQ + 1] = {};
    double ratio[MAXQ + 1];
    for (int i = 0; i <= MAXQ; ++i) ratio[i] = 1.0;
    total[0] = rc2[1];
    np[0] = 1;
    uint32_t d = 0;
    unsigned long long candidates = 0;
    for (;;) {
        if (pos[d] >= total[d]) {
            if (d == 0) break;
            --d;
            continue;
        }
        const bool emits = d < dmax;
        unsigned long long chunk = std::min<unsigned long long>(total[d] - pos[d], max_scan);
        if (emits) {
            const double allowed = (double)buf[d].cap / std::max(ratio[d], 1.0 / 8192.0);
            chunk = std::min<unsigned long long>(chunk, (unsigned long long)std::max<double>(allowed, TILE));
            chunk = std::min<unsigned long long>(chunk, kMaxEmitChunk);
        }
        const uint32_t ntiles = (uint32_t)div_up(chunk, TILE);
        StepArgs a{};
        a.g = gv;
        a.plans = d_plan;
        a.depth = d;
        if (d == 0) {
            a.pcstart = d_rcstart;
            a.pcoff = d_rcoff;
        } else {
            a.ptup = buf[d - 1].tup;
            a.pstride = buf[d - 1].cap;
            a.pcstart = buf[d - 1].cstart;
            a.pcoff = buf[d - 1].coff;
        }
        a.np = np[d];
        a.tile_parent = tile_parent;
        a.c0 = pos[d];
        a.cend = pos[d] + chunk;
        a.ntiles = ntiles;
        if (emits) {
            a.ctup = buf[d].tup;
            a.cstride = buf[d].cap;
            a.ccap = buf[d].cap;
            a.ccstart = buf[d].cstart;
            a.ccoff = buf[d].coff;
        }
        a.counts = d_count;
        a.result = d_result;
        a.rows_ctr = rows_ctr;
        a.root_rep = d_root_rep;
        // one query: a step either counts (last level) or emits, so a re-run
        // step never counts twice and the count goes straight to the total
        a.pcoff_end = total[d];
        k_partition<<<(unsigned)div_up((uint64_t)ntiles + 1, 256), 256, 0, st>>>(
            a.pcoff, a.np, a.pcoff_end, a.c0, chunk, ntiles, TILE, tile_parent, d_result, nullptr, 0);
        launch_step(0, d == 0, a, ntiles, st);
        if (cudaGetLastError() != cudaSuccess) return fail(GFSM_ERR_CUDA);
        StepResult r;
        if (cudaMemcpyAsync(&r, d_result, sizeof(r), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return fail(GFSM_ERR_CUDA);
        r.n_children = r.alloc >> kAllocShift;  // the step's totals are its allocator word
        r.total_next = r.alloc & kAllocMask;
        if (r.err) return GFSM_ERR_CUDA;
        if (emits && r.next_ovf && chunk <= TILE) return GFSM_ERR_TOO_LARGE;
        const bool retry = emits && (r.n_children > buf[d].cap || r.next_ovf);
        if (trace)
            fprintf(stderr, "gfsm-noalloc-step depth=%u cand=%llu children=%llu next=%llu tiles=%u retry=%d\n", d,
                    chunk, emits ? r.n_children : 0ull, emits ? r.total_next : 0ull, ntiles, retry ? 1 : 0);
        if (retry) {
            ratio[d] = std::max(ratio[d] * 4.0, 2.0 * (double)r.n_children / (double)chunk);
            continue;
        }
        // the candidate cap of the data graph's context, as gfsm_match_count applies it
        candidates += chunk;
        if (lim.max_candidates && candidates > lim.max_candidates) return GFSM_ERR_TOO_LARGE;
        pos[d] += chunk;
        if (emits) {
            ratio[d] = std::max(2.0 * (double)r.n_children / (double)chunk, ratio[d] * 0.5);
            if (r.n_children > 0 && r.total_next > 0) {
                np[d + 1] = r.n_children;
                total[d + 1] = r.total_next;
                pos[d + 1] = 0;
                ++d;
            }
        }
    }
    unsigned long long c = 0;
    if (cudaMemcpyAsync(&c, d_count, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(GFSM_ERR_CUDA);
    *count = c;
    return GFSM_OK;
}
