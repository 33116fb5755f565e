// builder.cu -- device CCSR builder.
//
// Replaces the reference's serial host builder (HnHelper.cuh:383-478:
// Dynamic2D rows, std::sort of (degree, id), per-row std::sort, remap of
// targets to row offsets) with device passes over the edge list:
//   1. degree histogram (atomics);
//   2. vertex order = sort of (label group, degree descending, id ascending)
//      -- the reference's row order, grouped by vertex label when labels are
//      matched so that every label is one contiguous id range;
//   3. row pointers = exclusive scan of the degrees in that order;
//   4. entries bucketed by (source row, target row, edge label) with one
//      64-bit key sort -- rows come out contiguous and sorted by target,
//      which is the reference's per-row order;
//   5. flags: symmetric structure, duplicate (u,v) entries, label count.
// Targets are stored as row indices (not packed row offsets), so the 24-bit
// CCSRVertSize limit of the packed format does not apply.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cstdio>

#include "gfsm_internal.h"

namespace gfsm {

namespace {

#define BCHECK(x)                                                                 \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            err = std::string(#x) + ": " + cudaGetErrorString(e_);                \
            rc = (e_ == cudaErrorMemoryAllocation) ? GFSM_ERR_NOMEM : GFSM_ERR_CUDA; \
            goto done;                                                            \
        }                                                                         \
    } while (0)

__global__ void k_degree(const uint32_t *src, uint64_t m, uint32_t *deg) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&deg[src[i]], 1u);
}

// key = group << 32 | (~degree); value = vertex id (ascending input ->
// the stable radix sort keeps ids ascending inside equal keys).
__global__ void k_vertex_keys(const uint32_t *deg, const uint32_t *group, uint32_t n,
                              unsigned long long *key, uint32_t *val) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        unsigned long long g = group ? group[v] : 0u;
        key[v] = (g << 32) | (unsigned long long)(0xffffffffu - deg[v]);
        val[v] = v;
    }
}

__global__ void k_invert(const uint32_t *order, uint32_t n, const uint32_t *deg, uint32_t *inv,
                         uint32_t *deg_sorted) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t v = order[i];
        inv[v] = i;
        deg_sorted[i] = deg[v];
    }
}

__global__ void k_edge_keys(const uint32_t *src, const uint32_t *dst, uint64_t m, const uint32_t *inv,
                            uint32_t bits, unsigned long long *key) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x)
        key[i] = ((unsigned long long)inv[src[i]] << bits) | inv[dst[i]];
}

__global__ void k_unpack(const unsigned long long *key, uint64_t m, uint32_t bits, uint32_t *adj,
                         const uint8_t *lab, uint32_t *flags) {
    const unsigned long long mask = (1ull << bits) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long k = key[i];
        adj[i] = (uint32_t)(k & mask);
        if (i > 0 && key[i - 1] == k) atomicOr(&flags[0], 1u);      // duplicate (u,v)
        if (i > 0 && lab[i] != lab[0]) atomicOr(&flags[1], 1u);     // more than one label
    }
}

// Symmetric structure check: for entry u->v, v's row must contain u.
__global__ void k_symmetric(const unsigned long long *key, uint64_t m, uint32_t bits,
                            const uint32_t *rowptr, const uint32_t *adj, uint32_t *flags) {
    const unsigned long long mask = (1ull << bits) - 1ull;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        unsigned long long k = key[i];
        uint32_t u = (uint32_t)(k >> bits), v = (uint32_t)(k & mask);
        uint32_t lo = rowptr[v], hi = rowptr[v + 1];
        while (lo < hi) {
            uint32_t mid = lo + ((hi - lo) >> 1);
            if (adj[mid] < u) lo = mid + 1; else hi = mid;
        }
        if (lo >= rowptr[v + 1] || adj[lo] != u) atomicOr(&flags[2], 1u);
    }
}

inline unsigned grid_for(uint64_t n, unsigned threads) {
    uint64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 32));
}

}  // namespace

void free_device_graph(DeviceGraph &g) {
    if (g.block) cudaFree(g.block);
    g.block = nullptr;
    g.rowptr = g.adj = g.order = nullptr;
    g.elab = nullptr;
}

// Host side of the build.  The outputs (rowptr, adj, order, elab) live in one
// persistent allocation; every temporary (edge copies, keys, degrees, CUB
// scratch) is carved from one stream-ordered workspace allocation released
// with cudaFreeAsync, so the build holds no device-wide synchronisation
// besides its final stream sync.  Events split the build into allocation,
// host-to-device copies, device passes and the copies back.
gfsm_status build_device_graph(const HostGraph &h, int device, bool vl_mode, DeviceGraph &out,
                               std::string &err) {
    gfsm_status rc = GFSM_OK;
    const uint32_t n = h.n;
    const uint64_t m = h.src.size();
    out = DeviceGraph();
    out.device = device;
    out.n = n;
    out.m = m;
    out.vl_grouped = vl_mode;
    if (m >= (1ull << 32) || n >= 0xffffffffu) return GFSM_ERR_TOO_LARGE;

    uint32_t bits = 1;
    while ((1ull << bits) < (uint64_t)std::max<uint32_t>(n, 2)) ++bits;
    const uint64_t n1 = std::max<uint32_t>(n, 1), m1 = std::max<uint64_t>(m, 1);
    auto al = [](uint64_t b) { return (b + 255) & ~255ull; };

    char *ws = nullptr;
    uint32_t h_flags[3] = {0, 0, 0};
    std::vector<uint32_t> group;  // per vertex, when grouping by label
    cudaStream_t st = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    uint32_t *d_src, *d_dst, *d_deg, *d_group, *d_inv, *d_degs, *d_val, *d_flags;
    unsigned long long *d_vkey, *d_vkey2, *d_ekey, *d_ekey2;
    uint8_t *d_lab, *d_lab2;
    void *d_tmp;
    size_t tmp_bytes = 0, need = 0;
    int gbits = 0;
    auto t_host0 = std::chrono::steady_clock::now();

    BCHECK(cudaSetDevice(device));
    BCHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (cudaEvent_t &e : ev) BCHECK(cudaEventCreate(&e));
    if (vl_mode) {
        // label value -> group (labels ascending): a table over the value
        // range when it is small (the usual case), else a sort of the values
        uint32_t mx = 0;
        for (uint32_t v = 0; v < n; ++v) mx = std::max(mx, h.vlabel[v]);
        std::vector<uint32_t> vals;
        group.resize(n);
        if (mx < (1u << 22)) {
            std::vector<uint32_t> idx((size_t)mx + 1, 0);
            for (uint32_t v = 0; v < n; ++v) idx[h.vlabel[v]] = 1;
            for (uint32_t x = 0; x <= mx; ++x)
                if (idx[x]) {
                    idx[x] = (uint32_t)vals.size();
                    vals.push_back(x);
                }
            for (uint32_t v = 0; v < n; ++v) group[v] = idx[h.vlabel[v]];
        } else {
            vals.assign(h.vlabel.begin(), h.vlabel.end());
            std::sort(vals.begin(), vals.end());
            vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
            for (uint32_t v = 0; v < n; ++v)
                group[v] = (uint32_t)(std::lower_bound(vals.begin(), vals.end(), h.vlabel[v]) - vals.begin());
        }
        std::vector<uint32_t> cnt(vals.size() + 1, 0);
        for (uint32_t v = 0; v < n; ++v) cnt[group[v] + 1]++;
        for (size_t i = 0; i < vals.size(); ++i) cnt[i + 1] += cnt[i];
        out.group_value = vals;
        out.group_start = cnt;
    } else {
        out.group_value = {0};
        out.group_start = {0, n};
    }
    while ((1ull << gbits) < out.group_value.size()) ++gbits;

    // scratch sizes of the CUB passes (queried with null pointers)
    BCHECK(cub::DeviceRadixSort::SortPairs(nullptr, need, (unsigned long long *)nullptr,
                                           (unsigned long long *)nullptr, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                           (int)n1, 0, 32 + gbits, st));
    tmp_bytes = need;
    BCHECK(cub::DeviceScan::ExclusiveSum(nullptr, need, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n1 + 1, st));
    tmp_bytes = std::max(tmp_bytes, need);
    BCHECK(cub::DeviceRadixSort::SortPairs(nullptr, need, (unsigned long long *)nullptr,
                                           (unsigned long long *)nullptr, (uint8_t *)nullptr, (uint8_t *)nullptr,
                                           (int64_t)m1, 0, 2 * bits, st));
    tmp_bytes = std::max(tmp_bytes, need);

    BCHECK(cudaEventRecord(ev[0], st));
    {
        // persistent outputs: rowptr | adj | order | elab
        const uint64_t o_rowptr = 0, o_adj = al((n1 + 1) * 4), o_order = o_adj + al(m1 * 4),
                       o_elab = o_order + al(n1 * 4), o_end = o_elab + al(m1);
        BCHECK(cudaMalloc(&out.block, o_end));
        char *b = static_cast<char *>(out.block);
        out.rowptr = reinterpret_cast<uint32_t *>(b + o_rowptr);
        out.adj = reinterpret_cast<uint32_t *>(b + o_adj);
        out.order = reinterpret_cast<uint32_t *>(b + o_order);
        d_lab2 = reinterpret_cast<uint8_t *>(b + o_elab);  // becomes out.elab when labels differ
        // workspace
        const uint64_t sizes[] = {m1 * 4, m1 * 4, m1, n1 * 4, n1 * 4, n1 * 4, (n1 + 1) * 4, n1 * 4, 64,
                                  n1 * 8, n1 * 8, m1 * 8, m1 * 8, tmp_bytes};
        uint64_t total = 0;
        for (uint64_t x : sizes) total += al(x);
        // the device's default pool keeps up to 4 GiB of freed workspace
        // reserved for this process (the pool releases everything at each
        // synchronisation otherwise), so a second build does not map its
        // workspace again: builds of the same graph measured 28 ms to 0.9 s
        // with the mapping redone every time
        {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
                uint64_t keep = 4ull << 30, cur = 0;
                if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur) == cudaSuccess &&
                    cur < keep)
                    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
        }
        BCHECK(cudaMallocAsync(reinterpret_cast<void **>(&ws), total, st));
        char *w = ws;
        auto take = [&](uint64_t bytes) {
            char *r = w;
            w += al(bytes);
            return r;
        };
        d_src = reinterpret_cast<uint32_t *>(take(sizes[0]));
        d_dst = reinterpret_cast<uint32_t *>(take(sizes[1]));
        d_lab = reinterpret_cast<uint8_t *>(take(sizes[2]));
        d_deg = reinterpret_cast<uint32_t *>(take(sizes[3]));
        d_group = reinterpret_cast<uint32_t *>(take(sizes[4]));
        d_inv = reinterpret_cast<uint32_t *>(take(sizes[5]));
        d_degs = reinterpret_cast<uint32_t *>(take(sizes[6]));
        d_val = reinterpret_cast<uint32_t *>(take(sizes[7]));
        d_flags = reinterpret_cast<uint32_t *>(take(sizes[8]));
        d_vkey = reinterpret_cast<unsigned long long *>(take(sizes[9]));
        d_vkey2 = reinterpret_cast<unsigned long long *>(take(sizes[10]));
        d_ekey = reinterpret_cast<unsigned long long *>(take(sizes[11]));
        d_ekey2 = reinterpret_cast<unsigned long long *>(take(sizes[12]));
        d_tmp = take(sizes[13]);
    }
    BCHECK(cudaEventRecord(ev[1], st));

    // 1. edges in, degree histogram
    if (m) {
        BCHECK(cudaMemcpyAsync(d_src, h.src.data(), m * 4, cudaMemcpyHostToDevice, st));
        BCHECK(cudaMemcpyAsync(d_dst, h.dst.data(), m * 4, cudaMemcpyHostToDevice, st));
        BCHECK(cudaMemcpyAsync(d_lab, h.lab.data(), m, cudaMemcpyHostToDevice, st));
    }
    if (vl_mode && n) BCHECK(cudaMemcpyAsync(d_group, group.data(), (uint64_t)n * 4, cudaMemcpyHostToDevice, st));
    BCHECK(cudaEventRecord(ev[2], st));
    BCHECK(cudaMemsetAsync(d_deg, 0, n1 * 4, st));
    BCHECK(cudaMemsetAsync(d_flags, 0, 16, st));
    if (m) k_degree<<<grid_for(m, 256), 256, 0, st>>>(d_src, m, d_deg);

    // 2. vertex order, 3. row pointers
    if (n) {
        k_vertex_keys<<<grid_for(n, 256), 256, 0, st>>>(d_deg, vl_mode ? d_group : nullptr, n, d_vkey, d_val);
        BCHECK(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_vkey, d_vkey2, d_val, out.order, (int)n, 0,
                                               32 + gbits, st));
        k_invert<<<grid_for(n, 256), 256, 0, st>>>(out.order, n, d_deg, d_inv, d_degs);
        BCHECK(cudaMemsetAsync(d_degs + n, 0, 4, st));
        BCHECK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_degs, out.rowptr, (int)n + 1, st));
    } else {
        BCHECK(cudaMemsetAsync(out.rowptr, 0, 4, st));
    }

    // 4. entries keyed (row(src), row(dst)), labels carried as values
    if (m) {
        k_edge_keys<<<grid_for(m, 256), 256, 0, st>>>(d_src, d_dst, m, d_inv, bits, d_ekey);
        BCHECK(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_ekey, d_ekey2, d_lab, d_lab2, (int64_t)m, 0,
                                               2 * bits, st));
        k_unpack<<<grid_for(m, 256), 256, 0, st>>>(d_ekey2, m, bits, out.adj, d_lab2, d_flags);
        k_symmetric<<<grid_for(m, 256), 256, 0, st>>>(d_ekey2, m, bits, out.rowptr, out.adj, d_flags);
    }
    BCHECK(cudaGetLastError());
    BCHECK(cudaEventRecord(ev[3], st));
    BCHECK(cudaMemcpyAsync(h_flags, d_flags, 12, cudaMemcpyDeviceToHost, st));
    out.h_rowptr.resize((uint64_t)n + 1);
    out.h_order.resize(n);
    BCHECK(cudaMemcpyAsync(out.h_rowptr.data(), out.rowptr, ((uint64_t)n + 1) * 4, cudaMemcpyDeviceToHost, st));
    if (n) BCHECK(cudaMemcpyAsync(out.h_order.data(), out.order, (uint64_t)n * 4, cudaMemcpyDeviceToHost, st));
    BCHECK(cudaEventRecord(ev[4], st));
    BCHECK(cudaFreeAsync(ws, st));
    ws = nullptr;
    BCHECK(cudaStreamSynchronize(st));
    {
        float a = 0.f, b = 0.f, c = 0.f, d = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        cudaEventElapsedTime(&c, ev[2], ev[3]);
        cudaEventElapsedTime(&d, ev[3], ev[4]);
        out.build_ms[0] = a;
        out.build_ms[1] = b;
        out.build_ms[2] = c;
        out.build_ms[3] = d;
    }
    out.multi = h_flags[0] != 0;
    out.symmetric = m == 0 || h_flags[2] == 0;
    if (m == 0) {
        out.n_edge_labels = 0;
        out.single_label = 0;
    } else if (h_flags[1]) {
        std::vector<uint8_t> seen(256, 0);
        for (uint8_t l : h.lab) seen[l] = 1;
        out.n_edge_labels = 0;
        for (int i = 0; i < 256; ++i) out.n_edge_labels += seen[i];
        out.elab = d_lab2;
    } else {
        out.n_edge_labels = 1;
        out.single_label = h.lab[0];
    }
    out.rows = 0;
    out.max_degree = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t d = out.h_rowptr[i + 1] - out.h_rowptr[i];
        if (d) out.rows++;
        out.max_degree = std::max(out.max_degree, d);
    }
    {
        // the degree window of every (label group, degree bound < 17): a
        // query vertex's degree bound is below its query's size (at most 16)
        const uint32_t ng = (uint32_t)out.group_value.size(), K = DeviceGraph::kCutDeltas;
        out.deg_cut.assign((size_t)ng * K, 0);
        for (uint32_t gi = 0; gi < ng; ++gi) {
            const uint32_t glo = out.group_start[gi], ghi = out.group_start[gi + 1];
            out.deg_cut[(size_t)gi * K] = ghi;  // delta 0: the whole group
            for (uint32_t delta = 1; delta < K; ++delta) {
                uint32_t a = glo, b = ghi;  // ids are degree-descending inside the group
                while (a < b) {
                    const uint32_t mid = a + (b - a) / 2;
                    if (out.h_rowptr[mid + 1] - out.h_rowptr[mid] >= delta) a = mid + 1; else b = mid;
                }
                out.deg_cut[(size_t)gi * K + delta] = a;
            }
        }
    }
    out.bytes = ((uint64_t)n + 1) * 4 + m * 4 + (out.elab ? m : 0) + (uint64_t)n * 4;
    out.build_wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_host0).count();

done:
    if (ws) {
        cudaFreeAsync(ws, st);
        cudaStreamSynchronize(st);
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
    if (rc != GFSM_OK) free_device_graph(out);
    return rc;
}

}  // namespace gfsm
