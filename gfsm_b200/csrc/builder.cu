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
    if (g.rowptr) cudaFree(g.rowptr);
    if (g.adj) cudaFree(g.adj);
    if (g.elab) cudaFree(g.elab);
    if (g.order) cudaFree(g.order);
    g.rowptr = g.adj = g.order = nullptr;
    g.elab = nullptr;
}

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

    uint32_t *d_src = nullptr, *d_dst = nullptr, *d_deg = nullptr, *d_group = nullptr;
    uint32_t *d_inv = nullptr, *d_degs = nullptr, *d_val = nullptr, *d_order = nullptr, *d_flags = nullptr;
    unsigned long long *d_vkey = nullptr, *d_vkey2 = nullptr, *d_ekey = nullptr, *d_ekey2 = nullptr;
    uint8_t *d_lab = nullptr, *d_lab2 = nullptr;
    void *d_tmp = nullptr;
    size_t tmp_bytes = 0, need = 0;
    uint32_t h_flags[3] = {0, 0, 0};
    std::vector<uint32_t> group;  // per vertex, when grouping by label
    cudaStream_t st = nullptr;

    BCHECK(cudaSetDevice(device));
    BCHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (vl_mode) {
        std::vector<uint32_t> vals(h.vlabel.begin(), h.vlabel.end());
        std::sort(vals.begin(), vals.end());
        vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
        out.group_value = vals;
        group.resize(n);
        std::vector<uint32_t> cnt(vals.size() + 1, 0);
        for (uint32_t v = 0; v < n; ++v) {
            group[v] = (uint32_t)(std::lower_bound(vals.begin(), vals.end(), h.vlabel[v]) - vals.begin());
            cnt[group[v] + 1]++;
        }
        for (size_t i = 0; i < vals.size(); ++i) cnt[i + 1] += cnt[i];
        out.group_start = cnt;
    } else {
        out.group_value = {0};
        out.group_start = {0, n};
    }

    BCHECK(cudaMalloc(&d_src, std::max<uint64_t>(m, 1) * 4));
    BCHECK(cudaMalloc(&d_dst, std::max<uint64_t>(m, 1) * 4));
    BCHECK(cudaMalloc(&d_lab, std::max<uint64_t>(m, 1)));
    BCHECK(cudaMalloc(&d_lab2, std::max<uint64_t>(m, 1)));
    BCHECK(cudaMalloc(&d_deg, (uint64_t)std::max<uint32_t>(n, 1) * 4));
    BCHECK(cudaMalloc(&d_flags, 16));
    if (m) {
        BCHECK(cudaMemcpyAsync(d_src, h.src.data(), m * 4, cudaMemcpyHostToDevice, st));
        BCHECK(cudaMemcpyAsync(d_dst, h.dst.data(), m * 4, cudaMemcpyHostToDevice, st));
        BCHECK(cudaMemcpyAsync(d_lab, h.lab.data(), m, cudaMemcpyHostToDevice, st));
    }
    BCHECK(cudaMemsetAsync(d_deg, 0, (uint64_t)std::max<uint32_t>(n, 1) * 4, st));
    BCHECK(cudaMemsetAsync(d_flags, 0, 16, st));
    if (vl_mode && n) {
        BCHECK(cudaMalloc(&d_group, (uint64_t)n * 4));
        BCHECK(cudaMemcpyAsync(d_group, group.data(), (uint64_t)n * 4, cudaMemcpyHostToDevice, st));
    }
    if (m) k_degree<<<grid_for(m, 256), 256, 0, st>>>(d_src, m, d_deg);

    // 2. vertex order
    BCHECK(cudaMalloc(&d_vkey, (uint64_t)std::max<uint32_t>(n, 1) * 8));
    BCHECK(cudaMalloc(&d_vkey2, (uint64_t)std::max<uint32_t>(n, 1) * 8));
    BCHECK(cudaMalloc(&d_val, (uint64_t)std::max<uint32_t>(n, 1) * 4));
    BCHECK(cudaMalloc(&d_order, (uint64_t)std::max<uint32_t>(n, 1) * 4));
    BCHECK(cudaMalloc(&d_inv, (uint64_t)std::max<uint32_t>(n, 1) * 4));
    BCHECK(cudaMalloc(&d_degs, ((uint64_t)n + 1) * 4));
    BCHECK(cudaMalloc(&out.rowptr, ((uint64_t)n + 1) * 4));
    if (n) {
        int gbits = 0;
        while ((1ull << gbits) < out.group_value.size()) ++gbits;
        k_vertex_keys<<<grid_for(n, 256), 256, 0, st>>>(d_deg, d_group, n, d_vkey, d_val);
        BCHECK(cub::DeviceRadixSort::SortPairs(nullptr, need, d_vkey, d_vkey2, d_val, d_order, (int)n, 0,
                                               32 + gbits, st));
        tmp_bytes = need;
        BCHECK(cub::DeviceScan::ExclusiveSum(nullptr, need, d_degs, out.rowptr, (int)n + 1, st));
        tmp_bytes = std::max(tmp_bytes, need);
        BCHECK(cub::DeviceRadixSort::SortPairs(nullptr, need, d_ekey, d_ekey2, d_lab, d_lab2,
                                               (int64_t)std::max<uint64_t>(m, 1), 0, 2 * bits, st));
        tmp_bytes = std::max(tmp_bytes, need);
        BCHECK(cudaMalloc(&d_tmp, tmp_bytes));
        BCHECK(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_vkey, d_vkey2, d_val, d_order, (int)n, 0,
                                               32 + gbits, st));
        k_invert<<<grid_for(n, 256), 256, 0, st>>>(d_order, n, d_deg, d_inv, d_degs);
        BCHECK(cudaMemsetAsync(d_degs + n, 0, 4, st));
        // 3. row pointers
        BCHECK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_degs, out.rowptr, (int)n + 1, st));
    } else {
        BCHECK(cudaMemsetAsync(out.rowptr, 0, 4, st));
    }
    cudaFree(d_vkey); d_vkey = nullptr;
    cudaFree(d_vkey2); d_vkey2 = nullptr;
    cudaFree(d_val); d_val = nullptr;

    // 4. entries keyed (row(src), row(dst)), labels carried as values
    BCHECK(cudaMalloc(&out.adj, std::max<uint64_t>(m, 1) * 4));
    if (m) {
        BCHECK(cudaMalloc(&d_ekey, m * 8));
        BCHECK(cudaMalloc(&d_ekey2, m * 8));
        k_edge_keys<<<grid_for(m, 256), 256, 0, st>>>(d_src, d_dst, m, d_inv, bits, d_ekey);
        BCHECK(cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_ekey, d_ekey2, d_lab, d_lab2, (int64_t)m, 0,
                                               2 * bits, st));
        k_unpack<<<grid_for(m, 256), 256, 0, st>>>(d_ekey2, m, bits, out.adj, d_lab2, d_flags);
        k_symmetric<<<grid_for(m, 256), 256, 0, st>>>(d_ekey2, m, bits, out.rowptr, out.adj, d_flags);
    }
    BCHECK(cudaMemcpyAsync(h_flags, d_flags, 12, cudaMemcpyDeviceToHost, st));
    out.h_rowptr.resize((uint64_t)n + 1);
    out.h_order.resize(n);
    BCHECK(cudaMemcpyAsync(out.h_rowptr.data(), out.rowptr, ((uint64_t)n + 1) * 4, cudaMemcpyDeviceToHost, st));
    if (n) BCHECK(cudaMemcpyAsync(out.h_order.data(), d_order, (uint64_t)n * 4, cudaMemcpyDeviceToHost, st));
    BCHECK(cudaStreamSynchronize(st));
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
        d_lab2 = nullptr;
    } else {
        out.n_edge_labels = 1;
        out.single_label = h.lab[0];
    }
    out.order = d_order;
    d_order = nullptr;
    out.rows = 0;
    out.max_degree = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t d = out.h_rowptr[i + 1] - out.h_rowptr[i];
        if (d) out.rows++;
        out.max_degree = std::max(out.max_degree, d);
    }
    out.bytes = ((uint64_t)n + 1) * 4 + m * 4 + (out.elab ? m : 0) + (uint64_t)n * 4;

done:
    if (d_src) cudaFree(d_src);
    if (d_dst) cudaFree(d_dst);
    if (d_lab) cudaFree(d_lab);
    if (d_lab2) cudaFree(d_lab2);
    if (d_deg) cudaFree(d_deg);
    if (d_group) cudaFree(d_group);
    if (d_inv) cudaFree(d_inv);
    if (d_degs) cudaFree(d_degs);
    if (d_val) cudaFree(d_val);
    if (d_order) cudaFree(d_order);
    if (d_flags) cudaFree(d_flags);
    if (d_vkey) cudaFree(d_vkey);
    if (d_vkey2) cudaFree(d_vkey2);
    if (d_ekey) cudaFree(d_ekey);
    if (d_ekey2) cudaFree(d_ekey2);
    if (d_tmp) cudaFree(d_tmp);
    if (st) cudaStreamDestroy(st);
    if (rc != GFSM_OK) free_device_graph(out);
    return rc;
}

}  // namespace gfsm
