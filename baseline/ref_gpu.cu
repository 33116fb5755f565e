// ref_gpu.cu -- the reference GFSM build's FFS, run on sm_100a for comparison.
//
// NOT PART OF THE PRODUCT.  Built by baseline/Makefile into baseline/_ref/
// (git-ignored) from the reference's own sources where they lie: its parser
// (HnHelper.cuh fileParse), planner (ccsr.cpp, HnGPU.cu preProcessQuery) and
// level-step kernels hnInit / hnGen / hnCheck / hnRemove with updateHeader
// (HnGPU.cu:76-334), compiled unchanged.  What the reference cannot run on
// sm_100a is its level driver: hnSolve / hnLoop / hnScan (HnGPU.cu:336-669)
// launch kernels, synchronise and call CUB from device code (CDP1, absent on
// sm_90+).  This file restates that driver on the host, step for step, with
// host-side cub::DeviceScan::ExclusiveSum and the same kernel arguments:
//
//   hnSolve root (HnGPU.cu:474-513): hnInit per row length, scan, hnRemove,
//     updateHeader, scan of the degrees;
//   per depth (HnGPU.cu:518-667, the non-batching branch): the frontier
//     prediction predFuncCount and its SOLN_LIMIT test, then hnLoop
//     (HnGPU.cu:371-439): hnGen, updateHeader, hnCheck, scan, hnRemove,
//     updateHeader, scan of the degrees; stop at an empty frontier.
//
// Inputs outside the reference's valid domain are not run: the host tests,
// before every launch, the same bounds the reference's buffers imply (the
// forest and the candidate level below SOLN_LIMIT / SCAN_LIMIT), and a query
// whose frontier would need the reference's batching path (HnGPU.cu:529-627)
// is reported as "overflow" instead.  The reference's device-side checks that
// end in __trap() (GPUDEBUG / PREDICTCHECK / OVERFLOWCHECK, Environment.h:17-20)
// are compiled out; the host checks above keep every index in bounds.
//
//   ref_gpu <data.g> <out.jsonl> <query.g>...
//
// The data graph is parsed and copied to the device once; each query is then
// parsed, planned, its tables copied in, and its FFS run.  Per query one JSON
// line: count (the reference's "Function Count", HnGPU.cu:999-1000), status,
// kernel_ms (CUDA events around the level loop: the reference's "Kernel
// Time", HnGPU.cu:951) and gpu_ms (planning + table copies + level loop +
// count read: the reference's "GPU Time", HnGPU.cu:736, without its per-query
// cudaMalloc/copy/cudaFree of the data graph and without hnWrite).
#include "Environment.h"
#undef GPUDEBUG
#undef PREDICTCHECK
#undef OVERFLOWCHECK
#include "HnHelper.cuh"
#include "hngpu_kernels.inc"
#include "hngpu_plan.inc"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

__global__ void k_update_header(uint32_t *h) { HnGPU::updateHeader(h); }

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "ref_gpu: %s: %s\n", #x, cudaGetErrorString(e_));                 \
            exit(3);                                                                           \
        }                                                                                      \
    } while (0)

struct Buffers {
    HnFunction *front = nullptr, *back = nullptr;
    uint32_t *functCounts = nullptr, *functionDegrees = nullptr, *bBfrFunctionDegrees = nullptr,
             *scanBfr = nullptr, *header = nullptr;
    void *cubTemp = nullptr;
    size_t cubBytes = 0;
    uint32_t *reqs = nullptr, *reqHeader = nullptr;
    size_t soln = 0, scan = 0;
};

// HnSetup::preinit (HnGPU.cu:847-862), once.
void preinit(Buffers &b, size_t soln, size_t scan) {
    b.soln = soln;
    b.scan = scan;
    CK(cudaMalloc(&b.front, sizeof(HnFunction) * soln));
    CK(cudaMalloc(&b.back, sizeof(HnFunction) * soln));
    CK(cudaMalloc(&b.functCounts, sizeof(uint32_t) * scan));
    CK(cudaMalloc(&b.functionDegrees, sizeof(uint32_t) * scan));
    CK(cudaMalloc(&b.bBfrFunctionDegrees, sizeof(uint32_t) * scan));
    CK(cudaMalloc(&b.scanBfr, sizeof(uint32_t) * scan));
    CK(cudaMalloc(&b.header, sizeof(uint32_t) * 8));
    CK(cub::DeviceScan::ExclusiveSum(nullptr, b.cubBytes, b.functCounts, b.scanBfr, (int)scan));
    CK(cudaMalloc(&b.cubTemp, b.cubBytes));
    CK(cudaMalloc(&b.reqs, sizeof(uint32_t) * 4096));
    CK(cudaMalloc(&b.reqHeader, sizeof(uint32_t) * 1024));
}

uint32_t read_word(const uint32_t *p) {
    uint32_t v = 0;
    CK(cudaMemcpy(&v, p, 4, cudaMemcpyDeviceToHost));
    return v;
}

void scan(Buffers &b, const uint32_t *in, uint32_t n) {
    CK(cub::DeviceScan::ExclusiveSum(b.cubTemp, b.cubBytes, in, b.scanBfr, (int)n));
}

enum Status { OK, OVERFLOW, TOO_LARGE };

// hnSolve + hnLoop on the host.  Returns the final count in *count.
Status solve(Buffers &b, CCSRSegment *data, const CCSR::CCSRStagger &ds, uint32_t maxValencyData,
             const CCSR::CCSRGraph &q, const std::vector<uint32_t> &rh, uint32_t *count) {
    using namespace HnGPU;
    const uint32_t depthTarget = q.count - 1;
    CK(cudaMemset(b.header, 0, sizeof(uint32_t) * 8));
    // root candidates: one hnInit launch per CCSR row length (HnGPU.cu:474-495)
    uint32_t graphOffset = 0, solutionOffset = 0, roots = 0;
    for (int spacing = (int)ds.size + 1; spacing > 1; spacing--) {
        const uint32_t stagger = ds.staggers[spacing - 2];
        const uint32_t genFuncs = stagger / spacing;
        if ((uint64_t)solutionOffset + genFuncs > b.scan || (uint64_t)solutionOffset + genFuncs > b.soln)
            return TOO_LARGE;
        if (genFuncs)
            hnInit<<<getBlockCount(genFuncs, HBLOCKSIZE), HBLOCKSIZE>>>(
                data, b.back, b.bBfrFunctionDegrees, b.header, b.functCounts, spacing, solutionOffset, graphOffset,
                b.reqs, rh[HNREQS_H_NUM], genFuncs);
        solutionOffset += genFuncs;
        if (stagger) graphOffset += stagger;
        roots += genFuncs;
    }
    CK(cudaMemcpy(b.header + HNFUNC_COUNT, &roots, 4, cudaMemcpyHostToDevice));
    CK(cudaGetLastError());
    if (roots == 0) {
        *count = 0;
        return OK;
    }
    scan(b, b.functCounts, roots);
    hnRemove<<<getBlockCount(roots, HBLOCKSIZE), HBLOCKSIZE>>>(b.front, b.back, b.functionDegrees,
                                                              b.bBfrFunctionDegrees, b.header, b.scanBfr, 0);
    k_update_header<<<1, 1>>>(b.header);
    uint32_t cnt = read_word(b.header + HNFUNC_COUNT);
    if (cnt) scan(b, b.functionDegrees, cnt);
    for (uint32_t depth = 0; depth < depthTarget && cnt; depth++) {
        // frontier prediction and its limit (HnGPU.cu:518-527)
        const uint32_t off = read_word(b.header + HNFUNC_OFFSET);
        const uint64_t pred =
            (uint64_t)read_word(b.scanBfr + cnt - 1) + (uint64_t)read_word(b.functionDegrees + cnt - 1);
        // (hnGen writes a parent's whole row from its predicted offset: one
        // row of margin keeps even a misprediction inside the buffer)
        if (pred + cnt + off + maxValencyData >= b.soln || pred > b.scan) return OVERFLOW;  // its batching path
        // hnLoop (HnGPU.cu:371-439)
        const uint32_t reqIndex = (depth + 1) * 3;
        const uint32_t nextReqIndex = reqIndex + (depth != depthTarget) * 3;
        hnGen<<<getBlockCount(cnt, HBLOCKSIZE), HBLOCKSIZE>>>(data, b.front, b.back, b.functionDegrees, b.scanBfr,
                                                             b.header, b.functCounts, maxValencyData,
                                                             rh[HNREQS_H_FIRSTQVERTEX + reqIndex], 0);
        k_update_header<<<1, 1>>>(b.header);
        const uint32_t cand = read_word(b.header + HNFUNC_COUNT);
        if (cand != pred) return TOO_LARGE;  // cannot happen on valid data; stop rather than run past it
        if (cand == 0) {
            cnt = 0;
            break;
        }
        hnCheck<<<getBlockCount(cand, HBLOCKSIZE), HBLOCKSIZE>>>(
            data, b.front, b.back, b.bBfrFunctionDegrees, b.header, b.functCounts, b.scanBfr, b.reqs,
            rh[HNREQS_H_NUM + reqIndex], rh[HNREQS_H_INDEX + reqIndex], depth, rh[HNREQS_H_FIRSTQVERTEX + nextReqIndex]);
        scan(b, b.functCounts, cand);
        hnRemove<<<getBlockCount(cand, HBLOCKSIZE), HBLOCKSIZE>>>(b.front, b.back, b.functionDegrees,
                                                                 b.bBfrFunctionDegrees, b.header, b.scanBfr, 0);
        k_update_header<<<1, 1>>>(b.header);
        cnt = read_word(b.header + HNFUNC_COUNT);
        if (cnt) scan(b, b.functionDegrees, cnt);
        CK(cudaGetLastError());
    }
    *count = cnt;
    return OK;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <data.g> <out.jsonl> <query.g>...\n", argv[0]);
        return 2;
    }
    CK(cudaFree(nullptr));
    Buffers b;
    preinit(b, MAXSOLNSIZE, MAXSCANSIZE);
    auto t0 = std::chrono::steady_clock::now();
    CCSR::CCSRStagger dst;
    CCSR::CCSRGraph dg = fileParse(std::string(argv[1]), false, &dst);
    const double parse_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if ((uint64_t)dg.size >= (1ull << CCSRVertSize)) {
        fprintf(stderr, "ref_gpu: data CCSR of %u words exceeds the %d-bit offset field\n", dg.size, CCSRVertSize);
        return 4;
    }
    const uint32_t maxValencyData = CCSR::getMaxValency(dg);
    CCSRSegment *data = nullptr;
    CK(cudaMalloc(&data, sizeof(CCSRSegment) * dg.size));
    CK(cudaMemcpy(data, dg.segments, sizeof(CCSRSegment) * dg.size, cudaMemcpyHostToDevice));
    FILE *out = fopen(argv[2], "w");
    if (!out) return 3;
    fprintf(out, "{\"data\": \"%s\", \"parse_s\": %.6f, \"ccsr_words\": %u, \"vertices\": %u}\n", argv[1], parse_s,
            dg.size, dg.count);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int i = 3; i < argc; i++) {
        CCSR::CCSRStagger qst;
        CCSR::CCSRGraph q = fileParse(std::string(argv[i]), false, &qst);
        auto g0 = std::chrono::steady_clock::now();
        uint32_t *reqs = nullptr, *header = nullptr;
        int32_t *mapping = nullptr;
        const uint32_t maxValencyQuery = HnSetup::preProcessQuery(q, &reqs, &header, &mapping);
        const size_t nreq = 2ull * maxValencyQuery * q.count, nh = 3ull * q.count;
        // the level after the last reads one requirement-header row past the
        // table (HnGPU.cu:380, depth == depthTarget - 1): padded with zeros
        std::vector<uint32_t> rh(nh + 3, 0u);
        for (size_t j = 0; j < nh; j++) rh[j] = header[j];
        if (nreq > 4096 || nh + 3 > 1024) {
            fprintf(out, "{\"query\": \"%s\", \"k\": %u, \"status\": \"too_large\"}\n", argv[i], q.count);
            continue;
        }
        CK(cudaMemcpy(b.reqs, reqs, sizeof(uint32_t) * nreq, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(b.reqHeader, rh.data(), sizeof(uint32_t) * rh.size(), cudaMemcpyHostToDevice));
        uint32_t count = 0;
        CK(cudaEventRecord(e0));
        const Status st = solve(b, data, dst, maxValencyData, q, rh, &count);
        CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1));
        const double gpu_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - g0).count();
        float kms = 0.f;
        CK(cudaEventElapsedTime(&kms, e0, e1));
        if (st == OK)
            fprintf(out, "{\"query\": \"%s\", \"k\": %u, \"status\": \"ok\", \"count\": %u, \"kernel_ms\": %.4f, "
                         "\"gpu_ms\": %.4f}\n", argv[i], q.count, count, kms, gpu_ms);
        else
            fprintf(out, "{\"query\": \"%s\", \"k\": %u, \"status\": \"%s\"}\n", argv[i], q.count,
                    st == OVERFLOW ? "overflow" : "too_large");
        fflush(out);
        free(reqs);
        free(header);
        free(mapping);
    }
    fclose(out);
    return 0;
}
