// ref_frontend.cu -- TEST INFRASTRUCTURE ONLY.
//
// A small driver, compiled together with the reference's own sources where
// they lie (HnHelper.cuh fileParse, ccsr.cpp genereateCCSRRequirements /
// getMaxValency, HnGPU.cu preProcessQuery), that dumps the reference's CCSR
// and query plan so the oracle's restatement can be compared bit for bit.
// No kernel is launched; only the reference's host code runs.
//
//   ref_frontend <graph.g> <out.bin> [plan]
//
// out.bin holds little-endian uint32 words:
//   count, size, segments[size], verticeLocs[count], invVerticeLocs[count],
//   staggerSize, staggers[staggerSize], staggerInfo[2*staggerSize],
//   and with "plan": maxValency, requirements[2*maxValency*count],
//   requirementHeader[3*count], mappingData[count] (after preProcessQuery).
#include "HnHelper.cuh"
#include "HnGPU.cuh"
#include <cstdio>
#include <cstdlib>
#include <cstring>

static void put(FILE* f, uint32_t v) { fwrite(&v, 4, 1, f); }
static void putn(FILE* f, const uint32_t* p, size_t n) { if (n) fwrite(p, 4, n, f); }

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <graph.g> <out.bin> [plan]\n", argv[0]);
        return 2;
    }
    CCSR::CCSRStagger st;
    CCSR::CCSRGraph g = fileParse(std::string(argv[1]), false, &st);
    FILE* f = fopen(argv[2], "wb");
    if (!f) return 3;
    put(f, g.count);
    put(f, g.size);
    putn(f, g.segments, g.size);
    putn(f, g.verticeLocs, g.count);
    putn(f, g.invVerticeLocs, g.count);
    put(f, st.size);
    putn(f, st.staggers, st.size);
    for (uint32_t i = 0; i < st.size; i++) {
        put(f, st.staggersInfo[i].offset);
        put(f, st.staggersInfo[i].normOffset);
    }
    if (argc > 3 && !strcmp(argv[3], "plan")) {
        fflush(f);  // the planner may exit(1); keep what was written
        uint32_t *reqs = nullptr, *header = nullptr;
        int32_t* mapping = nullptr;
        uint32_t maxv = HnSetup::preProcessQuery(g, &reqs, &header, &mapping);
        put(f, maxv);
        putn(f, reqs, 2ull * maxv * g.count);
        putn(f, header, 3ull * g.count);
        putn(f, reinterpret_cast<uint32_t*>(mapping), g.count);
    }
    fclose(f);
    return 0;
}
