// cli.cpp -- the `GFSM <query> <data>` command (drop-in for main.cu:56-65).
//
// Prints the reference's CSV line (columns as in mainscripts/runLabel.sh:20:
// Query, Data, Preallocate, Query Parse, Data Parse, Kernel, Reallocate,
// ReKernel, Function Count, Solution Write, GPU Time, End to End) and exits
// with the reference's codes on failure (232/233/234 file errors, 1 for an
// unplannable query).  Knobs come from the Environment.h names as GFSM_*
// environment variables.  GFSM_OUTPUT=1 also writes the mappings to
// output.fs in the reference's binary layout (HnGPU.cu:1081-1091:
// u32 count, u32 width, u32[count*width]), columns = query vertex ids.
// GFSM_PLANNER=data plans the query for the data graph (data-aware matching
// order where the count cannot depend on the order); the default is the
// reference's order.
#include <cstring>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/gfsm.h"

namespace {

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

std::string base_name(const std::string &p) {
    size_t i = p.find_last_of('/');
    return i == std::string::npos ? p : p.substr(i + 1);
}

int fail(gfsm_ctx *ctx, gfsm_status rc) {
    fprintf(stderr, "GFSM: %s%s%s\n", gfsm_status_str(rc), ctx ? ": " : "", ctx ? gfsm_last_error(ctx) : "");
    fflush(stdout);
    return rc > 255 ? 255 : (int)rc;
}

int run(const std::string &qpath, const std::string &dpath) {
    printf("\n%s,%s,", base_name(qpath).c_str(), base_name(dpath).c_str());
    auto t0 = Clock::now();
    gfsm_ctx *ctx = nullptr;
    gfsm_status rc = gfsm_init(&ctx, nullptr, 0);
    if (rc != GFSM_OK) return fail(nullptr, rc);
    auto t1 = Clock::now();
    printf("%fs,", secs(t0, t1));  // Preallocate
    auto start = Clock::now();

    gfsm_graph *q = nullptr, *d = nullptr;
    auto a = Clock::now();
    rc = gfsm_graph_load_text(ctx, qpath.c_str(), &q);
    if (rc != GFSM_OK) return fail(ctx, rc);
    printf("%fs,", secs(a, Clock::now()));  // Query Parse
    a = Clock::now();
    rc = gfsm_graph_load_text(ctx, dpath.c_str(), &d);
    if (rc == GFSM_OK) rc = gfsm_graph_to_device(ctx, d);
    if (rc != GFSM_OK) return fail(ctx, rc);
    printf("%fs,", secs(a, Clock::now()));  // Data Parse (text + device CCSR)

    auto solve0 = Clock::now();
    gfsm_plan *plan = nullptr;
    const char *planner = getenv("GFSM_PLANNER");
    rc = planner && !strcmp(planner, "data") ? gfsm_query_prepare_for(ctx, q, d, &plan)
                                             : gfsm_query_prepare(ctx, q, &plan);
    if (rc != GFSM_OK) return fail(ctx, rc);
    uint64_t count = 0;
    gfsm_stats st{};
    a = Clock::now();
    const char *out = getenv("GFSM_OUTPUT");
    const bool write_out = out && *out && *out != '0';
    std::vector<uint32_t> rows;
    uint32_t k = 0;
    gfsm_plan_tables(plan, &k, nullptr, nullptr, nullptr, nullptr);
    if (write_out) {
        rc = gfsm_match_count(ctx, plan, d, &count, &st);
        if (rc == GFSM_OK) {
            rows.resize(count * k);
            uint64_t nr = 0;
            rc = gfsm_match_mappings(ctx, plan, d, rows.data(), count, &nr, &count, &st);
        }
    } else {
        rc = gfsm_match_count(ctx, plan, d, &count, &st);
    }
    if (rc != GFSM_OK) return fail(ctx, rc);
    printf("%fs,", secs(a, Clock::now()));  // Kernel
    printf("n/a,n/a,");                        // Reallocate, ReKernel: chunking never restarts
    printf("%llu,", (unsigned long long)count);  // Function Count
    a = Clock::now();
    if (write_out) {
        FILE *f = fopen("output.fs", "wb");
        if (f) {
            uint32_t c32 = (uint32_t)count;
            fwrite(&c32, 4, 1, f);
            fwrite(&k, 4, 1, f);
            if (!rows.empty()) fwrite(rows.data(), 4, rows.size(), f);
            fclose(f);
        }
    }
    printf("%fs,", secs(a, Clock::now()));          // Solution Write
    printf("%fs,", secs(solve0, Clock::now()));     // GPU Time
    printf("%fs,", secs(start, Clock::now()));      // End to End
    fflush(stdout);
    gfsm_plan_destroy(plan);
    gfsm_graph_destroy(q);
    gfsm_graph_destroy(d);
    gfsm_destroy(ctx);
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc == 3) return run(argv[1], argv[2]);
    return run("query/_5_road5.g", "data/roadNet-PA.g");  // main.cu:49-54
}
