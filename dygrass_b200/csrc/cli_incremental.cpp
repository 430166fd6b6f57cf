// incremental_update -- drop-in for the reference's incremental updater CLI
// (random_walk_incremental/main.cu:240-362).
//
//   incremental_update <graph_name> <distortion_threshold> <#walkers> [--key=value ...]
//
// Reads ../dataset/<g>/adj_sparse.mtx (ids as written, weighted) and
// ../dataset/<g>/ext.mtx (1-based, weighted), tests the insertions in
// batches of ceil(N/10) on the device, and writes
// ../dataset/<g>/updated_adj_sparse.mtx: the original lines, then the added
// edges in input order, 1-based (gpu_graph.cuh:427-454).
// Options: --dataset-dir=DIR (default ../dataset), --max-steps=N (100),
// --seed=S, --batch=B (0 = ceil(N/10)), --transition=uniform|weighted.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "dyg.h"
#include "dyg_io.h"

static int fail(const char *what, dyg_status s) {
    fprintf(stderr, "%s failed (status %d): %s\n", what, (int)s, dyg_last_error_string());
    return 1;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        printf("Input: ./incremental_update <1.graph name> <2.distortion_threshold> <3.# of walkers>\n");
        return 0;
    }
    std::string dir = "../dataset";
    dyg_walk_params p;
    dyg_walk_params_default(&p);
    p.threshold = (float)atof(argv[2]);
    p.walkers = (uint32_t)atoi(argv[3]);
    uint32_t batch = 0;
    for (int i = 4; i < argc; ++i) {
        const char *a = argv[i];
        if (!strncmp(a, "--dataset-dir=", 14)) dir = a + 14;
        else if (!strncmp(a, "--max-steps=", 12)) p.max_steps = (uint32_t)atoi(a + 12);
        else if (!strncmp(a, "--seed=", 7)) p.seed = strtoull(a + 7, nullptr, 10);
        else if (!strncmp(a, "--batch=", 8)) batch = (uint32_t)atoi(a + 8);
        else if (!strcmp(a, "--transition=weighted")) p.transition = DYG_TRANSITION_WEIGHTED;
        else if (!strcmp(a, "--transition=uniform")) p.transition = DYG_TRANSITION_UNIFORM;
        else {
            fprintf(stderr, "unknown option %s\n", a);
            return 2;
        }
    }
    const std::string base = dir + "/" + argv[1] + "/";
    const std::string graph_file = base + "adj_sparse.mtx";
    const std::string target_file = base + "ext.mtx";
    const std::string output_file = base + "updated_adj_sparse.mtx";

    uint64_t m = 0, k = 0;
    uint32_t *gs, *gd, *es, *ed, mx_g = 0, mx_e = 0;
    float *gw, *ew;
    dyg_status s = dyg_mtx_read(graph_file.c_str(), 0, 1, &m, &gs, &gd, &gw, &mx_g);
    if (s) return fail("reading adj_sparse.mtx", s);
    s = dyg_mtx_read(target_file.c_str(), 1, 1, &k, &es, &ed, &ew, &mx_e);
    if (s) return fail("reading ext.mtx", s);
    uint32_t n = (m ? mx_g + 1 : 0);
    if (k && mx_e + 1 > n) n = mx_e + 1;
    printf("after read_targets\n");

    dyg_graph *H = nullptr;
    s = dyg_graph_create_from_edges(n, m, gs, gd, gw, nullptr, &H);
    if (s) return fail("dyg_graph_create_from_edges", s);
    printf("Graph copied to GPU\n");

    std::vector<int32_t> found(k);
    std::vector<float> cond(k);
    std::vector<uint8_t> acc(k);
    const auto t0 = std::chrono::high_resolution_clock::now();
    s = dyg_incremental_stream(H, nullptr, es, ed, ew, (uint32_t)k, batch, &p, found.data(),
                               cond.data(), acc.data(), nullptr);
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (s) return fail("dyg_incremental_stream", s);
    const long long ms = std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count();
    printf("Time taken: %lld milliseconds\n", ms);
    uint64_t added = 0;
    std::vector<uint32_t> as, ad;
    std::vector<float> aw;
    for (uint64_t i = 0; i < k; ++i)
        if (acc[i]) {
            ++added;
            as.push_back(es[i]);
            ad.push_back(ed[i]);
            aw.push_back(ew[i]);
        }
    printf("No path %%: %g\n", k ? (double)(float)((float)added / (float)k * 100.0f) : 0.0);
    printf("Edges added: %llu out of %llu samples\n", (unsigned long long)added,
           (unsigned long long)k);
    printf("saving mtx to %s\n", output_file.c_str());
    s = dyg_mtx_write(output_file.c_str(), 0, m, gs, gd, gw, 1);
    if (!s) s = dyg_mtx_write(output_file.c_str(), 1, added, as.data(), ad.data(), aw.data(), 1);
    if (s) return fail("writing updated_adj_sparse.mtx", s);
    printf("Updated graph saved to %s\n", output_file.c_str());
    dyg_graph_destroy(H);
    dyg_mtx_free(gs); dyg_mtx_free(gd); dyg_mtx_free(gw);
    dyg_mtx_free(es); dyg_mtx_free(ed); dyg_mtx_free(ew);
    printf("Incremental graph sparsification completed successfully!\n");
    return 0;
}
