// decremental_update -- drop-in for the reference's decremental updater CLI
// (random_walk_decremental/main.cu:318-468).
//
//   decremental_update <graph_name> [--key=value ...]
//
// Reads ../dataset/<g>/updated_dense.mtx (G after insertions, 1-based,
// weighted), ../dataset/<g>/updated_adj_sparse.mtx (H, 1-based, weighted) and
// ../dataset/<g>/del.mtx (1-based, unweighted); deletes in batches of
// ceil(N/10) with the reference's fixed parameters (100 steps, 512 walkers,
// 16 fallback walkers per endpoint, main.cu:332-335) and writes
// ../dataset/<g>/added_edges.mtx: "min+1 max+1" per recovered edge, in
// commit order.  Fallback-walk edges are written too (the reference keeps
// them out of the file, gpu_graph.cuh:599-601, so its final sparsifier
// loses them).
// Options: --dataset-dir=DIR, --max-steps=N, --walkers=N, --seed=S, --batch=B,
// --fallback-walkers=N, --path-edges-only, --snapshot-dir=DIR (also write
// the final G and H there as adj_dense.mtx / adj_sparse.mtx, the format of
// dyg_graph_save: what the reference's evaluation rebuilds from
// added_edges.mtx, dyGRASS.jl:516-541).
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
    if (argc < 2) {
        printf("Input: ./decremental_update <1. graph name>\n");
        return 0;
    }
    std::string dir = "../dataset";
    dyg_walk_params p;
    dyg_walk_params_default(&p);
    p.max_steps = 100;
    p.walkers = 512;
    p.heuristic_walkers = 16;
    uint32_t batch = 0;
    bool path_only = false;
    std::string snapshot;
    for (int i = 2; i < argc; ++i) {
        const char *a = argv[i];
        if (!strncmp(a, "--dataset-dir=", 14)) dir = a + 14;
        else if (!strncmp(a, "--max-steps=", 12)) p.max_steps = (uint32_t)atoi(a + 12);
        else if (!strncmp(a, "--walkers=", 10)) p.walkers = (uint32_t)atoi(a + 10);
        else if (!strncmp(a, "--seed=", 7)) p.seed = strtoull(a + 7, nullptr, 10);
        else if (!strncmp(a, "--batch=", 8)) batch = (uint32_t)atoi(a + 8);
        else if (!strncmp(a, "--fallback-walkers=", 19)) p.heuristic_walkers = (uint32_t)atoi(a + 19);
        else if (!strcmp(a, "--path-edges-only")) path_only = true;
        else if (!strncmp(a, "--snapshot-dir=", 15)) snapshot = a + 15;
        else {
            fprintf(stderr, "unknown option %s\n", a);
            return 2;
        }
    }
    const std::string base = dir + "/" + argv[1] + "/";
    const std::string sparse_file = base + "updated_adj_sparse.mtx";
    const std::string dense_file = base + "updated_dense.mtx";
    const std::string del_file = base + "del.mtx";
    const std::string output_file = base + "added_edges.mtx";

    printf("Read graph and sparsifier\n");
    uint64_t mg = 0, mh = 0, md = 0;
    uint32_t *gs, *gd, *hs, *hd, *ds, *dd, mxg = 0, mxh = 0, mxd = 0;
    float *gw, *hw, *unused = nullptr;
    dyg_status s = dyg_mtx_read(dense_file.c_str(), 1, 1, &mg, &gs, &gd, &gw, &mxg);
    if (s) return fail("reading updated_dense.mtx", s);
    s = dyg_mtx_read(sparse_file.c_str(), 1, 1, &mh, &hs, &hd, &hw, &mxh);
    if (s) return fail("reading updated_adj_sparse.mtx", s);
    printf("Read targets\n");
    s = dyg_mtx_read(del_file.c_str(), 1, 0, &md, &ds, &dd, &unused, &mxd);
    if (s) return fail("reading del.mtx", s);
    // vertex count = largest id + 1 (the reference's v_max undercounts by one,
    // random_walk_decremental/functions.cpp:123)
    uint32_t n = 0;
    if (mg && mxg + 1 > n) n = mxg + 1;
    if (mh && mxh + 1 > n) n = mxh + 1;
    if (md && mxd + 1 > n) n = mxd + 1;

    dyg_graph *G = nullptr, *H = nullptr;
    s = dyg_graph_create_from_edges(n, mg, gs, gd, gw, nullptr, &G);
    if (s) return fail("creating G", s);
    s = dyg_graph_create_from_edges(n, mh, hs, hd, hw, nullptr, &H);
    if (s) return fail("creating H", s);
    uint64_t h_slots0 = 0;
    dyg_graph_info(H, nullptr, &h_slots0, nullptr, nullptr);
    printf("Graph copied to GPU\n");

    std::vector<int32_t> status(md);
    const uint64_t cap = md * (uint64_t)(p.max_steps + 4u * p.heuristic_walkers) + 16;
    std::vector<uint32_t> rx(cap), ry(cap);
    std::vector<uint8_t> rk(cap);
    uint64_t nrec = 0;
    const auto t0 = std::chrono::high_resolution_clock::now();
    s = dyg_decremental_stream(G, H, ds, dd, (uint32_t)md, batch, &p, status.data(), nullptr,
                               rx.data(), ry.data(), rk.data(), cap, &nrec, nullptr);
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (s) return fail("dyg_decremental_stream", s);
    const long long ms = std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count();
    printf("Time taken: %lld milliseconds\n", ms);
    uint64_t h_slots1 = 0;
    dyg_graph_info(H, nullptr, &h_slots1, nullptr, nullptr);
    const long long e0 = (long long)(h_slots0 / 2), e1 = (long long)(h_slots1 / 2);
    printf("Increased edges number: %lld\n", e1 - e0);
    printf("Density: %g %%\n", n ? (double)(float)((float)(e1 - (long long)n) / (float)n * 100.0f) : 0.0);
    std::vector<uint32_t> ox, oy;
    for (uint64_t i = 0; i < nrec; ++i) {
        if (path_only && rk[i] != DYG_REC_PATH) continue;
        ox.push_back(rx[i] < ry[i] ? rx[i] : ry[i]);
        oy.push_back(rx[i] < ry[i] ? ry[i] : rx[i]);
    }
    printf("Size of added edges: %zu\n", ox.size());
    s = dyg_mtx_write(output_file.c_str(), 0, ox.size(), ox.data(), oy.data(), nullptr, 1);
    if (s) return fail("writing added_edges.mtx", s);
    printf("Added edges saved to: %s\n", output_file.c_str());
    if (!snapshot.empty()) {
        s = dyg_graph_save(G, (snapshot + "/adj_dense.mtx").c_str());
        if (s) return fail("writing adj_dense.mtx", s);
        s = dyg_graph_save(H, (snapshot + "/adj_sparse.mtx").c_str());
        if (s) return fail("writing adj_sparse.mtx", s);
    }
    dyg_graph_destroy(G);
    dyg_graph_destroy(H);
    dyg_mtx_free(gs); dyg_mtx_free(gd); dyg_mtx_free(gw);
    dyg_mtx_free(hs); dyg_mtx_free(hd); dyg_mtx_free(hw);
    dyg_mtx_free(ds); dyg_mtx_free(dd);
    printf("Decremental graph sparsification completed successfully!\n");
    return 0;
}
