// dynamic_update -- drop-in for the reference's mixed-stream updater CLI
// (dynamic_update/main.cu:26-136).
//
//   dynamic_update <graph_name> <distortion_threshold>
//                  [inc_steps dec_steps inc_walkers dec_walkers] [--key=value ...]
//
// Reads ./dataset/<g>/new_adj_dense.mtx (G) and ./dataset/<g>/new_adj_sparse.mtx
// (H) with the format detection of dynamic_update/functions.cpp:35-291 (header,
// dimensions line, weight column, Laplacian, triangular or full, base), then
// every regular file of ./dataset/<g>/stream_edges/ whose name starts with
// "stream_" and contains ".mtx", in name order (functions.cpp:589-629); a
// name with "insert"/"inc" inserts, one with "delete"/"dec" deletes
// (688-692).  Each file goes through dyg_stream_file: weight merges of
// edges already in G, then walks in chunks of max(5% |V|, 10000) with the
// sparsifier updated after each chunk.  Defaults: 100 steps and 512 walkers
// for both operations (main.cu:50-54), 16 fallback walkers per endpoint
// (gpu_graph.cuh:228).  Writes ./output/<g>/<timestamp>/adj_dense.mtx and
// adj_sparse.mtx: one line "u+1 v+1 w" per undirected edge (u <= v), sorted
// (the reference writes its hash maps in their iteration order,
// gpu_graph.cuh:725-763).  The reference asks before every file on standard
// input (main.cu:96-101, functions.cpp:647-668); this tool applies them all.
// Options: --dataset-dir=DIR, --output-dir=DIR, --timestamp=T, --seed=S,
// --chunk=N, --fallback-walkers=N.
#include <dirent.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "dyg.h"
#include "dyg_io.h"

namespace {

int fail(const char *what, dyg_status s) {
    fprintf(stderr, "%s failed (status %d): %s\n", what, (int)s, dyg_last_error_string());
    return 1;
}

struct Loaded {
    dyg_mtx_info info;
    uint64_t m = 0;
    uint32_t *src = nullptr, *dst = nullptr;
    float *w = nullptr;
    ~Loaded() {
        dyg_mtx_free(src);
        dyg_mtx_free(dst);
        dyg_mtx_free(w);
    }
};

// A triangular file lists each undirected edge once: both rows get it.  A
// full one lists both directions: each record fills its source's row only.
dyg_status build_graph(const Loaded &L, uint32_t n, dyg_graph **out) {
    if (L.info.triangular) return dyg_graph_create_from_edges(n, L.m, L.src, L.dst, L.w, nullptr, out);
    std::vector<uint64_t> rp((size_t)n + 1, 0);
    for (uint64_t i = 0; i < L.m; ++i) {
        if (L.src[i] >= n || L.dst[i] >= n) return DYG_EINVAL;
        rp[L.src[i] + 1]++;
    }
    for (uint32_t v = 0; v < n; ++v) rp[v + 1] += rp[v];
    std::vector<uint64_t> fill(rp.begin(), rp.end() - 1);
    std::vector<uint32_t> col(L.m ? L.m : 1);
    std::vector<float> w(L.m ? L.m : 1);
    for (uint64_t i = 0; i < L.m; ++i) {
        const uint64_t p = fill[L.src[i]]++;
        col[p] = L.dst[i];
        w[p] = L.w[i];
    }
    return dyg_graph_create_from_csr(n, rp.data(), col.data(), w.data(), nullptr, out);
}

void mkdirs(const std::string &path) {
    for (size_t i = 1; i <= path.size(); ++i)
        if (i == path.size() || path[i] == '/') mkdir(path.substr(0, i).c_str(), 0755);
}

}  // namespace

int main(int argc, char **argv) {
    std::vector<const char *> pos;
    std::string dataset = "./dataset", output = "./output", stamp;
    uint64_t seed = 0;
    bool have_seed = false;
    uint32_t chunk = 0, hw = 16;
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        if (!strncmp(a, "--dataset-dir=", 14)) dataset = a + 14;
        else if (!strncmp(a, "--output-dir=", 13)) output = a + 13;
        else if (!strncmp(a, "--timestamp=", 12)) stamp = a + 12;
        else if (!strncmp(a, "--seed=", 7)) { seed = strtoull(a + 7, nullptr, 10); have_seed = true; }
        else if (!strncmp(a, "--chunk=", 8)) chunk = (uint32_t)atoi(a + 8);
        else if (!strncmp(a, "--fallback-walkers=", 19)) hw = (uint32_t)atoi(a + 19);
        else if (!strncmp(a, "--", 2)) {
            fprintf(stderr, "unknown option %s\n", a);
            return 2;
        } else pos.push_back(a);
    }
    if (pos.size() != 2 && pos.size() != 6) {
        printf("Input: .dynamic_update<1.graph name><2.distortion_threshold><3.incremental_steps>"
               "<4.decremental_steps><5.incremental_number_of_walkers>"
               "<6.decremental_number_of_walkers>\n");
        return 0;
    }
    const std::string name = pos[0];
    dyg_walk_params ip, dp;
    dyg_walk_params_default(&ip);
    ip.threshold = (float)atof(pos[1]);
    ip.max_steps = 100;
    ip.walkers = 512;
    ip.heuristic_walkers = hw;
    if (have_seed) ip.seed = seed;
    dp = ip;
    if (pos.size() == 6) {
        ip.max_steps = (uint32_t)atoi(pos[2]);
        dp.max_steps = (uint32_t)atoi(pos[3]);
        ip.walkers = (uint32_t)atoi(pos[4]);
        dp.walkers = (uint32_t)atoi(pos[5]);
    }
    if (stamp.empty()) {
        char buf[32];
        const time_t t = time(nullptr);
        strftime(buf, sizeof buf, "%Y%m%d_%H%M%S", localtime(&t));
        stamp = buf;
    }
    printf("Graph Name: %s\n", name.c_str());
    printf("Distortion Threshold: %g\n", (double)ip.threshold);
    printf("Incremental Steps: %u\n", ip.max_steps);
    printf("Decremental Steps: %u\n", dp.max_steps);
    printf("Incremental Number of Walkers: %u\n", ip.walkers);
    printf("Decremental Number of Walkers: %u\n", dp.walkers);

    const std::string dir = dataset + "/" + name + "/";
    printf("Read graph and sparsifier\n");
    Loaded D, S;
    dyg_status s = dyg_mtx_read_auto((dir + "new_adj_dense.mtx").c_str(), &D.info, &D.m, &D.src,
                                     &D.dst, &D.w);
    if (s) return fail("reading new_adj_dense.mtx", s);
    s = dyg_mtx_read_auto((dir + "new_adj_sparse.mtx").c_str(), &S.info, &S.m, &S.src, &S.dst,
                          &S.w);
    if (s) return fail("reading new_adj_sparse.mtx", s);
    if (D.info.base != S.info.base || D.info.v_max != S.info.v_max ||
        D.info.v_min != S.info.v_min) {
        fprintf(stderr, "the dense graph and the sparsifier differ in base or id range\n");
        return 1;
    }
    const uint32_t n = D.info.v_max - (uint32_t)D.info.base + 1u;
    dyg_graph *G = nullptr, *H = nullptr;
    s = build_graph(D, n, &G);
    if (s) return fail("creating G", s);
    s = build_graph(S, n, &H);
    if (s) return fail("creating H", s);

    const std::string sdir = dir + "stream_edges/";
    std::vector<std::string> files;
    if (DIR *dd = opendir(sdir.c_str())) {
        while (dirent *e = readdir(dd)) {
            const std::string f = e->d_name;
            struct stat st;
            if (stat((sdir + f).c_str(), &st) != 0 || !S_ISREG(st.st_mode)) continue;
            if (f.rfind("stream_", 0) == 0 && f.find(".mtx") != std::string::npos) files.push_back(f);
        }
        closedir(dd);
    } else {
        fprintf(stderr, "Error: Cannot open directory '%s'\n", sdir.c_str());
        return 1;
    }
    std::sort(files.begin(), files.end());
    printf("Found %zu stream updates files: \n", files.size());
    for (const auto &f : files) printf("  %s\n", f.c_str());

    uint32_t op = DYG_STREAM_INSERT;
    uint64_t uid = 0;
    double total_ms = 0;
    for (const auto &f : files) {
        op = dyg_stream_op_from_name(f.c_str(), op);
        printf("Next stream file: %s\n", f.c_str());
        uint64_t m = 0;
        uint32_t *es = nullptr, *ed = nullptr;
        float *ew = nullptr;
        int32_t weighted = 0;
        s = dyg_stream_read((sdir + f).c_str(), (uint32_t)D.info.base, &m, &es, &ed, &ew, &weighted);
        if (s) return fail("reading a stream file", s);
        printf("Loaded %llu edges (%s)\n", (unsigned long long)m,
               op == DYG_STREAM_INSERT ? "INSERT" : "DELETE");
        const dyg_walk_params &p = op == DYG_STREAM_INSERT ? ip : dp;
        std::vector<int32_t> status(m ? m : 1);
        const uint64_t cap = m * (uint64_t)(p.max_steps + 4u * p.heuristic_walkers) + 16;
        std::vector<uint32_t> rx(op == DYG_STREAM_DELETE ? cap : 1), ry(rx.size());
        std::vector<uint8_t> rk(rx.size());
        uint64_t nrec = 0;
        const auto t0 = std::chrono::high_resolution_clock::now();
        s = dyg_stream_file(G, H, op, es, ed, ew, (uint32_t)m, uid, chunk, &p, status.data(),
                            nullptr, op == DYG_STREAM_DELETE ? rx.data() : nullptr,
                            op == DYG_STREAM_DELETE ? ry.data() : nullptr,
                            op == DYG_STREAM_DELETE ? rk.data() : nullptr,
                            op == DYG_STREAM_DELETE ? cap : 0, &nrec, nullptr);
        const auto t1 = std::chrono::high_resolution_clock::now();
        if (s) return fail("dyg_stream_file", s);
        total_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        uint64_t skipped = 0, nopath = 0, added = 0;
        for (uint64_t i = 0; i < m; ++i) {
            const int32_t v = status[i];
            if (op == DYG_STREAM_INSERT) {
                if (v == DYG_INS_MERGED || v == DYG_INS_SELF_LOOP) ++skipped;
                if (v == -1) ++nopath, ++added;
            } else {
                if (v == DYG_DEL_NOT_IN_G || v == DYG_DEL_NOT_IN_H) ++skipped;
                if (v == DYG_DEL_NO_PATH) ++nopath;
            }
        }
        if (op == DYG_STREAM_DELETE) added = nrec;
        printf("Filtered out %llu edges during initial check.\n", (unsigned long long)skipped);
        printf("%s edges not found in NBRW: %llu\n",
               op == DYG_STREAM_INSERT ? "Incremental" : "Decremental", (unsigned long long)nopath);
        printf("Sparsifier updated with %llu edges from stream.\n", (unsigned long long)added);
        uid += m;
        dyg_mtx_free(es);
        dyg_mtx_free(ed);
        dyg_mtx_free(ew);
    }
    printf("Update time: %.3f milliseconds\n", total_ms);
    const std::string out = output + "/" + name + "/" + stamp;
    mkdirs(out);
    s = dyg_graph_save(G, (out + "/adj_dense.mtx").c_str());
    if (s) return fail("writing adj_dense.mtx", s);
    s = dyg_graph_save(H, (out + "/adj_sparse.mtx").c_str());
    if (s) return fail("writing adj_sparse.mtx", s);
    printf("Results saved to: %s\n", out.c_str());
    dyg_graph_destroy(G);
    dyg_graph_destroy(H);
    return 0;
}
