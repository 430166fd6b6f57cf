// graph.cu -- device-resident dynamic CSR: upload, arena growth, compaction
// and the small shared helpers (allocation, scans, scalar read-back).  Row
// updates live in rowops.cu.  Row moves (capacity exceeded) take space from a
// bump arena: offsets differ from run to run but contents never do.

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "dyg_internal.cuh"
#include "scan.cuh"

namespace dyg {

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int num_sms() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1) sms = 1;
    }
    return sms;
}

dyg_status ensure(Buf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return DYG_OK;
    if (b.p) {
        DYG_CUDA(cudaFree(b.p));
        b.p = nullptr;
        b.bytes = 0;
    }
    size_t want = bytes + bytes / 4;
    want = (want + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        set_error(std::string("cudaMalloc of ") + std::to_string(want) + " bytes failed: " +
                  cudaGetErrorString(e));
        return DYG_ENOMEM;
    }
    b.bytes = want;
    return DYG_OK;
}

dyg_status read_scalars(dyg_graph *G, cudaStream_t st) {
    Workspace &ws = G->ws;
    DYG_CUDA(cudaMemcpyAsync(ws.host_scalars, ws.scalars.p, S_NSCALARS * sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaMemcpyAsync(ws.host_counts, ws.counts.p, C_NCOUNTS * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    if (ws.host_scalars[S_LONG]) G->long_rows = true;
    return DYG_OK;
}

dyg_status read_scalars2(dyg_graph *A, dyg_graph *B, cudaStream_t st) {
    if (!B || B == A) return read_scalars(A, st);
    for (dyg_graph *G : {A, B}) {
        Workspace &ws = G->ws;
        DYG_CUDA(cudaMemcpyAsync(ws.host_scalars, ws.scalars.p,
                                 S_NSCALARS * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        DYG_CUDA(cudaMemcpyAsync(ws.host_counts, ws.counts.p, C_NCOUNTS * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
    }
    DYG_CUDA(cudaStreamSynchronize(st));
    for (dyg_graph *G : {A, B})
        if (G->ws.host_scalars[S_LONG]) G->long_rows = true;
    return DYG_OK;
}

// ------------------------------------------------------------------ upload

dyg_status upload_graph(dyg_graph *G, uint32_t n, const uint64_t *row_ptr, const uint32_t *col,
                        const float *w) {
    const uint64_t slots = row_ptr[n];
    std::string msg;
    uint2 *h_desc = (uint2 *)malloc(sizeof(uint2) * (size_t)(n ? n : 1));
    uint32_t *h_cap = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n ? n : 1));
    if (!h_desc || !h_cap) {
        free(h_desc);
        free(h_cap);
        set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    uint64_t off = 0;
    for (uint32_t v = 0; v < n; ++v) {
        const uint64_t deg = row_ptr[v + 1] - row_ptr[v];
        const uint64_t cap = deg + G->slack;
        if (deg > kBigRow) G->long_rows = true;
        h_desc[v] = make_uint2((uint32_t)off, (uint32_t)deg);
        h_cap[v] = (uint32_t)cap;
        off += cap;
    }
    const uint64_t used = off;
    uint64_t arena = used + (uint64_t)((double)slots * G->headroom) + 1024;
    if (arena >= 0xFFFFFFFFull) {
        free(h_desc);
        free(h_cap);
        set_error("graph too large for 32-bit slot offsets");
        return DYG_EINVAL;
    }
    uint2 *h_slots = (uint2 *)calloc((size_t)(used ? used : 1), sizeof(uint2));
    float *h_w = (float *)calloc((size_t)(used ? used : 1), sizeof(float));
    if (!h_slots || !h_w) {
        free(h_desc);
        free(h_cap);
        free(h_slots);
        free(h_w);
        set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    for (uint32_t v = 0; v < n; ++v) {
        const uint64_t o = h_desc[v].x;
        for (uint64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) {
            const float rw = 1.0f / w[j];   // IEEE division: equals __frcp_rn(w)
            uint32_t rb;
            memcpy(&rb, &rw, 4);
            h_slots[o + (j - row_ptr[v])] = make_uint2(col[j], rb);
            h_w[o + (j - row_ptr[v])] = w[j];
        }
    }
    dyg_status rc = DYG_OK;
    G->g.n = n;
    G->g.arena_cap = arena;
    if (cudaMalloc(&G->g.desc, sizeof(uint2) * (size_t)(n ? n : 1)) != cudaSuccess ||
        cudaMalloc(&G->g.cap, sizeof(uint32_t) * (size_t)(n ? n : 1)) != cudaSuccess ||
        cudaMalloc(&G->g.slots, sizeof(uint2) * (size_t)arena) != cudaSuccess ||
        cudaMalloc(&G->g.wts, sizeof(float) * (size_t)arena) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of the graph arena failed");
        rc = DYG_ENOMEM;
    }
    if (rc == DYG_OK) {
        cudaError_t e = cudaMemcpy(G->g.desc, h_desc, sizeof(uint2) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G->g.cap, h_cap, sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G->g.slots, h_slots, sizeof(uint2) * used, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G->g.wts, h_w, sizeof(float) * used, cudaMemcpyHostToDevice);
        unsigned long long top = used;
        if (e == cudaSuccess) e = cudaMemcpy(G->g.top, &top, sizeof(top), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = cuda_fail(e, "graph upload", __FILE__, __LINE__);
    }
    free(h_desc);
    free(h_cap);
    free(h_slots);
    free(h_w);
    return rc;
}

dyg_status grow_arena(dyg_graph *G, uint64_t min_cap, cudaStream_t st) {
    uint64_t cap = G->g.arena_cap + G->g.arena_cap / 2;
    if (cap < min_cap + min_cap / 4 + 1024) cap = min_cap + min_cap / 4 + 1024;
    if (cap >= 0xFFFFFFFFull) cap = 0xFFFFFFFEull;
    if (cap < min_cap) {
        set_error("arena would exceed 32-bit slot offsets");
        return DYG_ENOMEM;
    }
    uint2 *ns = nullptr;
    float *nw = nullptr;
    cudaError_t e = cudaMalloc(&ns, sizeof(uint2) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMalloc(&nw, sizeof(float) * (size_t)cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (ns) cudaFree(ns);
        set_error("cudaMalloc while growing the arena failed");
        return DYG_ENOMEM;
    }
    DYG_TRY(read_scalars(G, st));
    const unsigned long long top = G->ws.host_scalars[S_TOP];
    DYG_CUDA(cudaMemcpyAsync(ns, G->g.slots, sizeof(uint2) * (size_t)top, cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(nw, G->g.wts, sizeof(float) * (size_t)top, cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    DYG_CUDA(cudaFree(G->g.slots));
    DYG_CUDA(cudaFree(G->g.wts));
    G->g.slots = ns;
    G->g.wts = nw;
    G->g.arena_cap = cap;
    return DYG_OK;
}

// ---------------------------------------------------------- exclusive scan
namespace {
struct CopyScan {
    const uint32_t *in;
    uint32_t *out;
    __device__ uint32_t load(uint32_t i) const { return in[i]; }
    __device__ void store(uint32_t i, uint32_t excl, uint32_t) const { out[i] = excl; }
    __device__ void last(uint32_t) const {}
};
}  // namespace

dyg_status exclusive_scan_u32(Workspace &ws, const uint32_t *in, uint32_t *out, uint32_t m,
                              cudaStream_t st, const uint32_t *m_dev) {
    return scan_op(ws, CopyScan{in, out}, m, m_dev, nullptr, st);
}

// -------------------------------------------------------------- compaction

// Rows keep slack; a vertex with neither slots nor capacity (an unoccupied
// vertex of a pool graph) keeps none.
__global__ void k_new_caps(DevGraph g, uint32_t slack, uint32_t *caps) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= g.n) return;
    const uint32_t deg = g.desc[v].y;
    caps[v] = (deg == 0u && g.cap[v] == 0u) ? 0u : deg + slack;
}

// One warp per row: consecutive lanes copy consecutive slots into the new
// arena, four loads per lane issued before their stores (the new arena never
// overlaps the old one).  Lane 0 reads the descriptor and hands it to the
// warp before it rewrites it.
__global__ void k_move_rows(DevGraph g, uint2 *ns, float *nw, const uint32_t *off,
                            const uint32_t *caps) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < g.n; v += warps) {
        uint2 d = make_uint2(0u, 0u);
        if (lane == 0u) d = g.desc[v];
        d.x = __shfl_sync(kFull, d.x, 0);
        d.y = __shfl_sync(kFull, d.y, 0);
        const uint32_t o = off[v];
        for (uint32_t j0 = 0; j0 < d.y; j0 += 128u) {
            uint2 sv[4];
            float wv[4];
#pragma unroll
            for (uint32_t u = 0; u < 4u; ++u) {
                const uint32_t j = j0 + lane + 32u * u;
                if (j < d.y) {
                    sv[u] = g.slots[d.x + j];
                    wv[u] = g.wts[d.x + j];
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < 4u; ++u) {
                const uint32_t j = j0 + lane + 32u * u;
                if (j < d.y) {
                    ns[o + j] = sv[u];
                    nw[o + j] = wv[u];
                }
            }
        }
        if (lane == 0u) {
            g.desc[v] = make_uint2(o, d.y);
            g.cap[v] = caps[v];
        }
    }
}

dyg_status compact_graph(dyg_graph *G, cudaStream_t st) {
    Workspace &ws = G->ws;
    const uint32_t n = G->g.n;
    if (n == 0) return DYG_OK;
    DYG_TRY(ensure(ws.flags, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(ws.pos, sizeof(uint32_t) * (size_t)n));
    const int th = 256;
    const int gr = (int)((n + th - 1) / th);
    k_new_caps<<<gr, th, 0, st>>>(G->g, G->slack, ptr<uint32_t>(ws.flags));
    count_launch();
    DYG_TRY(exclusive_scan_u32(ws, ptr<uint32_t>(ws.flags), ptr<uint32_t>(ws.pos), n, st));
    uint32_t last_off = 0, last_cap = 0;
    DYG_CUDA(cudaMemcpyAsync(&last_off, ptr<uint32_t>(ws.pos) + n - 1, 4, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaMemcpyAsync(&last_cap, ptr<uint32_t>(ws.flags) + n - 1, 4, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    const uint64_t used = (uint64_t)last_off + last_cap;
    uint64_t cap = used + (uint64_t)((double)used * G->headroom) + 1024;
    if (cap < G->g.arena_cap / 2) cap = G->g.arena_cap / 2 > used ? G->g.arena_cap / 2 : cap;
    if (cap >= 0xFFFFFFFFull) cap = 0xFFFFFFFEull;
    uint2 *ns = nullptr;
    float *nw = nullptr;
    cudaError_t e = cudaMalloc(&ns, sizeof(uint2) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMalloc(&nw, sizeof(float) * (size_t)cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (ns) cudaFree(ns);
        set_error("cudaMalloc during compaction failed");
        return DYG_ENOMEM;
    }
    k_move_rows<<<num_sms() * 8, th, 0, st>>>(G->g, ns, nw, ptr<uint32_t>(ws.pos),
                                              ptr<uint32_t>(ws.flags));
    count_launch();
    DYG_CUDA(cudaGetLastError());
    unsigned long long top = used;
    DYG_CUDA(cudaMemcpyAsync(G->g.top, &top, sizeof(top), cudaMemcpyHostToDevice, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    DYG_CUDA(cudaFree(G->g.slots));
    DYG_CUDA(cudaFree(G->g.wts));
    G->g.slots = ns;
    G->g.wts = nw;
    G->g.arena_cap = cap;
    return DYG_OK;
}

// ----------------------------------------------------------- vertex ranges
// A graph that holds many graphs at vertex offsets (the serving pool) loads,
// saves and clears one graph's rows at a time.

// One warp per vertex: row v0 + i goes to [out_off[i], out_off[i] + deg) of
// col / w, with columns made local (minus v0).
__global__ void k_gather_rows(DevGraph g, uint32_t v0, uint32_t n, const unsigned long long *out_off,
                              uint32_t *col, float *w) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const uint2 d = g.desc[v0 + i];
        const unsigned long long o = out_off[i];
        for (uint32_t j = lane; j < d.y; j += 32u) {
            col[o + j] = g.slots[d.x + j].x - v0;
            w[o + j] = g.wts[d.x + j];
        }
    }
}

// One warp per vertex: row i of the staged CSR goes to the arena at
// top + rp[i] + slack * i, columns shifted by v0, with the correctly rounded
// 1/w beside each column.
__global__ void k_place_rows(DevGraph g, uint32_t v0, uint32_t n, unsigned long long top,
                             uint32_t slack, const unsigned long long *rp, const uint32_t *col,
                             const float *w, unsigned long long *long_flag) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n;
         i += (gridDim.x * blockDim.x) >> 5) {
        const unsigned long long a = rp[i];
        const uint32_t deg = (uint32_t)(rp[i + 1] - a);
        const unsigned long long off = top + a + (unsigned long long)slack * i;
        for (uint32_t j = lane; j < deg; j += 32u) {
            const float x = w[a + j];
            g.slots[off + j] = make_uint2(col[a + j] + v0, __float_as_uint(__frcp_rn(x)));
            g.wts[off + j] = x;
        }
        if (lane == 0u) {
            g.desc[v0 + i] = make_uint2((uint32_t)off, deg);
            g.cap[v0 + i] = deg + slack;
            if (deg > kBigRow) *long_flag = 1ull;
        }
    }
}

dyg_status load_range(dyg_graph *G, uint32_t v0, uint32_t n, const uint64_t *row_ptr,
                      const uint32_t *col, const float *w, cudaStream_t st) {
    if (n == 0) return DYG_OK;
    if ((uint64_t)v0 + n > G->g.n) {
        set_error("vertex range outside the graph");
        return DYG_EINVAL;
    }
    const uint64_t m = row_ptr[n];
    const uint64_t need = m + (uint64_t)G->slack * n;
    DYG_TRY(read_scalars(G, st));
    uint64_t top = G->ws.host_scalars[S_TOP];
    if (top + need > G->g.arena_cap) {
        // holes left by evicted graphs and moved rows go first
        DYG_TRY(compact_graph(G, st));
        DYG_TRY(read_scalars(G, st));
        top = G->ws.host_scalars[S_TOP];
        if (top + need > G->g.arena_cap) DYG_TRY(grow_arena(G, top + need, st));
    }
    if (top + need >= 0xFFFFFFFFull) {
        set_error("arena would exceed 32-bit slot offsets");
        return DYG_ENOMEM;
    }
    Workspace &ws = G->ws;
    DYG_TRY(ensure(ws.f_uid, sizeof(unsigned long long) * ((size_t)n + 1)));
    DYG_TRY(ensure(ws.cand_x, sizeof(uint32_t) * (m ? m : 1)));
    DYG_TRY(ensure(ws.cand_w, sizeof(float) * (m ? m : 1)));
    DYG_CUDA(cudaMemcpyAsync(ws.f_uid.p, row_ptr, sizeof(uint64_t) * ((size_t)n + 1),
                             cudaMemcpyHostToDevice, st));
    if (m) {
        DYG_CUDA(cudaMemcpyAsync(ws.cand_x.p, col, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, st));
        DYG_CUDA(cudaMemcpyAsync(ws.cand_w.p, w, sizeof(float) * m, cudaMemcpyHostToDevice, st));
    }
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    const int gr = (int)std::min<uint64_t>(((uint64_t)n * 32 + 255) / 256, (uint64_t)num_sms() * 16);
    k_place_rows<<<gr, 256, 0, st>>>(G->g, v0, n, top, G->slack, ptr<unsigned long long>(ws.f_uid),
                                     ptr<uint32_t>(ws.cand_x), ptr<float>(ws.cand_w), sc + S_LONG);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    const unsigned long long ntop = top + need;
    DYG_CUDA(cudaMemcpyAsync(G->g.top, &ntop, sizeof(ntop), cudaMemcpyHostToDevice, st));
    DYG_TRY(read_scalars(G, st));   // synchronizes; picks up a long row
    return DYG_OK;
}

dyg_status save_range(dyg_graph *G, uint32_t v0, uint32_t n, std::vector<uint64_t> &row_ptr,
                      std::vector<uint32_t> &col, std::vector<float> &w, cudaStream_t st) {
    row_ptr.assign((size_t)n + 1, 0);
    col.clear();
    w.clear();
    if (n == 0) return DYG_OK;
    std::vector<uint2> h_desc(n);
    DYG_CUDA(cudaMemcpyAsync(h_desc.data(), G->g.desc + v0, sizeof(uint2) * n, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    std::vector<unsigned long long> off(n);
    for (uint32_t v = 0; v < n; ++v) {
        off[v] = row_ptr[v];
        row_ptr[v + 1] = row_ptr[v] + h_desc[v].y;
    }
    const uint64_t m = row_ptr[n];
    col.resize(m);
    w.resize(m);
    if (m == 0) return DYG_OK;
    Workspace &ws = G->ws;
    DYG_TRY(ensure(ws.f_uid, sizeof(unsigned long long) * n));
    DYG_TRY(ensure(ws.cand_x, sizeof(uint32_t) * m));
    DYG_TRY(ensure(ws.cand_w, sizeof(float) * m));
    DYG_CUDA(cudaMemcpyAsync(ws.f_uid.p, off.data(), sizeof(unsigned long long) * n,
                             cudaMemcpyHostToDevice, st));
    const int gr = (int)std::min<uint64_t>(((uint64_t)n * 32 + 255) / 256, (uint64_t)num_sms() * 16);
    k_gather_rows<<<gr, 256, 0, st>>>(G->g, v0, n, ptr<unsigned long long>(ws.f_uid),
                                      ptr<uint32_t>(ws.cand_x), ptr<float>(ws.cand_w));
    count_launch();
    DYG_CUDA(cudaGetLastError());
    DYG_CUDA(cudaMemcpyAsync(col.data(), ws.cand_x.p, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaMemcpyAsync(w.data(), ws.cand_w.p, sizeof(float) * m, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    return DYG_OK;
}

dyg_status clear_range(dyg_graph *G, uint32_t v0, uint32_t n, cudaStream_t st) {
    if (n == 0) return DYG_OK;
    DYG_CUDA(cudaMemsetAsync(G->g.desc + v0, 0, sizeof(uint2) * n, st));
    DYG_CUDA(cudaMemsetAsync(G->g.cap + v0, 0, sizeof(uint32_t) * n, st));
    return DYG_OK;
}

}  // namespace dyg

extern "C" uint64_t dyg_kernel_launches(void) { return dyg::g_launches.load(); }
