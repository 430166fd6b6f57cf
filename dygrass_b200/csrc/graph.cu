// graph.cu -- device-resident dynamic CSR: upload, in-order append, swap-with-
// last delete, compaction, and the dedup used by decremental recovery.
//
// Every update is applied on the device in the order the reference applies it
// on the host, so row contents (and therefore later walks) are identical:
//   append:  half-edges are listed in commit order (edge e: u<-v then v<-u,
//            random_walk_incremental/gpu_graph.cuh:320-325), stably sorted by
//            row, and each row's run is appended by one thread in list order.
//   delete:  each row's deletions run in input order; a deleted slot takes
//            the row's last live slot (random_walk_decremental/gpu_graph.cuh:359-399).
// Row moves (capacity exceeded) take space from a bump arena: offsets differ
// from run to run but contents never do.
#include <cub/cub.cuh>

#include <atomic>

#include "dyg_internal.cuh"

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

// ------------------------------------------------------------ cub wrappers

dyg_status sort_pairs_u32(Workspace &ws, const uint32_t *keys_in, uint32_t *keys_out,
                          const uint32_t *vals_in, uint32_t *vals_out, uint32_t m,
                          uint32_t key_bits, cudaStream_t st) {
    size_t tmp = 0;
    DYG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys_in, keys_out, vals_in, vals_out,
                                             (int)m, 0, (int)key_bits, st));
    DYG_TRY(ensure(ws.cub_tmp, tmp));
    tmp = ws.cub_tmp.bytes;
    DYG_CUDA(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.p, tmp, keys_in, keys_out, vals_in, vals_out,
                                             (int)m, 0, (int)key_bits, st));
    return DYG_OK;
}

dyg_status exclusive_scan_u32(Workspace &ws, const uint32_t *in, uint32_t *out, uint32_t m,
                              cudaStream_t st) {
    size_t tmp = 0;
    DYG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, in, out, (int)m, st));
    DYG_TRY(ensure(ws.cub_tmp, tmp));
    tmp = ws.cub_tmp.bytes;
    DYG_CUDA(cub::DeviceScan::ExclusiveSum(ws.cub_tmp.p, tmp, in, out, (int)m, st));
    return DYG_OK;
}

uint32_t bits_for(uint32_t n) {
    uint32_t b = 1;
    while (b < 32 && (1ull << b) < (unsigned long long)n) ++b;
    return b;
}

__global__ void k_iota(uint32_t *v, uint32_t m) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) v[i] = i;
}

// ------------------------------------------------------------------ append

__device__ __forceinline__ bool run_head(const uint32_t *k, uint32_t p) {
    return p == 0 || k[p] != k[p - 1];
}
__device__ __forceinline__ uint32_t run_len(const uint32_t *k, uint32_t p, uint32_t m) {
    uint32_t q = p + 1;
    while (q < m && k[q] == k[p]) ++q;
    return q - p;
}

__global__ void k_append_prepare(DevGraph g, const uint32_t *rows, uint32_t m, uint32_t slack,
                                 uint32_t *need, unsigned long long *scalars) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m) return;
    need[p] = 0;
    if (!run_head(rows, p)) return;
    const uint32_t x = rows[p];
    if (x >= g.n) return;
    const uint32_t k = run_len(rows, p, m);
    const uint2 d = g.desc[x];
    const uint32_t newdeg = d.y + k;
    if (newdeg > g.cap[x]) {
        uint32_t nc = max(2u * newdeg, newdeg + slack);
        nc = (nc + 1u) & ~1u;
        need[p] = nc;
        atomicAdd(scalars + S_NEED, (unsigned long long)nc);
    }
}

__global__ void k_append_apply(DevGraph g, const uint32_t *rows, const uint32_t *idx, uint32_t m,
                               const uint32_t *hy, const float *hw, const uint32_t *need) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m || !run_head(rows, p)) return;
    const uint32_t x = rows[p];
    if (x >= g.n) return;
    const uint32_t k = run_len(rows, p, m);
    const uint2 d = g.desc[x];
    uint32_t off = d.x;
    if (need[p]) {
        off = (uint32_t)atomicAdd(g.top, (unsigned long long)need[p]);
        for (uint32_t j = 0; j < d.y; ++j) {
            g.slots[off + j] = g.slots[d.x + j];
            g.wts[off + j] = g.wts[d.x + j];
        }
        g.cap[x] = need[p];
    }
    for (uint32_t q = 0; q < k; ++q) {
        const uint32_t i = idx[p + q];
        g.slots[off + d.y + q] = make_uint2(hy[i], __float_as_uint(__frcp_rn(hw[i])));
        g.wts[off + d.y + q] = hw[i];
    }
    g.desc[x] = make_uint2(off, d.y + k);
}

// Phase 1 of an append: sort the half-edge list by row (stable, so list order
// is kept within a row) and compute each overflowing row's new capacity.
// Entries whose row is >= n (0xFFFFFFFF) sort last and are ignored, so a list
// may be sized by an upper bound.  The relocation total lands in S_NEED.
dyg_status commit_prepare(dyg_graph *G, const uint32_t *hx, uint32_t m, cudaStream_t st) {
    Workspace &ws = G->ws;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    DYG_CUDA(cudaMemsetAsync(sc + S_NEED, 0, sizeof(unsigned long long), st));
    if (m == 0) return DYG_OK;
    DYG_TRY(ensure(ws.skeys, sizeof(uint32_t) * m));
    DYG_TRY(ensure(ws.svals, sizeof(uint32_t) * m));
    DYG_TRY(ensure(ws.need, sizeof(uint32_t) * m * 2));
    uint32_t *iota = ptr<uint32_t>(ws.need) + m;
    const int th = 256;
    const int gr = (int)((m + th - 1) / th);
    k_iota<<<gr, th, 0, st>>>(iota, m);
    count_launch();
    DYG_TRY(sort_pairs_u32(ws, hx, ptr<uint32_t>(ws.skeys), iota, ptr<uint32_t>(ws.svals), m,
                           bits_for(G->g.n + 1u), st));
    k_append_prepare<<<gr, th, 0, st>>>(G->g, ptr<uint32_t>(ws.skeys), m, G->slack,
                                        ptr<uint32_t>(ws.need), sc);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// Phase 2: after the caller has read the scalars (read_scalars), grow the
// arena if the relocations do not fit, then write the rows.
dyg_status commit_finish(dyg_graph *G, const uint32_t *hy, const float *hw, uint32_t m,
                         cudaStream_t st) {
    if (m == 0) return DYG_OK;
    Workspace &ws = G->ws;
    const unsigned long long need = ws.host_scalars[S_NEED];
    const unsigned long long top = ws.host_scalars[S_TOP];
    if (top + need > G->g.arena_cap) DYG_TRY(grow_arena(G, top + need, st));
    const int th = 256;
    const int gr = (int)((m + th - 1) / th);
    k_append_apply<<<gr, th, 0, st>>>(G->g, ptr<uint32_t>(ws.skeys), ptr<uint32_t>(ws.svals), m,
                                      hy, hw, ptr<uint32_t>(ws.need));
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status commit_append(dyg_graph *G, const uint32_t *hx, const uint32_t *hy,
                         const float *hw, uint32_t m, cudaStream_t st) {
    if (m == 0) return DYG_OK;
    DYG_TRY(commit_prepare(G, hx, m, st));
    DYG_TRY(read_scalars(G, st));
    return commit_finish(G, hy, hw, m, st);
}

// ------------------------------------------------------------------ delete

// Half-edge i = 2e + side removes column hy[i] from row rows[p]; runs of one
// row are processed in list order by one thread.  When `mask` is given only
// half-edges whose edge was found on both sides of `mask` are processed.
__global__ void k_delete(DevGraph g, const uint32_t *rows, const uint32_t *idx, uint32_t m,
                         const uint32_t *hy, const uint8_t *mask, uint8_t *found) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m || !run_head(rows, p)) return;
    const uint32_t x = rows[p];
    const uint32_t k = run_len(rows, p, m);
    const uint2 d = g.desc[x];
    uint32_t deg = d.y;
    for (uint32_t q = 0; q < k; ++q) {
        const uint32_t i = idx[p + q];
        if (mask && !(mask[i & ~1u] && mask[i | 1u])) continue;
        const uint32_t y = hy[i];
        for (uint32_t j = 0; j < deg; ++j) {
            if (g.slots[d.x + j].x == y) {
                g.slots[d.x + j] = g.slots[d.x + deg - 1u];
                g.wts[d.x + j] = g.wts[d.x + deg - 1u];
                --deg;
                found[i] = 1;
                break;
            }
        }
    }
    g.desc[x] = make_uint2(d.x, deg);
}

dyg_status delete_half_edges(dyg_graph *G, const uint32_t *sorted_row,
                             const uint32_t *sorted_idx, const uint32_t *hy, uint32_t m,
                             const uint8_t *mask_found, uint8_t *found, cudaStream_t st) {
    if (m == 0) return DYG_OK;
    DYG_CUDA(cudaMemsetAsync(found, 0, m, st));
    const int th = 256;
    k_delete<<<(m + th - 1) / th, th, 0, st>>>(G->g, sorted_row, sorted_idx, m, hy, mask_found, found);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// -------------------------------------------------------------- compaction

__global__ void k_new_caps(DevGraph g, uint32_t slack, uint32_t *caps) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < g.n) caps[v] = g.desc[v].y + slack;
}

__global__ void k_move_rows(DevGraph g, uint2 *ns, float *nw, const uint32_t *off,
                            const uint32_t *caps) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= g.n) return;
    const uint2 d = g.desc[v];
    for (uint32_t j = 0; j < d.y; ++j) {
        ns[off[v] + j] = g.slots[d.x + j];
        nw[off[v] + j] = g.wts[d.x + j];
    }
    g.desc[v] = make_uint2(off[v], d.y);
    g.cap[v] = caps[v];
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
    k_move_rows<<<gr, th, 0, st>>>(G->g, ns, nw, ptr<uint32_t>(ws.pos), ptr<uint32_t>(ws.flags));
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

// ------------------------------------------------------------------- dedup

__device__ __forceinline__ unsigned long long ekey(uint32_t x, uint32_t y) {
    const uint32_t a = min(x, y), b = max(x, y);
    return ((unsigned long long)a << 32) | b;
}
__device__ __forceinline__ uint32_t hslot(unsigned long long k, uint32_t mask) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k & mask;
}

__global__ void k_hash_insert(const uint32_t *cx, const uint32_t *cy, uint32_t m,
                              unsigned long long *tk, uint32_t *tv, uint32_t mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = cx[i], y = cy[i];
    if (x == ~0u || y == ~0u || x == y) return;
    const unsigned long long k = ekey(x, y);
    uint32_t h = hslot(k, mask);
    while (true) {
        const unsigned long long prev = atomicCAS(tk + h, ~0ull, k);
        if (prev == ~0ull || prev == k) {
            atomicMin(tv + h, i);
            return;
        }
        h = (h + 1u) & mask;
    }
}

// keep[i] = candidate i is the first occurrence of its edge and the edge is
// not in H (gpu_graph.cuh:534-538 and 599-601 test sparse_map the same way).
__global__ void k_hash_keep(DevGraph h, const uint32_t *cx, const uint32_t *cy, uint32_t m,
                            const unsigned long long *tk, const uint32_t *tv, uint32_t mask,
                            uint32_t *keep) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t x = cx[i], y = cy[i];
    uint32_t kp = 0;
    if (x != ~0u && y != ~0u && x != y) {
        const unsigned long long k = ekey(x, y);
        uint32_t s = hslot(k, mask);
        while (tk[s] != k) s = (s + 1u) & mask;
        if (tv[s] == i) {
            kp = 1;
            if (x < h.n) {
                const uint2 d = h.desc[x];
                for (uint32_t j = 0; j < d.y; ++j)
                    if (h.slots[d.x + j].x == y) {
                        kp = 0;
                        break;
                    }
            }
        }
    }
    keep[i] = kp;
}

dyg_status dedup_keep(dyg_graph *H, const uint32_t *cx, const uint32_t *cy,
                      uint32_t m, uint32_t *keep, cudaStream_t st) {
    if (m == 0) return DYG_OK;
    Workspace &ws = H->ws;
    uint32_t T = 1024;
    while (T < 2u * m) T <<= 1;
    DYG_TRY(ensure(ws.htab_k, sizeof(unsigned long long) * T));
    DYG_TRY(ensure(ws.htab_v, sizeof(uint32_t) * T));
    DYG_CUDA(cudaMemsetAsync(ws.htab_k.p, 0xFF, sizeof(unsigned long long) * T, st));
    DYG_CUDA(cudaMemsetAsync(ws.htab_v.p, 0xFF, sizeof(uint32_t) * T, st));
    const int th = 256;
    const int gr = (int)((m + th - 1) / th);
    k_hash_insert<<<gr, th, 0, st>>>(cx, cy, m, ptr<unsigned long long>(ws.htab_k),
                                     ptr<uint32_t>(ws.htab_v), T - 1);
    count_launch();
    k_hash_keep<<<gr, th, 0, st>>>(H->g, cx, cy, m, ptr<unsigned long long>(ws.htab_k),
                                   ptr<uint32_t>(ws.htab_v), T - 1, keep);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

}  // namespace dyg

extern "C" uint64_t dyg_kernel_launches(void) { return dyg::g_launches.load(); }
