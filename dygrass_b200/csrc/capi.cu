// capi.cu -- the extern "C" boundary (include/dyg.h): graph handles and the
// incremental / decremental batch and stream entry points.
//
// Batch flow, incremental (one iteration of random_walk_incremental/main.cu:314-340):
//   stage inputs -> walk H (persistent kernel, per-edge winner keys) ->
//   decode flags -> exclusive scan of the accept flags (input order) ->
//   append accepted half-edges to H [-> append every half-edge to G].
// Batch flow, decremental (random_walk_decremental/main.cu:413-444):
//   delete from G and H in input order -> compact the edges found in both ->
//   walk G -> replay winners for their paths -> dedup path edges, drop those
//   in H, append the rest in order -> 2-step fallback walks for the edges
//   without a path, same dedup and append.
#include <math.h>

#include <string>

#include "dyg_internal.cuh"

namespace dyg {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

dyg_status cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    cudaGetLastError();
    set_error(std::string(what) + " failed: " + cudaGetErrorString(e) + " (" + file + ":" +
              std::to_string(line) + ")");
    return DYG_ECUDA;
}

namespace {

struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
            changed = cudaSetDevice(dev) == cudaSuccess;
        }
        cudaGetLastError();
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

bool on_device(const void *p) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

template <typename T>
dyg_status stage_in(Buf &b, const T *p, size_t n, cudaStream_t st, const T **out) {
    if (!p) {
        *out = nullptr;
        return DYG_OK;
    }
    if (on_device(p)) {
        *out = p;
        return DYG_OK;
    }
    DYG_TRY(ensure(b, sizeof(T) * n));
    DYG_CUDA(cudaMemcpyAsync(b.p, p, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    *out = ptr<T>(b);
    return DYG_OK;
}

template <typename T>
dyg_status copy_out(T *dst, const T *src_dev, size_t n, cudaStream_t st, bool *host_out) {
    if (!dst || n == 0) return DYG_OK;
    const bool dev = on_device(dst);
    if (!dev) *host_out = true;
    DYG_CUDA(cudaMemcpyAsync(dst, src_dev, sizeof(T) * n,
                             dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    return DYG_OK;
}

dyg_status check_params(const dyg_walk_params *p) {
    if (!p) {
        set_error("walk params are NULL");
        return DYG_EINVAL;
    }
    if (p->walkers == 0 || p->walkers % 32 != 0 || p->walkers > 1024) {
        set_error("walkers must be a positive multiple of 32 and <= 1024");
        return DYG_EINVAL;
    }
    if (p->max_steps < 1 || p->max_steps > 0x3FFFFF) {
        set_error("max_steps must be in [1, 4194303]");
        return DYG_EINVAL;
    }
    if (p->transition > DYG_TRANSITION_WEIGHTED) {
        set_error("unknown transition rule");
        return DYG_EINVAL;
    }
    if (p->heuristic_walkers > 1024) {
        set_error("heuristic_walkers must be <= 1024");
        return DYG_EINVAL;
    }
    return DYG_OK;
}

dyg_status check_host_ids(const uint32_t *v, size_t n, uint32_t nv, const char *what) {
    if (!v || on_device(v)) return DYG_OK;
    for (size_t i = 0; i < n; ++i)
        if (v[i] >= nv) {
            set_error(std::string(what) + "[" + std::to_string(i) + "] = " + std::to_string(v[i]) +
                      " is not a vertex (n = " + std::to_string(nv) + ")");
            return DYG_EINVAL;
        }
    return DYG_OK;
}

dyg_status check_host_weights(const float *w, size_t n) {
    if (!w || on_device(w)) return DYG_OK;
    for (size_t i = 0; i < n; ++i)
        if (!(w[i] > 0.0f) || !isfinite(w[i])) {
            set_error("weight[" + std::to_string(i) + "] is not finite and > 0");
            return DYG_EINVAL;
        }
    return DYG_OK;
}

dyg_status check_device_errors(dyg_graph *G, cudaStream_t st) {
    DYG_TRY(read_scalars(G, st));
    const unsigned long long err = G->ws.host_scalars[S_ERR];
    if (err) {
        unsigned long long zero = 0;
        DYG_CUDA(cudaMemcpy(ptr<unsigned long long>(G->ws.scalars) + S_ERR, &zero, sizeof(zero),
                            cudaMemcpyHostToDevice));
        if (err & kErrVertex) {
            set_error("a batch endpoint is not a vertex of the graph");
            return DYG_EINVAL;
        }
        set_error("internal consistency check failed (device error bits " + std::to_string(err) + ")");
        return DYG_ESTATE;
    }
    return DYG_OK;
}

// ----------------------------------------------------------- small kernels

__global__ void k_incr_decode(const unsigned long long *keys, uint32_t n, int32_t *found,
                              float *cond, uint8_t *acc, uint32_t *flags) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const unsigned long long k = keys[e];
    found[e] = key_found(k);
    cond[e] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
    acc[e] = k ? 0 : 1;
    flags[e] = k ? 0u : 1u;
}

// Half-edges of the accepted edges, in input order (u gets v, then v gets u:
// random_walk_incremental/gpu_graph.cuh:320-325).  flags == null: all edges.
__global__ void k_half_edges(const uint32_t *src, const uint32_t *dst, const float *w, uint32_t n,
                             const uint32_t *flags, const uint32_t *pos, uint32_t *hx, uint32_t *hy,
                             float *hw, uint32_t *count) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (flags && e == n - 1 && count) *count = pos[e] + flags[e];
    if (flags && !flags[e]) return;
    const uint32_t q = flags ? pos[e] : e;
    const uint32_t u = src[e], v = dst[e];
    const float ww = w[e];
    hx[2 * q] = u;
    hy[2 * q] = v;
    hw[2 * q] = ww;
    hx[2 * q + 1] = v;
    hy[2 * q + 1] = u;
    hw[2 * q + 1] = ww;
}

// Deletion half-edges with endpoints ordered min -> max
// (random_walk_decremental/gpu_graph.cuh:340-343).
__global__ void k_del_half_edges(const uint32_t *src, const uint32_t *dst, uint32_t n,
                                 uint32_t nv, uint32_t *hx, uint32_t *hy,
                                 unsigned long long *scalars) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    uint32_t a = src[e], b = dst[e];
    if (a > b) {
        const uint32_t t = a;
        a = b;
        b = t;
    }
    if (b >= nv) {
        atomicOr(scalars + S_ERR, (unsigned long long)kErrVertex);
        a = b = nv ? nv - 1 : 0;   // harmless self-pair: never found
    }
    hx[2 * e] = a;
    hy[2 * e] = b;
    hx[2 * e + 1] = b;
    hy[2 * e + 1] = a;
}

__global__ void k_del_filter(const uint8_t *fG, const uint8_t *fH, uint32_t n, uint32_t *flags,
                             int32_t *status, float *cond) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const bool inG = fG[2 * e] && fG[2 * e + 1];
    const bool inH = inG && fH[2 * e] && fH[2 * e + 1];
    flags[e] = inH ? 1u : 0u;
    status[e] = !inG ? DYG_DEL_NOT_IN_G : (!inH ? DYG_DEL_NOT_IN_H : DYG_DEL_NO_PATH);
    cond[e] = 0.f;
}

__global__ void k_del_compact(const uint32_t *hx, const uint32_t *hy, uint32_t n,
                              const uint32_t *flags, const uint32_t *pos,
                              unsigned long long uid0, uint32_t *f_src, uint32_t *f_dst,
                              unsigned long long *f_uid, uint32_t *f_idx, uint32_t *count) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (e == n - 1) *count = pos[e] + flags[e];
    if (!flags[e]) return;
    const uint32_t f = pos[e];
    f_src[f] = hx[2 * e];   // min
    f_dst[f] = hy[2 * e];   // max
    f_uid[f] = uid0 + e;
    f_idx[f] = e;
}

// Per filtered edge: status / conductance, path-candidate counts and the
// no-path flags (for f >= F everything is zero).
__global__ void k_decr_results(const unsigned long long *keys, const int32_t *plen,
                               const uint32_t *f_idx, const uint32_t *F_dev, uint32_t n,
                               int32_t *status, float *cond, uint32_t *clen, uint32_t *noflag) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    const uint32_t F = *F_dev;
    if (f >= F) {
        clen[f] = 0;
        noflag[f] = 0;
        return;
    }
    const uint32_t e = f_idx[f];
    const int32_t L = plen[f];
    const unsigned long long k = keys[f];
    status[e] = L > 0 ? L : DYG_DEL_NO_PATH;
    cond[e] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
    clen[f] = L > 0 ? (uint32_t)L : 0u;
    noflag[f] = L > 0 ? 0u : 1u;
}

__global__ void k_path_cands(const uint32_t *pv, const float *pw, uint32_t stride,
                             const uint32_t *clen, const uint32_t *coff, uint32_t n,
                             const uint32_t *noflag, const uint32_t *nopos, uint32_t *cx,
                             uint32_t *cy, float *cw, uint32_t *nop, uint32_t *counts) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
    if (f == n - 1) {
        counts[C_CANDS] = coff[f] + clen[f];
        counts[C_NOPATH] = nopos[f] + noflag[f];
    }
    if (noflag[f]) nop[nopos[f]] = f;
    const uint32_t L = clen[f];
    const uint32_t base = coff[f];
    const uint32_t *v = pv + (size_t)f * stride;
    const float *w = pw + (size_t)f * stride;
    for (uint32_t j = 0; j < L; ++j) {
        cx[base + j] = v[j];
        cy[base + j] = v[j + 1];
        cw[base + j] = w[j + 1];
    }
}

// Kept candidates -> half-edges (x gets y, then y gets x) and the recovered
// edge record.
__global__ void k_emit_kept(const uint32_t *cx, const uint32_t *cy, const float *cw, uint32_t m,
                            const uint32_t *keep, const uint32_t *kpos, uint8_t kind,
                            uint32_t rec_base, uint32_t *hx, uint32_t *hy, float *hw,
                            uint32_t *rx, uint32_t *ry, uint8_t *rk, uint32_t *counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (i == m - 1) counts[C_KEPT] = kpos[i] + keep[i];
    if (!keep[i]) return;
    const uint32_t q = kpos[i];
    const uint32_t x = cx[i], y = cy[i];
    const float w = cw[i];
    hx[2 * q] = x;
    hy[2 * q] = y;
    hw[2 * q] = w;
    hx[2 * q + 1] = y;
    hy[2 * q + 1] = x;
    hw[2 * q + 1] = w;
    rx[rec_base + q] = x;
    ry[rec_base + q] = y;
    rk[rec_base + q] = kind;
}

inline int blocks(uint64_t n, int th) { return (int)((n + th - 1) / th); }

// Dedup + membership + append of one candidate list; appends the recovered
// edges after rec_base in the stream-level record buffers.
dyg_status recover_round(dyg_graph *G, dyg_graph *H, const uint32_t *cx, const uint32_t *cy,
                         const float *cw, uint32_t m, uint8_t kind, uint32_t rec_base,
                         uint32_t *rx, uint32_t *ry, uint8_t *rk, uint32_t *kept, cudaStream_t st) {
    *kept = 0;
    if (m == 0) return DYG_OK;
    Workspace &ws = G->ws;
    DYG_TRY(ensure(ws.keep, sizeof(uint32_t) * (size_t)m * 2));
    uint32_t *keep = ptr<uint32_t>(ws.keep);
    uint32_t *kpos = keep + m;
    DYG_TRY(dedup_keep(H, cx, cy, m, keep, st));
    DYG_TRY(exclusive_scan_u32(ws, keep, kpos, m, st));
    DYG_TRY(ensure(ws.hx, sizeof(uint32_t) * (size_t)m * 2));
    DYG_TRY(ensure(ws.hy, sizeof(uint32_t) * (size_t)m * 2));
    DYG_TRY(ensure(ws.hw, sizeof(float) * (size_t)m * 2));
    k_emit_kept<<<blocks(m, 256), 256, 0, st>>>(cx, cy, cw, m, keep, kpos, kind, rec_base,
                                                 ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy),
                                                 ptr<float>(ws.hw), rx, ry, rk,
                                                 ptr<uint32_t>(ws.counts));
    count_launch();
    DYG_CUDA(cudaGetLastError());
    DYG_TRY(read_scalars(G, st));
    *kept = ws.host_counts[C_KEPT];
    DYG_TRY(commit_append(H, ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw),
                          2u * *kept, st));
    return DYG_OK;
}

dyg_status graph_alloc_scalars(dyg_graph *G) {
    DYG_TRY(ensure(G->ws.scalars, sizeof(unsigned long long) * S_NSCALARS));
    DYG_TRY(ensure(G->ws.counts, sizeof(uint32_t) * C_NCOUNTS));
    DYG_CUDA(cudaMemset(G->ws.scalars.p, 0, sizeof(unsigned long long) * S_NSCALARS));
    DYG_CUDA(cudaMemset(G->ws.counts.p, 0, sizeof(uint32_t) * C_NCOUNTS));
    DYG_CUDA(cudaMallocHost(&G->ws.host_scalars, sizeof(unsigned long long) * S_NSCALARS));
    DYG_CUDA(cudaMallocHost(&G->ws.host_counts, sizeof(uint32_t) * C_NCOUNTS));
    G->g.top = ptr<unsigned long long>(G->ws.scalars) + S_TOP;
    return DYG_OK;
}

void free_buf(Buf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

void free_graph(dyg_graph *G) {
    if (!G) return;
    DeviceGuard dg(G->device);
    Workspace &ws = G->ws;
    Buf *bufs[] = {&ws.in_src, &ws.in_dst, &ws.in_w, &ws.keys, &ws.work, &ws.flags, &ws.pos,
                   &ws.f_src, &ws.f_dst, &ws.f_idx, &ws.f_uid, &ws.found, &ws.hx, &ws.hy,
                   &ws.hw, &ws.hseq, &ws.skeys, &ws.svals, &ws.need, &ws.path_v, &ws.path_w,
                   &ws.path_len, &ws.cand_x, &ws.cand_y, &ws.cand_w, &ws.keep, &ws.htab_k,
                   &ws.htab_v, &ws.nop, &ws.rec_x, &ws.rec_y, &ws.rec_k, &ws.out_found,
                   &ws.out_cond, &ws.out_acc, &ws.out_status, &ws.cub_tmp, &ws.s_src, &ws.s_dst,
                   &ws.s_w, &ws.s_o1, &ws.s_o2, &ws.s_o3, &ws.rx2, &ws.ry2, &ws.rk2,
                   &ws.scalars, &ws.counts};
    for (Buf *b : bufs) free_buf(*b);
    if (ws.host_scalars) cudaFreeHost(ws.host_scalars);
    if (ws.host_counts) cudaFreeHost(ws.host_counts);
    if (G->g.desc) cudaFree(G->g.desc);
    if (G->g.cap) cudaFree(G->g.cap);
    if (G->g.slots) cudaFree(G->g.slots);
    if (G->g.wts) cudaFree(G->g.wts);
    cudaGetLastError();
    delete G;
}

// ------------------------------------------------------------ incremental

dyg_status incremental_batch_dev(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n, uint64_t uid0,
                                 const dyg_walk_params &p, cudaStream_t st) {
    Workspace &ws = H->ws;
    DYG_TRY(ensure(ws.keys, sizeof(unsigned long long) * n));
    DYG_TRY(ensure(ws.flags, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.pos, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.out_found, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.out_cond, sizeof(float) * n));
    DYG_TRY(ensure(ws.out_acc, sizeof(uint8_t) * n));
    DYG_TRY(ensure(ws.hx, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(ws.hy, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(ws.hw, sizeof(float) * (size_t)n * 2));
    unsigned long long *keys = ptr<unsigned long long>(ws.keys);
    DYG_CUDA(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * n, st));
    // unused entries of the accepted half-edge list stay 0xFFFFFFFF (ignored)
    DYG_CUDA(cudaMemsetAsync(ws.hx.p, 0xFF, sizeof(uint32_t) * (size_t)n * 2, st));
    WalkJob job{src, dst, w, nullptr, (unsigned long long)uid0, nullptr, n, kDomainIncr};
    DYG_TRY(launch_walk(H, job, p, true, keys, st));
    k_incr_decode<<<blocks(n, 256), 256, 0, st>>>(keys, n, ptr<int32_t>(ws.out_found),
                                                   ptr<float>(ws.out_cond), ptr<uint8_t>(ws.out_acc),
                                                   ptr<uint32_t>(ws.flags));
    count_launch();
    DYG_TRY(exclusive_scan_u32(ws, ptr<uint32_t>(ws.flags), ptr<uint32_t>(ws.pos), n, st));
    k_half_edges<<<blocks(n, 256), 256, 0, st>>>(src, dst, w, n, ptr<uint32_t>(ws.flags),
                                                  ptr<uint32_t>(ws.pos), ptr<uint32_t>(ws.hx),
                                                  ptr<uint32_t>(ws.hy), ptr<float>(ws.hw),
                                                  ptr<uint32_t>(ws.counts) + C_ACCEPTED);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    // both commits are sized by the upper bound 2n, so one synchronize serves
    // the error check and both arena checks
    DYG_TRY(commit_prepare(H, ptr<uint32_t>(ws.hx), 2u * n, st));
    if (G) {
        Workspace &wg = G->ws;
        DYG_TRY(ensure(wg.hx, sizeof(uint32_t) * (size_t)n * 2));
        DYG_TRY(ensure(wg.hy, sizeof(uint32_t) * (size_t)n * 2));
        DYG_TRY(ensure(wg.hw, sizeof(float) * (size_t)n * 2));
        k_half_edges<<<blocks(n, 256), 256, 0, st>>>(src, dst, w, n, nullptr, nullptr,
                                                      ptr<uint32_t>(wg.hx), ptr<uint32_t>(wg.hy),
                                                      ptr<float>(wg.hw), nullptr);
        count_launch();
        DYG_CUDA(cudaGetLastError());
        DYG_TRY(commit_prepare(G, ptr<uint32_t>(wg.hx), 2u * n, st));
    }
    DYG_TRY(read_scalars2(H, G, st));
    const unsigned long long err = ws.host_scalars[S_ERR];
    if (err) DYG_TRY(check_device_errors(H, st));
    DYG_TRY(commit_finish(H, ptr<uint32_t>(ws.hy), ptr<float>(ws.hw), 2u * n, st));
    if (G) DYG_TRY(commit_finish(G, ptr<uint32_t>(G->ws.hy), ptr<float>(G->ws.hw), 2u * n, st));
    return DYG_OK;
}

// ------------------------------------------------------------ decremental

dyg_status decremental_batch_dev(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                 const uint32_t *dst, uint32_t n, uint64_t uid0,
                                 const dyg_walk_params &p, uint32_t rec_base, uint32_t *rx,
                                 uint32_t *ry, uint8_t *rk, uint32_t *n_rec, cudaStream_t st) {
    Workspace &ws = G->ws;
    *n_rec = 0;
    const uint32_t m = 2u * n;
    const uint32_t stride = p.max_steps > 2 ? p.max_steps : 2;
    DYG_TRY(ensure(ws.hx, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.hy, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.skeys, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.svals, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.need, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.found, (size_t)m * 2));
    DYG_TRY(ensure(ws.flags, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.pos, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_src, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_dst, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_idx, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_uid, sizeof(unsigned long long) * n));
    DYG_TRY(ensure(ws.keys, sizeof(unsigned long long) * n));
    DYG_TRY(ensure(ws.out_status, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.out_cond, sizeof(float) * n));
    DYG_TRY(ensure(ws.path_v, sizeof(uint32_t) * (size_t)n * stride));
    DYG_TRY(ensure(ws.path_w, sizeof(float) * (size_t)n * stride));
    DYG_TRY(ensure(ws.path_len, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.nop, sizeof(uint32_t) * (size_t)n * 4));
    uint32_t *hx = ptr<uint32_t>(ws.hx), *hy = ptr<uint32_t>(ws.hy);
    uint8_t *fG = ptr<uint8_t>(ws.found), *fH = fG + m;
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);

    // 1. delete from G, then from H the edges found in G (gpu_graph.cuh:338-458)
    k_del_half_edges<<<blocks(n, 256), 256, 0, st>>>(src, dst, n, G->g.n, hx, hy, sc);
    count_launch();
    k_iota<<<blocks(m, 256), 256, 0, st>>>(ptr<uint32_t>(ws.need), m);
    count_launch();
    DYG_TRY(sort_pairs_u32(ws, hx, ptr<uint32_t>(ws.skeys), ptr<uint32_t>(ws.need),
                           ptr<uint32_t>(ws.svals), m, bits_for(G->g.n), st));
    DYG_TRY(delete_half_edges(G, ptr<uint32_t>(ws.skeys), ptr<uint32_t>(ws.svals), hy, m, nullptr,
                              fG, st));
    DYG_TRY(delete_half_edges(H, ptr<uint32_t>(ws.skeys), ptr<uint32_t>(ws.svals), hy, m, fG, fH,
                              st));
    int32_t *status = ptr<int32_t>(ws.out_status);
    float *cond = ptr<float>(ws.out_cond);
    k_del_filter<<<blocks(n, 256), 256, 0, st>>>(fG, fH, n, ptr<uint32_t>(ws.flags), status, cond);
    count_launch();
    DYG_TRY(exclusive_scan_u32(ws, ptr<uint32_t>(ws.flags), ptr<uint32_t>(ws.pos), n, st));
    k_del_compact<<<blocks(n, 256), 256, 0, st>>>(hx, hy, n, ptr<uint32_t>(ws.flags),
                                                   ptr<uint32_t>(ws.pos), uid0,
                                                   ptr<uint32_t>(ws.f_src), ptr<uint32_t>(ws.f_dst),
                                                   ptr<unsigned long long>(ws.f_uid),
                                                   ptr<uint32_t>(ws.f_idx), counts + C_FILTERED);
    count_launch();
    DYG_CUDA(cudaGetLastError());

    // 2. walks on the updated G (main.cu:392, 420); F stays on the device
    unsigned long long *keys = ptr<unsigned long long>(ws.keys);
    DYG_CUDA(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * n, st));
    WalkJob job{ptr<uint32_t>(ws.f_src), ptr<uint32_t>(ws.f_dst), nullptr,
                ptr<unsigned long long>(ws.f_uid), 0ull, counts + C_FILTERED, n, kDomainDecr};
    DYG_TRY(launch_walk(G, job, p, false, keys, st));
    DYG_TRY(launch_winner_paths(G, job, p, keys, n, stride, ptr<uint32_t>(ws.path_v),
                                ptr<float>(ws.path_w), ptr<int32_t>(ws.path_len), st));

    // 3. path candidates in (edge, step) order; no-path list
    uint32_t *clen = ptr<uint32_t>(ws.nop) + n, *coff = clen + n, *noflag = coff + n,
             *nopos = ptr<uint32_t>(ws.flags);
    k_decr_results<<<blocks(n, 256), 256, 0, st>>>(keys, ptr<int32_t>(ws.path_len),
                                                    ptr<uint32_t>(ws.f_idx), counts + C_FILTERED, n,
                                                    status, cond, clen, noflag);
    count_launch();
    DYG_TRY(exclusive_scan_u32(ws, clen, coff, n, st));
    DYG_TRY(exclusive_scan_u32(ws, noflag, nopos, n, st));
    DYG_TRY(check_device_errors(G, st));   // syncs; needs the candidate-buffer size next
    // candidate count upper bound: F * (stride - 1)
    const uint32_t F = ws.host_counts[C_FILTERED];
    const size_t cmax = (size_t)(F ? F : 1) * stride;
    DYG_TRY(ensure(ws.cand_x, sizeof(uint32_t) * cmax));
    DYG_TRY(ensure(ws.cand_y, sizeof(uint32_t) * cmax));
    DYG_TRY(ensure(ws.cand_w, sizeof(float) * cmax));
    k_path_cands<<<blocks(n, 256), 256, 0, st>>>(ptr<uint32_t>(ws.path_v), ptr<float>(ws.path_w),
                                                  stride, clen, coff, n, noflag, nopos,
                                                  ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                                                  ptr<float>(ws.cand_w), ptr<uint32_t>(ws.nop), counts);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    DYG_TRY(read_scalars(G, st));
    const uint32_t M = ws.host_counts[C_CANDS];
    const uint32_t NOP = ws.host_counts[C_NOPATH];

    // 4. path recovery (gpu_graph.cuh:514-552)
    uint32_t kept1 = 0, kept2 = 0;
    DYG_TRY(recover_round(G, H, ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                          ptr<float>(ws.cand_w), M, DYG_REC_PATH, rec_base, rx, ry, rk, &kept1, st));

    // 5. fallback walks for edges without a path (main.cu:400-408, 428-436)
    if (NOP > 0 && p.heuristic_walkers > 0) {
        const size_t hm = (size_t)NOP * 4u * p.heuristic_walkers;
        DYG_TRY(ensure(ws.cand_x, sizeof(uint32_t) * hm));
        DYG_TRY(ensure(ws.cand_y, sizeof(uint32_t) * hm));
        DYG_TRY(ensure(ws.cand_w, sizeof(float) * hm));
        DYG_TRY(launch_fallback_walks(G, ptr<uint32_t>(ws.f_src), ptr<uint32_t>(ws.f_dst),
                                      ptr<unsigned long long>(ws.f_uid), ptr<uint32_t>(ws.nop), NOP,
                                      p, ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                                      ptr<float>(ws.cand_w), st));
        DYG_TRY(recover_round(G, H, ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                              ptr<float>(ws.cand_w), (uint32_t)hm, DYG_REC_FALLBACK,
                              rec_base + kept1, rx, ry, rk, &kept2, st));
    }
    *n_rec = kept1 + kept2;
    return DYG_OK;
}

// Grows b to `bytes`, keeping its first `used` bytes.
dyg_status grow_keep(Buf &b, size_t bytes, size_t used, cudaStream_t st) {
    if (b.bytes >= bytes) return DYG_OK;
    Buf nb;
    DYG_TRY(ensure(nb, bytes));
    if (used && b.p) {
        DYG_CUDA(cudaMemcpyAsync(nb.p, b.p, used, cudaMemcpyDeviceToDevice, st));
        DYG_CUDA(cudaStreamSynchronize(st));
    }
    free_buf(b);
    b = nb;
    return DYG_OK;
}

dyg_status ensure_records(Workspace &ws, uint64_t used, uint64_t need, cudaStream_t st) {
    DYG_TRY(grow_keep(ws.rx2, sizeof(uint32_t) * need, sizeof(uint32_t) * used, st));
    DYG_TRY(grow_keep(ws.ry2, sizeof(uint32_t) * need, sizeof(uint32_t) * used, st));
    DYG_TRY(grow_keep(ws.rk2, need, used, st));
    return DYG_OK;
}

}  // namespace
}  // namespace dyg

using namespace dyg;

// ======================================================================= ABI

extern "C" {

const char *dyg_version(void) { return "dygrass_b200 0.1.0 (sm_100a)"; }

const char *dyg_last_error_string(void) { return g_last_error.c_str(); }

void dyg_walk_params_default(dyg_walk_params *p) {
    if (!p) return;
    p->threshold = 100.0f;
    p->walkers = 512;
    p->max_steps = 100;
    p->transition = DYG_TRANSITION_UNIFORM;
    p->heuristic_walkers = 16;
    p->flags = 0;
    p->seed = 20251203ull;
}

void dyg_graph_opts_default(dyg_graph_opts *o) {
    if (!o) return;
    o->slack_per_row = 2;
    o->reserved = 0;
    o->arena_headroom = 0.5;
    o->device = -1;
    o->pad = 0;
}

uint32_t dyg_reference_batch_size(uint32_t n) {
    const uint32_t b = (uint32_t)(((uint64_t)n + 9u) / 10u);
    return b ? b : 1u;
}

dyg_status dyg_graph_create_from_edges(uint32_t n_vertices, uint64_t n_edges, const uint32_t *src,
                                       const uint32_t *dst, const float *w,
                                       const dyg_graph_opts *opts, dyg_graph **out) {
    set_error("");
    if (!out || (n_edges && (!src || !dst || !w))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    *out = nullptr;
    if (n_edges > 0x7FFFFFFFull) {
        set_error("too many edges");
        return DYG_EINVAL;
    }
    DYG_TRY(check_host_ids(src, n_edges, n_vertices, "src"));
    DYG_TRY(check_host_ids(dst, n_edges, n_vertices, "dst"));
    DYG_TRY(check_host_weights(w, n_edges));
    dyg_graph_opts o;
    dyg_graph_opts_default(&o);
    if (opts) o = *opts;
    int dev = o.device;
    if (dev < 0) DYG_CUDA(cudaGetDevice(&dev));
    DeviceGuard dg(dev);
    // rows in file order (functions.cpp:130-232): count, prefix, fill
    uint64_t *row_ptr = (uint64_t *)calloc((size_t)n_vertices + 1, sizeof(uint64_t));
    uint32_t *col = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(2 * n_edges + 1));
    float *ww = (float *)malloc(sizeof(float) * (size_t)(2 * n_edges + 1));
    uint64_t *fill = (uint64_t *)calloc((size_t)n_vertices + 1, sizeof(uint64_t));
    if (!row_ptr || !col || !ww || !fill) {
        free(row_ptr); free(col); free(ww); free(fill);
        set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    for (uint64_t i = 0; i < n_edges; ++i) {
        row_ptr[src[i] + 1]++;
        row_ptr[dst[i] + 1]++;
    }
    for (uint32_t v = 0; v < n_vertices; ++v) row_ptr[v + 1] += row_ptr[v];
    for (uint64_t i = 0; i < n_edges; ++i) {
        const uint32_t s = src[i], d = dst[i];
        uint64_t ps = row_ptr[s] + fill[s]++;
        col[ps] = d;
        ww[ps] = w[i];
        uint64_t pd = row_ptr[d] + fill[d]++;
        col[pd] = s;
        ww[pd] = w[i];
    }
    dyg_graph *G = new dyg_graph();
    G->device = dev;
    G->slack = o.slack_per_row;
    G->headroom = o.arena_headroom > 0 ? o.arena_headroom : 0.0;
    dyg_status rc = graph_alloc_scalars(G);
    if (rc == DYG_OK) rc = upload_graph(G, n_vertices, row_ptr, col, ww);
    free(row_ptr); free(col); free(ww); free(fill);
    if (rc != DYG_OK) {
        free_graph(G);
        return rc;
    }
    *out = G;
    return DYG_OK;
}

dyg_status dyg_graph_copy_from(dyg_graph *dst, const dyg_graph *src, dyg_stream_t stream) {
    set_error("");
    if (!dst || !src || dst->g.n != src->g.n || dst->device != src->device) {
        set_error("copy_from needs two graphs with the same vertex count on one device");
        return DYG_EINVAL;
    }
    DeviceGuard dg(dst->device);
    cudaStream_t st = (cudaStream_t)stream;
    dyg_graph *s = const_cast<dyg_graph *>(src);
    DYG_TRY(read_scalars(s, st));
    const unsigned long long top = s->ws.host_scalars[S_TOP];
    if (dst->g.arena_cap < top) {
        uint2 *ns = nullptr;
        float *nw = nullptr;
        if (cudaMalloc(&ns, sizeof(uint2) * (size_t)src->g.arena_cap) != cudaSuccess ||
            cudaMalloc(&nw, sizeof(float) * (size_t)src->g.arena_cap) != cudaSuccess) {
            cudaGetLastError();
            if (ns) cudaFree(ns);
            set_error("cudaMalloc in copy_from failed");
            return DYG_ENOMEM;
        }
        DYG_CUDA(cudaFree(dst->g.slots));
        DYG_CUDA(cudaFree(dst->g.wts));
        dst->g.slots = ns;
        dst->g.wts = nw;
        dst->g.arena_cap = src->g.arena_cap;
    }
    const uint32_t n = src->g.n;
    DYG_CUDA(cudaMemcpyAsync(dst->g.desc, src->g.desc, sizeof(uint2) * n, cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(dst->g.cap, src->g.cap, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(dst->g.slots, src->g.slots, sizeof(uint2) * (size_t)top,
                             cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(dst->g.wts, src->g.wts, sizeof(float) * (size_t)top,
                             cudaMemcpyDeviceToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(dst->g.top, src->g.top, sizeof(unsigned long long),
                             cudaMemcpyDeviceToDevice, st));
    dst->slack = src->slack;
    dst->headroom = src->headroom;
    return DYG_OK;
}

dyg_status dyg_graph_clone(const dyg_graph *g, dyg_graph **out) {
    set_error("");
    if (!g || !out) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DeviceGuard dg(g->device);
    dyg_graph *G = new dyg_graph();
    G->device = g->device;
    G->slack = g->slack;
    G->headroom = g->headroom;
    G->g.n = g->g.n;
    G->g.arena_cap = g->g.arena_cap;
    dyg_status rc = graph_alloc_scalars(G);
    if (rc == DYG_OK &&
        (cudaMalloc(&G->g.desc, sizeof(uint2) * (size_t)(g->g.n ? g->g.n : 1)) != cudaSuccess ||
         cudaMalloc(&G->g.cap, sizeof(uint32_t) * (size_t)(g->g.n ? g->g.n : 1)) != cudaSuccess ||
         cudaMalloc(&G->g.slots, sizeof(uint2) * (size_t)g->g.arena_cap) != cudaSuccess ||
         cudaMalloc(&G->g.wts, sizeof(float) * (size_t)g->g.arena_cap) != cudaSuccess)) {
        cudaGetLastError();
        set_error("cudaMalloc in clone failed");
        rc = DYG_ENOMEM;
    }
    if (rc == DYG_OK) rc = dyg_graph_copy_from(G, g, nullptr);
    if (rc == DYG_OK && cudaDeviceSynchronize() != cudaSuccess) rc = cuda_fail(cudaGetLastError(), "clone", __FILE__, __LINE__);
    if (rc != DYG_OK) {
        free_graph(G);
        return rc;
    }
    *out = G;
    return DYG_OK;
}

dyg_status dyg_graph_destroy(dyg_graph *g) {
    if (!g) return DYG_OK;
    {
        DeviceGuard dg(g->device);
        cudaDeviceSynchronize();
    }
    free_graph(g);
    return DYG_OK;
}

dyg_status dyg_graph_info(const dyg_graph *g, uint32_t *n_vertices, uint64_t *n_slots,
                          uint64_t *arena_used, uint64_t *arena_cap) {
    set_error("");
    if (!g) {
        set_error("NULL graph");
        return DYG_EINVAL;
    }
    DeviceGuard dg(g->device);
    dyg_graph *G = const_cast<dyg_graph *>(g);
    DYG_TRY(read_scalars(G, nullptr));
    if (n_vertices) *n_vertices = g->g.n;
    if (arena_used) *arena_used = G->ws.host_scalars[S_TOP];
    if (arena_cap) *arena_cap = g->g.arena_cap;
    if (n_slots) {
        uint2 *h = (uint2 *)malloc(sizeof(uint2) * (size_t)(g->g.n ? g->g.n : 1));
        if (!h) {
            set_error("host allocation failed");
            return DYG_ENOMEM;
        }
        cudaError_t e = cudaMemcpy(h, g->g.desc, sizeof(uint2) * g->g.n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            free(h);
            return cuda_fail(e, "info", __FILE__, __LINE__);
        }
        uint64_t s = 0;
        for (uint32_t v = 0; v < g->g.n; ++v) s += h[v].y;
        free(h);
        *n_slots = s;
    }
    return DYG_OK;
}

dyg_status dyg_graph_export(dyg_graph *g, uint64_t *row_ptr, uint32_t *col, float *w,
                            uint64_t slot_cap) {
    set_error("");
    if (!g || !row_ptr) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DeviceGuard dg(g->device);
    DYG_CUDA(cudaDeviceSynchronize());
    DYG_TRY(read_scalars(g, nullptr));
    const unsigned long long top = g->ws.host_scalars[S_TOP];
    const uint32_t n = g->g.n;
    uint2 *hd = (uint2 *)malloc(sizeof(uint2) * (size_t)(n ? n : 1));
    uint2 *hs = (uint2 *)malloc(sizeof(uint2) * (size_t)(top ? top : 1));
    float *hw = (float *)malloc(sizeof(float) * (size_t)(top ? top : 1));
    if (!hd || !hs || !hw) {
        free(hd); free(hs); free(hw);
        set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    cudaError_t e = cudaMemcpy(hd, g->g.desc, sizeof(uint2) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hs, g->g.slots, sizeof(uint2) * (size_t)top, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hw, g->g.wts, sizeof(float) * (size_t)top, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        free(hd); free(hs); free(hw);
        return cuda_fail(e, "export", __FILE__, __LINE__);
    }
    uint64_t o = 0;
    dyg_status rc = DYG_OK;
    for (uint32_t v = 0; v < n; ++v) {
        row_ptr[v] = o;
        for (uint32_t j = 0; j < hd[v].y; ++j) {
            if (o + j < slot_cap) {
                if (col) col[o + j] = hs[hd[v].x + j].x;
                if (w) w[o + j] = hw[hd[v].x + j];
            } else {
                rc = DYG_ERANGE;
            }
        }
        o += hd[v].y;
    }
    row_ptr[n] = o;
    free(hd);
    free(hs);
    free(hw);
    if (rc != DYG_OK) set_error("slot_cap smaller than the number of slots");
    return rc;
}

dyg_status dyg_graph_compact(dyg_graph *g, dyg_stream_t stream) {
    set_error("");
    if (!g) {
        set_error("NULL graph");
        return DYG_EINVAL;
    }
    DeviceGuard dg(g->device);
    return compact_graph(g, (cudaStream_t)stream);
}

dyg_status dyg_graph_counters(const dyg_graph *g, uint64_t *walker_moves, uint64_t *walks) {
    set_error("");
    if (!g) {
        set_error("NULL graph");
        return DYG_EINVAL;
    }
    DeviceGuard dg(g->device);
    dyg_graph *G = const_cast<dyg_graph *>(g);
    DYG_CUDA(cudaDeviceSynchronize());
    DYG_TRY(read_scalars(G, nullptr));
    if (walker_moves) *walker_moves = G->ws.host_scalars[S_MOVES];
    if (walks) *walks = G->ws.host_scalars[S_WALKS];
    return DYG_OK;
}

dyg_status dyg_incremental_batch(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n,
                                 uint64_t first_update_id, const dyg_walk_params *p,
                                 int32_t *found_at, float *conductance, uint8_t *accepted,
                                 dyg_stream_t stream) {
    set_error("");
    if (!H || (n && (!src || !dst || !w))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DYG_TRY(check_params(p));
    if (G && (G->g.n != H->g.n || G->device != H->device)) {
        set_error("G and H must have the same vertex count and device");
        return DYG_EINVAL;
    }
    if (n == 0) return DYG_OK;
    DeviceGuard dg(H->device);
    cudaStream_t st = (cudaStream_t)stream;
    DYG_TRY(check_host_ids(src, n, H->g.n, "src"));
    DYG_TRY(check_host_ids(dst, n, H->g.n, "dst"));
    DYG_TRY(check_host_weights(w, n));
    Workspace &ws = H->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w;
    DYG_TRY(stage_in(ws.in_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.in_dst, dst, n, st, &d_dst));
    DYG_TRY(stage_in(ws.in_w, w, n, st, &d_w));
    DYG_TRY(incremental_batch_dev(H, G, d_src, d_dst, d_w, n, first_update_id, *p, st));
    bool host_out = false;
    DYG_TRY(copy_out(found_at, ptr<int32_t>(ws.out_found), n, st, &host_out));
    DYG_TRY(copy_out(conductance, ptr<float>(ws.out_cond), n, st, &host_out));
    DYG_TRY(copy_out(accepted, ptr<uint8_t>(ws.out_acc), n, st, &host_out));
    if (host_out) DYG_CUDA(cudaStreamSynchronize(st));
    return DYG_OK;
}

dyg_status dyg_incremental_stream(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                  const uint32_t *dst, const float *w, uint32_t n,
                                  uint32_t batch_size, const dyg_walk_params *p,
                                  int32_t *found_at, float *conductance, uint8_t *accepted,
                                  dyg_stream_t stream) {
    set_error("");
    if (!H || (n && (!src || !dst || !w))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DYG_TRY(check_params(p));
    if (G && (G->g.n != H->g.n || G->device != H->device)) {
        set_error("G and H must have the same vertex count and device");
        return DYG_EINVAL;
    }
    if (n == 0) return DYG_OK;
    DeviceGuard dg(H->device);
    cudaStream_t st = (cudaStream_t)stream;
    DYG_TRY(check_host_ids(src, n, H->g.n, "src"));
    DYG_TRY(check_host_ids(dst, n, H->g.n, "dst"));
    DYG_TRY(check_host_weights(w, n));
    Workspace &ws = H->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w;
    DYG_TRY(stage_in(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.s_dst, dst, n, st, &d_dst));
    DYG_TRY(stage_in(ws.s_w, w, n, st, &d_w));
    DYG_TRY(ensure(ws.s_o1, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.s_o2, sizeof(float) * n));
    DYG_TRY(ensure(ws.s_o3, sizeof(uint8_t) * n));
    const uint32_t B = batch_size ? batch_size : dyg_reference_batch_size(n);
    for (uint32_t b0 = 0; b0 < n; b0 += B) {
        const uint32_t nb = (n - b0 < B) ? n - b0 : B;
        DYG_TRY(incremental_batch_dev(H, G, d_src + b0, d_dst + b0, d_w + b0, nb, b0, *p, st));
        DYG_CUDA(cudaMemcpyAsync(ptr<int32_t>(ws.s_o1) + b0, ws.out_found.p, sizeof(int32_t) * nb,
                                 cudaMemcpyDeviceToDevice, st));
        DYG_CUDA(cudaMemcpyAsync(ptr<float>(ws.s_o2) + b0, ws.out_cond.p, sizeof(float) * nb,
                                 cudaMemcpyDeviceToDevice, st));
        DYG_CUDA(cudaMemcpyAsync(ptr<uint8_t>(ws.s_o3) + b0, ws.out_acc.p, nb,
                                 cudaMemcpyDeviceToDevice, st));
    }
    bool host_out = false;
    DYG_TRY(copy_out(found_at, ptr<int32_t>(ws.s_o1), n, st, &host_out));
    DYG_TRY(copy_out(conductance, ptr<float>(ws.s_o2), n, st, &host_out));
    DYG_TRY(copy_out(accepted, ptr<uint8_t>(ws.s_o3), n, st, &host_out));
    if (host_out) DYG_CUDA(cudaStreamSynchronize(st));
    return DYG_OK;
}

static dyg_status decremental_common(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                     const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                     uint64_t uid_base, const dyg_walk_params *p, int32_t *status,
                                     float *conductance, uint32_t *rec_src, uint32_t *rec_dst,
                                     uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec,
                                     dyg_stream_t stream) {
    set_error("");
    if (!G || !H || (n && (!src || !dst))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DYG_TRY(check_params(p));
    if (G->g.n != H->g.n || G->device != H->device) {
        set_error("G and H must have the same vertex count and device");
        return DYG_EINVAL;
    }
    if (n_rec) *n_rec = 0;
    if (n == 0) return DYG_OK;
    DeviceGuard dg(G->device);
    cudaStream_t st = (cudaStream_t)stream;
    DYG_TRY(check_host_ids(src, n, G->g.n, "src"));
    DYG_TRY(check_host_ids(dst, n, G->g.n, "dst"));
    Workspace &ws = G->ws;
    const uint32_t *d_src, *d_dst;
    DYG_TRY(stage_in(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.s_dst, dst, n, st, &d_dst));
    DYG_TRY(ensure(ws.s_o1, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.s_o2, sizeof(float) * n));
    const uint32_t B = batch_size ? batch_size : dyg_reference_batch_size(n);
    const uint32_t hw = p->heuristic_walkers;
    const uint32_t stride = p->max_steps > 2 ? p->max_steps : 2;
    uint64_t total = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += B) {
        const uint32_t nb = (n - b0 < B) ? n - b0 : B;
        // worst case recovered edges of this batch
        const uint64_t worst = (uint64_t)nb * (stride + 4ull * hw);
        DYG_TRY(ensure_records(ws, total, total + worst, st));
        uint32_t got = 0;
        DYG_TRY(decremental_batch_dev(G, H, d_src + b0, d_dst + b0, nb, uid_base + b0, *p,
                                      (uint32_t)total, ptr<uint32_t>(ws.rx2), ptr<uint32_t>(ws.ry2),
                                      ptr<uint8_t>(ws.rk2), &got, st));
        DYG_CUDA(cudaMemcpyAsync(ptr<int32_t>(ws.s_o1) + b0, ws.out_status.p, sizeof(int32_t) * nb,
                                 cudaMemcpyDeviceToDevice, st));
        DYG_CUDA(cudaMemcpyAsync(ptr<float>(ws.s_o2) + b0, ws.out_cond.p, sizeof(float) * nb,
                                 cudaMemcpyDeviceToDevice, st));
        total += got;
    }
    DYG_TRY(check_device_errors(G, st));
    bool host_out = false;
    DYG_TRY(copy_out(status, ptr<int32_t>(ws.s_o1), n, st, &host_out));
    DYG_TRY(copy_out(conductance, ptr<float>(ws.s_o2), n, st, &host_out));
    const uint64_t nout = total < rec_cap ? total : rec_cap;
    DYG_TRY(copy_out(rec_src, ptr<uint32_t>(ws.rx2), nout, st, &host_out));
    DYG_TRY(copy_out(rec_dst, ptr<uint32_t>(ws.ry2), nout, st, &host_out));
    DYG_TRY(copy_out(rec_kind, ptr<uint8_t>(ws.rk2), nout, st, &host_out));
    if (host_out) DYG_CUDA(cudaStreamSynchronize(st));
    if (n_rec) *n_rec = total;
    if (total > rec_cap && (rec_src || rec_dst || rec_kind)) {
        set_error("more recovered edges than rec_cap");
        return DYG_ERANGE;
    }
    return DYG_OK;
}

dyg_status dyg_decremental_batch(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                 const uint32_t *dst, uint32_t n, uint64_t first_update_id,
                                 const dyg_walk_params *p, int32_t *status, float *conductance,
                                 uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                                 uint64_t rec_cap, uint64_t *n_rec, dyg_stream_t stream) {
    return decremental_common(G, H, src, dst, n, n ? n : 1, first_update_id, p, status, conductance,
                              rec_src, rec_dst, rec_kind, rec_cap, n_rec, stream);
}

dyg_status dyg_decremental_stream(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                  const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                  const dyg_walk_params *p, int32_t *status, float *conductance,
                                  uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                                  uint64_t rec_cap, uint64_t *n_rec, dyg_stream_t stream) {
    return decremental_common(G, H, src, dst, n, batch_size, 0, p, status, conductance, rec_src,
                              rec_dst, rec_kind, rec_cap, n_rec, stream);
}

}  // extern "C"
