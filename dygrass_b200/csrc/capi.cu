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

PtrPlace ptr_place(const void *p, int device) {
    if (!p) return kOnHost;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return kOnHost;
    }
    if (at.type == cudaMemoryTypeManaged) return kOnDevice;
    if (at.type == cudaMemoryTypeDevice) return at.device == device ? kOnDevice : kOnOtherDevice;
    return kOnHost;
}

dyg_status check_same_device(int device, const void *const *ptrs, const char *const *names,
                             int count) {
    for (int i = 0; i < count; ++i)
        if (ptrs[i] && ptr_place(ptrs[i], device) == kOnOtherDevice) {
            set_error(std::string(names[i]) + " is device memory of another GPU than the graph's (device " +
                      std::to_string(device) + ")");
            return DYG_EINVAL;
        }
    return DYG_OK;
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

// Host batches up to this size are checked on the host (the message names
// the entry); larger ones are staged first and checked by k_validate on the
// device, like device batches, instead of by a serial host loop.
constexpr uint32_t kHostCheckMax = 65536;

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
        if (err & kErrWeight) {
            set_error("a batch weight is not finite and > 0");
            return DYG_EINVAL;
        }
        if (err & kErrScan) {
            set_error("a prefix scan tile timed out waiting for its predecessor");
            return DYG_ESTATE;
        }
        set_error("internal consistency check failed (device error bits " + std::to_string(err) + ")");
        return DYG_ESTATE;
    }
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
    Buf *bufs[] = {&ws.keys, &ws.flags, &ws.pos, &ws.f_src, &ws.f_dst, &ws.f_idx, &ws.f_uid,
                   &ws.f_w, &ws.found, &ws.hx, &ws.hy, &ws.hw, &ws.path_v, &ws.path_s,
                   &ws.path_len, &ws.cand_x, &ws.cand_y, &ws.cand_w, &ws.keep, &ws.htab_k,
                   &ws.htab_v, &ws.nop, &ws.cub_tmp, &ws.scan_status, &ws.s_src, &ws.s_dst, &ws.s_w, &ws.s_o1,
                   &ws.s_o2, &ws.s_o3, &ws.rx2, &ws.ry2, &ws.rk2, &ws.rank, &ws.lneed, &ws.dtmp,
                   &ws.rowcnt, &ws.rowtmp, &ws.tmask, &ws.del_hx, &ws.del_hy,
                   &ws.st_key, &ws.st_val, &ws.st_pos, &ws.st_wapp, &ws.big, &ws.s_uid, &ws.scalars,
                   &ws.counts};
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

}  // namespace

dyg_status check_walk_params(const dyg_walk_params *p) { return check_params(p); }

dyg_status create_empty_graph(uint32_t n, uint64_t arena_slots, int device, uint32_t slack,
                              double headroom, dyg_graph **out) {
    *out = nullptr;
    if (arena_slots < 1024) arena_slots = 1024;
    if (arena_slots >= 0xFFFFFFFFull) {
        set_error("arena would exceed 32-bit slot offsets");
        return DYG_EINVAL;
    }
    DeviceGuard dg(device);
    dyg_graph *G = new dyg_graph();
    G->device = device;
    G->slack = slack;
    G->headroom = headroom;
    G->g.n = n;
    G->g.arena_cap = arena_slots;
    dyg_status rc = graph_alloc_scalars(G);
    if (rc == DYG_OK &&
        (cudaMalloc(&G->g.desc, sizeof(uint2) * (size_t)(n ? n : 1)) != cudaSuccess ||
         cudaMalloc(&G->g.cap, sizeof(uint32_t) * (size_t)(n ? n : 1)) != cudaSuccess ||
         cudaMalloc(&G->g.slots, sizeof(uint2) * (size_t)arena_slots) != cudaSuccess ||
         cudaMalloc(&G->g.wts, sizeof(float) * (size_t)arena_slots) != cudaSuccess)) {
        cudaGetLastError();
        set_error("cudaMalloc of a pool graph failed");
        rc = DYG_ENOMEM;
    }
    if (rc == DYG_OK && (cudaMemset(G->g.desc, 0, sizeof(uint2) * (size_t)(n ? n : 1)) != cudaSuccess ||
                         cudaMemset(G->g.cap, 0, sizeof(uint32_t) * (size_t)(n ? n : 1)) != cudaSuccess))
        rc = cuda_fail(cudaGetLastError(), "cudaMemset", __FILE__, __LINE__);
    if (rc != DYG_OK) {
        free_graph(G);
        return rc;
    }
    *out = G;
    return DYG_OK;
}

void destroy_graph(dyg_graph *G) {
    if (!G) return;
    {
        DeviceGuard dg(G->device);
        cudaDeviceSynchronize();
    }
    free_graph(G);
}

dyg_status device_errors(dyg_graph *G, cudaStream_t st) {
    return G->ws.host_scalars[S_ERR] ? check_device_errors(G, st) : DYG_OK;
}

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

dyg_status dyg_graph_create_from_csr(uint32_t n_vertices, const uint64_t *row_ptr,
                                     const uint32_t *col, const float *w,
                                     const dyg_graph_opts *opts, dyg_graph **out) {
    set_error("");
    if (!out || !row_ptr) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    *out = nullptr;
    const uint64_t m = row_ptr[n_vertices];
    if (m && (!col || !w)) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    if (row_ptr[0] != 0 || m > 0xFFFFFFFFull) {
        set_error("row_ptr must start at 0 and hold at most 2^32 - 1 slots");
        return DYG_EINVAL;
    }
    for (uint32_t v = 0; v < n_vertices; ++v)
        if (row_ptr[v + 1] < row_ptr[v]) {
            set_error("row_ptr must be non-decreasing");
            return DYG_EINVAL;
        }
    DYG_TRY(check_host_ids(col, m, n_vertices, "col"));
    DYG_TRY(check_host_weights(w, m));
    dyg_graph_opts o;
    dyg_graph_opts_default(&o);
    if (opts) o = *opts;
    int dev = o.device;
    if (dev < 0) DYG_CUDA(cudaGetDevice(&dev));
    DeviceGuard dg(dev);
    dyg_graph *G = new dyg_graph();
    G->device = dev;
    G->slack = o.slack_per_row;
    G->headroom = o.arena_headroom > 0 ? o.arena_headroom : 0.0;
    dyg_status rc = graph_alloc_scalars(G);
    if (rc == DYG_OK) rc = upload_graph(G, n_vertices, row_ptr, col, w);
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
    DYG_CUDA(cudaMemsetAsync(ptr<unsigned long long>(dst->ws.scalars) + S_LONG, 0,
                             sizeof(unsigned long long), st));
    dst->slack = src->slack;
    dst->headroom = src->headroom;
    dst->long_rows = src->long_rows;
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

static dyg_status incremental_common(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                     const uint32_t *dst, const float *w, uint32_t n,
                                     uint32_t batch_size, uint64_t uid_base, const uint64_t *uids,
                                     const dyg_walk_params *p, int32_t *found_at,
                                     float *conductance, uint8_t *accepted, dyg_stream_t stream) {
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
    {
        const void *ps[] = {src, dst, w, uids, found_at, conductance, accepted};
        const char *nm[] = {"src", "dst", "w", "update_ids", "found_at", "conductance", "accepted"};
        DYG_TRY(check_same_device(H->device, ps, nm, 7));
    }
    const bool host_check = n <= kHostCheckMax;
    if (host_check) {
        DYG_TRY(check_host_ids(src, n, H->g.n, "src"));
        DYG_TRY(check_host_ids(dst, n, H->g.n, "dst"));
        DYG_TRY(check_host_weights(w, n));
    }
    Workspace &ws = H->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w;
    DYG_TRY(stage_in(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.s_dst, dst, n, st, &d_dst));
    DYG_TRY(stage_in(ws.s_w, w, n, st, &d_w));
    const uint64_t *d_uid = nullptr;
    DYG_TRY(stage_in(ws.s_uid, uids, n, st, &d_uid));
    // device outputs are written in place; host outputs go through staging
    int32_t *o_found = found_at && on_device(found_at) ? found_at : nullptr;
    float *o_cond = conductance && on_device(conductance) ? conductance : nullptr;
    uint8_t *o_acc = accepted && on_device(accepted) ? accepted : nullptr;
    if (found_at && !o_found) {
        DYG_TRY(ensure(ws.s_o1, sizeof(int32_t) * n));
        o_found = ptr<int32_t>(ws.s_o1);
    }
    if (conductance && !o_cond) {
        DYG_TRY(ensure(ws.s_o2, sizeof(float) * n));
        o_cond = ptr<float>(ws.s_o2);
    }
    if (accepted && !o_acc) {
        DYG_TRY(ensure(ws.s_o3, sizeof(uint8_t) * n));
        o_acc = ptr<uint8_t>(ws.s_o3);
    }
    const uint32_t B = batch_size ? batch_size : dyg_reference_batch_size(n);
    // inputs read in place from device memory were not checked on the host
    const bool dev_in = !host_check || d_src == src || d_dst == dst || d_w == w;
    DYG_TRY(incremental_run(H, G, d_src, d_dst, d_w, n, B, uid_base,
                            (const unsigned long long *)d_uid, *p, o_found, o_cond, o_acc,
                            st, dev_in));
    if (H->ws.host_scalars[S_ERR]) DYG_TRY(check_device_errors(H, st));
    bool host_out = false;
    if (found_at && o_found != found_at) DYG_TRY(copy_out(found_at, (const int32_t *)o_found, n, st, &host_out));
    if (conductance && o_cond != conductance) DYG_TRY(copy_out(conductance, (const float *)o_cond, n, st, &host_out));
    if (accepted && o_acc != accepted) DYG_TRY(copy_out(accepted, (const uint8_t *)o_acc, n, st, &host_out));
    if (host_out) DYG_CUDA(cudaStreamSynchronize(st));
    return DYG_OK;
}

dyg_status dyg_incremental_batch(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n,
                                 uint64_t first_update_id, const dyg_walk_params *p,
                                 int32_t *found_at, float *conductance, uint8_t *accepted,
                                 dyg_stream_t stream) {
    return incremental_common(H, G, src, dst, w, n, n ? n : 1, first_update_id, nullptr, p,
                              found_at, conductance, accepted, stream);
}

dyg_status dyg_incremental_stream(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                  const uint32_t *dst, const float *w, uint32_t n,
                                  uint32_t batch_size, const dyg_walk_params *p,
                                  int32_t *found_at, float *conductance, uint8_t *accepted,
                                  dyg_stream_t stream) {
    return incremental_common(H, G, src, dst, w, n, batch_size, 0, nullptr, p, found_at,
                              conductance, accepted, stream);
}

static dyg_status decremental_common(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                     const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                     uint64_t uid_base, const uint64_t *uids,
                                     const dyg_walk_params *p, int32_t *status,
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
    {
        const void *ps[] = {src, dst, uids, status, conductance, rec_src, rec_dst, rec_kind};
        const char *nm[] = {"src", "dst", "update_ids", "status", "conductance",
                            "rec_src", "rec_dst", "rec_kind"};
        DYG_TRY(check_same_device(G->device, ps, nm, 8));
    }
    const bool host_check = n <= kHostCheckMax;
    if (host_check) {
        DYG_TRY(check_host_ids(src, n, G->g.n, "src"));
        DYG_TRY(check_host_ids(dst, n, G->g.n, "dst"));
    }
    Workspace &ws = G->ws;
    const uint32_t *d_src, *d_dst;
    DYG_TRY(stage_in(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.s_dst, dst, n, st, &d_dst));
    const uint64_t *d_uid = nullptr;
    DYG_TRY(stage_in(ws.s_uid, uids, n, st, &d_uid));
    int32_t *o_st = status && on_device(status) ? status : nullptr;
    float *o_cd = conductance && on_device(conductance) ? conductance : nullptr;
    if (!o_st) {
        DYG_TRY(ensure(ws.s_o1, sizeof(int32_t) * n));
        o_st = ptr<int32_t>(ws.s_o1);
    }
    if (!o_cd) {
        DYG_TRY(ensure(ws.s_o2, sizeof(float) * n));
        o_cd = ptr<float>(ws.s_o2);
    }
    const uint32_t B = batch_size ? batch_size : dyg_reference_batch_size(n);
    uint64_t total = 0;
    const bool dev_in = !host_check || d_src == src || d_dst == dst;
    G->last_rec = 0;
    DYG_TRY(decremental_run(G, H, d_src, d_dst, n, B, uid_base, (const unsigned long long *)d_uid,
                            *p, o_st, o_cd, &total, st, dev_in));
    G->last_rec = total;
    if (G->ws.host_scalars[S_ERR]) DYG_TRY(check_device_errors(G, st));
    bool host_out = false;
    if (status && o_st != status) DYG_TRY(copy_out(status, (const int32_t *)o_st, n, st, &host_out));
    if (conductance && o_cd != conductance) DYG_TRY(copy_out(conductance, (const float *)o_cd, n, st, &host_out));
    const uint64_t nout = total < rec_cap ? total : rec_cap;
    DYG_TRY(copy_out(rec_src, (const uint32_t *)ptr<uint32_t>(ws.rx2), nout, st, &host_out));
    DYG_TRY(copy_out(rec_dst, (const uint32_t *)ptr<uint32_t>(ws.ry2), nout, st, &host_out));
    DYG_TRY(copy_out(rec_kind, (const uint8_t *)ptr<uint8_t>(ws.rk2), nout, st, &host_out));
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
    return decremental_common(G, H, src, dst, n, n ? n : 1, first_update_id, nullptr, p, status,
                              conductance, rec_src, rec_dst, rec_kind, rec_cap, n_rec, stream);
}

dyg_status dyg_decremental_stream(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                  const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                  const dyg_walk_params *p, int32_t *status, float *conductance,
                                  uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                                  uint64_t rec_cap, uint64_t *n_rec, dyg_stream_t stream) {
    return decremental_common(G, H, src, dst, n, batch_size, 0, nullptr, p, status, conductance,
                              rec_src, rec_dst, rec_kind, rec_cap, n_rec, stream);
}

dyg_status dyg_incremental_batch_ids(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                     const uint32_t *dst, const float *w,
                                     const uint64_t *update_ids, uint32_t n,
                                     const dyg_walk_params *p, int32_t *found_at,
                                     float *conductance, uint8_t *accepted, dyg_stream_t stream) {
    if (n && !update_ids) {
        set_error("NULL update_ids");
        return DYG_EINVAL;
    }
    return incremental_common(H, G, src, dst, w, n, n ? n : 1, 0, update_ids, p, found_at,
                              conductance, accepted, stream);
}

dyg_status dyg_decremental_batch_ids(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                     const uint32_t *dst, const uint64_t *update_ids, uint32_t n,
                                     const dyg_walk_params *p, int32_t *status,
                                     float *conductance, uint32_t *rec_src, uint32_t *rec_dst,
                                     uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec,
                                     dyg_stream_t stream) {
    if (n && !update_ids) {
        set_error("NULL update_ids");
        return DYG_EINVAL;
    }
    return decremental_common(G, H, src, dst, n, n ? n : 1, 0, update_ids, p, status, conductance,
                              rec_src, rec_dst, rec_kind, rec_cap, n_rec, stream);
}

dyg_status dyg_recovered_read(const dyg_graph *g, uint64_t first, uint64_t count,
                              uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind) {
    set_error("");
    if (!g) {
        set_error("NULL graph");
        return DYG_EINVAL;
    }
    if (first > g->last_rec || count > g->last_rec - first) {
        set_error("records [" + std::to_string(first) + ", " + std::to_string(first + count) +
                  ") are not all among the last call's " + std::to_string(g->last_rec));
        return DYG_ERANGE;
    }
    if (count == 0) return DYG_OK;
    DeviceGuard dg(g->device);
    const Workspace &ws = g->ws;
    const void *ps[] = {rec_src, rec_dst, rec_kind};
    const char *nm[] = {"rec_src", "rec_dst", "rec_kind"};
    DYG_TRY(check_same_device(g->device, ps, nm, 3));
    if (rec_src)
        DYG_CUDA(cudaMemcpy(rec_src, ptr<uint32_t>(ws.rx2) + first, sizeof(uint32_t) * count,
                            cudaMemcpyDefault));
    if (rec_dst)
        DYG_CUDA(cudaMemcpy(rec_dst, ptr<uint32_t>(ws.ry2) + first, sizeof(uint32_t) * count,
                            cudaMemcpyDefault));
    if (rec_kind)
        DYG_CUDA(cudaMemcpy(rec_kind, ptr<uint8_t>(ws.rk2) + first, count, cudaMemcpyDefault));
    return DYG_OK;
}

uint32_t dyg_stream_default_chunk(uint32_t n_vertices) {
    return stream_default_chunk(n_vertices);
}

dyg_status dyg_stream_file(dyg_graph *G, dyg_graph *H, uint32_t op, const uint32_t *src,
                           const uint32_t *dst, const float *w, uint32_t n,
                           uint64_t first_update_id, uint32_t chunk, const dyg_walk_params *p,
                           int32_t *status, float *conductance, uint32_t *rec_src,
                           uint32_t *rec_dst, uint8_t *rec_kind, uint64_t rec_cap,
                           uint64_t *n_rec, dyg_stream_t stream) {
    set_error("");
    const bool ins = op == DYG_STREAM_INSERT;
    if (!G || !H || (n && (!src || !dst || (ins && !w)))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    if (op != DYG_STREAM_INSERT && op != DYG_STREAM_DELETE) {
        set_error("op must be DYG_STREAM_INSERT or DYG_STREAM_DELETE");
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
    {
        const void *ps[] = {src, dst, w, status, conductance, rec_src, rec_dst, rec_kind};
        const char *nm[] = {"src", "dst", "w", "status", "conductance", "rec_src", "rec_dst",
                            "rec_kind"};
        DYG_TRY(check_same_device(G->device, ps, nm, 8));
    }
    const bool host_check = n <= kHostCheckMax;
    if (host_check) {
        DYG_TRY(check_host_ids(src, n, G->g.n, "src"));
        DYG_TRY(check_host_ids(dst, n, G->g.n, "dst"));
        if (ins) DYG_TRY(check_host_weights(w, n));
    }
    Workspace &ws = G->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w = nullptr;
    DYG_TRY(stage_in(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage_in(ws.s_dst, dst, n, st, &d_dst));
    if (ins) DYG_TRY(stage_in(ws.s_w, w, n, st, &d_w));
    int32_t *o_st = status && on_device(status) ? status : nullptr;
    float *o_cd = conductance && on_device(conductance) ? conductance : nullptr;
    if (!o_st) {
        DYG_TRY(ensure(ws.s_o1, sizeof(int32_t) * n));
        o_st = ptr<int32_t>(ws.s_o1);
    }
    if (!o_cd) {
        DYG_TRY(ensure(ws.s_o2, sizeof(float) * n));
        o_cd = ptr<float>(ws.s_o2);
    }
    uint64_t total = 0;
    const bool dev_in = !host_check || d_src == src || d_dst == dst || (ins && d_w == w);
    if (!ins) G->last_rec = 0;
    DYG_TRY(stream_file_run(G, H, op, d_src, d_dst, d_w, n, first_update_id, chunk, *p, o_st, o_cd,
                            &total, st, dev_in));
    if (!ins) G->last_rec = total;
    if (G->ws.host_scalars[S_ERR]) DYG_TRY(check_device_errors(G, st));
    bool host_out = false;
    if (status && o_st != status) DYG_TRY(copy_out(status, (const int32_t *)o_st, n, st, &host_out));
    if (conductance && o_cd != conductance)
        DYG_TRY(copy_out(conductance, (const float *)o_cd, n, st, &host_out));
    const uint64_t nout = total < rec_cap ? total : rec_cap;
    if (!ins) {
        DYG_TRY(copy_out(rec_src, (const uint32_t *)ptr<uint32_t>(ws.rx2), nout, st, &host_out));
        DYG_TRY(copy_out(rec_dst, (const uint32_t *)ptr<uint32_t>(ws.ry2), nout, st, &host_out));
        DYG_TRY(copy_out(rec_kind, (const uint8_t *)ptr<uint8_t>(ws.rk2), nout, st, &host_out));
    }
    if (host_out) DYG_CUDA(cudaStreamSynchronize(st));
    if (n_rec) *n_rec = total;
    if (total > rec_cap && (rec_src || rec_dst || rec_kind)) {
        set_error("more recovered edges than rec_cap");
        return DYG_ERANGE;
    }
    return DYG_OK;
}

}  // extern "C"
