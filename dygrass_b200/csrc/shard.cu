// shard.cu -- a batch split over processes (one per GPU), each holding a
// replica of G and H: every rank walks a contiguous range of the batch and
// writes the winner keys of that range; the ranks combine the keys (an
// element-wise max over the ranks' arrays, whose other entries are zero) and
// every rank then commits the whole batch identically.  The split calls give
// exactly what the whole-batch calls give (dyg_incremental_batch,
// dyg_decremental_batch): the keys are the same numbers, and the commit is the
// same code.
#include "dyg_internal.cuh"

namespace dyg {
namespace {

bool dev_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

template <typename T>
dyg_status stage(Buf &b, const T *p, size_t n, cudaStream_t st, const T **out) {
    if (!p || dev_ptr(p)) {
        *out = p;
        return DYG_OK;
    }
    DYG_TRY(ensure(b, sizeof(T) * (n ? n : 1)));
    DYG_CUDA(cudaMemcpyAsync(b.p, p, sizeof(T) * n, cudaMemcpyHostToDevice, st));
    *out = ptr<T>(b);
    return DYG_OK;
}

struct Guard {
    int prev = -1;
    bool changed = false;
    explicit Guard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = cudaSetDevice(dev) == cudaSuccess;
        cudaGetLastError();
    }
    ~Guard() {
        if (changed) cudaSetDevice(prev);
    }
};

dyg_status check_walk(const dyg_walk_params *p) {
    if (!p || p->walkers == 0 || p->walkers % 32 != 0 || p->walkers > 1024 || p->max_steps < 1 ||
        p->max_steps > 0x3FFFFF || p->transition > DYG_TRANSITION_WEIGHTED) {
        set_error("invalid walk parameters");
        return DYG_EINVAL;
    }
    return DYG_OK;
}

dyg_status clear_halt_of(dyg_graph *D, cudaStream_t st) {
    DYG_CUDA(cudaMemsetAsync(ptr<unsigned long long>(D->ws.scalars) + S_HALT, 0,
                             sizeof(unsigned long long), st));
    return DYG_OK;
}

}  // namespace
}  // namespace dyg

using namespace dyg;

extern "C" {

dyg_status dyg_walk_keys(dyg_graph *X, const uint32_t *src, const uint32_t *dst, const float *w,
                         const uint64_t *update_ids, uint64_t first_update_id, uint32_t n,
                         uint32_t lo, uint32_t hi, uint32_t incremental,
                         const dyg_walk_params *p, uint64_t *keys, dyg_stream_t stream) {
    set_error("");
    if (!X || !keys || lo > hi || hi > n || (n && (!src || !dst || (incremental && !w)))) {
        set_error("dyg_walk_keys: bad arguments (need lo <= hi <= n and device keys)");
        return DYG_EINVAL;
    }
    DYG_TRY(check_walk(p));
    if (lo == hi) return DYG_OK;
    Guard g(X->device);
    if (!dev_ptr(keys)) {
        set_error("dyg_walk_keys: keys must be a device array");
        return DYG_EINVAL;
    }
    {
        const void *ps[] = {src, dst, w, update_ids};
        const char *nm[] = {"src", "dst", "w", "update_ids"};
        DYG_TRY(check_same_device(X->device, ps, nm, 4));
    }
    cudaStream_t st = (cudaStream_t)stream;
    Workspace &ws = X->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w = nullptr;
    const uint64_t *d_ids = nullptr;
    DYG_TRY(stage(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage(ws.s_dst, dst, n, st, &d_dst));
    if (incremental) DYG_TRY(stage(ws.s_w, w, n, st, &d_w));
    DYG_TRY(stage(ws.s_uid, update_ids, n, st, &d_ids));
    unsigned long long *k = (unsigned long long *)keys + lo;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    DYG_TRY(clear_halt_of(X, st));
    // the range is checked on the device before it walks (host arrays too:
    // they are staged whole, and this call reads only [lo, hi))
    DYG_TRY(validate_enqueue(sc + S_HALT, sc + S_ERR, d_src + lo, d_dst + lo,
                             incremental ? d_w + lo : nullptr, hi - lo, X->g.n, st));
    DYG_CUDA(cudaMemsetAsync(k, 0, sizeof(unsigned long long) * (hi - lo), st));
    WalkJob job{sc + S_HALT, d_src + lo, d_dst + lo, incremental ? d_w + lo : nullptr,
                d_ids ? (const unsigned long long *)d_ids + lo : nullptr,
                (unsigned long long)(first_update_id + lo), nullptr, hi - lo,
                incremental ? kDomainIncr : kDomainDecr};
    DYG_TRY(launch_walk(X, job, *p, incremental != 0, k, st));
    DYG_TRY(read_scalars(X, st));
    if (ws.host_scalars[S_HALT]) return rejected_inputs(X, st);
    return DYG_OK;
}

dyg_status dyg_incremental_commit_keys(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                       const uint32_t *dst, const float *w, uint32_t n,
                                       const uint64_t *keys, int32_t *found_at,
                                       float *conductance, uint8_t *accepted,
                                       dyg_stream_t stream) {
    set_error("");
    if (!H || (n && (!src || !dst || !w || !keys))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    if (G && (G->g.n != H->g.n || G->device != H->device)) {
        set_error("G and H must have the same vertex count and device");
        return DYG_EINVAL;
    }
    if (n == 0) return DYG_OK;
    Guard gd(H->device);
    const bool outs_dev = (!found_at || dev_ptr(found_at)) && (!conductance || dev_ptr(conductance)) &&
                          (!accepted || dev_ptr(accepted));
    if (!dev_ptr(keys) || !outs_dev) {
        set_error("dyg_incremental_commit_keys: keys and outputs must be device arrays");
        return DYG_EINVAL;
    }
    {
        const void *ps[] = {src, dst, w, keys, found_at, conductance, accepted};
        const char *nm[] = {"src", "dst", "w", "keys", "found_at", "conductance", "accepted"};
        DYG_TRY(check_same_device(H->device, ps, nm, 7));
    }
    cudaStream_t st = (cudaStream_t)stream;
    Workspace &ws = H->ws;
    const uint32_t *d_src, *d_dst;
    const float *d_w;
    DYG_TRY(stage(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage(ws.s_dst, dst, n, st, &d_dst));
    DYG_TRY(stage(ws.s_w, w, n, st, &d_w));
    unsigned long long *halt = ptr<unsigned long long>(ws.scalars) + S_HALT;
    for (int round = 0; round < 64; ++round) {
        DYG_TRY(clear_halt_of(H, st));
        if (round == 0)
            DYG_TRY(validate_enqueue(halt, ptr<unsigned long long>(ws.scalars) + S_ERR, d_src, d_dst,
                                     d_w, n, H->g.n, st));
        DYG_TRY(incr_commit_enqueue(H, G, d_src, d_dst, d_w, n, (const unsigned long long *)keys,
                                    halt, 0, found_at, conductance, accepted, st));
        DYG_TRY(read_scalars2(H, G, st));
        const unsigned long long h = H->ws.host_scalars[S_HALT];
        if (!h) return DYG_OK;
        if (((h >> 4) & 0xF) == kHaltInvalid) return rejected_inputs(H, st);
        DYG_TRY(grow_arena(H, H->g.arena_cap * 2, st));
        if (G) DYG_TRY(grow_arena(G, G->g.arena_cap * 2, st));
    }
    set_error("incremental commit: too many arena regrowths");
    return DYG_ENOMEM;
}

dyg_status dyg_decremental_delete(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                  const uint32_t *dst, const uint64_t *update_ids,
                                  uint64_t first_update_id, uint32_t n, int32_t *status,
                                  float *conductance, uint32_t *n_walk, dyg_stream_t stream) {
    set_error("");
    if (!G || !H || !n_walk || (n && (!src || !dst || !status || !conductance))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    if (G->g.n != H->g.n || G->device != H->device) {
        set_error("G and H must have the same vertex count and device");
        return DYG_EINVAL;
    }
    *n_walk = 0;
    if (n == 0) return DYG_OK;
    Guard gd(G->device);
    if (!dev_ptr(status) || !dev_ptr(conductance)) {
        set_error("dyg_decremental_delete: status and conductance must be device arrays");
        return DYG_EINVAL;
    }
    {
        const void *ps[] = {src, dst, update_ids, status, conductance};
        const char *nm[] = {"src", "dst", "update_ids", "status", "conductance"};
        DYG_TRY(check_same_device(G->device, ps, nm, 5));
    }
    cudaStream_t st = (cudaStream_t)stream;
    Workspace &ws = G->ws;
    const uint32_t *d_src, *d_dst;
    const uint64_t *d_ids = nullptr;
    DYG_TRY(stage(ws.s_src, src, n, st, &d_src));
    DYG_TRY(stage(ws.s_dst, dst, n, st, &d_dst));
    DYG_TRY(stage(ws.s_uid, update_ids, n, st, &d_ids));
    unsigned long long *halt = ptr<unsigned long long>(ws.scalars) + S_HALT;
    DYG_TRY(clear_halt_of(G, st));
    DYG_TRY(validate_enqueue(halt, ptr<unsigned long long>(ws.scalars) + S_ERR, d_src, d_dst,
                             nullptr, n, G->g.n, st));
    DYG_TRY(decr_delete_enqueue(G, H, d_src, d_dst, n, first_update_id,
                                (const unsigned long long *)d_ids, false, halt, status,
                                conductance, st));
    DYG_TRY(read_scalars2(G, H, st));
    if (ws.host_scalars[S_HALT]) return rejected_inputs(G, st);
    if (ws.host_scalars[S_ERR]) {
        set_error("a deletion endpoint is not a vertex of the graph");
        return DYG_EINVAL;
    }
    *n_walk = ws.host_counts[C_FILTERED];
    return DYG_OK;
}

dyg_status dyg_decremental_walk_keys(dyg_graph *G, uint32_t lo, uint32_t hi,
                                     const dyg_walk_params *p, uint64_t *keys,
                                     dyg_stream_t stream) {
    set_error("");
    if (!G || !keys || lo > hi) {
        set_error("dyg_decremental_walk_keys: bad arguments");
        return DYG_EINVAL;
    }
    DYG_TRY(check_walk(p));
    if (lo == hi) return DYG_OK;
    Guard gd(G->device);
    Workspace &ws = G->ws;
    if (!dev_ptr(keys) || ws.f_src.bytes < sizeof(uint32_t) * (size_t)hi) {
        set_error("dyg_decremental_walk_keys: device keys and a range inside the walk list needed");
        return DYG_EINVAL;
    }
    {
        const void *ps[] = {keys};
        const char *nm[] = {"keys"};
        DYG_TRY(check_same_device(G->device, ps, nm, 1));
    }
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long *k = (unsigned long long *)keys + lo;
    DYG_CUDA(cudaMemsetAsync(k, 0, sizeof(unsigned long long) * (hi - lo), st));
    WalkJob job{nullptr, ptr<uint32_t>(ws.f_src) + lo, ptr<uint32_t>(ws.f_dst) + lo, nullptr,
                ptr<unsigned long long>(ws.f_uid) + lo, 0ull, nullptr, hi - lo, kDomainDecr};
    DYG_TRY(launch_walk(G, job, *p, false, k, st));
    DYG_CUDA(cudaStreamSynchronize(st));
    return DYG_OK;
}

dyg_status dyg_decremental_commit_keys(dyg_graph *G, dyg_graph *H, const dyg_walk_params *p,
                                       const uint64_t *keys, uint32_t n_walk, int32_t *status,
                                       float *conductance, uint32_t *rec_src, uint32_t *rec_dst,
                                       uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec,
                                       dyg_stream_t stream) {
    set_error("");
    if (!G || !H || (n_walk && !keys)) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    DYG_TRY(check_walk(p));
    if (n_rec) *n_rec = 0;
    if (n_walk == 0) return DYG_OK;
    Guard gd(G->device);
    if (!dev_ptr(keys) || !dev_ptr(status) || !dev_ptr(conductance)) {
        set_error("dyg_decremental_commit_keys: keys, status and conductance must be device arrays");
        return DYG_EINVAL;
    }
    {
        const void *ps[] = {keys, status, conductance, rec_src, rec_dst, rec_kind};
        const char *nm[] = {"keys", "status", "conductance", "rec_src", "rec_dst", "rec_kind"};
        DYG_TRY(check_same_device(G->device, ps, nm, 6));
    }
    cudaStream_t st = (cudaStream_t)stream;
    Workspace &ws = G->ws;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    unsigned long long *halt = sc + S_HALT;
    const uint64_t want = (uint64_t)n_walk * 4 + 1024;
    DYG_TRY(ensure(ws.rx2, sizeof(uint32_t) * want));
    DYG_TRY(ensure(ws.ry2, sizeof(uint32_t) * want));
    DYG_TRY(ensure(ws.rk2, want));
    uint64_t cap = ws.rx2.bytes / 4;
    if (ws.ry2.bytes / 4 < cap) cap = ws.ry2.bytes / 4;
    if (ws.rk2.bytes < cap) cap = ws.rk2.bytes;
    unsigned long long init[2] = {0ull, cap};   // S_RECCNT, S_RECCAP
    DYG_CUDA(cudaMemcpyAsync(sc + S_RECCNT, init, sizeof(init), cudaMemcpyHostToDevice, st));
    uint32_t phase = 0;
    uint64_t total = 0;
    int round = 0;
    G->last_rec = 0;
    for (; round < 64; ++round) {
        DYG_TRY(clear_halt_of(G, st));
        DYG_TRY(decr_walk_enqueue(G, H, 0, n_walk, nullptr, *p, halt, 0, phase, status,
                                  conductance, st, (const unsigned long long *)keys));
        DYG_TRY(read_scalars2(G, H, st));
        const unsigned long long h = ws.host_scalars[S_HALT];
        if (!h) {
            total = ws.host_scalars[S_RECCNT];
            break;
        }
        const uint32_t kind = (uint32_t)((h >> 4) & 0xF);
        phase = (uint32_t)(h & 0xF);
        if (kind == kHaltRecords) {
            const uint64_t used = ws.host_scalars[S_RECCNT];
            const uint64_t ncap = cap * 2;
            DYG_TRY(grow_keep(ws.rx2, sizeof(uint32_t) * ncap, sizeof(uint32_t) * used, st));
            DYG_TRY(grow_keep(ws.ry2, sizeof(uint32_t) * ncap, sizeof(uint32_t) * used, st));
            DYG_TRY(grow_keep(ws.rk2, ncap, used, st));
            cap = ncap;
            DYG_CUDA(cudaMemcpyAsync(sc + S_RECCAP, &cap, sizeof(cap), cudaMemcpyHostToDevice, st));
            DYG_CUDA(cudaStreamSynchronize(st));
        } else {
            DYG_TRY(grow_arena(H, H->g.arena_cap * 2, st));
        }
    }
    if (round == 64) {
        set_error("decremental commit: too many buffer regrowths");
        return DYG_ENOMEM;
    }
    G->last_rec = total;
    const uint64_t nout = total < rec_cap ? total : rec_cap;
    const bool any_host = (rec_src && !dev_ptr(rec_src)) || (rec_dst && !dev_ptr(rec_dst)) ||
                          (rec_kind && !dev_ptr(rec_kind));
    if (nout) {
        if (rec_src)
            DYG_CUDA(cudaMemcpyAsync(rec_src, ws.rx2.p, sizeof(uint32_t) * nout, cudaMemcpyDefault, st));
        if (rec_dst)
            DYG_CUDA(cudaMemcpyAsync(rec_dst, ws.ry2.p, sizeof(uint32_t) * nout, cudaMemcpyDefault, st));
        if (rec_kind) DYG_CUDA(cudaMemcpyAsync(rec_kind, ws.rk2.p, nout, cudaMemcpyDefault, st));
    }
    if (any_host || nout) DYG_CUDA(cudaStreamSynchronize(st));
    if (n_rec) *n_rec = total;
    if (total > rec_cap && (rec_src || rec_dst || rec_kind)) {
        set_error("more recovered edges than rec_cap");
        return DYG_ERANGE;
    }
    return DYG_OK;
}

}  // extern "C"
