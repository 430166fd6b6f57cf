// pipeline.cu -- the incremental and decremental update pipelines.
//
// A whole update stream is enqueued on one CUDA stream with no host
// round-trip: counts stay on the device (grid-stride loops bounded by device
// counts), row updates go through rowops.cu, and the only host check is a
// single synchronize at the end.  A reservation that does not fit (arena or
// record buffers) halts every later kernel; the host then grows the buffer and
// resumes at the halted batch and phase, which reproduces the same results
// because no kernel changed anything after the halt.
//
// Incremental batch (one iteration of random_walk_incremental/main.cu:314-340):
//   walk H -> decode winner keys -> exclusive scan of accept flags (input
//   order) -> accepted half-edges to H [and every half-edge to G], reserved
//   together.  Resumes at the batch start (nothing of the batch changed).
// Decremental batch (random_walk_decremental/main.cu:413-444), phases:
//   0: delete from G and H in input order, compact the edges found in both,
//      walk G, replay winners, path candidates in (edge, step) order, then
//      the 2-step fallback walks' candidates for the edges without a path;
//   1: dedup all candidates (first occurrence), drop those in H, append the
//      rest in order (path edges, then fallback edges).
#include "dyg_internal.cuh"
#include "scan.cuh"

namespace dyg {

namespace {

inline int blocks(uint64_t n, int th) { return (int)((n + th - 1) / th); }

int grid_for(uint64_t m) {
    const uint64_t b = (m + 255) / 256;
    const uint64_t cap = (uint64_t)num_sms() * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

__device__ __forceinline__ uint32_t dcount(const uint32_t *dev, uint32_t host) {
    return dev ? min(*dev, host) : host;
}

#define HALTED(h) ((h) && *(h))
#define GSTRIDE(i, m) \
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (m); i += gridDim.x * blockDim.x)

// ------------------------------------------------------- input check

__global__ void k_validate(unsigned long long *halt, const uint32_t *src, const uint32_t *dst,
                           const float *w, uint32_t n, uint32_t nv, unsigned long long *err) {
    GSTRIDE(e, n) {
        unsigned long long bits = 0ull;
        if (src[e] >= nv || dst[e] >= nv) bits |= kErrVertex;
        if (w) {
            const float x = w[e];
            if (!(x > 0.0f) || !isfinite(x)) bits |= kErrWeight;
        }
        if (bits) {
            atomicOr(err, bits);
            atomicCAS(halt, 0ull, halt_code(0, (uint32_t)kHaltInvalid, 0));
        }
    }
}

// --------------------------------------------------------- incremental

// Incremental commit of one batch in one scan: element e is decoded from its
// winner key (found step, conductance, accept flag; keys[e] = 0: no walker
// connected the edge), the accept flags are scanned in input order, and the
// accepted edge goes to H's half-edge list at its scanned position -- u gets
// v, then v gets u (random_walk_incremental/gpu_graph.cuh:320-325).  With G,
// every edge also goes to G's list at its input position.
struct IncrCommitOp {
    const unsigned long long *keys;
    const uint32_t *src, *dst;
    const float *w;
    int32_t *found;
    float *cond;
    uint8_t *acc;
    uint32_t *hx, *hy;   // H: accepted edges, compacted
    float *hw;
    uint32_t *gx, *gy;   // G: every edge (null: no G)
    float *gw;
    uint32_t *half_count;   // 2 * accepted
    __device__ uint32_t load(uint32_t e) const {
        const unsigned long long k = keys[e];
        if (found) found[e] = key_found(k);
        if (cond) cond[e] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
        if (acc) acc[e] = k ? 0 : 1;
        return k ? 0u : 1u;
    }
    __device__ void store(uint32_t e, uint32_t q, uint32_t v) const {
        const uint32_t u = src[e], x = dst[e];
        const float ww = w[e];
        if (gx) {
            gx[2 * e] = u;
            gy[2 * e] = x;
            gw[2 * e] = ww;
            gx[2 * e + 1] = x;
            gy[2 * e + 1] = u;
            gw[2 * e + 1] = ww;
        }
        if (!v) return;
        hx[2 * q] = u;
        hy[2 * q] = x;
        hw[2 * q] = ww;
        hx[2 * q + 1] = x;
        hy[2 * q + 1] = u;
        hw[2 * q + 1] = ww;
    }
    __device__ void last(uint32_t total) const { *half_count = 2u * total; }
};

// ---------------------------------------------------------- decremental

// Deletion half-edges with endpoints ordered min -> max
// (random_walk_decremental/gpu_graph.cuh:340-343).
__global__ void k_del_half_edges(const unsigned long long *halt, const uint32_t *src,
                                 const uint32_t *dst, uint32_t n, uint32_t nv, uint32_t *hx,
                                 uint32_t *hy, unsigned long long *err) {
    if (HALTED(halt)) return;
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    uint32_t a = src[e], b = dst[e];
    if (a > b) {
        const uint32_t t = a;
        a = b;
        b = t;
    }
    if (b >= nv) {
        atomicOr(err, (unsigned long long)kErrVertex);
        a = b = 0xFFFFFFFFu;   // ignored by the row operations: never found
    }
    hx[2 * e] = a;
    hy[2 * e] = b;
    hx[2 * e + 1] = b;
    hy[2 * e + 1] = a;
}

// Deletion e found in G and in H goes to the walk list at its scanned
// position f: min -> max, or with osrc/odst the file orientation; every
// deletion gets its status code.
struct DelFilterOp {
    const uint8_t *fG, *fH;
    int32_t *status;
    float *cond;
    const uint32_t *hx, *hy, *osrc, *odst;
    unsigned long long uid0;
    const unsigned long long *uids;
    uint32_t *f_src, *f_dst;
    unsigned long long *f_uid;
    uint32_t *f_idx, *count;
    __device__ uint32_t load(uint32_t e) const {
        const bool inG = fG[2 * e] && fG[2 * e + 1];
        const bool inH = inG && fH[2 * e] && fH[2 * e + 1];
        status[e] = !inG ? DYG_DEL_NOT_IN_G : (!inH ? DYG_DEL_NOT_IN_H : DYG_DEL_NO_PATH);
        cond[e] = 0.f;
        return inH ? 1u : 0u;
    }
    __device__ void store(uint32_t e, uint32_t f, uint32_t v) const {
        if (!v) return;
        f_src[f] = osrc ? osrc[e] : hx[2 * e];
        f_dst[f] = odst ? odst[e] : hy[2 * e];
        f_uid[f] = uids ? uids[e] : uid0 + e;
        f_idx[f] = e;
    }
    __device__ void last(uint32_t total) const { *count = total; }
};

__global__ void k_range_count(const unsigned long long *halt, const uint32_t *F_dev, uint32_t f0,
                              uint32_t nf, uint32_t *out) {
    if (HALTED(halt)) return;
    const uint32_t F = *F_dev;
    *out = F > f0 ? min(F - f0, nf) : 0u;
}

// Per walk-list entry f (f < F; zero past it): status and conductance of its
// deletion, and its path length as the value scanned into the candidate
// offsets coff; the no-path flags go to noflag for the second scan.
struct DecrResultsOp {
    const unsigned long long *keys;
    const int32_t *plen;
    const uint32_t *f_idx, *F_dev;
    int32_t *status;
    float *cond;
    uint32_t *clen, *coff, *noflag, *counts;
    __device__ uint32_t load(uint32_t f) const {
        const uint32_t F = F_dev ? *F_dev : 0xFFFFFFFFu;
        if (f >= F) {
            noflag[f] = 0u;
            return 0u;
        }
        const uint32_t e = f_idx[f];
        const int32_t L = plen[f];
        const unsigned long long k = keys[f];
        status[e] = L > 0 ? L : DYG_DEL_NO_PATH;
        cond[e] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
        noflag[f] = L > 0 ? 0u : 1u;
        return L > 0 ? (uint32_t)L : 0u;
    }
    __device__ void store(uint32_t f, uint32_t excl, uint32_t v) const {
        coff[f] = excl;
        clen[f] = v;
    }
    __device__ void last(uint32_t total) const { counts[C_CANDS] = total; }
};

// The edges without a path, in walk-list order, for the fallback walks.
struct NoPathOp {
    const uint32_t *noflag;
    uint32_t *nop, *counts;
    uint32_t hw;
    __device__ uint32_t load(uint32_t f) const { return noflag[f]; }
    __device__ void store(uint32_t f, uint32_t q, uint32_t v) const {
        if (v) nop[q] = f;
    }
    __device__ void last(uint32_t total) const {
        counts[C_NOPATH] = total;
        counts[C_CANDS2] = total * 4u * hw;
        counts[C_CANDS_ALL] = counts[C_CANDS] + total * 4u * hw;
    }
};

// Path edges of walk-list entry f as recovery candidates at coff[f], one warp
// per path (consecutive lanes copy consecutive path edges); each edge's
// weight is read from the G slot the replay took (G is unchanged since).
__global__ void k_path_cands(const unsigned long long *halt, const uint32_t *pv, const uint32_t *ps,
                             const float *wts, uint32_t stride, const uint32_t *clen,
                             const uint32_t *coff, uint32_t n, uint32_t *cx, uint32_t *cy,
                             float *cw) {
    if (HALTED(halt)) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; f < n; f += warps) {
        const uint32_t L = clen[f];
        const uint32_t base = coff[f];
        const uint32_t *v = pv + (size_t)f * stride;
        const uint32_t *sl = ps + (size_t)f * stride;
        for (uint32_t j = lane; j < L; j += 32u) {
            cx[base + j] = v[j];
            cy[base + j] = v[j + 1];
            cw[base + j] = wts[sl[j + 1]];
        }
    }
}

// ------------------------------------------------------------- recovery

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

// Table of T = the smallest power of two >= max(1024, 2M) slots cleared; its
// mask and the kept count reset by the first thread.
__global__ void k_hash_clear(const unsigned long long *halt, const uint32_t *M_dev, uint32_t M_host,
                             unsigned long long *tk, uint32_t *tv, uint32_t *tmask,
                             uint32_t *counts) {
    if (HALTED(halt)) return;
    const uint32_t M = dcount(M_dev, M_host);
    uint32_t T = 1024u;
    while (T < 2u * M) T <<= 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *tmask = T - 1u;
        counts[C_KEPT] = 0u;
    }
    GSTRIDE(i, T) {
        tk[i] = ~0ull;
        tv[i] = ~0u;
    }
}

__global__ void k_hash_insert(const unsigned long long *halt, const uint32_t *cx,
                              const uint32_t *cy, const uint32_t *M_dev, uint32_t M_host,
                              unsigned long long *tk, uint32_t *tv, const uint32_t *tmask) {
    if (HALTED(halt)) return;
    const uint32_t M = dcount(M_dev, M_host), mask = *tmask;
    GSTRIDE(i, M) {
        const uint32_t x = cx[i], y = cy[i];
        if (x == ~0u || y == ~0u || x == y) continue;
        const unsigned long long k = ekey(x, y);
        uint32_t h = hslot(k, mask);
        while (true) {
            const unsigned long long prev = atomicCAS(tk + h, ~0ull, k);
            if (prev == ~0ull || prev == k) {
                atomicMin(tv + h, i);
                break;
            }
            h = (h + 1u) & mask;
        }
    }
}

// keep[i] = candidate i is the first occurrence of its edge and the edge is
// not in H (gpu_graph.cuh:534-538 and 599-601 test sparse_map the same way);
// zero for M <= i < M_host.  H membership scans the shorter of the two rows;
// when that row is longer than kBigRow the candidate goes to the big list and
// k_keep_big decides.
__global__ void k_hash_keep(const unsigned long long *halt, DevGraph h, const uint32_t *cx,
                            const uint32_t *cy, const uint32_t *M_dev, uint32_t M_host,
                            const unsigned long long *tk, const uint32_t *tv,
                            const uint32_t *tmask, uint32_t *keep, uint4 *big,
                            unsigned long long *nbig, bool big_ok) {
    if (HALTED(halt)) return;
    const uint32_t M = dcount(M_dev, M_host), mask = *tmask;
    GSTRIDE(i, M_host) {
        uint32_t kp = 0;
        if (i < M) {
            const uint32_t x = cx[i], y = cy[i];
            if (x != ~0u && y != ~0u && x != y) {
                const unsigned long long k = ekey(x, y);
                uint32_t s = hslot(k, mask);
                while (tk[s] != k) s = (s + 1u) & mask;
                if (tv[s] == i) {
                    kp = 1;
                    if (x < h.n && y < h.n) {
                        const uint2 dx = h.desc[x], dy = h.desc[y];
                        const bool xs = dx.y <= dy.y;
                        const uint2 d = xs ? dx : dy;
                        const uint32_t other = xs ? y : x;
                        if (big_ok && d.y > kBigRow) {
                            big[atomicAdd(nbig, 1ull)] = make_uint4(i, xs ? x : y, other, 0u);
                        } else {
                            // eight columns loaded before they are compared
                            for (uint32_t j0 = 0; j0 < d.y && kp; j0 += 8u) {
                                uint32_t cv[8];
#pragma unroll
                                for (uint32_t u = 0; u < 8u; ++u)
                                    cv[u] = j0 + u < d.y ? h.slots[d.x + j0 + u].x : ~0u;
#pragma unroll
                                for (uint32_t u = 0; u < 8u; ++u)
                                    if (cv[u] == other) kp = 0;
                            }
                        }
                    }
                }
            }
        }
        keep[i] = kp;
    }
}

// One block per long-row candidate: {candidate, row, column}.
__global__ void k_keep_big(const unsigned long long *halt, DevGraph h, const uint4 *big,
                           const unsigned long long *nbig, uint32_t *keep) {
    __shared__ uint32_t s_best;
    if (HALTED(halt)) return;
    const uint32_t nb = (uint32_t)*nbig;
    for (uint32_t q = blockIdx.x; q < nb; q += gridDim.x) {
        const uint4 e = big[q];
        const uint2 d = h.desc[e.y];
        const uint32_t j = block_find(h.slots, d.x, d.y, e.z, &s_best);
        if (threadIdx.x == 0 && j != ~0u) keep[e.x] = 0;
    }
}

// Kept candidates -> half-edges (x gets y, then y gets x), in candidate order,
// and the recovered-edge records after the ones recorded so far.  The kept
// edges must fit the record buffers: the records past them are not written
// and the last candidate halts the batch (it is resumed with larger buffers).
struct KeepEmitOp {
    const uint32_t *keep, *cx, *cy;
    const float *cw;
    uint8_t kind, kind_after;
    const uint32_t *split;   // candidates from *split on get kind_after (null: none)
    const unsigned long long *sc;
    unsigned long long *halt;
    unsigned long long code;
    uint32_t *hx, *hy;
    float *hw;
    uint32_t *rx, *ry;
    uint8_t *rk;
    uint32_t *counts;
    __device__ uint32_t load(uint32_t i) const { return keep[i]; }
    __device__ void store(uint32_t i, uint32_t q, uint32_t v) const {
        if (!v) return;
        const uint32_t x = cx[i], y = cy[i];
        const float w = cw[i];
        hx[2 * q] = x;
        hy[2 * q] = y;
        hw[2 * q] = w;
        hx[2 * q + 1] = y;
        hy[2 * q + 1] = x;
        hw[2 * q + 1] = w;
        const unsigned long long r = sc[S_RECCNT] + q;
        if (r < sc[S_RECCAP]) {
            rx[r] = x;
            ry[r] = y;
            rk[r] = (split && i >= *split) ? kind_after : kind;
        }
    }
    __device__ void last(uint32_t total) const {
        counts[C_KEPT] = 2u * total;
        if (sc[S_RECCNT] + total > sc[S_RECCAP]) atomicCAS(halt, 0ull, code);
    }
};

__global__ void k_rec_advance(const unsigned long long *halt, const uint32_t *counts,
                              unsigned long long *sc) {
    if (HALTED(halt)) return;
    sc[S_RECCNT] += counts[C_KEPT] / 2u;
}

// Dedup + membership + ordered append of one candidate list; candidates
// before *split (device, may be null) are recorded with `kind`, the rest with
// `kind_after`.
dyg_status recover_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *cx, const uint32_t *cy,
                           const float *cw, const uint32_t *M_dev, uint32_t M_host, uint8_t kind,
                           const uint32_t *split, uint8_t kind_after,
                           unsigned long long *halt, uint32_t batch, uint32_t phase,
                           cudaStream_t st) {
    if (M_host == 0) return DYG_OK;
    Workspace &ws = G->ws;
    uint32_t T = 1024;
    while (T < 2u * M_host) T <<= 1;
    DYG_TRY(ensure(ws.htab_k, sizeof(unsigned long long) * T));
    DYG_TRY(ensure(ws.htab_v, sizeof(uint32_t) * T));
    DYG_TRY(ensure(ws.tmask, sizeof(uint32_t)));
    DYG_TRY(ensure(ws.keep, sizeof(uint32_t) * (size_t)M_host));
    DYG_TRY(ensure(ws.big, sizeof(uint4) * (size_t)M_host));
    DYG_TRY(ensure(ws.hx, sizeof(uint32_t) * (size_t)M_host * 2));
    DYG_TRY(ensure(ws.hy, sizeof(uint32_t) * (size_t)M_host * 2));
    DYG_TRY(ensure(ws.hw, sizeof(float) * (size_t)M_host * 2));
    uint32_t *keep = ptr<uint32_t>(ws.keep);
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    const int gr = grid_for(M_host);
    k_hash_clear<<<grid_for((uint64_t)T), 256, 0, st>>>(halt, M_dev, M_host,
                                                        ptr<unsigned long long>(ws.htab_k),
                                                        ptr<uint32_t>(ws.htab_v),
                                                        ptr<uint32_t>(ws.tmask), counts);
    count_launch();
    k_hash_insert<<<gr, 256, 0, st>>>(halt, cx, cy, M_dev, M_host, ptr<unsigned long long>(ws.htab_k),
                                      ptr<uint32_t>(ws.htab_v), ptr<uint32_t>(ws.tmask));
    count_launch();
    const bool big_ok = H->long_rows;
    if (big_ok) DYG_CUDA(cudaMemsetAsync(sc + S_NBIG, 0, sizeof(unsigned long long), st));
    k_hash_keep<<<gr, 256, 0, st>>>(halt, H->g, cx, cy, M_dev, M_host,
                                    ptr<unsigned long long>(ws.htab_k), ptr<uint32_t>(ws.htab_v),
                                    ptr<uint32_t>(ws.tmask), keep, ptr<uint4>(ws.big), sc + S_NBIG,
                                    big_ok);
    count_launch();
    if (big_ok) {
        k_keep_big<<<num_sms() * 2, kBigThreads, 0, st>>>(halt, H->g, ptr<uint4>(ws.big),
                                                          sc + S_NBIG, keep);
        count_launch();
    }
    const KeepEmitOp op{keep, cx, cy, cw, kind, kind_after, split, sc, halt,
                        halt_code(batch, (uint32_t)kHaltRecords, phase),
                        ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw),
                        ptr<uint32_t>(ws.rx2), ptr<uint32_t>(ws.ry2), ptr<uint8_t>(ws.rk2), counts};
    DYG_TRY(scan_op(ws, op, M_host, M_dev, halt, st));
    DYG_CUDA(cudaGetLastError());
    AppendList L{ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw), counts + C_KEPT,
                 2u * M_host};
    DYG_TRY(append_enqueue(H, L, nullptr, nullptr, halt,
                           halt_code(batch, (uint32_t)kHaltArena, phase), st));
    k_rec_advance<<<1, 1, 0, st>>>(halt, counts, sc);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

}  // namespace

dyg_status validate_enqueue(unsigned long long *halt, unsigned long long *err,
                            const uint32_t *src, const uint32_t *dst, const float *w, uint32_t n,
                            uint32_t nv, cudaStream_t st) {
    if (n == 0) return DYG_OK;
    k_validate<<<grid_for(n), 256, 0, st>>>(halt, src, dst, w, n, nv, err);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// A call whose device-resident inputs failed k_validate: clear the halt and
// the error bits, and report which check failed.  Nothing was changed.
dyg_status rejected_inputs(dyg_graph *D, cudaStream_t st) {
    const unsigned long long err = D->ws.host_scalars[S_ERR];
    DYG_CUDA(cudaMemsetAsync(ptr<unsigned long long>(D->ws.scalars) + S_ERR, 0,
                             sizeof(unsigned long long), st));
    DYG_CUDA(cudaMemsetAsync(ptr<unsigned long long>(D->ws.scalars) + S_HALT, 0,
                             sizeof(unsigned long long), st));
    DYG_CUDA(cudaStreamSynchronize(st));
    D->ws.host_scalars[S_ERR] = 0ull;
    D->ws.host_scalars[S_HALT] = 0ull;
    if (err & kErrVertex)
        set_error("a batch endpoint is not a vertex of the graph (the call changed nothing)");
    else
        set_error("a batch weight is not finite and > 0 (the call changed nothing)");
    return DYG_EINVAL;
}

dyg_status grow_keep(Buf &b, size_t bytes, size_t used, cudaStream_t st) {
    if (b.bytes >= bytes) return DYG_OK;
    Buf nb;
    DYG_TRY(ensure(nb, bytes));
    if (used && b.p) {
        DYG_CUDA(cudaMemcpyAsync(nb.p, b.p, used, cudaMemcpyDeviceToDevice, st));
        DYG_CUDA(cudaStreamSynchronize(st));
    }
    if (b.p) cudaFree(b.p);
    b = nb;
    return DYG_OK;
}

// ------------------------------------------------------------ batches

// Enqueues incremental batch `batch` (edges src/dst/w[0, n), update ids
// uid0 + e).  Outputs go to found/cond/acc (device, may be null).
// Commit half of an incremental batch from its winner keys (keys[e] = 0: no
// walker connected edge e): decode, scan of the accept flags in input order,
// accepted half-edges to H [and every half-edge to G], reserved together.
dyg_status incr_commit_enqueue(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                               const uint32_t *dst, const float *w, uint32_t n,
                               const unsigned long long *keys, unsigned long long *halt,
                               uint32_t batch, int32_t *found, float *cond, uint8_t *acc,
                               cudaStream_t st) {
    Workspace &ws = H->ws;
    DYG_TRY(ensure(ws.hx, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(ws.hy, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(ws.hw, sizeof(float) * (size_t)n * 2));
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    IncrCommitOp op{keys, src, dst, w, found, cond, acc, ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy),
                    ptr<float>(ws.hw), nullptr, nullptr, nullptr, counts + C_HHALF};
    AppendList LH{ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw), counts + C_HHALF,
                  2u * n};
    AppendList LG{};
    if (G) {
        Workspace &wg = G->ws;
        DYG_TRY(ensure(wg.hx, sizeof(uint32_t) * (size_t)n * 2));
        DYG_TRY(ensure(wg.hy, sizeof(uint32_t) * (size_t)n * 2));
        DYG_TRY(ensure(wg.hw, sizeof(float) * (size_t)n * 2));
        op.gx = ptr<uint32_t>(wg.hx);
        op.gy = ptr<uint32_t>(wg.hy);
        op.gw = ptr<float>(wg.hw);
        LG = AppendList{op.gx, op.gy, op.gw, nullptr, 2u * n};
    }
    DYG_TRY(scan_op(ws, op, n, nullptr, halt, st));
    return append_enqueue(H, LH, G, G ? &LG : nullptr, halt,
                          halt_code(batch, (uint32_t)kHaltArena, 0), st);
}

dyg_status incr_enqueue(dyg_graph *H, dyg_graph *G, const uint32_t *src, const uint32_t *dst,
                        const float *w, uint32_t n, uint64_t uid0,
                        const unsigned long long *uids, const dyg_walk_params &p,
                        unsigned long long *halt, uint32_t batch, int32_t *found, float *cond,
                        uint8_t *acc, cudaStream_t st) {
    Workspace &ws = H->ws;
    DYG_TRY(ensure(ws.keys, sizeof(unsigned long long) * n));
    unsigned long long *keys = ptr<unsigned long long>(ws.keys);
    DYG_CUDA(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * n, st));
    WalkJob job{halt, src, dst, w, uids, (unsigned long long)uid0, nullptr, n, kDomainIncr};
    DYG_TRY(launch_walk(H, job, p, true, keys, st));
    return incr_commit_enqueue(H, G, src, dst, w, n, keys, halt, batch, found, cond, acc, st);
}

// Deletion stage of a decremental batch: delete every edge from G (swap with
// the row's last slot, in input order), erase the ones also in H, and compact
// the edges found in both into the walk list f_* (gpu_graph.cuh:338-458), each
// walked min -> max (random_walk_decremental/gpu_graph.cuh:342) or, with
// file_orient, src -> dst (dynamic_update/gpu_graph.cuh:874-875).
// status/cond (device, length n) get the per-deletion codes.
dyg_status decr_delete_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                               const uint32_t *dst, uint32_t n, uint64_t uid0,
                               const unsigned long long *uids, bool file_orient,
                               unsigned long long *halt, int32_t *status, float *cond,
                               cudaStream_t st) {
    Workspace &ws = G->ws;
    const uint32_t m = 2u * n;
    DYG_TRY(ensure(ws.del_hx, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.del_hy, sizeof(uint32_t) * (size_t)m));
    DYG_TRY(ensure(ws.found, (size_t)m * 2));
    DYG_TRY(ensure(ws.f_src, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_dst, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_idx, sizeof(uint32_t) * n));
    DYG_TRY(ensure(ws.f_uid, sizeof(unsigned long long) * n));
    uint32_t *hx = ptr<uint32_t>(ws.del_hx), *hy = ptr<uint32_t>(ws.del_hy);
    uint8_t *fG = ptr<uint8_t>(ws.found), *fH = fG + m;
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    k_del_half_edges<<<blocks(n, 256), 256, 0, st>>>(halt, src, dst, n, G->g.n, hx, hy,
                                                      sc + S_ERR);
    count_launch();
    DYG_TRY(delete_pair_enqueue(G, H, hx, hy, m, fG, fH, halt, st));
    const DelFilterOp op{fG, fH, status, cond, hx, hy, file_orient ? src : nullptr,
                         file_orient ? dst : nullptr, (unsigned long long)uid0, uids,
                         ptr<uint32_t>(ws.f_src), ptr<uint32_t>(ws.f_dst),
                         ptr<unsigned long long>(ws.f_uid), ptr<uint32_t>(ws.f_idx),
                         counts + C_FILTERED};
    DYG_TRY(scan_op(ws, op, n, nullptr, halt, st));
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// Walk-and-recover stage over walk-list entries [f0, f0 + nf) (nf a host
// bound; F_dev, if given, is the device count of the whole list), from phase
// `phase0` (0 = walks, 1 = path recovery, 2 = fallback).
dyg_status decr_walk_enqueue(dyg_graph *G, dyg_graph *H, uint32_t f0, uint32_t nf,
                             const uint32_t *F_dev, const dyg_walk_params &p,
                             unsigned long long *halt, uint32_t batch, uint32_t phase0,
                             int32_t *status, float *cond, cudaStream_t st,
                             const unsigned long long *keys_given) {
    if (nf == 0) return DYG_OK;
    Workspace &ws = G->ws;
    const uint32_t n = nf;
    const uint32_t stride = p.max_steps > 2 ? p.max_steps : 2;
    const uint32_t hwk = p.heuristic_walkers;
    DYG_TRY(ensure(ws.keys, sizeof(unsigned long long) * n));
    DYG_TRY(ensure(ws.path_v, sizeof(uint32_t) * (size_t)n * stride));
    DYG_TRY(ensure(ws.path_s, sizeof(uint32_t) * (size_t)n * stride));
    DYG_TRY(ensure(ws.path_len, sizeof(int32_t) * n));
    DYG_TRY(ensure(ws.nop, sizeof(uint32_t) * (size_t)n * 4));
    // path candidates at [0, C_CANDS), then the fallback candidates
    const size_t n_path = (size_t)n * (stride - 1u), n_fb = (size_t)n * 4u * hwk;
    DYG_TRY(ensure(ws.cand_x, sizeof(uint32_t) * (n_path + n_fb)));
    DYG_TRY(ensure(ws.cand_y, sizeof(uint32_t) * (n_path + n_fb)));
    DYG_TRY(ensure(ws.cand_w, sizeof(float) * (n_path + n_fb)));
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    uint32_t *clen = ptr<uint32_t>(ws.nop) + n, *coff = clen + n, *noflag = coff + n;
    const uint32_t *fsrc = ptr<uint32_t>(ws.f_src) + f0, *fdst = ptr<uint32_t>(ws.f_dst) + f0;
    const unsigned long long *fuid = ptr<unsigned long long>(ws.f_uid) + f0;
    const uint32_t *fidx = ptr<uint32_t>(ws.f_idx) + f0;
    // device count of this range: min(F - f0, nf) when F lives on the device
    const uint32_t *cnt_dev = nullptr;
    if (F_dev) {
        k_range_count<<<1, 1, 0, st>>>(halt, F_dev, f0, nf, counts + C_RANGE);
        count_launch();
        cnt_dev = counts + C_RANGE;
    }
    WalkJob job{halt, fsrc, fdst, nullptr, fuid, 0ull, cnt_dev, n, kDomainDecr};

    if (phase0 <= 0) {
        // walks on the updated G (main.cu:392, 420)
        const unsigned long long *keys = keys_given;
        if (!keys) {
            unsigned long long *k = ptr<unsigned long long>(ws.keys);
            DYG_CUDA(cudaMemsetAsync(k, 0, sizeof(unsigned long long) * n, st));
            DYG_TRY(launch_walk(G, job, p, false, k, st));
            keys = k;
        }
        DYG_TRY(launch_winner_paths(G, job, p, keys, n, stride, ptr<uint32_t>(ws.path_v),
                                    ptr<uint32_t>(ws.path_s), ptr<int32_t>(ws.path_len), st));
        const DecrResultsOp rop{keys, ptr<int32_t>(ws.path_len), fidx, cnt_dev, status, cond,
                                clen, coff, noflag, counts};
        DYG_TRY(scan_op(ws, rop, n, nullptr, halt, st));
        const NoPathOp nop_op{noflag, ptr<uint32_t>(ws.nop), counts, hwk};
        DYG_TRY(scan_op(ws, nop_op, n, nullptr, halt, st));
        k_path_cands<<<grid_for((uint64_t)n * 32u), 256, 0, st>>>(
            halt, ptr<uint32_t>(ws.path_v), ptr<uint32_t>(ws.path_s), G->g.wts, stride, clen, coff, n,
            ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y), ptr<float>(ws.cand_w));
        count_launch();
        DYG_CUDA(cudaGetLastError());
        if (hwk > 0) {
            // 2-step fallback walks for the edges without a path
            // (main.cu:400-408, 428-436); their candidates follow the path
            // candidates.  They read G only, which recovery does not change.
            DYG_TRY(launch_fallback_walks(G, halt, fsrc, fdst, fuid, ptr<uint32_t>(ws.nop),
                                          counts + C_NOPATH, n, p, counts + C_CANDS,
                                          ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                                          ptr<float>(ws.cand_w), st));
        }
    }
    if (phase0 <= 1) {
        // Path recovery (gpu_graph.cuh:514-552) and the fallback edges
        // (gpu_graph.cuh:577-615) in one pass over [path candidates, fallback
        // candidates].  It keeps what the two passes in turn keep: a fallback
        // edge equal to an earlier candidate is a repeat (dropped, as the
        // second pass drops it for being in H once the first appended it or
        // found it there), every other one is tested against H as before, and
        // appends and records follow candidate order.
        DYG_TRY(recover_enqueue(G, H, ptr<uint32_t>(ws.cand_x), ptr<uint32_t>(ws.cand_y),
                                ptr<float>(ws.cand_w), counts + C_CANDS_ALL,
                                (uint32_t)(n_path + n_fb), DYG_REC_PATH, counts + C_CANDS,
                                DYG_REC_FALLBACK, halt, batch, 1, st));
    }
    return DYG_OK;
}

// Decremental batch `batch` of the standalone updater: deletion stage, then
// walks over the batch's whole walk list.
dyg_status decr_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *src, const uint32_t *dst,
                        uint32_t n, uint64_t uid0, const unsigned long long *uids,
                        const dyg_walk_params &p,
                        unsigned long long *halt, uint32_t batch, uint32_t phase0,
                        int32_t *status, float *cond, cudaStream_t st) {
    if (phase0 <= 0)
        DYG_TRY(decr_delete_enqueue(G, H, src, dst, n, uid0, uids, false, halt, status, cond, st));
    return decr_walk_enqueue(G, H, 0, n, ptr<uint32_t>(G->ws.counts) + C_FILTERED, p, halt, batch,
                             phase0, status, cond, st);
}

// --------------------------------------------------------- stream drivers

namespace {

struct HaltInfo {
    uint32_t batch, kind, phase;
};

HaltInfo decode_halt(unsigned long long h) {
    return HaltInfo{(uint32_t)(h >> 8) - 1u, (uint32_t)((h >> 4) & 0xF), (uint32_t)(h & 0xF)};
}

dyg_status clear_halt(dyg_graph *D, cudaStream_t st) {
    DYG_CUDA(cudaMemsetAsync(ptr<unsigned long long>(D->ws.scalars) + S_HALT, 0,
                             sizeof(unsigned long long), st));
    return DYG_OK;
}

dyg_status grow_for_halt(dyg_graph *A, dyg_graph *B, cudaStream_t st) {
    DYG_TRY(grow_arena(A, A->g.arena_cap * 2, st));
    if (B) DYG_TRY(grow_arena(B, B->g.arena_cap * 2, st));
    return DYG_OK;
}

}  // namespace

dyg_status incremental_run(dyg_graph *H, dyg_graph *G, const uint32_t *src, const uint32_t *dst,
                           const float *w, uint32_t n, uint32_t B, uint64_t uid_base,
                           const unsigned long long *uids, const dyg_walk_params &p, int32_t *found, float *cond, uint8_t *acc,
                           cudaStream_t st, bool check_inputs,
                           const std::function<void()> *during) {
    unsigned long long *sc = ptr<unsigned long long>(H->ws.scalars);
    unsigned long long *halt = sc + S_HALT;
    DYG_TRY(clear_halt(H, st));
    if (check_inputs) DYG_TRY(validate_enqueue(halt, sc + S_ERR, src, dst, w, n, H->g.n, st));
    uint32_t b_start = 0;
    for (int round = 0; round < 64; ++round) {
        for (uint32_t b = b_start; (uint64_t)b * B < n; ++b) {
            const uint32_t b0 = b * B, nb = (n - b0 < B) ? n - b0 : B;
            DYG_TRY(incr_enqueue(H, G, src + b0, dst + b0, w + b0, nb, uid_base + b0,
                                 uids ? uids + b0 : nullptr, p, halt, b,
                                 found ? found + b0 : nullptr, cond ? cond + b0 : nullptr,
                                 acc ? acc + b0 : nullptr, st));
        }
        if (during && round == 0) (*during)();
        DYG_TRY(read_scalars2(H, G, st));
        const unsigned long long h = H->ws.host_scalars[S_HALT];
        if (!h) return DYG_OK;
        const HaltInfo hi = decode_halt(h);
        if (hi.kind == kHaltInvalid) return rejected_inputs(H, st);
        DYG_TRY(grow_for_halt(H, G, st));
        DYG_TRY(clear_halt(H, st));
        b_start = hi.batch;   // nothing of the halted batch changed: redo it whole
    }
    set_error("incremental stream: too many arena regrowths");
    return DYG_ENOMEM;
}

dyg_status decremental_run(dyg_graph *G, dyg_graph *H, const uint32_t *src, const uint32_t *dst,
                           uint32_t n, uint32_t B, uint64_t uid_base,
                           const unsigned long long *uids, const dyg_walk_params &p,
                           int32_t *status, float *cond, uint64_t *n_rec, cudaStream_t st,
                           bool check_inputs, const std::function<void()> *during) {
    Workspace &ws = G->ws;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    unsigned long long *halt = sc + S_HALT;
    // record buffers: start at 4 per deletion, grown on demand (halt + resume)
    const uint64_t want = (uint64_t)n * 4 + 1024;
    DYG_TRY(ensure(ws.rx2, sizeof(uint32_t) * want));
    DYG_TRY(ensure(ws.ry2, sizeof(uint32_t) * want));
    DYG_TRY(ensure(ws.rk2, want));
    uint64_t cap = ws.rx2.bytes / 4;
    if (ws.ry2.bytes / 4 < cap) cap = ws.ry2.bytes / 4;
    if (ws.rk2.bytes < cap) cap = ws.rk2.bytes;
    unsigned long long init[2] = {0ull, cap};   // S_RECCNT, S_RECCAP
    DYG_CUDA(cudaMemcpyAsync(sc + S_RECCNT, init, sizeof(init), cudaMemcpyHostToDevice, st));
    DYG_TRY(clear_halt(G, st));
    if (check_inputs) DYG_TRY(validate_enqueue(halt, sc + S_ERR, src, dst, nullptr, n, G->g.n, st));
    uint32_t b_start = 0, ph_start = 0;
    for (int round = 0; round < 64; ++round) {
        for (uint32_t b = b_start; (uint64_t)b * B < n; ++b) {
            const uint32_t b0 = b * B, nb = (n - b0 < B) ? n - b0 : B;
            DYG_TRY(decr_enqueue(G, H, src + b0, dst + b0, nb, uid_base + b0,
                                 uids ? uids + b0 : nullptr, p, halt, b,
                                 b == b_start ? ph_start : 0, status + b0, cond + b0, st));
        }
        if (during && round == 0) (*during)();
        DYG_TRY(read_scalars2(G, H, st));
        const unsigned long long h = ws.host_scalars[S_HALT];
        if (!h) {
            *n_rec = ws.host_scalars[S_RECCNT];
            return DYG_OK;
        }
        const HaltInfo hi = decode_halt(h);
        if (hi.kind == kHaltInvalid) return rejected_inputs(G, st);
        if (hi.kind == kHaltRecords) {
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
        DYG_TRY(clear_halt(G, st));
        b_start = hi.batch;
        ph_start = hi.phase;   // deletions and walks of this batch are done: resume there
    }
    set_error("decremental stream: too many buffer regrowths");
    return DYG_ENOMEM;
}

}  // namespace dyg
