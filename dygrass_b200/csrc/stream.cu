// stream.cu -- one file of the mixed insert/delete edge stream
// (dynamic_update/main.cu:96-126: preprocessStreamEdges, then walks in
// chunks with the sparsifier updated after each chunk).
//
// Insert file (gpu_graph.cuh:373-396, 620-643), all on the device:
//   probe    every edge's slot positions in G and H (rows scanned by groups
//            of 8 lanes, the shorter row first);
//   sort     (min, max) keys with their file indices (stable radix sort), so
//            the occurrences of one edge sit together in file order;
//   merge    one thread per edge group: an edge already in G adds every
//            occurrence's weight to G (and H) in file order; a new edge's
//            first occurrence enters G with the later occurrences' weights
//            folded in, and is listed for walking;
//   append   the new edges to G in file order (row order as the reference's
//            edgeInsertion produces);
//   chunks   of the walk list: walk H, then append the accepted edges to H
//            with their stream weight before the next chunk walks.
// Delete file (gpu_graph.cuh:398-431, 645-700): the whole file is deleted
// from G and H, then the walk list is walked on G and recovered in chunks.
// One host synchronize per file; a reservation that does not fit halts every
// later kernel and the file resumes at the halted stage after the arena or
// record buffers grew (nothing changed after the halt; the weight merges
// come before any reservation and are not repeated).
#include <cub/cub.cuh>

#include "dyg_internal.cuh"
#include "scan.cuh"

namespace dyg {

namespace {

constexpr uint32_t kProbeLanes = 8;

inline int blocks(uint64_t n, int th) { return (int)((n + th - 1) / th); }

#define HALTED(h) ((h) && *(h))

// Arena index of the first slot of row x holding y, or ~0u.  Called by the
// kProbeLanes lanes of one group together (`gmask` = the group's lanes).
__device__ __forceinline__ uint32_t group_find(const DevGraph &g, uint32_t x, uint32_t y,
                                               uint32_t lane, uint32_t gbase, uint32_t gmask) {
    const uint2 d = g.desc[x];
    constexpr uint32_t U = 4;   // a group's tile: U loads per lane issued before any compare
    for (uint32_t t0 = 0; t0 < d.y; t0 += U * kProbeLanes) {
        uint32_t cv[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t j = t0 + u * kProbeLanes + lane;
            cv[u] = j < d.y ? g.slots[d.x + j].x : ~0u;   // vertex ids are never ~0u
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t bits =
                (__ballot_sync(gmask, cv[u] == y) >> gbase) & ((1u << kProbeLanes) - 1u);
            if (bits) return d.x + t0 + u * kProbeLanes + (uint32_t)(__ffs(bits) - 1);
        }
    }
    return ~0u;
}

// Slots of edge {a, b} in g: .x in row a, .y in row b (~0u when absent).
__device__ __forceinline__ uint2 group_edge(const DevGraph &g, uint32_t a, uint32_t b,
                                            uint32_t lane, uint32_t gbase, uint32_t gmask) {
    const bool a_short = g.desc[a].y <= g.desc[b].y;
    const uint32_t s = a_short ? a : b, l = a_short ? b : a;
    const uint32_t ps = group_find(g, s, l, lane, gbase, gmask);
    if (ps == ~0u) return make_uint2(~0u, ~0u);
    const uint32_t pl = group_find(g, l, s, lane, gbase, gmask);
    return a_short ? make_uint2(ps, pl) : make_uint2(pl, ps);
}

__device__ __forceinline__ bool long_rows(const DevGraph &g, uint32_t a, uint32_t b) {
    return g.desc[a].y > kBigRow || g.desc[b].y > kBigRow;
}

// group_edge for an edge with a row longer than kBigRow: the group searches
// the shorter row when it has at most kBigRow slots, which settles an absent
// edge; *open is set when a search of a long row remains (the edge is in the
// short row, whose slot is returned, or both rows are long).
__device__ __forceinline__ uint2 group_edge_short(const DevGraph &g, uint32_t a, uint32_t b,
                                                  uint32_t lane, uint32_t gbase, uint32_t gmask,
                                                  bool *open) {
    const uint2 da = g.desc[a], db = g.desc[b];
    const bool a_short = da.y <= db.y;
    *open = false;
    if ((a_short ? db.y : da.y) <= kBigRow) return group_edge(g, a, b, lane, gbase, gmask);
    if ((a_short ? da.y : db.y) > kBigRow) {
        *open = true;
        return make_uint2(~0u, ~0u);
    }
    const uint32_t ps = group_find(g, a_short ? a : b, a_short ? b : a, lane, gbase, gmask);
    *open = ps != ~0u;
    return a_short ? make_uint2(ps, ~0u) : make_uint2(~0u, ps);
}

// One group of kProbeLanes lanes per edge: slot positions in G and H, the
// sort key (min << nb | max) and index; self-loops and invalid endpoints get
// key ~0 (sorted last, never merged or walked).  An edge with a row longer
// than kBigRow in G or H has its short rows searched here
// (group_edge_short); if a long row remains to be searched it goes to the big
// list for k_st_probe_big, with bit 0 (G) and bit 1 (H) of .w naming the
// graphs whose search is open.
__global__ void k_st_probe(const unsigned long long *halt, DevGraph G, DevGraph H,
                           const uint32_t *src, const uint32_t *dst, uint32_t n, uint32_t nb,
                           unsigned long long *key, uint32_t *val, uint4 *pos, uint32_t *nflag,
                           int32_t *status, float *cond, uint4 *big, unsigned long long *nbig,
                           bool big_ok, unsigned long long *err) {
    if (HALTED(halt)) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = t / kProbeLanes;
    const uint32_t lane = t % kProbeLanes;
    const uint32_t gbase = (threadIdx.x & 31u) & ~(kProbeLanes - 1u);
    const uint32_t gmask = ((1u << kProbeLanes) - 1u) << gbase;
    if (i >= n) return;   // whole groups leave together (n is per group)
    uint32_t a = src[i], b = dst[i];
    if (a > b) {
        const uint32_t x = a;
        a = b;
        b = x;
    }
    if (a == b || b >= G.n) {
        if (lane == 0) {
            if (b >= G.n) atomicOr(err, (unsigned long long)kErrVertex);
            key[i] = ~0ull;
            val[i] = i;
            pos[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
            nflag[i] = 0;
            status[i] = DYG_INS_SELF_LOOP;
            cond[i] = 0.f;
        }
        return;
    }
    if (lane == 0) {
        key[i] = ((unsigned long long)a << nb) | b;
        val[i] = i;
        nflag[i] = 0;
    }
    if (big_ok && (long_rows(G, a, b) || long_rows(H, a, b))) {
        bool og, oh;
        const uint2 pg = group_edge_short(G, a, b, lane, gbase, gmask, &og);
        const uint2 ph = group_edge_short(H, a, b, lane, gbase, gmask, &oh);
        if (lane == 0) {
            pos[i] = make_uint4(pg.x, pg.y, ph.x, ph.y);
            if (og || oh)
                big[atomicAdd(nbig, 1ull)] = make_uint4(i, a, b, (og ? 1u : 0u) | (oh ? 2u : 0u));
        }
        return;
    }
    const uint2 pg = group_edge(G, a, b, lane, gbase, gmask);
    const uint2 ph = group_edge(H, a, b, lane, gbase, gmask);
    if (lane == 0) pos[i] = make_uint4(pg.x, pg.y, ph.x, ph.y);
}

// Finishes group_edge_short's search of edge {a, b} in g by block-wide
// scans: `part` is its result (the short row's slot when only the long row
// remains).
__device__ uint2 block_edge(const DevGraph &g, uint32_t a, uint32_t b, uint2 part,
                            uint32_t *s_best) {
    const uint2 da = g.desc[a], db = g.desc[b];
    const bool a_short = da.y <= db.y;
    const uint2 ds = a_short ? da : db, dl = a_short ? db : da;
    const uint32_t s = a_short ? a : b, l = a_short ? b : a;
    uint32_t ps = a_short ? part.x : part.y;
    if (ds.y > kBigRow) {
        const uint32_t js = block_find(g.slots, ds.x, ds.y, l, s_best);
        if (js == ~0u) return make_uint2(~0u, ~0u);
        ps = ds.x + js;
    }
    const uint32_t jl = block_find(g.slots, dl.x, dl.y, s, s_best);
    const uint32_t pl = jl == ~0u ? ~0u : dl.x + jl;
    return a_short ? make_uint2(ps, pl) : make_uint2(pl, ps);
}

// One block per edge on the big list: the long-row searches k_st_probe left.
__global__ void k_st_probe_big(const unsigned long long *halt, DevGraph G, DevGraph H,
                               const uint4 *big, const unsigned long long *nbig, uint4 *pos) {
    __shared__ uint32_t s_best;
    if (HALTED(halt)) return;
    const uint32_t nbl = (uint32_t)*nbig;
    for (uint32_t q = blockIdx.x; q < nbl; q += gridDim.x) {
        const uint4 e = big[q];
        uint4 p = pos[e.x];
        if (e.w & 1u) {
            const uint2 pg = block_edge(G, e.y, e.z, make_uint2(p.x, p.y), &s_best);
            p.x = pg.x;
            p.y = pg.y;
        }
        if (e.w & 2u) {
            const uint2 ph = block_edge(H, e.y, e.z, make_uint2(p.z, p.w), &s_best);
            p.z = ph.x;
            p.w = ph.y;
        }
        if (threadIdx.x == 0) pos[e.x] = p;   // each edge is on the list once
    }
}

__device__ __forceinline__ void set_weight(DevGraph &g, uint32_t slot, float w) {
    g.wts[slot] = w;
    g.slots[slot].y = __float_as_uint(__frcp_rn(w));
}

// One thread per group of equal keys (dynamic_update/gpu_graph.cuh:373-396,
// 452-465): weights are folded in file order, one float add per occurrence.
__global__ void k_st_merge(const unsigned long long *halt, DevGraph G, DevGraph H,
                           const unsigned long long *skey, const uint32_t *sval, uint32_t n,
                           const uint4 *pos, const float *w, uint32_t *nflag, float *wapp,
                           int32_t *status, float *cond) {
    if (HALTED(halt)) return;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const unsigned long long k = skey[j];
    if (k == ~0ull || (j > 0 && skey[j - 1] == k)) return;
    uint32_t e = j + 1;
    while (e < n && skey[e] == k) ++e;
    const uint32_t i0 = sval[j];
    const uint4 p = pos[i0];
    const bool inH = p.z != ~0u;
    float ha = inH ? H.wts[p.z] : 0.f, hb = (inH && p.w != ~0u) ? H.wts[p.w] : 0.f;
    if (p.x != ~0u) {
        // already in G: every occurrence adds its weight to G and (if there) H
        float ga = G.wts[p.x], gb = p.y != ~0u ? G.wts[p.y] : 0.f;
        for (uint32_t q = j; q < e; ++q) {
            const uint32_t i = sval[q];
            const float wi = w[i];
            ga = __fadd_rn(ga, wi);
            gb = __fadd_rn(gb, wi);
            if (inH) {
                ha = __fadd_rn(ha, wi);
                hb = __fadd_rn(hb, wi);
            }
            status[i] = DYG_INS_MERGED;
            cond[i] = 0.f;
        }
        set_weight(G, p.x, ga);
        if (p.y != ~0u) set_weight(G, p.y, gb);
    } else {
        // new: the first occurrence enters G and is walked; the later ones
        // add their weights to its G copy (and to H's, if H has the edge)
        float wa = w[i0];
        for (uint32_t q = j + 1; q < e; ++q) {
            const uint32_t i = sval[q];
            const float wi = w[i];
            wa = __fadd_rn(wa, wi);
            if (inH) {
                ha = __fadd_rn(ha, wi);
                hb = __fadd_rn(hb, wi);
            }
            status[i] = DYG_INS_MERGED;
            cond[i] = 0.f;
        }
        nflag[i0] = 1u;
        wapp[i0] = wa;
    }
    if (inH) {
        set_weight(H, p.z, ha);
        if (p.w != ~0u) set_weight(H, p.w, hb);
    }
}

// New edges in file order: the walk list (file orientation, stream weight)
// and G's half-edges (src gets dst, dst gets src; merged weight), at the
// scanned positions of the new-edge flags.
struct StCompactOp {
    const uint32_t *nflag, *src, *dst;
    const float *w, *wapp;
    unsigned long long uid0;
    uint32_t *f_src, *f_dst;
    float *f_w;
    unsigned long long *f_uid;
    uint32_t *f_idx, *hx, *hy;
    float *hw;
    uint32_t *counts;
    __device__ uint32_t load(uint32_t i) const { return nflag[i]; }
    __device__ void store(uint32_t i, uint32_t q, uint32_t v) const {
        if (!v) return;
        const uint32_t u = src[i], x = dst[i];
        f_src[q] = u;
        f_dst[q] = x;
        f_w[q] = w[i];
        f_uid[q] = uid0 + i;
        f_idx[q] = i;
        const float wa = wapp[i];
        hx[2 * q] = u;
        hy[2 * q] = x;
        hw[2 * q] = wa;
        hx[2 * q + 1] = x;
        hy[2 * q + 1] = u;
        hw[2 * q + 1] = wa;
    }
    __device__ void last(uint32_t total) const {
        counts[C_WALKLIST] = total;
        counts[C_GHALF] = 2u * total;
    }
};

__global__ void k_st_range(const unsigned long long *halt, const uint32_t *F_dev, uint32_t f0,
                           uint32_t nf, uint32_t *out) {
    if (HALTED(halt)) return;
    const uint32_t F = *F_dev;
    *out = F > f0 ? min(F - f0, nf) : 0u;
}

// Chunk results: found_at / conductance by file index, and the accepted
// edges (no walker connected them) to H's half-edge list in chunk order;
// entries past the chunk's device count are not accepted.
struct StAcceptOp {
    const unsigned long long *keys;
    const uint32_t *f_idx, *cnt, *f_src, *f_dst;
    const float *f_w;
    int32_t *status;
    float *cond;
    uint32_t *hx, *hy;
    float *hw;
    uint32_t *counts;
    __device__ uint32_t load(uint32_t f) const {
        if (f >= *cnt) return 0u;
        const unsigned long long k = keys[f];
        const uint32_t i = f_idx[f];
        status[i] = key_found(k);
        cond[i] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
        return k ? 0u : 1u;
    }
    __device__ void store(uint32_t f, uint32_t q, uint32_t v) const {
        if (!v) return;
        const uint32_t u = f_src[f], x = f_dst[f];
        const float ww = f_w[f];
        hx[2 * q] = u;
        hy[2 * q] = x;
        hw[2 * q] = ww;
        hx[2 * q + 1] = x;
        hy[2 * q + 1] = u;
        hw[2 * q + 1] = ww;
    }
    __device__ void last(uint32_t total) const { counts[C_ACCEPTED] = 2u * total; }
};

// Files of up to kSortSmall edges are grouped by one block: a bitonic sort of
// words (key << 13 | file index), so equal keys stay in file order -- the
// order the radix sort of larger files gives -- and self-loop keys (~0),
// mapped to the largest 2nb-bit key, come last; in one launch instead of six.
// Each thread holds kSortE consecutive words: partners closer than kSortE
// are compared in registers, closer than 32 kSortE through warp shuffles,
// and only the farther ones through shared memory.
constexpr uint32_t kSortSmall = 8192;   // file indices fit 13 bits
constexpr uint32_t kSortE = 8;

__device__ __forceinline__ unsigned long long sort_keep(unsigned long long mine,
                                                        unsigned long long other, uint32_t i,
                                                        uint32_t j, uint32_t k) {
    // element i keeps the smaller word when it is the lower one of an
    // ascending pair or the upper one of a descending pair
    return (((i & j) == 0u) == ((i & k) == 0u)) ? min(mine, other) : max(mine, other);
}

template <uint32_t J>
__device__ __forceinline__ void sort_in_thread(unsigned long long (&v)[kSortE], uint32_t t,
                                               uint32_t k) {
#pragma unroll
    for (uint32_t e = 0; e < kSortE; ++e) {
        constexpr uint32_t kJ = J;
        const uint32_t p = e ^ kJ;
        if (p > e) {
            const bool asc = ((t * kSortE + e) & k) == 0u;
            const unsigned long long a = v[e], b = v[p];
            if ((a > b) == asc) {
                v[e] = b;
                v[p] = a;
            }
        }
    }
}

__global__ void __launch_bounds__(kSortSmall / kSortE)
k_sort_small(const unsigned long long *key, uint32_t n, uint32_t N, uint32_t kbits,
             unsigned long long *skey, uint32_t *sval) {
    extern __shared__ unsigned long long s_w[];   // N words
    const uint32_t t = threadIdx.x;
    const unsigned long long kmax = (1ull << kbits) - 1ull;   // above every real key
    for (uint32_t i = t; i < N; i += blockDim.x) {
        unsigned long long w = ~0ull;   // padding sorts after every entry
        if (i < n) {
            const unsigned long long k = key[i];
            w = ((k == ~0ull ? kmax : k) << 13) | i;
        }
        s_w[i] = w;
    }
    __syncthreads();
    unsigned long long v[kSortE];
#pragma unroll
    for (uint32_t e = 0; e < kSortE; ++e) v[e] = s_w[t * kSortE + e];
    for (uint32_t k = 2; k <= N; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32u * kSortE) {
                __syncthreads();   // the last readers of s_w are done
#pragma unroll
                for (uint32_t e = 0; e < kSortE; ++e) s_w[t * kSortE + e] = v[e];
                __syncthreads();
#pragma unroll
                for (uint32_t e = 0; e < kSortE; ++e) {
                    const uint32_t i = t * kSortE + e;
                    v[e] = sort_keep(v[e], s_w[i ^ j], i, j, k);
                }
            } else if (j >= kSortE) {
                const uint32_t d = j / kSortE;   // partner lane offset
#pragma unroll
                for (uint32_t e = 0; e < kSortE; ++e) {
                    const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, v[e], d);
                    v[e] = sort_keep(v[e], o, t * kSortE + e, j, k);
                }
            } else if (j == 4u) {
                sort_in_thread<4>(v, t, k);
            } else if (j == 2u) {
                sort_in_thread<2>(v, t, k);
            } else {
                sort_in_thread<1>(v, t, k);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (uint32_t e = 0; e < kSortE; ++e) s_w[t * kSortE + e] = v[e];
    __syncthreads();
    for (uint32_t i = t; i < n; i += blockDim.x) {
        const unsigned long long w = s_w[i];
        const unsigned long long k = w >> 13;
        skey[i] = k == kmax ? ~0ull : k;
        sval[i] = (uint32_t)(w & 0x1FFFu);
    }
}

// The one-block sort applies to files of up to kSortSmall edges whose keys
// (2 nb bits) and file indices (13 bits) fit one word below the padding.
bool sort_small_fits(uint32_t n, uint32_t nb) { return n <= kSortSmall && 2u * nb + 13u <= 63u; }

dyg_status sort_small_enqueue(const unsigned long long *key, uint32_t n, uint32_t nb,
                              unsigned long long *skey, uint32_t *sval, cudaStream_t st) {
    uint32_t N = 32u * kSortE;
    while (N < n) N <<= 1;
    const size_t bytes = (size_t)N * sizeof(unsigned long long);
    if (bytes > 48u * 1024u)   // the attribute belongs to the current device
        DYG_CUDA(cudaFuncSetAttribute(k_sort_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bytes));
    k_sort_small<<<1, N / kSortE, bytes, st>>>(key, n, N, 2u * nb, skey, sval);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

uint32_t key_bits(uint32_t nv) {
    uint32_t b = 1;
    while (b < 32 && (nv - 1u) >> b) ++b;
    return b;
}

// Probe, sort, merge and compact an insert file (no reservation: never halts).
dyg_status insert_prep_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                               const uint32_t *dst, const float *w, uint32_t n, uint64_t uid0,
                               unsigned long long *halt, int32_t *status, float *cond,
                               cudaStream_t st) {
    Workspace &ws = G->ws;
    const uint32_t nb = key_bits(G->g.n);
    unsigned long long *key = ptr<unsigned long long>(ws.st_key), *skey = key + n;
    uint32_t *val = ptr<uint32_t>(ws.st_val), *sval = val + n;
    uint32_t *nflag = ptr<uint32_t>(ws.flags);
    uint32_t *counts = ptr<uint32_t>(ws.counts);
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    const bool big_ok = G->long_rows || H->long_rows;
    if (big_ok) DYG_CUDA(cudaMemsetAsync(sc + S_NBIG, 0, sizeof(unsigned long long), st));
    k_st_probe<<<blocks((uint64_t)n * kProbeLanes, 256), 256, 0, st>>>(
        halt, G->g, H->g, src, dst, n, nb, key, val, ptr<uint4>(ws.st_pos), nflag, status, cond,
        ptr<uint4>(ws.big), sc + S_NBIG, big_ok, sc + S_ERR);
    count_launch();
    if (big_ok) {
        k_st_probe_big<<<num_sms() * 4, kBigThreads, 0, st>>>(halt, G->g, H->g, ptr<uint4>(ws.big),
                                                              sc + S_NBIG, ptr<uint4>(ws.st_pos));
        count_launch();
    }
    if (sort_small_fits(n, nb)) {
        DYG_TRY(sort_small_enqueue(key, n, nb, skey, sval, st));   // values are file indices
    } else {
        size_t tmp = 0;
        DYG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp, key, skey, val, sval, (int)n, 0,
                                                 (int)(2 * nb), st));
        DYG_TRY(ensure(ws.cub_tmp, tmp));
        tmp = ws.cub_tmp.bytes;
        // keys ~0 (self-loops) have all bits set: sorting on the low 2*nb
        // bits still places them after every real key (each real key is
        // < 2^(2nb) - 1)
        DYG_CUDA(cub::DeviceRadixSort::SortPairs(ws.cub_tmp.p, tmp, key, skey, val, sval, (int)n, 0,
                                                 (int)(2 * nb), st));
    }
    k_st_merge<<<blocks(n, 256), 256, 0, st>>>(halt, G->g, H->g, skey, sval, n,
                                                ptr<uint4>(ws.st_pos), w, nflag,
                                                ptr<float>(ws.st_wapp), status, cond);
    count_launch();
    const StCompactOp op{nflag, src, dst, w, ptr<float>(ws.st_wapp), (unsigned long long)uid0,
                         ptr<uint32_t>(ws.f_src), ptr<uint32_t>(ws.f_dst), ptr<float>(ws.f_w),
                         ptr<unsigned long long>(ws.f_uid), ptr<uint32_t>(ws.f_idx),
                         ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw), counts};
    DYG_TRY(scan_op(ws, op, n, nullptr, halt, st));
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status insert_gappend_enqueue(dyg_graph *G, uint32_t n, unsigned long long *halt,
                                  cudaStream_t st) {
    Workspace &ws = G->ws;
    AppendList L{ptr<uint32_t>(ws.hx), ptr<uint32_t>(ws.hy), ptr<float>(ws.hw),
                 ptr<uint32_t>(ws.counts) + C_GHALF, 2u * n};
    return append_enqueue(G, L, nullptr, nullptr, halt, halt_code(0, (uint32_t)kHaltArena, 1), st);
}

// Walks chunk c (walk-list entries [c*chunk, c*chunk + nc)) on H and appends
// its accepted edges to H.
dyg_status insert_chunk_enqueue(dyg_graph *G, dyg_graph *H, uint32_t c, uint32_t chunk,
                                uint32_t nc, const dyg_walk_params &p, unsigned long long *halt,
                                int32_t *status, float *cond, cudaStream_t st) {
    Workspace &wg = G->ws, &wh = H->ws;
    const uint32_t f0 = c * chunk;
    uint32_t *gcounts = ptr<uint32_t>(wg.counts), *hcounts = ptr<uint32_t>(wh.counts);
    k_st_range<<<1, 1, 0, st>>>(halt, gcounts + C_WALKLIST, f0, nc, gcounts + C_RANGE);
    count_launch();
    const uint32_t *cnt = gcounts + C_RANGE;
    const uint32_t *fsrc = ptr<uint32_t>(wg.f_src) + f0, *fdst = ptr<uint32_t>(wg.f_dst) + f0;
    const float *fw = ptr<float>(wg.f_w) + f0;
    unsigned long long *keys = ptr<unsigned long long>(wh.keys);
    DYG_CUDA(cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * nc, st));
    WalkJob job{halt, fsrc, fdst, fw, ptr<unsigned long long>(wg.f_uid) + f0, 0ull, cnt, nc,
                kDomainIncr};
    DYG_TRY(launch_walk(H, job, p, true, keys, st));
    const StAcceptOp op{keys, ptr<uint32_t>(wg.f_idx) + f0, cnt, fsrc, fdst, fw, status, cond,
                        ptr<uint32_t>(wh.hx), ptr<uint32_t>(wh.hy), ptr<float>(wh.hw), hcounts};
    DYG_TRY(scan_op(wh, op, nc, nullptr, halt, st));
    DYG_CUDA(cudaGetLastError());
    AppendList L{ptr<uint32_t>(wh.hx), ptr<uint32_t>(wh.hy), ptr<float>(wh.hw),
                 hcounts + C_ACCEPTED, 2u * nc};
    return append_enqueue(H, L, nullptr, nullptr, halt,
                          halt_code(c + 1, (uint32_t)kHaltArena, 0), st);
}

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

dyg_status insert_file_run(dyg_graph *G, dyg_graph *H, const uint32_t *src, const uint32_t *dst,
                           const float *w, uint32_t n, uint64_t uid0, uint32_t chunk,
                           const dyg_walk_params &p, int32_t *status, float *cond,
                           cudaStream_t st, bool check_inputs) {
    Workspace &wg = G->ws, &wh = H->ws;
    const uint32_t nc_max = n < chunk ? n : chunk;
    // every buffer at its final size before anything is enqueued: a resumed
    // stage finds the earlier stages' lists where they were left
    DYG_TRY(ensure(wg.st_key, sizeof(unsigned long long) * (size_t)n * 2));
    DYG_TRY(ensure(wg.st_val, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(wg.st_pos, sizeof(uint4) * (size_t)n));
    DYG_TRY(ensure(wg.st_wapp, sizeof(float) * (size_t)n));
    DYG_TRY(ensure(wg.big, sizeof(uint4) * (size_t)n * 2));   // probe, then the G append
    DYG_TRY(ensure(wg.dtmp, sizeof(uint32_t) * (size_t)n * 4));
    DYG_TRY(ensure(wg.rank, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(wg.lneed, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(wg.flags, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(wg.pos, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(wg.f_src, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(wg.f_dst, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(wg.f_w, sizeof(float) * (size_t)n));
    DYG_TRY(ensure(wg.f_uid, sizeof(unsigned long long) * (size_t)n));
    DYG_TRY(ensure(wg.f_idx, sizeof(uint32_t) * (size_t)n));
    DYG_TRY(ensure(wg.hx, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(wg.hy, sizeof(uint32_t) * (size_t)n * 2));
    DYG_TRY(ensure(wg.hw, sizeof(float) * (size_t)n * 2));
    DYG_TRY(ensure(wh.keys, sizeof(unsigned long long) * (size_t)nc_max));
    DYG_TRY(ensure(wh.hx, sizeof(uint32_t) * (size_t)nc_max * 2));
    DYG_TRY(ensure(wh.hy, sizeof(uint32_t) * (size_t)nc_max * 2));
    DYG_TRY(ensure(wh.hw, sizeof(float) * (size_t)nc_max * 2));
    unsigned long long *halt = ptr<unsigned long long>(wg.scalars) + S_HALT;
    DYG_TRY(clear_halt(G, st));
    if (check_inputs)
        DYG_TRY(validate_enqueue(halt, ptr<unsigned long long>(wg.scalars) + S_ERR, src, dst, w, n,
                                 G->g.n, st));
    DYG_TRY(insert_prep_enqueue(G, H, src, dst, w, n, uid0, halt, status, cond, st));
    const uint32_t nchunks = (uint32_t)(((uint64_t)n + chunk - 1) / chunk);
    uint32_t start = 0;   // 0 = G append, c + 1 = chunk c
    for (int round = 0; round < 64; ++round) {
        if (start == 0) DYG_TRY(insert_gappend_enqueue(G, n, halt, st));
        for (uint32_t c = start ? start - 1 : 0; c < nchunks; ++c) {
            const uint32_t f0 = c * chunk;
            const uint32_t nc = n - f0 < chunk ? n - f0 : chunk;
            DYG_TRY(insert_chunk_enqueue(G, H, c, chunk, nc, p, halt, status, cond, st));
        }
        DYG_TRY(read_scalars2(G, H, st));
        const unsigned long long h = wg.host_scalars[S_HALT];
        if (!h) return DYG_OK;
        const HaltInfo hi = decode_halt(h);
        if (hi.kind == kHaltInvalid) return rejected_inputs(G, st);
        dyg_graph *grow = hi.batch == 0 ? G : H;
        DYG_TRY(grow_arena(grow, grow->g.arena_cap * 2, st));
        DYG_TRY(clear_halt(G, st));
        start = hi.batch;
    }
    set_error("insert file: too many arena regrowths");
    return DYG_ENOMEM;
}

dyg_status delete_file_run(dyg_graph *G, dyg_graph *H, const uint32_t *src, const uint32_t *dst,
                           uint32_t n, uint64_t uid0, uint32_t chunk, const dyg_walk_params &p,
                           int32_t *status, float *cond, uint64_t *n_rec, cudaStream_t st,
                           bool check_inputs) {
    Workspace &ws = G->ws;
    unsigned long long *sc = ptr<unsigned long long>(ws.scalars);
    unsigned long long *halt = sc + S_HALT;
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
    if (check_inputs)
        DYG_TRY(validate_enqueue(halt, sc + S_ERR, src, dst, nullptr, n, G->g.n, st));
    DYG_TRY(decr_delete_enqueue(G, H, src, dst, n, uid0, nullptr, true, halt, status, cond, st));
    const uint32_t nchunks = (uint32_t)(((uint64_t)n + chunk - 1) / chunk);
    uint32_t c_start = 0, ph_start = 0;
    for (int round = 0; round < 64; ++round) {
        for (uint32_t c = c_start; c < nchunks; ++c) {
            const uint32_t f0 = c * chunk;
            const uint32_t nc = n - f0 < chunk ? n - f0 : chunk;
            DYG_TRY(decr_walk_enqueue(G, H, f0, nc, ptr<uint32_t>(ws.counts) + C_FILTERED, p, halt,
                                      c, c == c_start ? ph_start : 0, status, cond, st));
        }
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
        c_start = hi.batch;
        ph_start = hi.phase;
    }
    set_error("delete file: too many buffer regrowths");
    return DYG_ENOMEM;
}

}  // namespace

uint32_t stream_default_chunk(uint32_t n_vertices) {
    const uint32_t c = (uint32_t)((double)n_vertices * 0.05);
    return c < 10000u ? 10000u : c;
}

dyg_status stream_file_run(dyg_graph *G, dyg_graph *H, uint32_t op, const uint32_t *src,
                           const uint32_t *dst, const float *w, uint32_t n, uint64_t uid0,
                           uint32_t chunk, const dyg_walk_params &p, int32_t *status, float *cond,
                           uint64_t *n_rec, cudaStream_t st, bool check_inputs) {
    *n_rec = 0;
    if (chunk == 0) chunk = stream_default_chunk(G->g.n);
    if (op == DYG_STREAM_INSERT)
        return insert_file_run(G, H, src, dst, w, n, uid0, chunk, p, status, cond, st,
                               check_inputs);
    return delete_file_run(G, H, src, dst, n, uid0, chunk, p, status, cond, n_rec, st,
                           check_inputs);
}

}  // namespace dyg
