// rowops.cu -- device-driven row updates of the dynamic CSR.
//
// Both operations take a half-edge list (row hx[i], column hy[i], weight
// hw[i], i < m) whose length may live on the device, and apply it in list
// order per row without sorting the list:
//   append: each entry takes a rank in its row with an atomic counter; the
//           row's leader (rank 0) sizes the row, moves it when it overflows,
//           and after the entries have written themselves into the row's tail
//           restores list order in that tail (the list index rides in the
//           slot's second word until then).  Row order is therefore exactly
//           the order the reference's host loop produces
//           (random_walk_incremental/gpu_graph.cuh:297-329).
//   delete: entries of a row are gathered into a scratch run, sorted by list
//           index, and removed one by one with swap-with-last
//           (random_walk_decremental/gpu_graph.cuh:359-399).
// Arena space for the moves of one or two graphs is reserved by one thread,
// all or nothing.  When it does not fit, that thread writes a halt code; every
// kernel that changes a graph (and every kernel of the batch pipelines) then
// returns at once, and the host grows the arena and resumes the stream at the
// halted phase.  Nothing here needs a host-visible count, so a whole update
// stream is enqueued with a single synchronize at its end.
#include "dyg_internal.cuh"

namespace dyg {

namespace {

__device__ __forceinline__ uint32_t dcount(const uint32_t *dev, uint32_t host) {
    return dev ? min(*dev, host) : host;
}

__device__ __forceinline__ void dev_rank(DevGraph g, const uint32_t *hx, const uint32_t *m_dev,
                                         uint32_t m_host, uint32_t *rank, uint32_t *rowcnt,
                                         const unsigned long long *halt, unsigned long long *ran) {
    if (*halt) return;
    if (blockIdx.x == 0 && threadIdx.x == 0 && ran) *ran = 1ull;
    const uint32_t m = dcount(m_dev, m_host);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t x = hx[i];
        rank[i] = (x < g.n) ? atomicAdd(rowcnt + x, 1u) : 0xFFFFFFFFu;
    }
}

// ------------------------------------------------------------------ append

// Leaders size their rows; returns the arena slots this thread's moves need.
__device__ __forceinline__ unsigned long long dev_app_need(DevGraph g, const uint32_t *hx,
                                                           const uint32_t *m_dev, uint32_t m_host,
                                                           const uint32_t *rank,
                                                           const uint32_t *rowcnt, uint32_t slack,
                                                           uint32_t *lneed) {
    const uint32_t m = dcount(m_dev, m_host);
    unsigned long long total = 0ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (rank[i] != 0u) continue;
        const uint32_t x = hx[i];
        const uint2 d = g.desc[x];
        const uint32_t nd = d.y + rowcnt[x];
        uint32_t need = 0u;
        if (nd > g.cap[x]) {
            need = max(2u * nd, nd + slack);
            need = (need + 1u) & ~1u;
            total += need;
        }
        lneed[i] = need;
    }
    return total;
}

// Reserves the moves of one or both graphs, all or nothing, or halts.
__device__ __forceinline__ void reserve_moves(const DevGraph &g1, unsigned long long *sc1,
                                              const DevGraph *g2, unsigned long long *sc2,
                                              unsigned long long *halt, unsigned long long code) {
    const unsigned long long need1 = __ldcg(sc1 + S_NEED);
    const unsigned long long need2 = g2 ? __ldcg(sc2 + S_NEED) : 0ull;
    const bool ok1 = *g1.top + need1 <= g1.arena_cap;
    const bool ok2 = !g2 || *g2->top + need2 <= g2->arena_cap;
    if (!(ok1 && ok2)) {
        *halt = code;
        return;
    }
    sc1[S_CURSOR] = *g1.top;
    *g1.top += need1;
    if (g2) {
        sc2[S_CURSOR] = *g2->top;
        *g2->top += need2;
    }
}

// Leaders that must move their row take a new offset; a row of up to 32
// slots is copied by its leader's lane, a longer one by the whole warp (rows
// longer than kBigRow, with big_ok, by k_app_move_big instead).  Every lane of a warp runs the same
// iterations.
__device__ __forceinline__ void dev_app_move(DevGraph g, const uint32_t *hx, const uint32_t *m_dev,
                                             uint32_t m_host, const uint32_t *rank,
                                             const uint32_t *lneed, unsigned long long *cursor,
                                             uint4 *big, unsigned long long *nbig, bool big_ok,
                                             const unsigned long long *halt) {
    if (*halt) return;
    const uint32_t m = dcount(m_dev, m_host);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t wb = first - lane; wb < m; wb += gridDim.x * blockDim.x) {
        const uint32_t i = wb + lane;
        bool mv = i < m && rank[i] == 0u && lneed[i] != 0u;
        uint32_t x = 0, off = 0;
        uint2 d = make_uint2(0u, 0u);
        if (mv) {
            x = hx[i];
            d = g.desc[x];
            off = (uint32_t)atomicAdd(cursor, (unsigned long long)lneed[i]);
            if (big_ok && d.y > kBigRow) {
                big[atomicAdd(nbig, 1ull)] = make_uint4(i, off, d.x, d.y);
                mv = false;
            }
        }
        // rows of up to 32 slots are copied by their own lane, eight slots
        // loaded before they are stored (the new range is fresh arena space,
        // so it never overlaps a row being read)
        if (mv && d.y <= 32u) {
            for (uint32_t j0 = 0; j0 < d.y; j0 += 8u) {
                uint2 sv[8];
                float wv[8];
#pragma unroll
                for (uint32_t u = 0; u < 8u; ++u)
                    if (j0 + u < d.y) {
                        sv[u] = g.slots[d.x + j0 + u];
                        wv[u] = g.wts[d.x + j0 + u];
                    }
#pragma unroll
                for (uint32_t u = 0; u < 8u; ++u)
                    if (j0 + u < d.y) {
                        g.slots[off + j0 + u] = sv[u];
                        g.wts[off + j0 + u] = wv[u];
                    }
            }
        }
        unsigned todo = __ballot_sync(kFull, mv && d.y > 32u);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1u;
            const uint32_t so = __shfl_sync(kFull, off, src);
            const uint32_t sx = __shfl_sync(kFull, d.x, src);
            const uint32_t sy = __shfl_sync(kFull, d.y, src);
            for (uint32_t j0 = 0; j0 < sy; j0 += 256u) {
                uint2 sv[8];
                float wv[8];
#pragma unroll
                for (uint32_t u = 0; u < 8u; ++u) {
                    const uint32_t j = j0 + lane + 32u * u;
                    if (j < sy) {
                        sv[u] = g.slots[sx + j];
                        wv[u] = g.wts[sx + j];
                    }
                }
#pragma unroll
                for (uint32_t u = 0; u < 8u; ++u) {
                    const uint32_t j = j0 + lane + 32u * u;
                    if (j < sy) {
                        g.slots[so + j] = sv[u];
                        g.wts[so + j] = wv[u];
                    }
                }
            }
        }
        if (mv) {
            g.cap[x] = lneed[i];
            g.desc[x] = make_uint2(off, d.y);
        }
    }
}

// One block per long row to move: {leader, new offset, old offset, degree}.
__global__ void k_app_move_big(DevGraph g, const uint32_t *hx, const uint32_t *lneed,
                               const uint4 *big, const unsigned long long *nbig,
                               const unsigned long long *halt) {
    if (*halt) return;
    const uint32_t nb = (uint32_t)*nbig;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint4 e = big[b];
        // the old and new ranges never overlap (the row moves to fresh arena
        // space), so a tile's loads are all issued before its stores
        constexpr uint32_t U = 8;
        for (uint32_t base = 0; base < e.w; base += U * blockDim.x) {
            uint2 sv[U];
            float wv[U];
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) {
                const uint32_t j = base + u * blockDim.x + threadIdx.x;
                if (j < e.w) {
                    sv[u] = g.slots[e.z + j];
                    wv[u] = g.wts[e.z + j];
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) {
                const uint32_t j = base + u * blockDim.x + threadIdx.x;
                if (j < e.w) {
                    g.slots[e.y + j] = sv[u];
                    g.wts[e.y + j] = wv[u];
                }
            }
        }
        if (threadIdx.x == 0) {
            const uint32_t x = hx[e.x];
            g.cap[x] = lneed[e.x];
            g.desc[x] = make_uint2(e.y, e.w);
        }
    }
}

__device__ __forceinline__ void dev_app_write(DevGraph g, const uint32_t *hx, const uint32_t *hy,
                                              const float *hw, const uint32_t *m_dev,
                                              uint32_t m_host, const uint32_t *rank,
                                              const unsigned long long *halt) {
    if (*halt) return;
    const uint32_t m = dcount(m_dev, m_host);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t x = hx[i];
        if (x >= g.n) continue;
        const uint2 d = g.desc[x];
        const uint32_t pos = d.x + d.y + rank[i];
        g.slots[pos] = make_uint2(hy[i], i);   // list index until the tail is ordered
        g.wts[pos] = hw[i];
    }
}

constexpr uint32_t kTailWarp = 256;   // new tails up to this length are ordered by a warp
constexpr uint32_t kTailLane = 8;     // ... and from this length on (shorter: by the leader)

// Leaders order their row's new tail by list index, store 1/w in place of the
// index, publish the degree and clear the row counter (also after a halt, if
// this operation's ranks were taken).  A tail of kTailLane+1..kTailWarp
// entries is ordered by the whole warp (each entry placed at its rank among
// the tail's list indices, which are distinct); other tails by the leader.
__device__ __forceinline__ void dev_app_finish(DevGraph g, const uint32_t *hx, const uint32_t *m_dev,
                                               uint32_t m_host, const uint32_t *rank,
                                               uint32_t *rowcnt, const unsigned long long *halt,
                                               const unsigned long long *ran,
                                               unsigned long long *long_flag) {
    const bool halted = *halt != 0ull;
    if (halted && !*ran) return;
    const uint32_t m = dcount(m_dev, m_host);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t wb = first - lane; wb < m; wb += gridDim.x * blockDim.x) {
        const uint32_t i = wb + lane;
        const bool lead = i < m && rank[i] == 0u;
        uint32_t x = 0, cnt = 0;
        if (lead) {
            x = hx[i];
            cnt = rowcnt[x];
            rowcnt[x] = 0u;
        }
        if (halted) continue;
        const uint2 d = lead ? g.desc[x] : make_uint2(0u, 0u);
        const uint32_t base = d.x + d.y;
        const bool coop = lead && cnt > kTailLane && cnt <= kTailWarp;
        if (lead && !coop && cnt <= kTailLane) {
            // a short tail: loaded at once, each entry written at its rank
            // among the tail's (distinct) list indices, with 1/w in place of
            // the index
            uint2 sv[kTailLane];
            float wv[kTailLane];
#pragma unroll
            for (uint32_t u = 0; u < kTailLane; ++u)
                if (u < cnt) {
                    sv[u] = g.slots[base + u];
                    wv[u] = g.wts[base + u];
                }
#pragma unroll
            for (uint32_t u = 0; u < kTailLane; ++u)
                if (u < cnt) {
                    uint32_t r = 0;
#pragma unroll
                    for (uint32_t v = 0; v < kTailLane; ++v)
                        if (v < cnt) r += sv[v].y < sv[u].y ? 1u : 0u;
                    g.slots[base + r] = make_uint2(sv[u].x, __float_as_uint(__frcp_rn(wv[u])));
                    g.wts[base + r] = wv[u];
                }
        } else if (lead && !coop) {
            for (uint32_t a = 1; a < cnt; ++a) {   // insertion sort by list index
                const uint2 sl = g.slots[base + a];
                const float w = g.wts[base + a];
                uint32_t b = a;
                while (b > 0 && g.slots[base + b - 1].y > sl.y) {
                    g.slots[base + b] = g.slots[base + b - 1];
                    g.wts[base + b] = g.wts[base + b - 1];
                    --b;
                }
                g.slots[base + b] = sl;
                g.wts[base + b] = w;
            }
            for (uint32_t a = 0; a < cnt; ++a)
                g.slots[base + a].y = __float_as_uint(__frcp_rn(g.wts[base + a]));
        }
        unsigned todo = __ballot_sync(kFull, coop);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1u;
            const uint32_t tb = __shfl_sync(kFull, base, src);
            const uint32_t c = __shfl_sync(kFull, cnt, src);
            uint32_t col[kTailWarp / 32], key[kTailWarp / 32], r[kTailWarp / 32];
            float w[kTailWarp / 32];
#pragma unroll
            for (uint32_t u = 0; u < kTailWarp / 32; ++u) {
                const uint32_t a = lane + 32u * u;
                key[u] = 0xFFFFFFFFu;
                r[u] = 0u;
                if (a < c) {
                    const uint2 sl = g.slots[tb + a];
                    col[u] = sl.x;
                    key[u] = sl.y;
                    w[u] = g.wts[tb + a];
                }
            }
#pragma unroll
            for (uint32_t cu = 0; cu < kTailWarp / 32; ++cu) {
                if (32u * cu >= c) break;
                for (uint32_t j = 0; j < 32u; ++j) {
                    const uint32_t kj = __shfl_sync(kFull, key[cu], j);
#pragma unroll
                    for (uint32_t u = 0; u < kTailWarp / 32; ++u) r[u] += kj < key[u] ? 1u : 0u;
                }
            }
            __syncwarp();
#pragma unroll
            for (uint32_t u = 0; u < kTailWarp / 32; ++u) {
                if (lane + 32u * u < c) {
                    g.slots[tb + r[u]] = make_uint2(col[u], __float_as_uint(__frcp_rn(w[u])));
                    g.wts[tb + r[u]] = w[u];
                }
            }
            __syncwarp();
        }
        if (lead) {
            g.desc[x] = make_uint2(d.x, d.y + cnt);
            if (d.y + cnt > kBigRow && d.y <= kBigRow) *long_flag = 1ull;
        }
    }
}

// One append list and its graph.  The append kernels take two and pick one
// by blockIdx.y, so the appends to H and to G of one batch share each launch.
struct AppSide {
    DevGraph g;
    const uint32_t *hx, *hy;
    const float *hw;
    const uint32_t *m_dev;
    uint32_t m_host;
    uint32_t slack;
    uint32_t *rank, *rowcnt, *lneed;
    unsigned long long *sc;   // the graph's scalars
    uint4 *big;
    bool big_ok;
};
struct AppSides {
    AppSide s[2];
};

__global__ void k_app_rank(AppSides A, const unsigned long long *halt) {
    const AppSide &a = A.s[blockIdx.y];
    dev_rank(a.g, a.hx, a.m_dev, a.m_host, a.rank, a.rowcnt, halt, a.sc + S_OPRAN);
}

// Row sizes and the graphs' arena needs; the block that finishes last (a
// ticket taken after its needs were added, no waiting) reserves the moves of
// both graphs, so no one-thread launch follows.
__global__ void k_app_need(AppSides A, unsigned long long *halt, unsigned long long code) {
    __shared__ unsigned long long s_need;
    __shared__ bool s_last;
    if (*halt) return;
    const AppSide &a = A.s[blockIdx.y];
    if (threadIdx.x == 0) s_need = 0ull;
    __syncthreads();
    const unsigned long long mine =
        dev_app_need(a.g, a.hx, a.m_dev, a.m_host, a.rank, a.rowcnt, a.slack, a.lneed);
    if (mine) atomicAdd(&s_need, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_need) atomicAdd(a.sc + S_NEED, s_need);
        __threadfence();   // this block's need is counted before its ticket
        unsigned long long *done = A.s[0].sc + S_BLOCKS;
        s_last = atomicAdd(done, 1ull) + 1ull == (unsigned long long)gridDim.x * gridDim.y;
        if (s_last) {
            __threadfence();   // every block's need is visible
            *done = 0ull;
            reserve_moves(A.s[0].g, A.s[0].sc, gridDim.y > 1 ? &A.s[1].g : nullptr,
                          A.s[1].sc, halt, code);
        }
    }
}

__global__ void k_app_move(AppSides A, const unsigned long long *halt) {
    const AppSide &a = A.s[blockIdx.y];
    dev_app_move(a.g, a.hx, a.m_dev, a.m_host, a.rank, a.lneed, a.sc + S_CURSOR, a.big,
                 a.sc + S_NBIG, a.big_ok, halt);
}

__global__ void k_app_write(AppSides A, const unsigned long long *halt) {
    const AppSide &a = A.s[blockIdx.y];
    dev_app_write(a.g, a.hx, a.hy, a.hw, a.m_dev, a.m_host, a.rank, halt);
}

__global__ void k_app_finish(AppSides A, const unsigned long long *halt) {
    const AppSide &a = A.s[blockIdx.y];
    dev_app_finish(a.g, a.hx, a.m_dev, a.m_host, a.rank, a.rowcnt, halt, a.sc + S_OPRAN,
                   a.sc + S_LONG);
}

// ------------------------------------------------------------------ delete

// Leaders take a run of `rowcnt[x]` scratch entries.  One atomic per warp:
// the warp's requests are prefix-summed with shuffles, lane 31 takes the sum.
__device__ __forceinline__ void dev_del_base(const uint32_t *hx, uint32_t m, const uint32_t *rank,
                                             const uint32_t *rowcnt, uint32_t *rowtmp,
                                             unsigned long long *cursor,
                                             const unsigned long long *halt) {
    if (*halt) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t warp0 = first - lane;
    for (uint32_t base = warp0; base < m; base += stride) {
        const uint32_t i = base + lane;
        const bool lead = i < m && rank[i] == 0u;
        const uint32_t x = lead ? hx[i] : 0u;
        const uint32_t want = lead ? rowcnt[x] : 0u;
        uint32_t incl = want;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, d);
            if (lane >= (uint32_t)d) incl += v;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        unsigned long long start = 0ull;
        if (lane == 31u && total) start = atomicAdd(cursor, (unsigned long long)total);
        start = __shfl_sync(kFull, start, 31);
        if (lead) rowtmp[x] = (uint32_t)start + incl - want;
    }
}

__device__ __forceinline__ void dev_del_scatter(DevGraph g, const uint32_t *hx, uint32_t m,
                                                const uint32_t *rank, const uint32_t *rowtmp,
                                                uint32_t *tmp, const unsigned long long *halt) {
    if (*halt) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t x = hx[i];
        if (x < g.n) tmp[rowtmp[x] + rank[i]] = i;
    }
}

// The deletion list's graphs (G, then H): their ranks, scratch runs and
// scatters do not depend on each other, so both share each launch
// (blockIdx.y picks the graph); only H's removal waits for G's found flags.
struct DelSide {
    DevGraph g;
    uint32_t *rank, *rowcnt, *rowtmp, *dtmp;
    unsigned long long *cursor;
};
struct DelSides {
    DelSide s[2];
};

__global__ void k_del_rank(DelSides D, const uint32_t *hx, uint32_t m,
                           const unsigned long long *halt) {
    const DelSide &d = D.s[blockIdx.y];
    dev_rank(d.g, hx, nullptr, m, d.rank, d.rowcnt, halt, nullptr);
}

__global__ void k_del_base(DelSides D, const uint32_t *hx, uint32_t m,
                           const unsigned long long *halt) {
    const DelSide &d = D.s[blockIdx.y];
    dev_del_base(hx, m, d.rank, d.rowcnt, d.rowtmp, d.cursor, halt);
}

__global__ void k_del_scatter(DelSides D, const uint32_t *hx, uint32_t m,
                              const unsigned long long *halt) {
    const DelSide &d = D.s[blockIdx.y];
    dev_del_scatter(d.g, hx, m, d.rank, d.rowtmp, d.dtmp, halt);
}

// One warp removes row x's cnt entries (its run in tmp at rowtmp[x]) in list
// order: the run is ordered by list index (each entry placed at its rank,
// into the second half of the scratch), then each deletion searches the row
// 32 slots at a time and moves the row's last slot into the hit.  With
// `mask`, entry i = 2e + side is applied only if edge e was found on both
// sides of `mask`.  Every lane calls it with the same arguments.
__device__ __forceinline__ void warp_del_row(const DevGraph &g, const uint32_t *hy, uint32_t m,
                                             uint32_t x, uint32_t cnt, uint2 d,
                                             const uint32_t *rowtmp, uint32_t *tmp,
                                             const uint8_t *mask, uint8_t *found, uint32_t lane) {
    const uint32_t off = d.x;
    uint32_t deg = d.y;
    const uint32_t *run = tmp + rowtmp[x];
    uint32_t *sorted = tmp + m + rowtmp[x];
    for (uint32_t a = lane; a < cnt; a += 32u) {   // each entry to its rank
        const uint32_t v = run[a];
        uint32_t r = 0;
        for (uint32_t c = 0; c < cnt; ++c) r += run[c] < v;
        sorted[r] = v;
    }
    __syncwarp();
    for (uint32_t a = 0; a < cnt; ++a) {
        const uint32_t k = sorted[a];
        if (mask && !(mask[k & ~1u] && mask[k | 1u])) continue;
        const uint32_t y = hy[k];
        uint32_t pos = ~0u;
        for (uint32_t j0 = 0; j0 < deg; j0 += 32u) {
            const uint32_t j = j0 + lane;
            const unsigned hit = __ballot_sync(kFull, j < deg && g.slots[off + j].x == y);
            if (hit) {
                pos = j0 + (uint32_t)(__ffs(hit) - 1);
                break;
            }
        }
        if (pos != ~0u) {
            if (lane == 0u) {
                g.slots[off + pos] = g.slots[off + deg - 1u];
                g.wts[off + pos] = g.wts[off + deg - 1u];
                found[k] = 1;
            }
            --deg;
            __syncwarp();   // the moved slot is visible to the next search
        }
    }
    if (lane == 0u) g.desc[x] = make_uint2(off, deg);
    __syncwarp();
}

// Leaders remove their row's entries in list order (mask as in
// warp_del_row).  A row of up to 32 slots is edited by its leader's lane.
// Without big_ok a longer one is edited by the whole warp; with big_ok (the
// graph has rows longer than kBigRow) rows longer than kBigRow go to the
// front of the big list and rows of 33..kBigRow slots to its back (counted in
// the high half of *nbig), both for k_del_apply_big, so that no warp edits
// several such rows one after another.  Every lane of a warp runs the same
// iterations.
__global__ void k_del_apply(DevGraph g, const uint32_t *hx, const uint32_t *hy, uint32_t m,
                            const uint32_t *rank, uint32_t *rowcnt, const uint32_t *rowtmp,
                            uint32_t *tmp, const uint8_t *mask, uint8_t *found, uint4 *big,
                            unsigned long long *nbig, bool big_ok,
                            const unsigned long long *halt) {
    if (*halt) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t wb = first - lane; wb < m; wb += gridDim.x * blockDim.x) {
        const uint32_t i = wb + lane;
        bool lead = i < m && rank[i] == 0u;
        uint32_t x = 0u, cnt = 0u;
        uint2 d = make_uint2(0u, 0u);
        if (lead) {
            x = hx[i];
            d = g.desc[x];
            if (big_ok && d.y > 32u) {
                if (d.y > kBigRow)   // the count of long rows is the low half
                    big[(uint32_t)atomicAdd(nbig, 1ull)] = make_uint4(i, 0u, 0u, 0u);
                else
                    big[m - 1u - (uint32_t)(atomicAdd(nbig, 1ull << 32) >> 32)] =
                        make_uint4(i, 0u, 0u, 0u);
                lead = false;
            } else {
                cnt = rowcnt[x];
                rowcnt[x] = 0u;
            }
        }
        const bool coop = lead && d.y > 32u;
        if (lead && !coop) {
            uint32_t *run = tmp + rowtmp[x];
            for (uint32_t a = 1; a < cnt; ++a) {
                const uint32_t v = run[a];
                uint32_t b = a;
                while (b > 0 && run[b - 1] > v) {
                    run[b] = run[b - 1];
                    --b;
                }
                run[b] = v;
            }
            uint32_t deg = d.y;
            for (uint32_t a = 0; a < cnt; ++a) {
                const uint32_t k = run[a];
                if (mask && !(mask[k & ~1u] && mask[k | 1u])) continue;
                const uint32_t y = hy[k];
                // first slot holding y, eight columns loaded before they are
                // compared (vertex ids are never ~0u)
                uint32_t pos = ~0u;
                for (uint32_t j0 = 0; j0 < deg && pos == ~0u; j0 += 8u) {
                    uint32_t cv[8];
#pragma unroll
                    for (uint32_t u = 0; u < 8u; ++u)
                        cv[u] = j0 + u < deg ? g.slots[d.x + j0 + u].x : ~0u;
#pragma unroll
                    for (uint32_t u = 0; u < 8u; ++u)
                        if (pos == ~0u && cv[u] == y) pos = j0 + u;
                }
                if (pos != ~0u) {
                    g.slots[d.x + pos] = g.slots[d.x + deg - 1u];
                    g.wts[d.x + pos] = g.wts[d.x + deg - 1u];
                    --deg;
                    found[k] = 1;
                }
            }
            g.desc[x] = make_uint2(d.x, deg);
        }
        unsigned todo = __ballot_sync(kFull, coop);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1u;
            const uint32_t sx = __shfl_sync(kFull, x, src);
            const uint32_t sc = __shfl_sync(kFull, cnt, src);
            const uint2 sd = make_uint2(__shfl_sync(kFull, d.x, src), __shfl_sync(kFull, d.y, src));
            warp_del_row(g, hy, m, sx, sc, sd, rowtmp, tmp, mask, found, lane);
        }
    }
}

constexpr uint32_t kTrackMax = 128;   // deletions per long row tracked in shared memory

// One block per long row.  The row's run is ordered by list index (each
// entry placed at its rank, into the second half of the scratch).  Then, if
// the row has at most kTrackMax deletions whose columns are distinct and each
// occur once in the row, one pass over the row finds every target's slot and
// one thread applies the swaps in order, following the single slot each swap
// moves (the row's last); otherwise every deletion is a block-wide search.
// Both give the one-thread path's result.  Then the rows of 33..kBigRow
// slots that k_del_apply left at the back of the list, one warp each.
__global__ void k_del_apply_big(DevGraph g, const uint32_t *hx, const uint32_t *hy, uint32_t m,
                                uint32_t *rowcnt, const uint32_t *rowtmp, uint32_t *tmp,
                                const uint8_t *mask, uint8_t *found, const uint4 *big,
                                const unsigned long long *nbig, const unsigned long long *halt) {
    __shared__ uint32_t s_best, s_ok, s_n;
    __shared__ uint32_t s_y[kTrackMax], s_pos[kTrackMax], s_occ[kTrackMax];
    __shared__ unsigned long long s_key[kTrackMax];   // (column << 8 | a), ascending
    if (*halt) return;
    const unsigned long long nboth = *nbig;
    const uint32_t nb = (uint32_t)nboth, nmid = (uint32_t)(nboth >> 32);
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t x = hx[big[b].x];
        const uint32_t cnt = rowcnt[x];
        const uint32_t *run = tmp + rowtmp[x];
        uint32_t *sorted = tmp + m + rowtmp[x];
        for (uint32_t a = threadIdx.x; a < cnt; a += blockDim.x) {
            const uint32_t v = run[a];
            uint32_t r = 0;
            for (uint32_t c = 0; c < cnt; ++c) r += run[c] < v;
            sorted[r] = v;
        }
        if (threadIdx.x == 0) s_ok = cnt <= kTrackMax ? 1u : 0u;
        __syncthreads();
        const uint2 d = g.desc[x];
        uint32_t deg = d.y;
        if (s_ok) {
            for (uint32_t a = threadIdx.x; a < cnt; a += blockDim.x) {
                const uint32_t k = sorted[a];
                const bool on = !mask || (mask[k & ~1u] && mask[k | 1u]);
                s_y[a] = on ? hy[k] : ~0u;
                s_pos[a] = ~0u;
                s_occ[a] = 0u;
            }
            __syncthreads();
            // the tracked columns sorted (rank by count, ties by index), so
            // each slot of the row finds its deletion by binary search instead
            // of comparing against all of them
            for (uint32_t a = threadIdx.x; a < cnt; a += blockDim.x) {
                const unsigned long long ka = ((unsigned long long)s_y[a] << 8) | a;
                uint32_t r = 0;
                for (uint32_t c = 0; c < cnt; ++c) {
                    const unsigned long long kc = ((unsigned long long)s_y[c] << 8) | c;
                    r += kc < ka;
                    if (c < a && s_y[a] != ~0u && s_y[c] == s_y[a]) s_ok = 0u;
                }
                s_key[r] = ka;
            }
            if (threadIdx.x == 0) {
                uint32_t live = 0;
                for (uint32_t a = 0; a < cnt; ++a) live += s_y[a] != ~0u;
                s_n = live;   // masked-off entries (column ~0u) sort last
            }
            __syncthreads();
            const uint32_t nlive = s_n;
            const uint32_t *cols = reinterpret_cast<const uint32_t *>(g.slots + d.x);
            for (uint32_t base = 0; base < deg; base += kFindUnroll * blockDim.x) {
                uint32_t v[kFindUnroll];   // a tile's loads are issued before any search
#pragma unroll
                for (uint32_t u = 0; u < kFindUnroll; ++u) {
                    const uint32_t j = base + u * blockDim.x + threadIdx.x;
                    v[u] = j < deg ? cols[2u * j] : ~0u;
                }
#pragma unroll
                for (uint32_t u = 0; u < kFindUnroll; ++u) {
                    const uint32_t col = v[u];
                    if (col == ~0u) continue;
                    uint32_t lo = 0, hi = nlive;
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if ((uint32_t)(s_key[mid] >> 8) < col) lo = mid + 1u;
                        else hi = mid;
                    }
                    if (lo < nlive && (uint32_t)(s_key[lo] >> 8) == col) {
                        const uint32_t a = (uint32_t)(s_key[lo] & 0xFFu);
                        atomicMin(&s_pos[a], base + u * blockDim.x + threadIdx.x);
                        atomicAdd(&s_occ[a], 1u);
                    }
                }
            }
            __syncthreads();
            for (uint32_t a = threadIdx.x; a < cnt; a += blockDim.x)
                if (s_occ[a] > 1u) s_ok = 0u;
            __syncthreads();
        }
        if (s_ok) {
            if (threadIdx.x == 0) {
                for (uint32_t a = 0; a < cnt; ++a) {
                    const uint32_t p = s_pos[a];
                    if (s_y[a] == ~0u || p == ~0u) continue;
                    const uint32_t last = deg - 1u;
                    g.slots[d.x + p] = g.slots[d.x + last];
                    g.wts[d.x + p] = g.wts[d.x + last];
                    --deg;
                    found[sorted[a]] = 1;
                    if (p != last)   // the slot from `last` now sits at p
                        for (uint32_t c = a + 1; c < cnt; ++c)
                            if (s_pos[c] == last) s_pos[c] = p;
                }
                g.desc[x] = make_uint2(d.x, deg);
            }
        } else {
            for (uint32_t a = 0; a < cnt; ++a) {
                const uint32_t k = sorted[a];
                if (mask && !(mask[k & ~1u] && mask[k | 1u])) continue;
                const uint32_t j = block_find(g.slots, d.x, deg, hy[k], &s_best);
                if (j != ~0u) {
                    if (threadIdx.x == 0) {
                        g.slots[d.x + j] = g.slots[d.x + deg - 1u];
                        g.wts[d.x + j] = g.wts[d.x + deg - 1u];
                        found[k] = 1;
                    }
                    --deg;
                    __syncthreads();   // the moved slot is visible to the next search
                }
            }
        }
        if (threadIdx.x == 0) {
            rowcnt[x] = 0u;
            if (!s_ok) g.desc[x] = make_uint2(d.x, deg);
        }
        __syncthreads();   // s_ok and the shared arrays are reused by the next row
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nmid; j += nw) {
        const uint32_t x = hx[big[m - 1u - j].x];
        const uint32_t cnt = rowcnt[x];
        warp_del_row(g, hy, m, x, cnt, g.desc[x], rowtmp, tmp, mask, found, lane);
        if (lane == 0u) rowcnt[x] = 0u;
    }
}

int grid_for(uint64_t m) {
    const uint64_t b = (m + 255) / 256;
    const uint64_t cap = (uint64_t)num_sms() * 8;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

dyg_status rowops_ensure(dyg_graph *G, uint32_t m_host) {
    Workspace &ws = G->ws;
    DYG_TRY(ensure(ws.rank, sizeof(uint32_t) * (size_t)(m_host ? m_host : 1)));
    DYG_TRY(ensure(ws.lneed, sizeof(uint32_t) * (size_t)(m_host ? m_host : 1)));
    DYG_TRY(ensure(ws.dtmp, sizeof(uint32_t) * (size_t)(m_host ? m_host : 1) * 2));
    DYG_TRY(ensure(ws.big, sizeof(uint4) * (size_t)(m_host ? m_host : 1)));
    if (!ws.rowcnt.p) {
        DYG_TRY(ensure(ws.rowcnt, sizeof(uint32_t) * (size_t)(G->g.n ? G->g.n : 1)));
        DYG_TRY(ensure(ws.rowtmp, sizeof(uint32_t) * (size_t)(G->g.n ? G->g.n : 1)));
        DYG_CUDA(cudaMemset(ws.rowcnt.p, 0, ws.rowcnt.bytes));
    }
    return DYG_OK;
}

// Appends list A to graph GA and (optionally) list B to GB; the arena space
// of both is reserved together, so either both appends happen or neither
// (halt = code).
dyg_status append_enqueue(dyg_graph *GA, const AppendList &A, dyg_graph *GB, const AppendList *B,
                          unsigned long long *halt, unsigned long long code, cudaStream_t st) {
    dyg_graph *gs[2] = {GA, B ? GB : nullptr};
    const AppendList *ls[2] = {&A, B};
    const int ns = gs[1] ? 2 : 1;
    AppSides S{};
    uint32_t m_max = 0;
    for (int k = 0; k < ns; ++k) {
        dyg_graph *G = gs[k];
        DYG_TRY(rowops_ensure(G, ls[k]->m_host));
        unsigned long long *sc = ptr<unsigned long long>(G->ws.scalars);
        // need, cursor, ran [, long-row count]
        DYG_CUDA(cudaMemsetAsync(sc + S_NEED, 0, sizeof(unsigned long long) * (G->long_rows ? 4 : 3),
                                 st));
        S.s[k] = AppSide{G->g, ls[k]->hx, ls[k]->hy, ls[k]->hw, ls[k]->m_dev, ls[k]->m_host,
                         G->slack, ptr<uint32_t>(G->ws.rank), ptr<uint32_t>(G->ws.rowcnt),
                         ptr<uint32_t>(G->ws.lneed), sc, ptr<uint4>(G->ws.big), G->long_rows};
        if (ls[k]->m_host > m_max) m_max = ls[k]->m_host;
    }
    if (m_max == 0) return DYG_OK;
    const dim3 grid(grid_for(m_max), ns);
    k_app_rank<<<grid, 256, 0, st>>>(S, halt);
    count_launch();
    k_app_need<<<grid, 256, 0, st>>>(S, halt, code);
    count_launch();
    k_app_move<<<grid, 256, 0, st>>>(S, halt);
    count_launch();
    for (int k = 0; k < ns; ++k) {
        dyg_graph *G = gs[k];
        if (!G->long_rows || ls[k]->m_host == 0) continue;
        unsigned long long *sc = ptr<unsigned long long>(G->ws.scalars);
        k_app_move_big<<<num_sms() * 2, kBigThreads, 0, st>>>(
            G->g, ls[k]->hx, ptr<uint32_t>(G->ws.lneed), ptr<uint4>(G->ws.big), sc + S_NBIG, halt);
        count_launch();
    }
    k_app_write<<<grid, 256, 0, st>>>(S, halt);
    count_launch();
    k_app_finish<<<grid, 256, 0, st>>>(S, halt);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// Deletes the half-edges of a list whose length m is known on the host.
dyg_status delete_pair_enqueue(dyg_graph *G, dyg_graph *H, const uint32_t *hx, const uint32_t *hy,
                               uint32_t m, uint8_t *fG, uint8_t *fH, unsigned long long *halt,
                               cudaStream_t st) {
    if (m == 0) return DYG_OK;
    dyg_graph *gs[2] = {G, H};
    DelSides D{};
    for (int k = 0; k < 2; ++k) {
        dyg_graph *X = gs[k];
        DYG_TRY(rowops_ensure(X, m));
        unsigned long long *sc = ptr<unsigned long long>(X->ws.scalars);
        // [long-row count,] scratch cursor
        if (X->long_rows)
            DYG_CUDA(cudaMemsetAsync(sc + S_NBIG, 0, sizeof(unsigned long long) * 2, st));
        else
            DYG_CUDA(cudaMemsetAsync(sc + S_TMPCUR, 0, sizeof(unsigned long long), st));
        D.s[k] = DelSide{X->g, ptr<uint32_t>(X->ws.rank), ptr<uint32_t>(X->ws.rowcnt),
                         ptr<uint32_t>(X->ws.rowtmp), ptr<uint32_t>(X->ws.dtmp), sc + S_TMPCUR};
    }
    DYG_CUDA(cudaMemsetAsync(fG, 0, m, st));
    DYG_CUDA(cudaMemsetAsync(fH, 0, m, st));
    const int gr = grid_for(m);
    const dim3 grid2(gr, 2);
    k_del_rank<<<grid2, 256, 0, st>>>(D, hx, m, halt);
    count_launch();
    k_del_base<<<grid2, 256, 0, st>>>(D, hx, m, halt);
    count_launch();
    k_del_scatter<<<grid2, 256, 0, st>>>(D, hx, m, halt);
    count_launch();
    for (int k = 0; k < 2; ++k) {
        // H's entries only where G found the edge on both sides
        dyg_graph *X = gs[k];
        const uint8_t *mask = k ? fG : nullptr;
        uint8_t *found = k ? fH : fG;
        unsigned long long *sc = ptr<unsigned long long>(X->ws.scalars);
        k_del_apply<<<gr, 256, 0, st>>>(X->g, hx, hy, m, ptr<uint32_t>(X->ws.rank),
                                        ptr<uint32_t>(X->ws.rowcnt), ptr<uint32_t>(X->ws.rowtmp),
                                        ptr<uint32_t>(X->ws.dtmp), mask, found,
                                        ptr<uint4>(X->ws.big), sc + S_NBIG, X->long_rows, halt);
        count_launch();
        if (X->long_rows) {
            k_del_apply_big<<<num_sms() * 4, kBigThreads, 0, st>>>(
                X->g, hx, hy, m, ptr<uint32_t>(X->ws.rowcnt), ptr<uint32_t>(X->ws.rowtmp),
                ptr<uint32_t>(X->ws.dtmp), mask, found, ptr<uint4>(X->ws.big), sc + S_NBIG, halt);
            count_launch();
        }
    }
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

}  // namespace dyg
