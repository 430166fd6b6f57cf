// walk.cu -- sm_100a random-walk kernels of the dyGRASS update path.
//
// One walker = one non-backtracking random walk from an edge's source towards
// its target (random_walk_incremental/main.cu:70-211 and
// random_walk_decremental/main.cu:77-220 restated).  Walk lengths differ by
// two orders of magnitude between walkers (dead ends after one step, full
// max_steps walks), so instead of the reference's one-block-per-edge with a
// 512-thread barrier tree, each warp of a persistent grid keeps its 32 lanes
// busy: a lane whose walker ends takes the next walker of the warp's current
// edge, and the warp pulls a new edge from a global counter when the current
// one is handed out.  The per-edge winner (max 1/R, lowest walker id) is a
// 64-bit key reduced with atomicMax, so no barrier and no global scratch
// arrays are needed.  Lanes refill in step with one another (every fourth
// warp iteration), so the random-number blocks are drawn by whole warps.
//
// Draw d of walker k of update u is word d&3 of
// Philox4x32-10({d>>2, k, u_lo, u_hi | domain<<24}, seed): any walker can be
// replayed, which is how the decremental winner's path is recovered without
// the reference's per-thread path[100] arrays.
#include <stdlib.h>

#include <mutex>
#include <vector>

#include <atomic>

#include "dyg_internal.cuh"

namespace dyg {

// ------------------------------------------------------------- profiling
namespace {
struct ProfEvent {
    cudaEvent_t a, b;
    int kind;  // 0 incremental walk, 1 decremental walk, 2 replay/fallback
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfEvent> g_prof_events;
dyg_profile g_prof_acc{};

void prof_flush_locked() {
    for (ProfEvent &e : g_prof_events) {
        float ms = 0.f;
        if (cudaEventSynchronize(e.b) == cudaSuccess && cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
            if (e.kind == 0) { g_prof_acc.incr_walk_ms += ms; g_prof_acc.incr_walk_launches++; }
            else if (e.kind == 1) { g_prof_acc.decr_walk_ms += ms; g_prof_acc.decr_walk_launches++; }
            else { g_prof_acc.other_walk_ms += ms; g_prof_acc.other_walk_launches++; }
        }
        cudaGetLastError();
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    g_prof_events.clear();
}

struct ProfScope {
    bool on = false;
    ProfEvent ev{};
    cudaStream_t st;
    ProfScope(int kind, cudaStream_t s) : st(s) {
        std::lock_guard<std::mutex> lk(g_prof_mu);
        if (!g_prof_on) return;
        ev.kind = kind;
        if (cudaEventCreate(&ev.a) != cudaSuccess || cudaEventCreate(&ev.b) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaEventRecord(ev.a, st);
        on = true;
    }
    ~ProfScope() {
        if (!on) return;
        cudaEventRecord(ev.b, st);
        std::lock_guard<std::mutex> lk(g_prof_mu);
        g_prof_events.push_back(ev);
        if (g_prof_events.size() > 4096) prof_flush_locked();
    }
};
}  // namespace

constexpr int kWalkThreads = 256;

struct WalkArgs {
    DevGraph g;
    WalkJob job;
    uint32_t walkers, max_steps;
    uint32_t prune;
    uint32_t prune_every;   // iterations between reads of the edge's best (a power of two)
    uint32_t chunk;   // walkers handed to a warp at a time
    float threshold;
    uint2 key;
    unsigned long long *keys;
    unsigned long long *scalars;
};

struct Walker {
    uint32_t cur, prev, step, tgt, walker, c2, c3, rblk;
    uint4 rbuf;
    float R, we;
};

enum : int { kContinue = 0, kFail = 1, kFound = 2 };

// Draw for the walker's current step: word (step-1)&3 of the Philox block
// (step-1)>>2, computed once per block of four draws.
__device__ __forceinline__ uint32_t draw_next(Walker &s, uint2 key) {
    const uint32_t di = s.step - 1u, b = di >> 2;
    if (b != s.rblk) {
        s.rbuf = philox4x32_10(make_uint4(b, s.walker, s.c2, s.c3), key);
        s.rblk = b;
    }
    return pick4(s.rbuf, di & 3u);
}

// The move's common end: R += 1/w; distortion test (incremental only, from
// step 2 on), then the target test; the walk ends when the step counter
// reaches max_steps (main.cu:116, 139-157).
template <bool INCR>
__device__ __forceinline__ int finish_move(Walker &s, uint2 sl, uint32_t at, bool first,
                                           uint32_t max_steps, float thr, bool *moved,
                                           uint2 *taken, uint32_t *taken_at) {
    *moved = true;
    *taken = sl;
    *taken_at = at;
    // the slot holds the correctly rounded 1/w: one add per move, as R += 1/w
    s.R = __fadd_rn(s.R, __uint_as_float(sl.y));
    if (INCR && !first && __fmul_rn(s.R, s.we) >= thr) return kFail;
    if (sl.x == s.tgt) return kFound;
    s.prev = s.cur;
    s.cur = sl.x;
    s.step += 1u;
    if (s.step >= max_steps) return kFail;
    return kContinue;
}

// Weight-proportional choice in row [lo, lo + deg) by one thread: the first
// slot, in row order, among those whose column is not `ex` (when has_ex),
// whose inclusive prefix of fixed-point weights wq(w) exceeds
// floor(r * total / 2^32).  ~0u when total is 0; *picked receives the chosen
// slot.  The row is read kPickGroup slots at a time with the group's loads
// issued together (the second pass reads the groups again, from L1 mostly),
// so a row of up to kPickGroup slots costs two rounds of loads, not 2 deg.
constexpr uint32_t kPickGroup = 4;
__device__ __forceinline__ uint32_t lane_pick_weighted(const uint2 *__restrict__ slots,
                                                       const float *__restrict__ wts, uint32_t lo,
                                                       uint32_t deg, uint32_t ex, bool has_ex,
                                                       uint32_t r, uint2 *picked) {
    unsigned long long total = 0ull;
    for (uint32_t j0 = 0; j0 < deg; j0 += kPickGroup) {
        uint2 c[kPickGroup];
        float w[kPickGroup];
#pragma unroll
        for (uint32_t u = 0; u < kPickGroup; ++u) {
            const bool in = j0 + u < deg;
            c[u] = in ? __ldg(slots + lo + j0 + u) : make_uint2(0u, 0u);
            w[u] = in ? __ldg(wts + lo + j0 + u) : 0.f;
        }
#pragma unroll
        for (uint32_t u = 0; u < kPickGroup; ++u)
            if (j0 + u < deg && !(has_ex && c[u].x == ex)) total += wq(w[u]);
    }
    if (total == 0ull) return ~0u;
    const unsigned long long target = mul_hi32(r, total);
    unsigned long long acc = 0ull;
    uint32_t last = deg;
    uint2 last_sl = make_uint2(0u, 0u);
    for (uint32_t j0 = 0; j0 < deg; j0 += kPickGroup) {
        uint2 c[kPickGroup];
        float w[kPickGroup];
#pragma unroll
        for (uint32_t u = 0; u < kPickGroup; ++u) {
            const bool in = j0 + u < deg;
            c[u] = in ? __ldg(slots + lo + j0 + u) : make_uint2(0u, 0u);
            w[u] = in ? __ldg(wts + lo + j0 + u) : 0.f;
        }
#pragma unroll
        for (uint32_t u = 0; u < kPickGroup; ++u) {
            if (j0 + u >= deg || (has_ex && c[u].x == ex)) continue;
            acc += wq(w[u]);
            last = j0 + u;
            last_sl = c[u];
            if (acc > target) {
                *picked = last_sl;
                return lo + last;
            }
        }
    }
    *picked = last_sl;
    return lo + last;
}

// The uniform move from row d (deg = d.y, past the dead-end test) with draw r.
template <bool INCR>
__device__ __forceinline__ int move_uniform(Walker &s, uint2 d, uint32_t r,
                                            const uint2 *__restrict__ slots, uint32_t max_steps,
                                            float thr, bool *moved, uint2 *taken,
                                            uint32_t *taken_at) {
    const bool first = (s.step == 1u);
    const uint32_t deg = d.y;
    uint32_t at = d.x + (first ? r % deg : r % (deg - 1u));
    uint2 sl = __ldg(slots + at);
    if (!first) {
        // the row's last slot is loaded beside the drawn one, not after it:
        // some lane of a warp lands on its previous vertex in almost every
        // step, and a dependent reload would hold the whole warp
        const uint32_t at_last = d.x + deg - 1u;
        const uint2 sl_last = __ldg(slots + at_last);
        if (sl.x == s.prev) {
            at = at_last;
            sl = sl_last;
        }
    }
    return finish_move<INCR>(s, sl, at, first, max_steps, thr, moved, taken, taken_at);
}

// One move of one walker, mirroring the reference loop body:
//   step 1:  any neighbour, r % deg                    (main.cu:99-106)
//   step >1: dead end if deg == 1; r % (deg - 1) and the last slot when the
//            draw lands on the previous vertex          (main.cu:118-137)
// then finish_move.  *moved is set when a neighbour was drawn; *taken
// receives its slot.  WEIGHTED rows are scanned by this thread alone (the
// walk kernel searches long rows with the whole warp instead).
template <bool INCR, bool WEIGHTED>
__device__ __forceinline__ int step_once(Walker &s, const uint2 *__restrict__ desc,
                                         const uint2 *__restrict__ slots,
                                         const float *__restrict__ wts, uint32_t max_steps,
                                         float thr, uint2 key, bool *moved, uint2 *taken,
                                         uint32_t *taken_at) {
    *moved = false;
    const uint2 d = __ldg(desc + s.cur);
    const uint32_t deg = d.y;
    const bool first = (s.step == 1u);
    if (first ? (deg == 0u) : (deg <= 1u)) return kFail;
    const uint32_t r = draw_next(s, key);
    if (!WEIGHTED) return move_uniform<INCR>(s, d, r, slots, max_steps, thr, moved, taken, taken_at);
    uint2 sl;
    const uint32_t at = lane_pick_weighted(slots, wts, d.x, deg, s.prev, !first, r, &sl);
    if (at == ~0u) return kFail;
    return finish_move<INCR>(s, sl, at, first, max_steps, thr, moved, taken, taken_at);
}

// ------------------------------------------------ weighted, warp-cooperative
// Rows longer than kCoopRow slots are searched by the whole warp, one lane's
// row at a time: each lane takes four consecutive slots per pass over 128
// slots (two 128-bit slot loads and one 128-bit weight load for a quad inside
// the row; the quad grid starts at the row start rounded down to four slots,
// so every vector load is 16-byte aligned), a warp reduction gives the sum of
// each 128-slot tile, and the sums of up to kSegs segments of tiles are kept
// in shared memory.  The second pass finds the segment holding the target
// from those sums and scans only its tiles with a warp prefix scan.  The
// choice is the per-thread scan's: prefix sums of the fixed-point weights are
// exact integers, so the order of additions does not matter; only when a sum
// wraps past 2^64 (weights near 2^32) are prefixes not monotone, and then the
// second pass scans the whole row from its start, as the per-thread scan does.
constexpr uint32_t kCoopRow = 32;
constexpr uint32_t kSegs = 64;

__device__ __forceinline__ unsigned long long wq_ex(uint32_t col, float w, uint32_t ex,
                                                    bool has_ex) {
    return (has_ex && col == ex) ? 0ull : wq(w);
}

// Fixed-point weights of slots [j, j + 4) inside row [lo, hi) (0 outside it
// or for the excluded column).
__device__ __forceinline__ void quad_weights(const uint2 *__restrict__ slots,
                                             const float *__restrict__ wts, uint32_t j,
                                             uint32_t lo, uint32_t hi, uint32_t ex, bool has_ex,
                                             unsigned long long q[4]) {
    if (j >= lo && j + 4u <= hi) {
        const uint4 s01 = __ldg(reinterpret_cast<const uint4 *>(slots + j));
        const uint4 s23 = __ldg(reinterpret_cast<const uint4 *>(slots + j + 2u));
        const float4 w4 = __ldg(reinterpret_cast<const float4 *>(wts + j));
        q[0] = wq_ex(s01.x, w4.x, ex, has_ex);
        q[1] = wq_ex(s01.z, w4.y, ex, has_ex);
        q[2] = wq_ex(s23.x, w4.z, ex, has_ex);
        q[3] = wq_ex(s23.z, w4.w, ex, has_ex);
    } else {
#pragma unroll
        for (uint32_t u = 0; u < 4u; ++u) {
            const uint32_t k = j + u;
            q[u] = (k >= lo && k < hi) ? wq_ex(__ldg(&slots[k].x), __ldg(wts + k), ex, has_ex) : 0ull;
        }
    }
}

// Sum over the warp with a wrap flag (any addition past 2^64).
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v, bool *wrap) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(kFull, v, o);
        const unsigned long long x = v + t;
        *wrap |= x < v;
        v = x;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_incl_scan_u64(unsigned long long v,
                                                                 uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(kFull, v, o);
        if (lane >= (uint32_t)o) v += t;
    }
    return v;
}

// Every lane of the warp calls this with the same row; returns the chosen
// slot (absolute index) on every lane, or ~0u when the total weight is 0.
__device__ __forceinline__ uint32_t warp_pick_weighted(const uint2 *__restrict__ slots,
                                                    const float *__restrict__ wts, uint32_t lo,
                                                    uint32_t deg, uint32_t ex, bool has_ex,
                                                    uint32_t r, unsigned long long *seg,
                                                    uint32_t lane) {
    const uint32_t hi = lo + deg;
    const uint32_t abase = lo & ~3u;
    const uint32_t ntile = (hi - abase + 127u) >> 7;
    uint32_t G = (ntile + kSegs - 1u) / kSegs;   // tiles per segment
    unsigned long long total = 0ull, segsum = 0ull;
    bool wrap = false;
    for (uint32_t t = 0; t < ntile; ++t) {
        unsigned long long q[4];
        quad_weights(slots, wts, abase + (t << 7) + 4u * lane, lo, hi, ex, has_ex, q);
        unsigned long long v = q[0] + q[1];
        wrap |= v < q[0];
        unsigned long long v2 = q[2] + q[3];
        wrap |= v2 < q[2];
        const unsigned long long v3 = v + v2;
        wrap |= v3 < v;
        v = warp_sum_u64(v3, &wrap);
        const unsigned long long nt = total + v;
        wrap |= nt < total;
        total = nt;
        segsum += v;
        if (t % G == G - 1u || t == ntile - 1u) {
            if (lane == 0u) seg[t / G] = segsum;
            segsum = 0ull;
        }
    }
    wrap = __any_sync(kFull, wrap);
    __syncwarp();
    if (total == 0ull) return ~0u;
    const unsigned long long target = mul_hi32(r, total);
    uint32_t t0 = 0u, t1 = ntile;
    unsigned long long base = 0ull;
    if (!wrap) {
        // the segment holding the target: lane l holds segments 2l and 2l+1
        const uint32_t nseg = (ntile + G - 1u) / G;
        const unsigned long long a = 2u * lane < nseg ? seg[2u * lane] : 0ull;
        const unsigned long long b = 2u * lane + 1u < nseg ? seg[2u * lane + 1u] : 0ull;
        const unsigned long long incl = warp_incl_scan_u64(a + b, lane);
        const unsigned long long excl = incl - (a + b);
        const uint32_t L = __ffs(__ballot_sync(kFull, incl > target)) - 1u;
        const bool in_a = excl + a > target;
        const uint32_t sidx = __shfl_sync(kFull, 2u * lane + (in_a ? 0u : 1u), L);
        base = __shfl_sync(kFull, in_a ? excl : excl + a, L);
        t0 = sidx * G;
        t1 = min(ntile, t0 + G);
    }
    __syncwarp();   // every lane read seg before a later row overwrites it
    for (uint32_t t = t0; t < t1; ++t) {
        const uint32_t j = abase + (t << 7) + 4u * lane;
        unsigned long long q[4];
        quad_weights(slots, wts, j, lo, hi, ex, has_ex, q);
        const unsigned long long v = q[0] + q[1] + q[2] + q[3];
        const unsigned long long incl = warp_incl_scan_u64(v, lane);
        // wrapped prefixes when `wrap`: then every tile is scanned in order
        // and the first slot whose prefix exceeds the target is the
        // per-thread scan's choice
        unsigned long long acc = base + incl - v;
        uint32_t hit = ~0u;
#pragma unroll
        for (uint32_t u = 0; u < 4u; ++u) {
            acc += q[u];
            if (hit == ~0u && j + u >= lo && j + u < hi && acc > target) hit = j + u;
        }
        const unsigned m = __ballot_sync(kFull, hit != ~0u);
        if (m) return __shfl_sync(kFull, hit, __ffs(m) - 1u);
        base += __shfl_sync(kFull, incl, 31);
    }
    return ~0u;
}

// One move of every active lane's walker, with rows longer than kCoopRow
// searched by the whole warp (all 32 lanes call this).  Returns the move's
// result for active lanes.
template <bool INCR>
__device__ __forceinline__ int step_weighted_warp(Walker &s, bool active, const DevGraph &g,
                                                  uint32_t max_steps, float thr, uint2 key,
                                                  unsigned long long *seg, uint32_t lane,
                                                  bool *moved, uint2 *taken, uint32_t *taken_at) {
    *moved = false;
    uint2 d = make_uint2(0u, 0u);
    bool first = false, pick = false;
    uint32_t r = 0u;
    if (active) {
        d = __ldg(g.desc + s.cur);
        first = (s.step == 1u);
        if (!(first ? (d.y == 0u) : (d.y <= 1u))) {
            r = draw_next(s, key);
            pick = true;
        }
    }
    uint32_t at = ~0u;
    uint2 sl = make_uint2(0u, 0u);
    const bool own_row = pick && d.y <= kCoopRow;   // chosen by this lane, slot in hand
    if (own_row) at = lane_pick_weighted(g.slots, g.wts, d.x, d.y, s.prev, !first, r, &sl);
    unsigned coop = __ballot_sync(kFull, pick && d.y > kCoopRow);
    while (coop) {
        const uint32_t L = __ffs(coop) - 1u;
        coop &= coop - 1u;
        const uint32_t lo = __shfl_sync(kFull, d.x, L), dg = __shfl_sync(kFull, d.y, L);
        const uint32_t ex = __shfl_sync(kFull, s.prev, L), rr = __shfl_sync(kFull, r, L);
        const bool hx = __shfl_sync(kFull, first ? 0u : 1u, L) != 0u;
        const uint32_t j = warp_pick_weighted(g.slots, g.wts, lo, dg, ex, hx, rr, seg, lane);
        if (lane == L) at = j;
    }
    if (!pick || at == ~0u) return kFail;
    if (!own_row) sl = __ldg(g.slots + at);
    return finish_move<INCR>(s, sl, at, first, max_steps, thr, moved, taken, taken_at);
}

// RN(1/R) < c for positive finite R, c, decided by one product where it can
// be: p = RN(R*c) is within 2^-24 of R*c, so p > 1 + 2^-21 gives
// 1/R < c (1 - 7 * 2^-24), below c by more than half an ulp of c, hence
// RN(1/R) < c; p < 1 - 2^-21 gives RN(1/R) > c the same way.  Only products
// inside that band take the correctly rounded reciprocal.
__device__ __forceinline__ bool below_best(float R, float c) {
    const float p = __fmul_rn(R, c);
    if (p > 1.0000004768371582f) return true;    // 1 + 2^-21
    if (p < 0.9999995231628418f) return false;   // 1 - 2^-21
    return __frcp_rn(R) < c;
}

// Resident blocks per SM the register budget is sized for: 6 (40 registers)
// for the uniform walks, 3 for the weighted ones (shared-memory segment sums).
template <bool INCR, bool WEIGHTED, int MOVES>
__global__ void __launch_bounds__(kWalkThreads, WEIGHTED ? 3 : 6) k_walk(WalkArgs a) {
    // per-warp segment sums of the cooperative weighted search
    __shared__ unsigned long long s_seg[WEIGHTED ? (kWalkThreads / 32) * kSegs : 1];
    if (a.job.halt && *a.job.halt) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t n = a.job.n_dev ? *a.job.n_dev : a.job.n_host;
    const uint32_t CW = a.chunk;                // walkers per chunk (divides walkers)
    const uint32_t cpe = a.walkers / CW;        // chunks per edge
    const uint32_t cpe_sh = (cpe & (cpe - 1u)) ? 32u : (uint32_t)(__ffs(cpe) - 1);
    const unsigned long long n_chunks = (unsigned long long)n * cpe;
    unsigned long long *work = a.scalars + S_WORK;

    // warp-uniform: the edge and walker range of the current chunk
    uint32_t ce = 0xFFFFFFFFu, c_next = 0u, c_end = 0u;
    bool exhausted = false;
    // best conductance bits seen in this warp for the current chunk's edge and
    // the previous one (warp-uniform)
    uint32_t ce_best = 0u, pe = 0xFFFFFFFFu, pe_best = 0u;

    bool active = false;
    uint32_t my_e = 0xFFFFFFFFu;
    uint32_t gbest = 0u;  // lane: last read of the edge's global best (cond bits)
    Walker s;
    s.cur = s.prev = s.step = s.tgt = s.walker = s.c2 = s.c3 = 0u;
    s.rblk = 0xFFFFFFFFu;
    s.rbuf = make_uint4(0u, 0u, 0u, 0u);
    s.R = 0.f;
    s.we = 0.f;
    uint32_t moves = 0u, walks = 0u;

    // Walkers start only on warp iterations that keep every walker of the
    // warp aligned to its 4-draw Philox blocks (each walker moves MOVES times
    // per iteration): then all of them draw their next block at the same
    // move, so the block (a quarter of the kernel's instructions when
    // computed) runs for the whole warp at once instead of for a few lanes at
    // a time, and refills are batched.  An empty warp refills at once.
    uint32_t T = 0u;
    while (true) {
        uint32_t free_mask = __ballot_sync(kFull, !active);
        if (free_mask == kFull) T = 0u;
        // walkers start when their steps stay aligned to the 4-draw Philox
        // blocks: every fourth iteration with one move per iteration, every
        // second with two, every iteration with four
        constexpr uint32_t kAlign = MOVES >= 4 ? 0u : (MOVES == 2 ? 1u : 3u);
        const bool refill = (T & kAlign) == 0u;
        while (free_mask != 0u && !exhausted && refill) {
            if (c_next >= c_end) {
                unsigned long long c = 0ull;
                if (lane == 0u) c = atomicAdd(work, 1ull);
                c = __shfl_sync(kFull, c, 0);
                if (c >= n_chunks) {
                    exhausted = true;
                    break;
                }
                // chunk c = edge e, part c mod cpe (cpe is a power of two
                // whenever the walker count is one)
                const uint32_t e = (c >> 32) ? (uint32_t)(c / cpe)
                                             : (cpe_sh < 32u ? (uint32_t)c >> cpe_sh
                                                             : (uint32_t)c / cpe);
                if (e != ce) {
                    pe = ce;
                    pe_best = ce_best;
                    ce = e;
                    ce_best = 0u;
                }
                c_next = (uint32_t)(c - (unsigned long long)e * cpe) * CW;
                c_end = c_next + CW;
            }
            const uint32_t take = min((uint32_t)__popc(free_mask), c_end - c_next);
            const uint32_t rank = __popc(free_mask & lt_mask);
            if (((free_mask >> lane) & 1u) && rank < take) {
                const uint32_t e = ce;
                my_e = e;
                s.walker = c_next + rank;
                s.cur = a.job.src[e];
                s.tgt = a.job.dst[e];
                s.we = INCR ? a.job.w[e] : 0.f;
                const unsigned long long uid = a.job.uid ? a.job.uid[e] : a.job.uid0 + e;
                s.c2 = (uint32_t)uid;
                s.c3 = ctr3_of(uid, a.job.domain);
                s.rblk = 0xFFFFFFFFu;
                s.step = 1u;
                s.R = 0.f;
                s.prev = 0u;
                gbest = a.prune ? (uint32_t)(*(volatile unsigned long long *)(a.keys + e) >> 32) : 0u;
                if (s.cur >= a.g.n || s.tgt >= a.g.n) {
                    atomicOr(a.scalars + S_ERR, (unsigned long long)kErrVertex);
                    ++walks;
                } else {
                    active = true;
                }
            }
            // the lanes that took a walker leave the free mask
            free_mask = __ballot_sync(kFull, ((free_mask >> lane) & 1u) && rank >= take);
            c_next += take;
        }
        if (!__any_sync(kFull, active)) break;
        uint32_t fc = 0u;  // conductance bits of a walker that found its target now
        // With four moves per iteration every walker enters an iteration at a
        // step = 1 (mod 4) (walkers start at the top of an iteration and move
        // four times in each one they stay in), so its Philox block for the
        // iteration is drawn once, up front, and word mv serves move mv.
        uint4 blk = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int mv = 0; mv < (WEIGHTED ? 1 : MOVES); ++mv) {
            int r = kContinue;
            bool moved = false;
            uint2 taken;
            uint32_t taken_at;
            if constexpr (WEIGHTED) {
                r = step_weighted_warp<INCR>(s, active, a.g, a.max_steps, a.threshold, a.key,
                                             s_seg + (threadIdx.x >> 5) * kSegs, lane, &moved,
                                             &taken, &taken_at);
            } else if (MOVES == 4 && active) {
                const uint2 d = __ldg(a.g.desc + s.cur);
                if (mv == 0)
                    blk = philox4x32_10(make_uint4((s.step - 1u) >> 2, s.walker, s.c2, s.c3), a.key);
                const uint32_t rd = mv == 0 ? blk.x : (mv == 1 ? blk.y : (mv == 2 ? blk.z : blk.w));
                r = (s.step == 1u ? d.y == 0u : d.y <= 1u)
                        ? kFail
                        : move_uniform<INCR>(s, d, rd, a.g.slots, a.max_steps, a.threshold, &moved,
                                             &taken, &taken_at);
            } else if (active) {
                r = step_once<INCR, false>(s, a.g.desc, a.g.slots, a.g.wts, a.max_steps,
                                           a.threshold, a.key, &moved, &taken, &taken_at);
            }
            if (active) {
                moves += moved ? 1u : 0u;
                if (r != kContinue) {
                    if (r == kFound) {
                        const float cond = __frcp_rn(s.R);
                        fc = __float_as_uint(cond);
                        // published at once, so walkers of this edge in other
                        // warps can stop early
                        atomicMax(a.keys + my_e, pack_key(cond, s.walker, s.step));
                    }
                    active = false;
                    ++walks;
                }
            }
        }
        if (a.prune) {
            // R only grows along a walk and 1/R is monotone, so a walker whose
            // 1/R is already below its edge's best success can neither win
            // nor tie: stopping it leaves every result unchanged.
            if (__any_sync(kFull, fc != 0u)) {
                ce_best = max(ce_best, __reduce_max_sync(kFull, (fc && my_e == ce) ? fc : 0u));
                pe_best = max(pe_best, __reduce_max_sync(kFull, (fc && my_e == pe) ? fc : 0u));
            }
            if (active) {
                // the edge's best is read again every fourth move
                constexpr uint32_t kEvery = MOVES >= 4 ? 1u : (MOVES == 2 ? 2u : 4u);
                const uint32_t pm = kEvery * a.prune_every - 1u;
                if ((T & pm) == pm)
                    gbest = max(gbest, (uint32_t)(*(volatile unsigned long long *)(a.keys + my_e) >> 32));
                const uint32_t known = max(gbest, (my_e == ce) ? ce_best
                                                  : (my_e == pe ? pe_best : 0u));
                if (known && below_best(s.R, __uint_as_float(known))) {
                    active = false;
                    ++walks;
                }
            }
        }
        ++T;
    }
    const uint32_t wm = __reduce_add_sync(kFull, moves);
    const uint32_t ww = __reduce_add_sync(kFull, walks);
    if (lane == 0u) {
        if (wm) atomicAdd(a.scalars + S_MOVES, (unsigned long long)wm);
        if (ww) atomicAdd(a.scalars + S_WALKS, (unsigned long long)ww);
    }
}

// Replays the winner of each decremental edge and writes its path
// (random_walk_decremental/main.cu:206-217 writes the same vertices from a
// per-thread local array).
template <bool WEIGHTED>
__global__ void k_winner_paths(DevGraph g, WalkJob job, uint32_t max_steps, uint2 key,
                               const unsigned long long *keys, uint32_t stride, uint32_t *pv,
                               uint32_t *ps, int32_t *plen, unsigned long long *scalars) {
    if (job.halt && *job.halt) return;
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = job.n_dev ? *job.n_dev : job.n_host;
    if (f >= n) return;
    const unsigned long long k = keys[f];
    if (!k) {
        plen[f] = -1;
        return;
    }
    Walker s;
    s.walker = key_walker(k);
    s.cur = job.src[f];
    s.tgt = job.dst[f];
    s.we = 0.f;
    const unsigned long long uid = job.uid ? job.uid[f] : job.uid0 + f;
    s.c2 = (uint32_t)uid;
    s.c3 = ctr3_of(uid, job.domain);
    s.rblk = 0xFFFFFFFFu;
    s.rbuf = make_uint4(0u, 0u, 0u, 0u);
    s.step = 1u;
    s.R = 0.f;
    s.prev = 0u;
    uint32_t *row_v = pv + (size_t)f * stride;
    uint32_t *row_s = ps + (size_t)f * stride;
    row_v[0] = s.cur;
    int r;
    do {
        const uint32_t at = s.step;
        bool moved;
        uint2 taken;
        uint32_t taken_at;
        r = step_once<false, WEIGHTED>(s, g.desc, g.slots, g.wts, max_steps, 0.f, key, &moved,
                                       &taken, &taken_at);
        if (moved && at < stride) {   // no load: a store waiting on one would stall the chain
            row_v[at] = taken.x;
            row_s[at] = taken_at;
        }
    } while (r == kContinue);
    const int32_t found = (r == kFound) ? (int32_t)s.step : -1;
    plen[f] = found;
    if (found != key_found(k)) atomicOr(scalars + S_ERR, (unsigned long long)kErrPath);
}

// Weighted winner replays, one warp per path: the walker lives in lane 0 and
// rows longer than kCoopRow are searched by the whole warp, as in the walk
// kernel (a replay through a hub row would otherwise scan it one slot at a
// time).
constexpr int kReplayThreads = 128;
__global__ void __launch_bounds__(kReplayThreads)
k_winner_paths_weighted(DevGraph g, WalkJob job, uint32_t max_steps, uint2 key,
                        const unsigned long long *keys, uint32_t stride, uint32_t *pv, uint32_t *ps,
                        int32_t *plen, unsigned long long *scalars) {
    __shared__ unsigned long long s_seg[(kReplayThreads / 32) * kSegs];
    if (job.halt && *job.halt) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t f = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n = job.n_dev ? *job.n_dev : job.n_host;
    if (f >= n) return;   // whole warps leave together
    const unsigned long long k = keys[f];
    if (!k) {
        if (lane == 0u) plen[f] = -1;
        return;
    }
    Walker s;
    s.walker = key_walker(k);
    s.cur = job.src[f];
    s.tgt = job.dst[f];
    s.we = 0.f;
    const unsigned long long uid = job.uid ? job.uid[f] : job.uid0 + f;
    s.c2 = (uint32_t)uid;
    s.c3 = ctr3_of(uid, job.domain);
    s.rblk = 0xFFFFFFFFu;
    s.rbuf = make_uint4(0u, 0u, 0u, 0u);
    s.step = 1u;
    s.R = 0.f;
    s.prev = 0u;
    uint32_t *row_v = pv + (size_t)f * stride;
    uint32_t *row_s = ps + (size_t)f * stride;
    if (lane == 0u) row_v[0] = s.cur;
    unsigned long long *seg = s_seg + (threadIdx.x >> 5) * kSegs;
    int r;
    do {
        const uint32_t at = s.step;
        bool moved;
        uint2 taken;
        uint32_t taken_at;
        r = step_weighted_warp<false>(s, lane == 0u, g, max_steps, 0.f, key, seg, lane, &moved,
                                      &taken, &taken_at);
        r = __shfl_sync(kFull, r, 0);
        if (lane == 0u && moved && at < stride) {
            row_v[at] = taken.x;
            row_s[at] = taken_at;
        }
    } while (r == kContinue);
    if (lane == 0u) {
        const int32_t found = (r == kFound) ? (int32_t)s.step : -1;
        plen[f] = found;
        if (found != key_found(k)) atomicOr(scalars + S_ERR, (unsigned long long)kErrPath);
    }
}

// 2-step fallback walks from both endpoints of each edge that found no path
// (random_walk_decremental/main.cu:243-290, with the second step reading the
// row of the vertex the walker stands on).  Candidate pair 2i, 2i+1 of item
// i = (q * 2 + side) * hw + j is (s0, x1), (x1, x2); x = ~0u marks none.
__global__ void k_fallback(DevGraph g, const unsigned long long *halt, const uint32_t *f_src,
                           const uint32_t *f_dst, const unsigned long long *f_uid,
                           const uint32_t *nop, const uint32_t *n_nop_dev, uint32_t hw, uint2 key,
                           const uint32_t *base_dev, uint32_t *cx, uint32_t *cy, float *cw) {
    if (halt && *halt) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t per = 2u * hw;
    if (i >= *n_nop_dev * per) return;
    const uint32_t b = *base_dev;
    cx += b;
    cy += b;
    cw += b;
    const uint32_t q = i / per, rem = i - q * per, side = rem / hw, j = rem - side * hw;
    const uint32_t f = nop[q];
    const uint32_t s0 = side ? f_dst[f] : f_src[f];
    const unsigned long long uid = f_uid[f];
    const uint4 rb = philox4x32_10(make_uint4(0u, side * hw + j, (uint32_t)uid,
                                              ctr3_of(uid, kDomainHeur)), key);
    uint32_t x1 = ~0u, x2 = ~0u;
    float w1 = 0.f, w2 = 0.f;
    const uint2 d0 = __ldg(g.desc + s0);
    if (d0.y != 0u) {
        const uint32_t i0 = d0.x + rb.x % d0.y;
        x1 = __ldg(&g.slots[i0].x);
        w1 = __ldg(g.wts + i0);
        const uint2 d1 = __ldg(g.desc + x1);
        if (d1.y != 0u) {
            uint32_t i1 = d1.x + rb.y % d1.y;
            if (__ldg(&g.slots[i1].x) == s0) i1 = d1.x + d1.y - 1u;
            x2 = __ldg(&g.slots[i1].x);
            w2 = __ldg(g.wts + i1);
        }
    }
    cx[2 * i] = (x1 == ~0u) ? ~0u : s0;
    cy[2 * i] = x1;
    cw[2 * i] = w1;
    cx[2 * i + 1] = (x2 == ~0u) ? ~0u : x1;
    cy[2 * i + 1] = x2;
    cw[2 * i + 1] = w2;
}

// Walkers handed to a warp at a time: 32 by default, so that the 512 walks
// of an edge nobody connects spread over 16 warps instead of running as 16
// waves on one.  DYG_WALK_CHUNK (a multiple of 32 dividing the walker count)
// overrides it for tuning sweeps.
// Launch shape of the walk kernel, process-wide (dyg_tune_set); 0 = default.
static std::atomic<uint32_t> g_tune_chunk{0}, g_tune_bpsm{0}, g_tune_prune{0};

// Iterations between reads of an edge's best result for pruning (1, 2 or 4).
static uint32_t prune_every() {
    const uint32_t t = g_tune_prune.load();
    return (t == 2u || t == 4u) ? t : 1u;
}

static uint32_t chunk_for(uint32_t walkers) {
    static int env = -1;
    if (env < 0) {
        const char *v = getenv("DYG_WALK_CHUNK");
        env = v ? atoi(v) : 0;
    }
    const uint32_t want = g_tune_chunk.load() ? g_tune_chunk.load() : (uint32_t)(env > 0 ? env : 0);
    uint32_t c = 32u;
    if (want > 0 && want % 32 == 0 && walkers % want == 0) c = want;
    return c;
}

// Resident blocks per SM, cached per kernel instance (the instances share one
// function type but not their launch bounds).
template <bool INCR, bool WTD, int MOVES>
static int persistent_blocks() {
    static int per_sm = 0;
    if (!per_sm) {
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_walk<INCR, WTD, MOVES>, kWalkThreads, 0);
        per_sm = nb < 1 ? 1 : nb;
    }
    const uint32_t t = g_tune_bpsm.load();
    const int b = (t && (int)t < per_sm) ? (int)t : per_sm;
    return b * num_sms();
}

// Moves per warp iteration of the uniform walk: 4 by default (the warp's
// refill, prune and loop bookkeeping then runs once per four moves; walk time
// per step on the 100^3 mesh: 11.08 ms with one move, 9.99 with two, 9.64 with
// four); DYG_WALK_MOVES = 1, 2 or 4 overrides it for tuning runs.  Results do
// not depend on it.
static int walk_moves() {
    static int m = 0;
    if (!m) {
        const char *v = getenv("DYG_WALK_MOVES");
        const int x = v ? atoi(v) : 4;
        m = (x == 1 || x == 2) ? x : 4;
    }
    return m;
}

template <bool INCR, bool WTD>
static void launch_walk_kernel(const WalkArgs &a, cudaStream_t st) {
    if constexpr (!WTD) {
        if (walk_moves() == 2) {
            const int grid = persistent_blocks<INCR, WTD, 2>();
            k_walk<INCR, WTD, 2><<<grid, kWalkThreads, 0, st>>>(a);
            return;
        }
        if (walk_moves() == 4) {
            const int grid = persistent_blocks<INCR, WTD, 4>();
            k_walk<INCR, WTD, 4><<<grid, kWalkThreads, 0, st>>>(a);
            return;
        }
    }
    const int grid = persistent_blocks<INCR, WTD, 1>();
    k_walk<INCR, WTD, 1><<<grid, kWalkThreads, 0, st>>>(a);
}

static void launch_walk_any(const WalkArgs &a, bool incremental, bool wtd, cudaStream_t st) {
    if (incremental) {
        if (wtd) launch_walk_kernel<true, true>(a, st);
        else launch_walk_kernel<true, false>(a, st);
    } else {
        if (wtd) launch_walk_kernel<false, true>(a, st);
        else launch_walk_kernel<false, false>(a, st);
    }
}

dyg_status launch_walk(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p, bool incremental,
                       unsigned long long *keys, cudaStream_t st) {
    WalkArgs a{};
    a.g = G->g;
    a.job = job;
    a.walkers = p.walkers;
    a.max_steps = p.max_steps;
    a.prune = (p.flags & DYG_FLAG_EXHAUSTIVE) ? 0u : 1u;
    a.prune_every = prune_every();
    a.chunk = chunk_for(p.walkers);
    a.threshold = p.threshold;
    a.key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    a.keys = keys;
    a.scalars = ptr<unsigned long long>(G->ws.scalars);
    DYG_CUDA(cudaMemsetAsync(a.scalars + S_WORK, 0, sizeof(unsigned long long), st));
    ProfScope prof(incremental ? 0 : 1, st);
    launch_walk_any(a, incremental, p.transition == DYG_TRANSITION_WEIGHTED, st);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// Same launch as launch_walk, with the kernel's counters (work chunks,
// error bits, move counts) at `scalars` instead of the handle's workspace, and
// without profiling events.
dyg_status launch_walk_scalars(const DevGraph &g, const WalkJob &job, const dyg_walk_params &p,
                               bool incremental, unsigned long long *keys,
                               unsigned long long *scalars, cudaStream_t st) {
    WalkArgs a{};
    a.g = g;
    a.job = job;
    a.walkers = p.walkers;
    a.max_steps = p.max_steps;
    a.prune = (p.flags & DYG_FLAG_EXHAUSTIVE) ? 0u : 1u;
    a.prune_every = prune_every();
    a.chunk = chunk_for(p.walkers);
    a.threshold = p.threshold;
    a.key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    a.keys = keys;
    a.scalars = scalars;
    launch_walk_any(a, incremental, p.transition == DYG_TRANSITION_WEIGHTED, st);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status launch_winner_paths(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p,
                               const unsigned long long *keys, uint32_t n_max, uint32_t stride,
                               uint32_t *path_v, uint32_t *path_s, int32_t *path_len, cudaStream_t st) {
    if (n_max == 0) return DYG_OK;
    const uint2 key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    const int threads = 128;
    const int grid = (int)((n_max + threads - 1) / threads);
    unsigned long long *sc = ptr<unsigned long long>(G->ws.scalars);
    ProfScope prof(2, st);
    if (p.transition == DYG_TRANSITION_WEIGHTED)
        k_winner_paths_weighted<<<(unsigned)(((uint64_t)n_max * 32 + kReplayThreads - 1) / kReplayThreads),
                                  kReplayThreads, 0, st>>>(G->g, job, p.max_steps, key, keys, stride,
                                                           path_v, path_s, path_len, sc);
    else
        k_winner_paths<false><<<grid, threads, 0, st>>>(G->g, job, p.max_steps, key, keys, stride,
                                                        path_v, path_s, path_len, sc);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status launch_fallback_walks(dyg_graph *G, const unsigned long long *halt,
                                 const uint32_t *f_src, const uint32_t *f_dst,
                                 const unsigned long long *f_uid, const uint32_t *nop,
                                 const uint32_t *n_nop_dev, uint32_t n_nop_max,
                                 const dyg_walk_params &p, const uint32_t *base_dev, uint32_t *cx,
                                 uint32_t *cy, float *cw, cudaStream_t st) {
    const uint64_t items = (uint64_t)n_nop_max * 2u * p.heuristic_walkers;
    if (items == 0) return DYG_OK;
    const uint2 key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    const int threads = 128;
    ProfScope prof(2, st);
    k_fallback<<<(unsigned)((items + threads - 1) / threads), threads, 0, st>>>(
        G->g, halt, f_src, f_dst, f_uid, nop, n_nop_dev, p.heuristic_walkers, key, base_dev, cx, cy,
        cw);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

}  // namespace dyg

extern "C" {

dyg_status dyg_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(dyg::g_prof_mu);
    dyg::g_prof_on = on != 0;
    return DYG_OK;
}

dyg_status dyg_profile_reset(void) {
    std::lock_guard<std::mutex> lk(dyg::g_prof_mu);
    dyg::prof_flush_locked();
    dyg::g_prof_acc = dyg_profile{};
    return DYG_OK;
}

dyg_status dyg_profile_read(dyg_profile *out) {
    if (!out) return DYG_EINVAL;
    std::lock_guard<std::mutex> lk(dyg::g_prof_mu);
    dyg::prof_flush_locked();
    *out = dyg::g_prof_acc;
    return DYG_OK;
}

}  // extern "C"

extern "C" void dyg_tune_set_prune_interval(uint32_t iterations) {
    dyg::g_tune_prune.store(iterations);
}

extern "C" void dyg_tune_set(uint32_t walk_chunk, uint32_t blocks_per_sm) {
    dyg::g_tune_chunk.store(walk_chunk);
    dyg::g_tune_bpsm.store(blocks_per_sm);
}
