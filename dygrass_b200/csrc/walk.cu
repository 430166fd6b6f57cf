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

// One move of one walker, mirroring the reference loop body:
//   step 1:  any neighbour, r % deg                    (main.cu:99-106)
//   step >1: dead end if deg == 1; r % (deg - 1) and the last slot when the
//            draw lands on the previous vertex          (main.cu:118-137)
//   R += 1/w; distortion test (incremental only, from step 2 on), then the
//   target test; walk ends when the step counter reaches max_steps
//                                                       (main.cu:116, 139-157)
// *moved is set when a neighbour was drawn; *taken receives its slot.
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
    const uint32_t di = s.step - 1u, b = di >> 2;
    if (b != s.rblk) {
        s.rbuf = philox4x32_10(make_uint4(b, s.walker, s.c2, s.c3), key);
        s.rblk = b;
    }
    const uint32_t r = pick4(s.rbuf, di & 3u);
    uint2 sl;
    uint32_t at;
    if (!WEIGHTED) {
        const uint32_t idx = first ? (r % deg) : (r % (deg - 1u));
        at = d.x + idx;
        sl = __ldg(slots + at);
        if (!first) {
            // the row's last slot is loaded beside the drawn one, not after
            // it: some lane of a warp lands on its previous vertex in almost
            // every step, and a dependent reload would hold the whole warp
            const uint32_t at_last = d.x + deg - 1u;
            const uint2 sl_last = __ldg(slots + at_last);
            if (sl.x == s.prev) {
                at = at_last;
                sl = sl_last;
            }
        }
    } else {
        unsigned long long total = 0ull;
        for (uint32_t j = 0; j < deg; ++j) {
            if (!first && __ldg(&slots[d.x + j].x) == s.prev) continue;
            total += wq(__ldg(wts + d.x + j));
        }
        if (total == 0ull) return kFail;
        const unsigned long long target = mul_hi32(r, total);
        unsigned long long acc = 0ull;
        uint32_t last = deg;
        for (uint32_t j = 0; j < deg; ++j) {
            if (!first && __ldg(&slots[d.x + j].x) == s.prev) continue;
            acc += wq(__ldg(wts + d.x + j));
            last = j;
            if (acc > target) break;
        }
        at = d.x + last;
        sl = __ldg(slots + at);
    }
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

template <bool INCR, bool WEIGHTED>
__global__ void __launch_bounds__(kWalkThreads) k_walk(WalkArgs a) {
    if (a.job.halt && *a.job.halt) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t n = a.job.n_dev ? *a.job.n_dev : a.job.n_host;
    const uint32_t CW = a.chunk;                // walkers per chunk (divides walkers)
    const uint32_t cpe = a.walkers / CW;        // chunks per edge
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

    // Walkers start only on warp iterations T = 0 mod 4.  Every walker moves
    // once per iteration, so all of a warp's walkers then stand at steps
    // 1 mod 4 together and draw their next Philox block in the same
    // iteration: the block (a quarter of the kernel's instructions when
    // computed) is run once per four iterations by the whole warp instead of
    // in almost every iteration for a few lanes, and refills are batched.
    // A lane waits at most three iterations; an empty warp refills at once.
    uint32_t T = 0u;
    while (true) {
        uint32_t free_mask = __ballot_sync(kFull, !active);
        if (free_mask == kFull) T = 0u;
        const bool refill = (T & 3u) == 0u;
        while (free_mask != 0u && !exhausted && refill) {
            if (c_next >= c_end) {
                unsigned long long c = 0ull;
                if (lane == 0u) c = atomicAdd(work, 1ull);
                c = __shfl_sync(kFull, c, 0);
                if (c >= n_chunks) {
                    exhausted = true;
                    break;
                }
                const uint32_t e = (uint32_t)(c / cpe);
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
            for (uint32_t i = 0; i < take; ++i) free_mask &= free_mask - 1u;
            c_next += take;
        }
        if (!__any_sync(kFull, active)) break;
        uint32_t fc = 0u;  // conductance bits of a walker that found its target now
        if (active) {
            bool moved;
            uint2 taken;
            uint32_t taken_at;
            const int r = step_once<INCR, WEIGHTED>(s, a.g.desc, a.g.slots, a.g.wts, a.max_steps,
                                                   a.threshold, a.key, &moved, &taken, &taken_at);
            moves += moved ? 1u : 0u;
            if (r != kContinue) {
                if (r == kFound) {
                    const float cond = __frcp_rn(s.R);
                    fc = __float_as_uint(cond);
                    // published at once, so walkers of this edge in other warps
                    // can stop early
                    atomicMax(a.keys + my_e, pack_key(cond, s.walker, s.step));
                }
                active = false;
                ++walks;
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
                if ((s.step & 3u) == 0u)
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
                               float *pw, int32_t *plen, unsigned long long *scalars) {
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
    float *row_w = pw + (size_t)f * stride;
    row_v[0] = s.cur;
    row_w[0] = 0.f;
    int r;
    do {
        const uint32_t at = s.step;
        bool moved;
        uint2 taken;
        uint32_t taken_at;
        r = step_once<false, WEIGHTED>(s, g.desc, g.slots, g.wts, max_steps, 0.f, key, &moved,
                                       &taken, &taken_at);
        if (moved && at < stride) {
            row_v[at] = taken.x;
            row_w[at] = g.wts[taken_at];
        }
    } while (r == kContinue);
    const int32_t found = (r == kFound) ? (int32_t)s.step : -1;
    plen[f] = found;
    if (found != key_found(k)) atomicOr(scalars + S_ERR, (unsigned long long)kErrPath);
}

// 2-step fallback walks from both endpoints of each edge that found no path
// (random_walk_decremental/main.cu:243-290, with the second step reading the
// row of the vertex the walker stands on).  Candidate pair 2i, 2i+1 of item
// i = (q * 2 + side) * hw + j is (s0, x1), (x1, x2); x = ~0u marks none.
__global__ void k_fallback(DevGraph g, const unsigned long long *halt, const uint32_t *f_src,
                           const uint32_t *f_dst, const unsigned long long *f_uid,
                           const uint32_t *nop, const uint32_t *n_nop_dev, uint32_t hw, uint2 key,
                           uint32_t *cx, uint32_t *cy, float *cw) {
    if (halt && *halt) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t per = 2u * hw;
    if (i >= *n_nop_dev * per) return;
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
static std::atomic<uint32_t> g_tune_chunk{0}, g_tune_bpsm{0};

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

template <typename K>
static int persistent_blocks(K kernel) {
    static int per_sm = 0;
    if (!per_sm) {
        int nb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kWalkThreads, 0);
        per_sm = nb < 1 ? 1 : nb;
    }
    const uint32_t t = g_tune_bpsm.load();
    const int b = (t && (int)t < per_sm) ? (int)t : per_sm;
    return b * num_sms();
}

dyg_status launch_walk(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p, bool incremental,
                       unsigned long long *keys, cudaStream_t st) {
    WalkArgs a;
    a.g = G->g;
    a.job = job;
    a.walkers = p.walkers;
    a.max_steps = p.max_steps;
    a.prune = (p.flags & DYG_FLAG_EXHAUSTIVE) ? 0u : 1u;
    a.chunk = chunk_for(p.walkers);
    a.threshold = p.threshold;
    a.key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    a.keys = keys;
    a.scalars = ptr<unsigned long long>(G->ws.scalars);
    DYG_CUDA(cudaMemsetAsync(a.scalars + S_WORK, 0, sizeof(unsigned long long), st));
    const bool wtd = p.transition == DYG_TRANSITION_WEIGHTED;
    int grid;
    ProfScope prof(incremental ? 0 : 1, st);
    if (incremental) {
        if (wtd) {
            grid = persistent_blocks(k_walk<true, true>);
            k_walk<true, true><<<grid, kWalkThreads, 0, st>>>(a);
            count_launch();
        } else {
            grid = persistent_blocks(k_walk<true, false>);
            k_walk<true, false><<<grid, kWalkThreads, 0, st>>>(a);
            count_launch();
        }
    } else {
        if (wtd) {
            grid = persistent_blocks(k_walk<false, true>);
            k_walk<false, true><<<grid, kWalkThreads, 0, st>>>(a);
            count_launch();
        } else {
            grid = persistent_blocks(k_walk<false, false>);
            k_walk<false, false><<<grid, kWalkThreads, 0, st>>>(a);
            count_launch();
        }
    }
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

// Same launch as launch_walk, with the kernel's counters (work chunks,
// error bits, move counts) at `scalars` instead of the handle's workspace, and
// without profiling events.
dyg_status launch_walk_scalars(const DevGraph &g, const WalkJob &job, const dyg_walk_params &p,
                               bool incremental, unsigned long long *keys,
                               unsigned long long *scalars, cudaStream_t st) {
    WalkArgs a;
    a.g = g;
    a.job = job;
    a.walkers = p.walkers;
    a.max_steps = p.max_steps;
    a.prune = (p.flags & DYG_FLAG_EXHAUSTIVE) ? 0u : 1u;
    a.chunk = chunk_for(p.walkers);
    a.threshold = p.threshold;
    a.key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    a.keys = keys;
    a.scalars = scalars;
    const bool wtd = p.transition == DYG_TRANSITION_WEIGHTED;
    int grid;
    if (incremental) {
        if (wtd) {
            grid = persistent_blocks(k_walk<true, true>);
            k_walk<true, true><<<grid, kWalkThreads, 0, st>>>(a);
        } else {
            grid = persistent_blocks(k_walk<true, false>);
            k_walk<true, false><<<grid, kWalkThreads, 0, st>>>(a);
        }
    } else {
        if (wtd) {
            grid = persistent_blocks(k_walk<false, true>);
            k_walk<false, true><<<grid, kWalkThreads, 0, st>>>(a);
        } else {
            grid = persistent_blocks(k_walk<false, false>);
            k_walk<false, false><<<grid, kWalkThreads, 0, st>>>(a);
        }
    }
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status launch_winner_paths(dyg_graph *G, const WalkJob &job, const dyg_walk_params &p,
                               const unsigned long long *keys, uint32_t n_max, uint32_t stride,
                               uint32_t *path_v, float *path_w, int32_t *path_len, cudaStream_t st) {
    if (n_max == 0) return DYG_OK;
    const uint2 key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    const int threads = 128;
    const int grid = (int)((n_max + threads - 1) / threads);
    unsigned long long *sc = ptr<unsigned long long>(G->ws.scalars);
    ProfScope prof(2, st);
    if (p.transition == DYG_TRANSITION_WEIGHTED)
        k_winner_paths<true><<<grid, threads, 0, st>>>(G->g, job, p.max_steps, key, keys, stride,
                                                       path_v, path_w, path_len, sc);
    else
        k_winner_paths<false><<<grid, threads, 0, st>>>(G->g, job, p.max_steps, key, keys, stride,
                                                        path_v, path_w, path_len, sc);
    count_launch();
    DYG_CUDA(cudaGetLastError());
    return DYG_OK;
}

dyg_status launch_fallback_walks(dyg_graph *G, const unsigned long long *halt,
                                 const uint32_t *f_src, const uint32_t *f_dst,
                                 const unsigned long long *f_uid, const uint32_t *nop,
                                 const uint32_t *n_nop_dev, uint32_t n_nop_max,
                                 const dyg_walk_params &p, uint32_t *cx, uint32_t *cy, float *cw,
                                 cudaStream_t st) {
    const uint64_t items = (uint64_t)n_nop_max * 2u * p.heuristic_walkers;
    if (items == 0) return DYG_OK;
    const uint2 key = make_uint2((uint32_t)p.seed, (uint32_t)(p.seed >> 32));
    const int threads = 128;
    ProfScope prof(2, st);
    k_fallback<<<(unsigned)((items + threads - 1) / threads), threads, 0, st>>>(
        G->g, halt, f_src, f_dst, f_uid, nop, n_nop_dev, p.heuristic_walkers, key, cx, cy, cw);
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

extern "C" void dyg_tune_set(uint32_t walk_chunk, uint32_t blocks_per_sm) {
    dyg::g_tune_chunk.store(walk_chunk);
    dyg::g_tune_bpsm.store(blocks_per_sm);
}
