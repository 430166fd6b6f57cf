// server.cu -- the continuous-batching server of include/dyg_serve.h.
//
// The reference runs one graph per process and one batch loop per run
// (random_walk_incremental/main.cu:314-340, random_walk_decremental/
// main.cu:395-444); it has no request loop.  Here many graphs stay resident
// in one union graph and requests for them are scheduled in steps.  A step
// takes the oldest pending request of every resident graph that has one,
// gathers the insertion requests into one batch and the deletion requests
// into another (global vertex ids = local id + the graph's offset; per-edge
// update ids = the graph's own update counter), stages both through
// page-locked memory, runs the incremental pipeline and then the decremental
// pipeline on the device (one host synchronize each, for the halt/resume
// protocol), and splits the results back per request: per-edge arrays by
// position, recovered edges by the graph whose vertex range holds them (each
// step runs at most one deletion request per graph, and a recovered edge
// joins two vertices of the graph it was recovered in).
//
// Graphs are disjoint in the union, every walk stays inside its own graph, and
// a graph's update ids do not depend on the other graphs, so each request's
// result equals the one it gets alone on its graph's own handles.
//
// Two ways to hold the graphs:
//   static (dyg_server_create): the caller builds the union; every graph is
//     resident for the server's life.
//   pool (dyg_server_create_pool): the server owns the union graphs and an
//     HBM budget for the graphs' estimated footprints.  Registered graphs live
//     in host memory until a request for them is scheduled; then, at the start
//     of a step, waiting graphs (oldest pending request first) are admitted
//     into a free vertex range while their footprint fits the budget, and to
//     make room the server evicts resident graphs -- idle ones least recently
//     used first; busy ones, whose oldest pending request is younger than the
//     waiting graph's, only once the waiting graph has waited kPatienceSteps
//     steps -- by copying their rows back to host memory.  A
//     graph's rows keep their order through eviction and admission, so its
//     results do not depend on where or how often it was resident.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <iterator>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "dyg_internal.cuh"
#include "../../include/dyg_serve.h"

namespace dyg {
namespace {

struct Request {
    std::vector<uint32_t> src, dst;   // local ids
    std::vector<float> w;
    uint64_t submit_step = 0;         // the server's step count when it was queued
    bool finished = false;
    dyg_server_done rec{};
    std::vector<int32_t> out_i;       // found_at (insertion) or status (deletion)
    std::vector<float> out_c;         // conductance
    std::vector<uint8_t> out_a;       // accepted (insertion)
    std::vector<uint32_t> rx, ry;     // recovered edges, local ids (deletion)
    std::vector<uint8_t> rk;
};

// The vertex range [lo, hi) of a deletion request's graph during its step.
struct Owner {
    uint32_t lo, hi;
    Request *r;
};

// A step whose results still sit in the page-locked result buffers; its
// requests complete once split_results has handed the results out (during
// the next step's device work, or at once).
struct StepResults {
    bool active = false;
    std::vector<Request *> heads;
    std::vector<Owner> owners;   // deletion requests, ascending lo
    uint64_t ni = 0, nrec = 0, t_start = 0, step = 0;
};

// Page-locked host staging; grows, contents not kept.
template <typename T>
struct Pinned {
    T *p = nullptr;
    size_t cap = 0;
    dyg_status ensure(size_t n) {
        if (n <= cap) return DYG_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = n + n / 2 + 64;
        DYG_CUDA(cudaHostAlloc((void **)&p, want * sizeof(T), cudaHostAllocDefault));
        cap = want;
        return DYG_OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

struct DevSet {
    int prev = -1;
    bool changed = false;
    explicit DevSet(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = cudaSetDevice(dev) == cudaSuccess;
        cudaGetLastError();
    }
    ~DevSet() {
        if (changed) cudaSetDevice(prev);
    }
};

// Rows of one graph in host memory (local ids, row order as on the device).
struct HostRows {
    std::vector<uint64_t> rp;
    std::vector<uint32_t> col;
    std::vector<float> w;
    void clear() {
        std::vector<uint64_t>().swap(rp);
        std::vector<uint32_t>().swap(col);
        std::vector<float>().swap(w);
    }
};

// A graph of a pool server.  `resident`, `v0` and the counters change only in
// the thread that runs steps (or in a call that needs an idle server), under
// the server's lock; host rows are touched only by those threads.
struct PoolGraph {
    uint32_t n = 0;
    bool resident = false;
    uint32_t v0 = 0;              // first vertex in the union while resident
    uint64_t footprint = 0;       // estimated device bytes (admission size)
    uint64_t last_step = 0;       // last step that ran one of its requests
    uint64_t admissions = 0, evictions = 0;
    HostRows g, h;                // while not resident
    HostRows g0, h0;              // the registered rows (reset), if kept
};

}  // namespace
}  // namespace dyg

struct dyg_server {
    dyg_graph *G = nullptr, *H = nullptr;
    bool pool = false;
    std::vector<uint32_t> off;            // static: n_graphs + 1 vertex offsets
    dyg_walk_params ip{}, dp{};
    cudaStream_t st = nullptr;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;                        // guards everything below up to `loop`
    std::condition_variable cv_work, cv_idle;
    std::vector<std::deque<dyg::Request *>> queues;
    std::vector<uint64_t> uid_next;
    std::unordered_map<uint64_t, dyg::Request *> by_tag;   // submitted, not fetched
    std::deque<dyg_server_done> done;
    uint32_t pending = 0;
    bool stepping = false, loop_on = false, stop = false;
    uint64_t steps = 0;
    // host wall time of the steps' phases (ns, cumulative): admission,
    // staging, insertion run, deletion run, result fetch, result split
    uint64_t ns_phase[6] = {};
    std::string err;
    std::thread loop;

    // pool mode (graph states: see PoolGraph)
    std::deque<dyg::PoolGraph> pg;        // stable addresses while it grows
    uint64_t budget = 0, resident_bytes = 0, admissions = 0, evictions = 0;
    uint32_t vcap = 0;
    bool keep_initial = false;
    std::vector<std::pair<uint32_t, uint32_t>> free_ranges;   // [a, b), ascending

    // owned by the thread that runs the step
    dyg::Pinned<uint32_t> h_src, h_dst, h_rx, h_ry;
    dyg::Pinned<float> h_w, h_cond;
    dyg::Pinned<unsigned long long> h_uid;
    dyg::Pinned<int32_t> h_out;
    dyg::Pinned<uint8_t> h_acc, h_rk;
    dyg::Buf d_src, d_dst, d_w, d_uid, d_out, d_cond, d_acc;
    dyg::StepResults split;   // a step whose results are not handed out yet
};

namespace {

using dyg::HostRows;
using dyg::Owner;
using dyg::StepResults;
using dyg::PoolGraph;
using dyg::Request;

uint64_t now_ns(const dyg_server *s) {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now() - s->t0).count();
}

dyg_status fail(dyg_server *s, dyg_status code, const std::string &msg) {
    dyg::set_error(msg);
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = msg;
    }
    return code;
}

uint32_t graph_count(const dyg_server *s) { return (uint32_t)s->queues.size(); }

// First vertex and vertex count of graph g in the union (pool: while resident).
uint32_t graph_base(const dyg_server *s, uint32_t g) { return s->pool ? s->pg[g].v0 : s->off[g]; }
uint32_t graph_size(const dyg_server *s, uint32_t g) {
    return s->pool ? s->pg[g].n : s->off[g + 1] - s->off[g];
}

// Estimated device bytes of a graph: per slot 12 B (slot + weight) with the
// arena's headroom and per-row slack, per vertex 12 B (descriptor + capacity),
// for G and H each.
uint64_t footprint_of(uint32_t n, uint64_t g_slots, uint64_t h_slots, uint32_t slack,
                      double headroom) {
    const double gs = ((double)g_slots + (double)slack * n) * (1.0 + headroom);
    const double hs = ((double)h_slots + (double)slack * n) * (1.0 + headroom);
    return (uint64_t)(12.0 * (gs + hs)) + 24ull * n;
}

// ------------------------------------------------------ vertex ranges (pool)

bool range_find(const dyg_server *s, uint32_t n, uint32_t *v0) {
    for (const auto &r : s->free_ranges)
        if (r.second - r.first >= n) {
            *v0 = r.first;
            return true;
        }
    return false;
}

void range_take(dyg_server *s, uint32_t v0, uint32_t n) {
    for (size_t i = 0; i < s->free_ranges.size(); ++i) {
        auto &r = s->free_ranges[i];
        if (r.first == v0) {
            r.first += n;
            if (r.first == r.second) s->free_ranges.erase(s->free_ranges.begin() + (long)i);
            return;
        }
    }
}

void range_free(dyg_server *s, uint32_t v0, uint32_t n) {
    if (n == 0) return;
    auto &fr = s->free_ranges;
    auto it = std::lower_bound(fr.begin(), fr.end(), std::make_pair(v0, v0));
    it = fr.insert(it, std::make_pair(v0, v0 + n));
    // merge with the following and the preceding range
    if (it + 1 != fr.end() && it->second == (it + 1)->first) {
        it->second = (it + 1)->second;
        fr.erase(it + 1);
    }
    if (it != fr.begin() && (it - 1)->second == it->first) {
        (it - 1)->second = it->second;
        fr.erase(it);
    }
}

// Copies a resident graph's rows to host memory and frees its range.
dyg_status evict(dyg_server *s, uint32_t g) {
    PoolGraph &p = s->pg[g];
    DYG_TRY(dyg::save_range(s->G, p.v0, p.n, p.g.rp, p.g.col, p.g.w, s->st));
    DYG_TRY(dyg::save_range(s->H, p.v0, p.n, p.h.rp, p.h.col, p.h.w, s->st));
    DYG_TRY(dyg::clear_range(s->G, p.v0, p.n, s->st));
    DYG_TRY(dyg::clear_range(s->H, p.v0, p.n, s->st));
    DYG_CUDA(cudaStreamSynchronize(s->st));
    std::lock_guard<std::mutex> lk(s->mu);
    range_free(s, p.v0, p.n);
    p.resident = false;
    s->resident_bytes -= p.footprint;
    p.footprint = footprint_of(p.n, p.g.col.size(), p.h.col.size(), s->G->slack, s->G->headroom);
    ++p.evictions;
    ++s->evictions;
    return DYG_OK;
}

// Loads a graph's host rows into [v0, v0 + n) of both union graphs.
dyg_status admit(dyg_server *s, uint32_t g, uint32_t v0) {
    PoolGraph &p = s->pg[g];
    dyg_status rc = dyg::load_range(s->G, v0, p.n, p.g.rp.data(), p.g.col.data(), p.g.w.data(), s->st);
    if (rc == DYG_OK) {
        rc = dyg::load_range(s->H, v0, p.n, p.h.rp.data(), p.h.col.data(), p.h.w.data(), s->st);
        if (rc != DYG_OK) {
            dyg::clear_range(s->G, v0, p.n, s->st);
            cudaStreamSynchronize(s->st);
        }
    }
    if (rc != DYG_OK) return rc;
    p.g.clear();
    p.h.clear();
    std::lock_guard<std::mutex> lk(s->mu);
    range_take(s, v0, p.n);
    p.v0 = v0;
    p.resident = true;
    s->resident_bytes += p.footprint;
    ++p.admissions;
    ++s->admissions;
    return DYG_OK;
}

// Steps a graph's oldest request waits before busy graphs (ones with requests
// pending) may be evicted for it.  Until then only idle graphs make room, so an
// oversubscribed server rotates graphs as their queues drain instead of
// trading them in and out on every step.
constexpr uint64_t kPatienceSteps = 32;

// Makes room for graph g (evicting in the victim order) and admits it; *ok
// is false when it does not fit yet.  `t_wait` is the arrival of its oldest
// pending request (busy graphs with an older one are never evicted for it,
// busy graphs at all only when allow_busy); `keep` marks graphs that must stay
// (admitted in this step).
dyg_status make_room_and_admit(dyg_server *s, uint32_t g, uint64_t t_wait, bool allow_busy,
                               const std::vector<char> &keep, bool *ok) {
    *ok = false;
    PoolGraph &p = s->pg[g];
    struct Victim {
        uint32_t g;
        bool busy;
        uint64_t head_t, last;
    };
    std::vector<Victim> vs;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t k = 0; k < graph_count(s); ++k) {
            if (!s->pg[k].resident || keep[k]) continue;
            const bool busy = !s->queues[k].empty();
            const uint64_t ht = busy ? s->queues[k].front()->rec.t_submit_ns : ~0ull;
            if (busy && (!allow_busy || ht <= t_wait)) continue;
            vs.push_back(Victim{k, busy, ht, s->pg[k].last_step});
        }
    }
    // idle graphs least recently used first, then busy graphs with the
    // youngest oldest request first
    std::sort(vs.begin(), vs.end(), [](const Victim &a, const Victim &b) {
        if (a.busy != b.busy) return !a.busy;
        if (!a.busy) return a.last < b.last;
        return a.head_t > b.head_t;
    });
    // would evicting every candidate make room?  Otherwise evict nothing.
    uint64_t freeable = 0;
    for (const Victim &v : vs) freeable += s->pg[v.g].footprint;
    if (s->resident_bytes - std::min(s->resident_bytes, freeable) + p.footprint > s->budget) return DYG_OK;
    size_t k = 0;
    uint32_t v0 = 0;
    while (!(s->resident_bytes + p.footprint <= s->budget && range_find(s, p.n, &v0))) {
        if (k == vs.size()) return DYG_OK;
        DYG_TRY(evict(s, vs[k++].g));
    }
    DYG_TRY(admit(s, g, v0));
    *ok = true;
    return DYG_OK;
}

// Pool admission at the start of a step.  Graphs whose admission fails for
// lack of memory, or whose footprint outgrew the budget, go to `failed` with
// the status their pending requests complete with.
dyg_status admit_waiting(dyg_server *s, std::vector<std::pair<uint32_t, dyg_status>> *failed) {
    struct Wait {
        uint64_t t;
        uint32_t g;
        bool patient;   // waited long enough to evict busy graphs
    };
    std::vector<Wait> waiting;
    std::vector<char> keep;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        keep.assign(graph_count(s), 0);
        for (uint32_t g = 0; g < graph_count(s); ++g)
            if (!s->pg[g].resident && !s->queues[g].empty()) {
                const Request *h = s->queues[g].front();
                waiting.push_back(Wait{h->rec.t_submit_ns, g,
                                       s->steps >= h->submit_step + kPatienceSteps});
            }
    }
    std::sort(waiting.begin(), waiting.end(), [](const Wait &a, const Wait &b) {
        return a.t != b.t ? a.t < b.t : a.g < b.g;
    });
    for (const Wait &w : waiting) {
        if (s->pg[w.g].footprint > s->budget) {
            dyg::set_error("graph " + std::to_string(w.g) + " outgrew the HBM budget");
            failed->push_back({w.g, DYG_ENOMEM});
            continue;
        }
        bool ok = false;
        const dyg_status rc = make_room_and_admit(s, w.g, w.t, w.patient, keep, &ok);
        if (rc == DYG_ENOMEM) {
            failed->push_back({w.g, rc});
            continue;
        }
        DYG_TRY(rc);
        if (ok) keep[w.g] = 1;
    }
    return DYG_OK;
}

// ------------------------------------------------------------------- steps

// Stages the step's batches, runs both pipelines and fetches the results
// into the page-locked result buffers; `out` describes them.  `during`
// (host work) runs while the first pipeline's kernels execute, and always
// before the fetch is enqueued.
dyg_status stage_and_run(dyg_server *s, const std::vector<Request *> &heads, uint64_t ni,
                         uint64_t nd, uint64_t *ns, const std::function<void()> &during,
                         StepResults *out) {
    using namespace dyg;
    const uint64_t nt = ni + nd;
    out->heads = heads;
    out->owners.clear();
    out->ni = ni;
    out->nrec = 0;
    if (nt == 0) return DYG_OK;
    uint64_t t = now_ns(s);
    auto lap = [&](int k) {
        const uint64_t u = now_ns(s);
        ns[k] += u - t;
        t = u;
    };
    if (ni > 0xFFFFFFFFull || nd > 0xFFFFFFFFull) {
        set_error("a step holds more than 2^32 - 1 updates of one kind");
        return DYG_EINVAL;
    }
    cudaStream_t st = s->st;
    DYG_TRY(s->h_src.ensure(nt));
    DYG_TRY(s->h_dst.ensure(nt));
    DYG_TRY(s->h_uid.ensure(nt));
    DYG_TRY(s->h_w.ensure(ni ? ni : 1));
    // insertions at [0, ni), deletions at [ni, nt), each in graph order
    uint64_t ki = 0, kd = ni;
    for (Request *r : heads) {
        const uint32_t n = r->rec.n;
        if (!n) continue;
        const uint32_t o = graph_base(s, r->rec.graph);
        const bool ins = r->rec.op == DYG_STREAM_INSERT;
        uint64_t &k = ins ? ki : kd;
        for (uint32_t i = 0; i < n; ++i) {
            s->h_src.p[k + i] = r->src[i] + o;
            s->h_dst.p[k + i] = r->dst[i] + o;
            s->h_uid.p[k + i] = r->rec.first_update_id + i;
        }
        if (ins) memcpy(s->h_w.p + k, r->w.data(), sizeof(float) * n);
        else out->owners.push_back(Owner{o, o + graph_size(s, r->rec.graph), r});
        k += n;
    }
    std::sort(out->owners.begin(), out->owners.end(),
              [](const Owner &a, const Owner &b) { return a.lo < b.lo; });
    DYG_TRY(ensure(s->d_src, sizeof(uint32_t) * nt));
    DYG_TRY(ensure(s->d_dst, sizeof(uint32_t) * nt));
    DYG_TRY(ensure(s->d_uid, sizeof(unsigned long long) * nt));
    DYG_TRY(ensure(s->d_w, sizeof(float) * (ni ? ni : 1)));
    DYG_TRY(ensure(s->d_out, sizeof(int32_t) * nt));
    DYG_TRY(ensure(s->d_cond, sizeof(float) * nt));
    DYG_TRY(ensure(s->d_acc, ni ? ni : 1));
    uint32_t *d_src = ptr<uint32_t>(s->d_src), *d_dst = ptr<uint32_t>(s->d_dst);
    unsigned long long *d_uid = ptr<unsigned long long>(s->d_uid);
    float *d_w = ptr<float>(s->d_w), *d_cond = ptr<float>(s->d_cond);
    int32_t *d_out = ptr<int32_t>(s->d_out);
    uint8_t *d_acc = ptr<uint8_t>(s->d_acc);
    DYG_CUDA(cudaMemcpyAsync(d_src, s->h_src.p, sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(d_dst, s->h_dst.p, sizeof(uint32_t) * nt, cudaMemcpyHostToDevice, st));
    DYG_CUDA(cudaMemcpyAsync(d_uid, s->h_uid.p, sizeof(unsigned long long) * nt,
                             cudaMemcpyHostToDevice, st));
    if (ni) DYG_CUDA(cudaMemcpyAsync(d_w, s->h_w.p, sizeof(float) * ni, cudaMemcpyHostToDevice, st));
    lap(1);
    if (ni) {
        DYG_TRY(incremental_run(s->H, s->G, d_src, d_dst, d_w, (uint32_t)ni, (uint32_t)ni, 0, d_uid,
                                s->ip, d_out, d_cond, d_acc, st, false, &during));
        DYG_TRY(device_errors(s->H, st));
    }
    lap(2);
    uint64_t nrec = 0;
    if (nd) {
        DYG_TRY(decremental_run(s->G, s->H, d_src + ni, d_dst + ni, (uint32_t)nd, (uint32_t)nd, 0,
                                d_uid + ni, s->dp, d_out + ni, d_cond + ni, &nrec, st, false,
                                &during));
        DYG_TRY(device_errors(s->G, st));
    }
    lap(3);
    during();   // (a no-op when a pipeline ran it) before the buffers are refilled
    DYG_TRY(s->h_out.ensure(nt));
    DYG_TRY(s->h_cond.ensure(nt));
    DYG_TRY(s->h_acc.ensure(ni ? ni : 1));
    DYG_CUDA(cudaMemcpyAsync(s->h_out.p, d_out, sizeof(int32_t) * nt, cudaMemcpyDeviceToHost, st));
    DYG_CUDA(cudaMemcpyAsync(s->h_cond.p, d_cond, sizeof(float) * nt, cudaMemcpyDeviceToHost, st));
    if (ni) DYG_CUDA(cudaMemcpyAsync(s->h_acc.p, d_acc, ni, cudaMemcpyDeviceToHost, st));
    if (nrec) {
        Workspace &ws = s->G->ws;
        DYG_TRY(s->h_rx.ensure(nrec));
        DYG_TRY(s->h_ry.ensure(nrec));
        DYG_TRY(s->h_rk.ensure(nrec));
        DYG_CUDA(cudaMemcpyAsync(s->h_rx.p, ws.rx2.p, sizeof(uint32_t) * nrec, cudaMemcpyDeviceToHost, st));
        DYG_CUDA(cudaMemcpyAsync(s->h_ry.p, ws.ry2.p, sizeof(uint32_t) * nrec, cudaMemcpyDeviceToHost, st));
        DYG_CUDA(cudaMemcpyAsync(s->h_rk.p, ws.rk2.p, nrec, cudaMemcpyDeviceToHost, st));
    }
    DYG_CUDA(cudaStreamSynchronize(st));
    out->nrec = nrec;
    lap(4);
    return DYG_OK;
}

// Hands a step's results out of the result buffers to its requests.
dyg_status split_results(dyg_server *s, const StepResults &R) {
    using namespace dyg;
    uint64_t ki = 0, kd = R.ni;
    for (Request *r : R.heads) {
        const uint32_t n = r->rec.n;
        if (!n) continue;
        const bool ins = r->rec.op == DYG_STREAM_INSERT;
        uint64_t &k = ins ? ki : kd;
        r->out_i.assign(s->h_out.p + k, s->h_out.p + k + n);
        r->out_c.assign(s->h_cond.p + k, s->h_cond.p + k + n);
        if (ins) r->out_a.assign(s->h_acc.p + k, s->h_acc.p + k + n);
        k += n;
    }
    const std::vector<Owner> &owners = R.owners;
    const uint64_t nrec = R.nrec;
    // Recovered edges come in walk-list order, i.e. in runs per request: the
    // last owner found is tried first.  One pass counts (and checks), so each
    // request's lists are sized once; the second pass fills them.
    std::vector<uint32_t> own(nrec), cnt(owners.size(), 0u);
    size_t last = owners.size();
    for (uint64_t j = 0; j < nrec; ++j) {
        const uint32_t x = s->h_rx.p[j], y = s->h_ry.p[j];
        if (last == owners.size() || x < owners[last].lo || x >= owners[last].hi) {
            auto it = std::upper_bound(owners.begin(), owners.end(), x,
                                       [](uint32_t v, const Owner &o) { return v < o.lo; });
            last = it == owners.begin() ? owners.size() : (size_t)(it - owners.begin()) - 1;
        }
        if (last == owners.size() || x >= owners[last].hi || y < owners[last].lo ||
            y >= owners[last].hi) {
            set_error("a recovered edge lies outside the graphs deleting in this step");
            return DYG_ESTATE;
        }
        own[j] = (uint32_t)last;
        ++cnt[last];
    }
    for (size_t o = 0; o < owners.size(); ++o) {
        Request *r = owners[o].r;
        r->rx.reserve(r->rx.size() + cnt[o]);
        r->ry.reserve(r->ry.size() + cnt[o]);
        r->rk.reserve(r->rk.size() + cnt[o]);
    }
    for (uint64_t j = 0; j < nrec; ++j) {
        const Owner &o = owners[own[j]];
        o.r->rx.push_back(s->h_rx.p[j] - o.lo);
        o.r->ry.push_back(s->h_ry.p[j] - o.lo);
        o.r->rk.push_back(s->h_rk.p[j]);
    }
    for (Request *r : R.heads) r->rec.n_rec = r->rx.size();
    return DYG_OK;
}

void complete(dyg_server *s, Request *r, dyg_status rc, uint64_t t_start, uint64_t t_done,
              uint64_t step) {
    r->rec.status = (int32_t)rc;
    r->rec.step = step;
    if (!r->rec.t_start_ns) r->rec.t_start_ns = t_start;
    r->rec.t_done_ns = t_done;
    r->finished = true;
    s->done.push_back(r->rec);
}

// Completes the step whose results were left in the result buffers (by the
// thread that holds the step; a no-op when there is none).
void finish_split(dyg_server *s, uint64_t *ns_split) {
    if (!s->split.active) return;
    StepResults R = std::move(s->split);
    s->split = StepResults{};
    const uint64_t t0 = now_ns(s);
    dyg_status rc;
    try {
        rc = split_results(s, R);
    } catch (const std::bad_alloc &) {
        dyg::set_error("host allocation failed while handing out results");
        rc = DYG_ENOMEM;
    }
    const uint64_t t_done = now_ns(s);
    if (ns_split) *ns_split += t_done - t0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Request *r : R.heads) complete(s, r, rc, R.t_start, t_done, R.step);
        if (rc != DYG_OK) s->err = dyg_last_error_string();
    }
    s->cv_idle.notify_all();
}

dyg_status run_step(dyg_server *s, uint32_t *n_done) {
    if (n_done) *n_done = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stepping) {
            dyg::set_error("another step (or an exclusive call) is running");
            return DYG_ESTATE;
        }
        if (s->pending == 0) return DYG_OK;
        s->stepping = true;
    }
    dyg::DevSet ds(s->H->device);
    const uint64_t t_start = now_ns(s);
    std::vector<std::pair<uint32_t, dyg_status>> failed;
    dyg_status arc = DYG_OK;
    std::string amsg;
    uint64_t ns[6] = {};
    if (s->pool) {
        try {
            arc = admit_waiting(s, &failed);
        } catch (const std::bad_alloc &) {
            dyg::set_error("host allocation failed while admitting graphs");
            arc = DYG_ENOMEM;
        }
        if (arc != DYG_OK || !failed.empty()) amsg = dyg_last_error_string();
        ns[0] = now_ns(s) - t_start;
    }
    std::vector<Request *> heads, dead;
    uint64_t ni = 0, nd = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t g = 0; g < graph_count(s); ++g) {
            auto &q = s->queues[g];
            if (q.empty() || (s->pool && !s->pg[g].resident)) continue;
            Request *r = q.front();
            q.pop_front();
            r->rec.first_update_id = s->uid_next[g];
            s->uid_next[g] += r->rec.n;
            r->rec.t_start_ns = t_start;
            if (s->pool) s->pg[g].last_step = s->steps;
            heads.push_back(r);
            if (r->rec.op == DYG_STREAM_INSERT) ni += r->rec.n;
            else nd += r->rec.n;
        }
        for (const auto &f : failed) {
            auto &q = s->queues[f.first];
            while (!q.empty()) {
                q.front()->rec.status = (int32_t)f.second;
                dead.push_back(q.front());
                q.pop_front();
            }
        }
        s->pending -= (uint32_t)(heads.size() + dead.size());
    }
    if (n_done) *n_done = (uint32_t)(heads.size() + dead.size());
    // The previous step's results (if it left them in the result buffers)
    // are handed out while this step's first pipeline runs on the device.
    const std::function<void()> during = [s, &ns] { finish_split(s, &ns[5]); };
    StepResults R;
    dyg_status rc = arc;
    if (rc == DYG_OK) {
        try {
            rc = stage_and_run(s, heads, ni, nd, ns, during, &R);
        } catch (const std::bad_alloc &) {
            dyg::set_error("host allocation failed in a server step");
            rc = DYG_ENOMEM;
        }
    }
    const std::string msg = rc == DYG_OK ? amsg : std::string(dyg_last_error_string());
    finish_split(s, &ns[5]);   // when no pipeline ran it
    uint64_t step;
    bool defer;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        step = s->steps;
        // under the loop thread, with requests still queued, this step's
        // results are handed out during the next step
        defer = rc == DYG_OK && s->loop_on && !s->stop && s->pending > 0 && !heads.empty();
    }
    dyg_status src = DYG_OK;
    if (defer) {
        R.active = true;
        R.t_start = t_start;
        R.step = step;
        s->split = std::move(R);
    } else if (rc == DYG_OK) {
        const uint64_t t0 = now_ns(s);
        try {
            src = split_results(s, R);
        } catch (const std::bad_alloc &) {
            dyg::set_error("host allocation failed while handing out results");
            src = DYG_ENOMEM;
        }
        ns[5] += now_ns(s) - t0;
        if (src != DYG_OK) rc = src;
    }
    const std::string emsg = src != DYG_OK ? std::string(dyg_last_error_string()) : msg;
    const uint64_t t_done = now_ns(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!defer)
            for (Request *r : heads) complete(s, r, rc, t_start, t_done, step);
        for (Request *r : dead) complete(s, r, (dyg_status)r->rec.status, t_start, t_done, step);
        ++s->steps;
        for (int k = 0; k < 6; ++k) s->ns_phase[k] += ns[k];
        s->stepping = false;
        if (!emsg.empty()) s->err = emsg;
    }
    s->cv_idle.notify_all();
    s->cv_work.notify_all();
    return rc;
}

void loop_main(dyg_server *s) {
    dyg::DevSet ds(s->H->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->pending == 0 || s->stepping) {   // stepping: an exclusive call holds the graphs
            s->cv_work.wait(lk);
            continue;
        }
        lk.unlock();
        run_step(s, nullptr);
        lk.lock();
    }
    // A step left for the next one to hand out is handed out now.  Another
    // holder of the step flag can only be a step (requests are queued while
    // results wait, so no exclusive call starts), and a step hands it out
    // itself.
    if (!s->stepping) {
        s->stepping = true;
        lk.unlock();
        finish_split(s, nullptr);
        lk.lock();
        s->stepping = false;
        s->cv_idle.notify_all();
        s->cv_work.notify_all();
    }
}

// The checks of one request (the lock held); "" when it is valid.
std::string check_request(const dyg_server *s, uint32_t graph, uint32_t op, const uint32_t *src,
                          const uint32_t *dst, const float *w, uint64_t n) {
    if (graph >= graph_count(s)) return "graph index out of range";
    if (op != DYG_STREAM_INSERT && op != DYG_STREAM_DELETE) return "unknown op";
    if (n > 0xFFFFFFFFull) return "a request holds more than 2^32 - 1 updates";
    if (n && (!src || !dst || (op == DYG_STREAM_INSERT && !w))) return "NULL array";
    const uint32_t nv = graph_size(s, graph);
    for (uint64_t i = 0; i < n; ++i) {
        if (src[i] >= nv || dst[i] >= nv)
            return "update " + std::to_string(i) + " names a vertex outside graph " +
                   std::to_string(graph) + " (n = " + std::to_string(nv) + ")";
        if (op == DYG_STREAM_INSERT && !(w[i] > 0.0f && isfinite(w[i])))
            return "weight " + std::to_string(i) + " is not finite and > 0";
    }
    return std::string();
}

Request *make_request(const dyg_server *s, uint64_t tag, uint32_t graph, uint32_t op,
                      const uint32_t *src, const uint32_t *dst, const float *w, uint32_t n) {
    Request *r = new Request;
    if (n) {
        r->src.assign(src, src + n);
        r->dst.assign(dst, dst + n);
        if (op == DYG_STREAM_INSERT) r->w.assign(w, w + n);
    }
    r->rec.tag = tag;
    r->rec.graph = graph;
    r->rec.op = op;
    r->rec.n = n;
    r->rec.status = DYG_OK;
    r->rec.t_submit_ns = now_ns(s);
    return r;
}

// Rows of an edge list in the order dyg_graph_create_from_edges gives them:
// for each edge (s, d), row s gets d, then row d gets s.
void rows_from_edges(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                     const float *w, HostRows *out) {
    out->rp.assign((size_t)n + 1, 0);
    for (uint64_t i = 0; i < m; ++i) {
        out->rp[src[i] + 1]++;
        out->rp[dst[i] + 1]++;
    }
    for (uint32_t v = 0; v < n; ++v) out->rp[v + 1] += out->rp[v];
    out->col.resize(out->rp[n]);
    out->w.resize(out->rp[n]);
    std::vector<uint64_t> fill(out->rp.begin(), out->rp.end() - 1);
    for (uint64_t i = 0; i < m; ++i) {
        const uint64_t a = fill[src[i]]++;
        out->col[a] = dst[i];
        out->w[a] = w[i];
        const uint64_t b = fill[dst[i]]++;
        out->col[b] = src[i];
        out->w[b] = w[i];
    }
}

// Exclusive access to the graphs for a call that needs an idle server:
// holds `stepping` so that no step starts meanwhile.
struct Exclusive {
    dyg_server *s;
    bool ok = false;
    explicit Exclusive(dyg_server *sv) : s(sv) {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stepping || s->pending) return;
        s->stepping = true;
        ok = true;
    }
    ~Exclusive() {
        if (!ok) return;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stepping = false;
        }
        s->cv_work.notify_all();
        s->cv_idle.notify_all();
    }
};

dyg_status server_alloc(dyg_graph *G, dyg_graph *H, const dyg_walk_params *ip,
                        const dyg_walk_params *dp, dyg_stream_t stream, dyg_server **out) {
    DYG_TRY(dyg::check_walk_params(ip));
    DYG_TRY(dyg::check_walk_params(dp));
    dyg_server *s = new dyg_server;
    s->G = G;
    s->H = H;
    s->ip = *ip;
    s->dp = *dp;
    s->st = (cudaStream_t)stream;
    s->t0 = std::chrono::steady_clock::now();
    *out = s;
    return DYG_OK;
}

}  // namespace

extern "C" {

dyg_status dyg_server_create(dyg_graph *G, dyg_graph *H, uint32_t n_graphs,
                             const uint32_t *vertex_offsets,
                             const dyg_walk_params *insert_params,
                             const dyg_walk_params *delete_params, dyg_stream_t stream,
                             dyg_server **out) {
    dyg::set_error("");
    if (!out) return fail(nullptr, DYG_EINVAL, "NULL out");
    *out = nullptr;
    if (!G || !H || !vertex_offsets || n_graphs == 0)
        return fail(nullptr, DYG_EINVAL, "NULL graph or offsets, or no graphs");
    if (G->g.n != H->g.n || G->device != H->device)
        return fail(nullptr, DYG_EINVAL, "G and H must have the same vertex count and device");
    for (uint32_t k = 0; k < n_graphs; ++k)
        if (vertex_offsets[k] > vertex_offsets[k + 1])
            return fail(nullptr, DYG_EINVAL, "vertex offsets must ascend");
    if (vertex_offsets[n_graphs] > G->g.n)
        return fail(nullptr, DYG_EINVAL, "vertex offsets exceed the vertex count");
    dyg_server *s = nullptr;
    DYG_TRY(server_alloc(G, H, insert_params, delete_params, stream, &s));
    s->off.assign(vertex_offsets, vertex_offsets + n_graphs + 1);
    s->queues.resize(n_graphs);
    s->uid_next.assign(n_graphs, 0);
    *out = s;
    return DYG_OK;
}

dyg_status dyg_server_create_pool(uint32_t vertex_capacity, uint64_t hbm_budget_bytes,
                                  const dyg_walk_params *insert_params,
                                  const dyg_walk_params *delete_params, int device,
                                  uint32_t keep_initial, dyg_stream_t stream, dyg_server **out) {
    dyg::set_error("");
    if (!out) return fail(nullptr, DYG_EINVAL, "NULL out");
    *out = nullptr;
    if (vertex_capacity == 0 || hbm_budget_bytes == 0)
        return fail(nullptr, DYG_EINVAL, "vertex capacity and budget must be positive");
    DYG_TRY(dyg::check_walk_params(insert_params));
    DYG_TRY(dyg::check_walk_params(delete_params));
    int dev = device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, DYG_ECUDA, "cudaGetDevice failed");
    }
    // arenas start small against the budget and grow on demand
    const uint64_t arena = std::max<uint64_t>(1 << 20, std::min<uint64_t>(hbm_budget_bytes / 12 / 16,
                                                                         0xF0000000ull));
    dyg_graph *G = nullptr, *H = nullptr;
    dyg_status rc = dyg::create_empty_graph(vertex_capacity, arena, dev, 2, 0.5, &G);
    if (rc == DYG_OK) rc = dyg::create_empty_graph(vertex_capacity, arena / 2, dev, 2, 0.5, &H);
    dyg_server *s = nullptr;
    if (rc == DYG_OK) rc = server_alloc(G, H, insert_params, delete_params, stream, &s);
    if (rc != DYG_OK) {
        dyg::destroy_graph(G);
        dyg::destroy_graph(H);
        return rc;
    }
    s->pool = true;
    s->budget = hbm_budget_bytes;
    s->vcap = vertex_capacity;
    s->keep_initial = keep_initial != 0;
    s->free_ranges.push_back({0u, vertex_capacity});
    *out = s;
    return DYG_OK;
}

dyg_status dyg_server_add_graph(dyg_server *s, uint32_t n_vertices, uint64_t g_edges,
                                const uint32_t *g_src, const uint32_t *g_dst, const float *g_w,
                                uint64_t h_edges, const uint32_t *h_src, const uint32_t *h_dst,
                                const float *h_w, uint32_t *graph) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    if (!s->pool) return fail(s, DYG_EINVAL, "graphs are added to pool servers only");
    if (!graph || n_vertices == 0 || (g_edges && (!g_src || !g_dst || !g_w)) ||
        (h_edges && (!h_src || !h_dst || !h_w)))
        return fail(s, DYG_EINVAL, "NULL argument or an empty graph");
    if (n_vertices > s->vcap) return fail(s, DYG_EINVAL, "graph has more vertices than the pool");
    for (uint64_t i = 0; i < g_edges; ++i)
        if (g_src[i] >= n_vertices || g_dst[i] >= n_vertices || !(g_w[i] > 0.0f && isfinite(g_w[i])))
            return fail(s, DYG_EINVAL, "G edge " + std::to_string(i) + " has a bad vertex or weight");
    for (uint64_t i = 0; i < h_edges; ++i)
        if (h_src[i] >= n_vertices || h_dst[i] >= n_vertices || !(h_w[i] > 0.0f && isfinite(h_w[i])))
            return fail(s, DYG_EINVAL, "H edge " + std::to_string(i) + " has a bad vertex or weight");
    const uint64_t fp = footprint_of(n_vertices, 2 * g_edges, 2 * h_edges, s->G->slack, s->G->headroom);
    if (fp > s->budget) return fail(s, DYG_ENOMEM, "the graph's footprint exceeds the HBM budget");
    PoolGraph p;
    try {
        rows_from_edges(n_vertices, g_edges, g_src, g_dst, g_w, &p.g);
        rows_from_edges(n_vertices, h_edges, h_src, h_dst, h_w, &p.h);
        if (s->keep_initial) {
            p.g0 = p.g;
            p.h0 = p.h;
        }
    } catch (const std::bad_alloc &) {
        return fail(s, DYG_ENOMEM, "host allocation failed while copying a graph");
    }
    p.n = n_vertices;
    p.footprint = fp;
    std::lock_guard<std::mutex> lk(s->mu);
    *graph = (uint32_t)s->queues.size();
    s->pg.push_back(std::move(p));
    s->queues.emplace_back();
    s->uid_next.push_back(0);
    return DYG_OK;
}

dyg_status dyg_server_prefetch(dyg_server *s, uint32_t graph, uint32_t *resident) {
    if (resident) *resident = 0;
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    if (!s->pool) return fail(s, DYG_EINVAL, "prefetch is for pool servers");
    Exclusive ex(s);
    if (!ex.ok) return fail(s, DYG_ESTATE, "prefetch needs an idle server");
    if (graph >= graph_count(s)) return fail(s, DYG_EINVAL, "graph index out of range");
    dyg::DevSet ds(s->H->device);
    if (!s->pg[graph].resident) {
        std::vector<char> keep(graph_count(s), 0);
        bool ok = false;
        // nothing is pending: only idle graphs are evicted
        DYG_TRY(make_room_and_admit(s, graph, 0, false, keep, &ok));
    }
    if (resident) *resident = s->pg[graph].resident ? 1u : 0u;
    return DYG_OK;
}

dyg_status dyg_server_stop(dyg_server *s) {
    if (!s) return DYG_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->loop_on) return DYG_OK;
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->loop.join();
    std::lock_guard<std::mutex> lk(s->mu);
    s->loop_on = false;
    s->stop = false;
    return DYG_OK;
}

dyg_status dyg_server_destroy(dyg_server *s) {
    if (!s) return DYG_OK;
    dyg_server_stop(s);
    for (auto &kv : s->by_tag) delete kv.second;   // every request, queued or done
    {
        dyg::DevSet ds(s->H->device);
        for (dyg::Buf *b : {&s->d_src, &s->d_dst, &s->d_w, &s->d_uid, &s->d_out, &s->d_cond, &s->d_acc})
            if (b->p) cudaFree(b->p);
        s->h_src.release();
        s->h_dst.release();
        s->h_rx.release();
        s->h_ry.release();
        s->h_w.release();
        s->h_cond.release();
        s->h_uid.release();
        s->h_out.release();
        s->h_acc.release();
        s->h_rk.release();
    }
    if (s->pool) {
        dyg::destroy_graph(s->G);
        dyg::destroy_graph(s->H);
    }
    delete s;
    return DYG_OK;
}

dyg_status dyg_server_submit_many(dyg_server *s, uint32_t n_req, const uint64_t *tags,
                                  const uint32_t *graphs, const uint32_t *ops,
                                  const uint64_t *offsets, const uint32_t *src,
                                  const uint32_t *dst, const float *w) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    if (n_req && (!tags || !graphs || !ops || !offsets))
        return fail(s, DYG_EINVAL, "NULL request arrays");
    std::vector<Request *> made;
    auto drop = [&made] {
        for (Request *r : made) delete r;
    };
    try {
        made.reserve(n_req);
        for (uint32_t j = 0; j < n_req; ++j) {
            const uint64_t a = offsets[j], b = offsets[j + 1];
            if (b < a) {
                drop();
                return fail(s, DYG_EINVAL, "request offsets must ascend");
            }
            const uint32_t *sj = src ? src + a : nullptr, *dj = dst ? dst + a : nullptr;
            const float *wj = (w && ops[j] == DYG_STREAM_INSERT) ? w + a : nullptr;
            std::string e;
            {
                // graphs only ever get added, and a graph's size never changes
                std::lock_guard<std::mutex> lk(s->mu);
                e = check_request(s, graphs[j], ops[j], sj, dj, wj, b - a);
            }
            if (!e.empty()) {
                drop();
                return fail(s, DYG_EINVAL, "request " + std::to_string(j) + ": " + e);
            }
            made.push_back(make_request(s, tags[j], graphs[j], ops[j], sj, dj, wj, (uint32_t)(b - a)));
        }
    } catch (const std::bad_alloc &) {
        drop();
        return fail(s, DYG_ENOMEM, "host allocation failed while copying requests");
    }
    std::unordered_set<uint64_t> seen;   // tags repeated within this call
    uint32_t rep = n_req;
    try {
        seen.reserve(n_req);
        for (uint32_t j = 0; j < n_req && rep == n_req; ++j)
            if (!seen.insert(tags[j]).second) rep = j;
    } catch (const std::bad_alloc &) {
        drop();
        return fail(s, DYG_ENOMEM, "host allocation failed while checking tags");
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t j = 0; j < n_req; ++j) {
            if (j == rep || s->by_tag.count(tags[j]) != 0) {
                drop();
                s->err = "tag " + std::to_string(tags[j]) + " is held by an unfetched request";
                dyg::set_error(s->err);
                return DYG_EINVAL;
            }
        }
        try {
            s->by_tag.reserve(s->by_tag.size() + n_req);
        } catch (const std::bad_alloc &) {
            drop();
            s->err = "host allocation failed while queueing requests";
            dyg::set_error(s->err);
            return DYG_ENOMEM;
        }
        for (uint32_t j = 0; j < n_req; ++j) {
            made[j]->submit_step = s->steps;
            s->by_tag[tags[j]] = made[j];
            s->queues[graphs[j]].push_back(made[j]);
        }
        s->pending += n_req;
    }
    s->cv_work.notify_one();
    return DYG_OK;
}

dyg_status dyg_server_submit(dyg_server *s, uint64_t tag, uint32_t graph, uint32_t op,
                             const uint32_t *src, const uint32_t *dst, const float *w,
                             uint32_t n) {
    const uint64_t offsets[2] = {0, n};
    return dyg_server_submit_many(s, 1, &tag, &graph, &op, offsets, src, dst, w);
}

dyg_status dyg_server_step(dyg_server *s, uint32_t *n_done) {
    if (n_done) *n_done = 0;
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->loop_on) {
            s->err = "the server's loop thread is running";
            dyg::set_error(s->err);
            return DYG_EINVAL;
        }
    }
    return run_step(s, n_done);
}

dyg_status dyg_server_start(dyg_server *s) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->loop_on) return DYG_OK;
    s->stop = false;
    s->loop_on = true;
    s->loop = std::thread(loop_main, s);
    return DYG_OK;
}

dyg_status dyg_server_drain(dyg_server *s, double timeout_s) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [s] { return s->pending == 0 && !s->stepping; };
    if (idle()) return DYG_OK;
    if (!s->loop_on && s->pending) {
        s->err = "requests are pending and the loop thread is not running";
        dyg::set_error(s->err);
        return DYG_ESTATE;
    }
    if (timeout_s < 0) {
        s->cv_idle.wait(lk, idle);
        return DYG_OK;
    }
    if (!s->cv_idle.wait_for(lk, std::chrono::duration<double>(timeout_s), idle)) {
        dyg::set_error("drain timed out");
        return DYG_ESTATE;
    }
    return DYG_OK;
}

uint32_t dyg_server_pending(dyg_server *s) {
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    return s->pending;
}

dyg_status dyg_server_poll(dyg_server *s, dyg_server_done *out, uint32_t cap, uint32_t *n) {
    if (n) *n = 0;
    if (!s || (cap && !out)) return fail(s, DYG_EINVAL, "NULL server or output");
    std::lock_guard<std::mutex> lk(s->mu);
    uint32_t k = 0;
    while (k < cap && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    if (n) *n = k;
    return DYG_OK;
}

dyg_status dyg_server_fetch(dyg_server *s, uint64_t tag, int32_t *found_or_status,
                            float *conductance, uint8_t *accepted, uint32_t *rec_src,
                            uint32_t *rec_dst, uint8_t *rec_kind, uint64_t rec_cap) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    Request *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->by_tag.find(tag);
        if (it == s->by_tag.end() || !it->second->finished) {
            s->err = "tag " + std::to_string(tag) + " is not a completed request";
            dyg::set_error(s->err);
            return DYG_EINVAL;
        }
        r = it->second;
        if ((rec_src || rec_dst || rec_kind) && r->rx.size() > rec_cap) {
            s->err = "more recovered edges than rec_cap";
            dyg::set_error(s->err);
            return DYG_ERANGE;
        }
        s->by_tag.erase(it);
    }
    if (found_or_status) std::copy(r->out_i.begin(), r->out_i.end(), found_or_status);
    if (conductance) std::copy(r->out_c.begin(), r->out_c.end(), conductance);
    if (accepted) std::copy(r->out_a.begin(), r->out_a.end(), accepted);
    if (rec_src) std::copy(r->rx.begin(), r->rx.end(), rec_src);
    if (rec_dst) std::copy(r->ry.begin(), r->ry.end(), rec_dst);
    if (rec_kind) std::copy(r->rk.begin(), r->rk.end(), rec_kind);
    delete r;
    return DYG_OK;
}

dyg_status dyg_server_reset(dyg_server *s) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    Exclusive ex(s);
    if (!ex.ok) return fail(s, DYG_ESTATE, "reset needs an idle server");
    if (s->pool) {
        if (!s->keep_initial)
            return fail(s, DYG_EINVAL, "a pool server resets only when it keeps the registered graphs");
        dyg::DevSet ds(s->H->device);
        for (uint32_t g = 0; g < graph_count(s); ++g) {
            PoolGraph &p = s->pg[g];
            if (p.resident) {
                DYG_TRY(dyg::clear_range(s->G, p.v0, p.n, s->st));
                DYG_TRY(dyg::clear_range(s->H, p.v0, p.n, s->st));
            }
            try {
                p.g = p.g0;
                p.h = p.h0;
            } catch (const std::bad_alloc &) {
                return fail(s, DYG_ENOMEM, "host allocation failed while restoring graphs");
            }
        }
        // no graph holds a row any more: the arenas start over at 0, keeping
        // the capacity they grew to (a replay after a reset then needs no
        // growth that the one before it did not need)
        const unsigned long long zero = 0ull;
        DYG_CUDA(cudaMemcpyAsync(s->G->g.top, &zero, sizeof(zero), cudaMemcpyHostToDevice, s->st));
        DYG_CUDA(cudaMemcpyAsync(s->H->g.top, &zero, sizeof(zero), cudaMemcpyHostToDevice, s->st));
        DYG_CUDA(cudaStreamSynchronize(s->st));
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t g = 0; g < graph_count(s); ++g) {
            PoolGraph &p = s->pg[g];
            p.resident = false;
            p.footprint = footprint_of(p.n, p.g.col.size(), p.h.col.size(), s->G->slack,
                                       s->G->headroom);
            p.last_step = 0;
        }
        s->free_ranges.assign(1, {0u, s->vcap});
        s->resident_bytes = 0;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto &kv : s->by_tag) delete kv.second;
    s->by_tag.clear();
    s->done.clear();
    std::fill(s->uid_next.begin(), s->uid_next.end(), 0ull);
    s->steps = 0;
    std::fill(std::begin(s->ns_phase), std::end(s->ns_phase), 0ull);
    return DYG_OK;
}

dyg_status dyg_server_stats_read(dyg_server *s, dyg_server_stats *out) {
    if (!s || !out) return fail(s, DYG_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    dyg_server_stats r{};
    r.graphs = graph_count(s);
    for (uint32_t g = 0; g < r.graphs; ++g) {
        const bool res = !s->pool || s->pg[g].resident;
        r.resident += res ? 1u : 0u;
        r.waiting += (!res && !s->queues[g].empty()) ? 1u : 0u;
    }
    r.resident_bytes = s->pool ? s->resident_bytes : 0;
    r.budget_bytes = s->pool ? s->budget : 0;
    r.admissions = s->admissions;
    r.evictions = s->evictions;
    r.steps = s->steps;
    r.pending = s->pending;
    r.ns_admit = s->ns_phase[0];
    r.ns_stage = s->ns_phase[1];
    r.ns_insert = s->ns_phase[2];
    r.ns_delete = s->ns_phase[3];
    r.ns_fetch = s->ns_phase[4];
    r.ns_split = s->ns_phase[5];
    *out = r;
    return DYG_OK;
}

dyg_status dyg_server_graph_info_read(dyg_server *s, uint32_t graph, dyg_server_graph_info *out) {
    if (!s || !out) return fail(s, DYG_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (graph >= graph_count(s)) {
        s->err = "graph index out of range";
        dyg::set_error(s->err);
        return DYG_EINVAL;
    }
    dyg_server_graph_info r{};
    r.n_vertices = graph_size(s, graph);
    r.resident = (!s->pool || s->pg[graph].resident) ? 1u : 0u;
    r.vertex_offset = r.resident ? graph_base(s, graph) : 0u;
    r.footprint_bytes = s->pool ? s->pg[graph].footprint : 0;
    r.updates = s->uid_next[graph];
    r.admissions = s->pool ? s->pg[graph].admissions : 0;
    r.evictions = s->pool ? s->pg[graph].evictions : 0;
    r.pending = s->queues[graph].size();
    *out = r;
    return DYG_OK;
}

dyg_status dyg_server_graph_export(dyg_server *s, uint32_t graph, uint32_t which,
                                   uint64_t *row_ptr, uint32_t *col, float *w, uint64_t slot_cap) {
    if (!s || !row_ptr) return fail(s, DYG_EINVAL, "NULL argument");
    if (which > 1) return fail(s, DYG_EINVAL, "which: 0 = G, 1 = H");
    Exclusive ex(s);
    if (!ex.ok) return fail(s, DYG_ESTATE, "export needs an idle server");
    if (graph >= graph_count(s)) return fail(s, DYG_EINVAL, "graph index out of range");
    HostRows tmp;
    const HostRows *rows = &tmp;
    if (!s->pool || s->pg[graph].resident) {
        dyg::DevSet ds(s->H->device);
        try {
            DYG_TRY(dyg::save_range(which ? s->H : s->G, graph_base(s, graph), graph_size(s, graph),
                                    tmp.rp, tmp.col, tmp.w, s->st));
        } catch (const std::bad_alloc &) {
            return fail(s, DYG_ENOMEM, "host allocation failed while exporting");
        }
    } else {
        rows = which ? &s->pg[graph].h : &s->pg[graph].g;
    }
    const uint32_t n = graph_size(s, graph);
    std::copy(rows->rp.begin(), rows->rp.begin() + n + 1, row_ptr);
    const uint64_t m = rows->rp[n];
    const uint64_t k = std::min(m, slot_cap);
    if (col) std::copy(rows->col.begin(), rows->col.begin() + (long)k, col);
    if (w) std::copy(rows->w.begin(), rows->w.begin() + (long)k, w);
    if (m > slot_cap && (col || w)) return fail(s, DYG_ERANGE, "slot_cap smaller than the graph's slots");
    return DYG_OK;
}

dyg_status dyg_server_counters(dyg_server *s, uint64_t *incr_moves, uint64_t *decr_moves) {
    if (!s) return fail(nullptr, DYG_EINVAL, "NULL server");
    Exclusive ex(s);
    if (!ex.ok) return fail(s, DYG_ESTATE, "counters need an idle server");
    dyg::DevSet ds(s->H->device);
    DYG_TRY(dyg::read_scalars(s->H, s->st));
    DYG_TRY(dyg::read_scalars(s->G, s->st));
    if (incr_moves) *incr_moves = s->H->ws.host_scalars[dyg::S_MOVES];
    if (decr_moves) *decr_moves = s->G->ws.host_scalars[dyg::S_MOVES];
    return DYG_OK;
}

uint64_t dyg_server_steps(const dyg_server *s) {
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(const_cast<dyg_server *>(s)->mu);
    return s->steps;
}

uint64_t dyg_server_now_ns(const dyg_server *s) { return s ? now_ns(s) : 0; }

const char *dyg_server_last_error(dyg_server *s) {
    static thread_local std::string copy;
    if (!s) return "";
    std::lock_guard<std::mutex> lk(s->mu);
    copy = s->err;
    return copy.c_str();
}

}  // extern "C"
