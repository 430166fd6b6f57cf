// server.cu -- the continuous-batching server of include/dyg_serve.h.
//
// The reference runs one graph per process and one batch loop per run
// (random_walk_incremental/main.cu:314-340, random_walk_decremental/
// main.cu:395-444); it has no request loop.  Here many graphs stay resident
// in one union graph and requests for them are scheduled in steps.  A step
// takes the oldest pending request of every graph that has one, gathers the
// insertion requests into one batch and the deletion requests into another
// (global vertex ids = local id + the graph's offset; per-edge update ids =
// the graph's own update counter), stages both through page-locked memory,
// runs the incremental pipeline and then the decremental pipeline on the
// device (one host synchronize each, for the halt/resume protocol), and
// splits the results back per request: per-edge arrays by position,
// recovered edges by the graph whose vertex range holds them (each step runs
// at most one deletion request per graph, and a recovered edge joins two
// vertices of the graph it was recovered in).
//
// Graphs are disjoint in the union, every walk stays inside its own graph, and
// a graph's update ids do not depend on the other graphs, so each request's
// result equals the one it gets alone on its graph's own handles.
#include <math.h>
#include <string.h>

#include <algorithm>
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
    bool finished = false;
    dyg_server_done rec{};
    std::vector<int32_t> out_i;       // found_at (insertion) or status (deletion)
    std::vector<float> out_c;         // conductance
    std::vector<uint8_t> out_a;       // accepted (insertion)
    std::vector<uint32_t> rx, ry;     // recovered edges, local ids (deletion)
    std::vector<uint8_t> rk;
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

}  // namespace
}  // namespace dyg

struct dyg_server {
    dyg_graph *G = nullptr, *H = nullptr;
    std::vector<uint32_t> off;            // n_graphs + 1 vertex offsets
    dyg_walk_params ip{}, dp{};
    cudaStream_t st = nullptr;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;                        // guards everything below up to `loop`
    std::condition_variable cv_work, cv_idle;
    std::vector<std::deque<dyg::Request *>> queues;
    std::unordered_map<uint64_t, dyg::Request *> by_tag;   // submitted, not fetched
    std::deque<dyg_server_done> done;
    uint32_t pending = 0;
    bool stepping = false, loop_on = false, stop = false;
    uint64_t steps = 0;
    std::string err;
    std::thread loop;

    // owned by the thread that runs the step
    std::vector<uint64_t> uid_next;
    std::vector<dyg::Request *> owner;
    dyg::Pinned<uint32_t> h_src, h_dst, h_rx, h_ry;
    dyg::Pinned<float> h_w, h_cond;
    dyg::Pinned<unsigned long long> h_uid;
    dyg::Pinned<int32_t> h_out;
    dyg::Pinned<uint8_t> h_acc, h_rk;
    dyg::Buf d_src, d_dst, d_w, d_uid, d_out, d_cond, d_acc;
};

namespace {

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

using dyg::Request;

// Stages the step's batches, runs both pipelines and splits the results.
dyg_status stage_and_run(dyg_server *s, const std::vector<Request *> &heads, uint64_t ni,
                         uint64_t nd) {
    using namespace dyg;
    const uint64_t nt = ni + nd;
    if (nt == 0) return DYG_OK;
    if (ni > 0xFFFFFFFFull || nd > 0xFFFFFFFFull) {
        set_error("a step holds more than 2^32 - 1 updates of one kind");
        return DYG_EINVAL;
    }
    DevSet ds(s->H->device);
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
        const uint32_t o = s->off[r->rec.graph];
        const bool ins = r->rec.op == DYG_STREAM_INSERT;
        uint64_t &k = ins ? ki : kd;
        for (uint32_t i = 0; i < n; ++i) {
            s->h_src.p[k + i] = r->src[i] + o;
            s->h_dst.p[k + i] = r->dst[i] + o;
            s->h_uid.p[k + i] = r->rec.first_update_id + i;
        }
        if (ins) memcpy(s->h_w.p + k, r->w.data(), sizeof(float) * n);
        k += n;
    }
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
    if (ni) {
        DYG_TRY(incremental_run(s->H, s->G, d_src, d_dst, d_w, (uint32_t)ni, (uint32_t)ni, 0, d_uid,
                                s->ip, d_out, d_cond, d_acc, st));
        DYG_TRY(device_errors(s->H, st));
    }
    uint64_t nrec = 0;
    if (nd) {
        DYG_TRY(decremental_run(s->G, s->H, d_src + ni, d_dst + ni, (uint32_t)nd, (uint32_t)nd, 0,
                                d_uid + ni, s->dp, d_out + ni, d_cond + ni, &nrec, st));
        DYG_TRY(device_errors(s->G, st));
    }
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
    std::fill(s->owner.begin(), s->owner.end(), nullptr);
    ki = 0;
    kd = ni;
    for (Request *r : heads) {
        const uint32_t n = r->rec.n;
        if (!n) continue;
        const bool ins = r->rec.op == DYG_STREAM_INSERT;
        uint64_t &k = ins ? ki : kd;
        r->out_i.assign(s->h_out.p + k, s->h_out.p + k + n);
        r->out_c.assign(s->h_cond.p + k, s->h_cond.p + k + n);
        if (ins) r->out_a.assign(s->h_acc.p + k, s->h_acc.p + k + n);
        else s->owner[r->rec.graph] = r;
        k += n;
    }
    for (uint64_t j = 0; j < nrec; ++j) {
        const uint32_t x = s->h_rx.p[j], y = s->h_ry.p[j];
        const size_t g = (size_t)(std::upper_bound(s->off.begin(), s->off.end(), x) - s->off.begin()) - 1;
        Request *r = g < s->owner.size() ? s->owner[g] : nullptr;
        if (!r || y < s->off[g] || y >= s->off[g + 1]) {
            set_error("a recovered edge lies outside the graphs deleting in this step");
            return DYG_ESTATE;
        }
        r->rx.push_back(x - s->off[g]);
        r->ry.push_back(y - s->off[g]);
        r->rk.push_back(s->h_rk.p[j]);
    }
    for (Request *r : heads) r->rec.n_rec = r->rx.size();
    return DYG_OK;
}

dyg_status run_step(dyg_server *s, uint32_t *n_done) {
    std::vector<Request *> heads;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stepping) {
            dyg::set_error("another step is running");
            return DYG_ESTATE;
        }
        for (auto &q : s->queues)
            if (!q.empty()) {
                heads.push_back(q.front());
                q.pop_front();
            }
        s->pending -= (uint32_t)heads.size();
        if (!heads.empty()) s->stepping = true;
    }
    if (n_done) *n_done = (uint32_t)heads.size();
    if (heads.empty()) return DYG_OK;
    const uint64_t t_start = now_ns(s);
    uint64_t ni = 0, nd = 0;
    for (Request *r : heads) {
        r->rec.first_update_id = s->uid_next[r->rec.graph];
        s->uid_next[r->rec.graph] += r->rec.n;
        r->rec.t_start_ns = t_start;
        if (r->rec.op == DYG_STREAM_INSERT) ni += r->rec.n;
        else nd += r->rec.n;
    }
    dyg_status rc;
    try {
        rc = stage_and_run(s, heads, ni, nd);
    } catch (const std::bad_alloc &) {
        dyg::set_error("host allocation failed in a server step");
        rc = DYG_ENOMEM;
    }
    const std::string msg = rc == DYG_OK ? std::string() : std::string(dyg_last_error_string());
    const uint64_t t_done = now_ns(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Request *r : heads) {
            r->rec.status = (int32_t)rc;
            r->rec.step = s->steps;
            r->rec.t_done_ns = t_done;
            r->finished = true;
            s->done.push_back(r->rec);
        }
        ++s->steps;
        s->stepping = false;
        if (rc != DYG_OK) s->err = msg;
    }
    s->cv_idle.notify_all();
    return rc;
}

void loop_main(dyg_server *s) {
    dyg::DevSet ds(s->H->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->pending == 0) {
            s->cv_work.wait(lk);
            continue;
        }
        lk.unlock();
        run_step(s, nullptr);
        lk.lock();
    }
}

// The checks of one request (no lock held); "" when it is valid.
std::string check_request(const dyg_server *s, uint32_t graph, uint32_t op, const uint32_t *src,
                          const uint32_t *dst, const float *w, uint64_t n) {
    if (graph >= s->queues.size()) return "graph index out of range";
    if (op != DYG_STREAM_INSERT && op != DYG_STREAM_DELETE) return "unknown op";
    if (n > 0xFFFFFFFFull) return "a request holds more than 2^32 - 1 updates";
    if (n && (!src || !dst || (op == DYG_STREAM_INSERT && !w))) return "NULL array";
    const uint32_t nv = s->off[graph + 1] - s->off[graph];
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
    DYG_TRY(dyg::check_walk_params(insert_params));
    DYG_TRY(dyg::check_walk_params(delete_params));
    dyg_server *s = new dyg_server;
    s->G = G;
    s->H = H;
    s->off.assign(vertex_offsets, vertex_offsets + n_graphs + 1);
    s->ip = *insert_params;
    s->dp = *delete_params;
    s->st = (cudaStream_t)stream;
    s->t0 = std::chrono::steady_clock::now();
    s->queues.resize(n_graphs);
    s->uid_next.assign(n_graphs, 0);
    s->owner.assign(n_graphs, nullptr);
    *out = s;
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
    for (auto &kv : s->by_tag) delete kv.second;
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
            const std::string e = check_request(s, graphs[j], ops[j], sj, dj, wj, b - a);
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
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->pending || s->stepping) {
        s->err = "reset needs an idle server";
        dyg::set_error(s->err);
        return DYG_ESTATE;
    }
    for (auto &kv : s->by_tag) delete kv.second;
    s->by_tag.clear();
    s->done.clear();
    std::fill(s->uid_next.begin(), s->uid_next.end(), 0ull);
    s->steps = 0;
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
