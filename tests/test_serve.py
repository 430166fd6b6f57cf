"""Continuous-batching server (include/dyg_serve.h, dygrass_b200/serve.py):
every request gets the result it gets alone on its graph's own handles, in
the native scheduler (stepped or in its loop thread) and in the Python one,
admission respects the HBM budget, and the C ABI reports misuse."""
import dataclasses

import numpy as np
import pytest

from dygrass_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dyg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import dygrass_b200
    dygrass_b200.lib()
    return dygrass_b200


def mixed_cases():
    cases, _ = W.rgg_many(k=4, n_lo=300, n_hi=3000, seed=21)
    cases += [W.mesh_3d(6, inserts=150, seed=22), W.grid_2d(20, 20, inserts=120, seed=23)]
    return cases


def same_request(a, b):
    assert a.first_update_id == b.first_update_id
    if a.op == 0:
        assert np.array_equal(a.found_at, b.found_at)
        assert np.array_equal(a.conductance.view(np.uint32), b.conductance.view(np.uint32))
        assert np.array_equal(a.accepted, b.accepted)
    else:
        assert np.array_equal(a.status, b.status)
        assert a.recovered == b.recovered


def rows_of(server, which, k):
    rp, col, w = (server.H if which == "H" else server.G).export()
    lo, hi = int(server.offsets[k]), int(server.offsets[k + 1])
    a, b = int(rp[lo]), int(rp[hi])
    return rp[lo:hi + 1] - rp[lo], col[a:b] - lo, w[a:b]


@pytest.mark.parametrize("native", [True, False])
def test_mixed_requests_match_alone(dyg, native):
    import torch
    from dygrass_b200.serve import PlainServer, Server, poisson_requests
    cases = mixed_cases()
    p = dyg.WalkParams.make(threshold=100.0, walkers=128)
    reqs = poisson_requests(cases, rate=1e7, count=80, seed=3, size_hi=200)
    alone = [dataclasses.replace(r) for r in reqs]
    S = Server(cases, p, p, native=native)
    done = S.serve(reqs, sync=torch.cuda.synchronize)
    assert len(done) == len(reqs) and S.steps < len(reqs)   # requests were batched
    P = PlainServer(cases, p, p)
    P.serve(alone)
    for a, b in zip(reqs, alone):
        same_request(a, b)
    for k in range(len(cases)):
        for which, mine in (("H", P.H[k]), ("G", P.G[k])):
            want = mine.export()
            got = rows_of(S, which, k)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
            assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32))
    assert any(r.op == 1 and r.recovered for r in reqs)
    S.close()
    P.close()


def test_admission_by_footprint(dyg):
    from dygrass_b200.serve import Server, footprint_bytes, poisson_requests
    cases = mixed_cases()
    fps = [footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in cases]
    budget = sum(fps[:3]) + fps[3] // 2
    p = dyg.WalkParams.make(walkers=64)
    S = Server(cases, p, p, hbm_budget=budget)
    want, used = [], 0
    for i, f in enumerate(fps):       # greedy in the given order
        if used + f <= budget:
            want.append(i)
            used += f
    assert S.admitted == want and 3 not in want
    assert S.footprint <= budget
    reqs = poisson_requests(cases, rate=1e7, count=30, seed=4, size_hi=50)
    done = S.serve(reqs)
    refused = [r for r in reqs if r.done < 0]
    assert refused and all(r.graph not in S.admitted for r in refused)
    assert all(r.graph in S.admitted for r in done)
    S.close()


def test_native_loop_with_arrivals_matches_alone(dyg):
    """Requests arriving while steps run (the loop thread) still get their
    results alone; latencies are measured on the server clock."""
    from dygrass_b200.serve import PlainServer, Server, poisson_requests
    cases = mixed_cases()
    p = dyg.WalkParams.make(threshold=100.0, walkers=64)
    reqs = poisson_requests(cases, rate=4000.0, count=60, seed=5, size_hi=100)
    alone = [dataclasses.replace(r) for r in reqs]
    S = Server(cases, p, p)
    S.snapshot()
    done = S.serve(reqs)
    assert len(done) == len(reqs)
    assert all(r.done >= r.arrival - 1e-3 for r in reqs)
    P = PlainServer(cases, p, p)
    P.serve(alone)
    for a, b in zip(reqs, alone):
        same_request(a, b)
    # the same replay again after restore: identical results
    again = [dataclasses.replace(r, found_at=None, status=None, rec_src=None) for r in reqs]
    S.restore()
    S.serve(again)
    for a, b in zip(again, alone):
        same_request(a, b)
    S.close()
    P.close()


def test_native_server_errors(dyg):
    import ctypes as C
    from dygrass_b200.serve import Server
    cases = mixed_cases()[:2]
    p = dyg.WalkParams.make(walkers=32)
    S = Server(cases, p, p)
    L, h = dyg.lib(), S._srv
    n0 = cases[0].n
    src = np.array([0, n0], np.uint32)          # n0 is outside graph 0
    dst = np.array([1, 2], np.uint32)
    w = np.ones(2, np.float32)
    assert L.dyg_server_submit(h, 1, 0, 0, dyg._ptr(src), dyg._ptr(dst), dyg._ptr(w), 2) == dyg.DYG_EINVAL
    assert b"outside graph 0" in L.dyg_server_last_error(h)
    assert L.dyg_server_submit(h, 1, 7, 0, dyg._ptr(src), dyg._ptr(dst), dyg._ptr(w), 1) == dyg.DYG_EINVAL
    bad_w = np.array([0.0], np.float32)
    assert L.dyg_server_submit(h, 1, 0, 0, dyg._ptr(src), dyg._ptr(dst), dyg._ptr(bad_w), 1) == dyg.DYG_EINVAL
    assert L.dyg_server_pending(h) == 0
    # a good deletion request; its tag cannot be reused until fetched
    c = cases[0]
    ds, dd = np.ascontiguousarray(c.g_src[:5], np.uint32), np.ascontiguousarray(c.g_dst[:5], np.uint32)
    assert L.dyg_server_submit(h, 9, 0, 1, dyg._ptr(ds), dyg._ptr(dd), None, 5) == 0
    assert L.dyg_server_submit(h, 9, 1, 1, dyg._ptr(ds), dyg._ptr(dd), None, 0) == dyg.DYG_EINVAL
    assert L.dyg_server_fetch(h, 9, None, None, None, None, None, None, 0) == dyg.DYG_EINVAL  # not run yet
    assert L.dyg_server_reset(h) == dyg.DYG_ESTATE            # not idle
    assert L.dyg_server_drain(h, 0.0) == dyg.DYG_ESTATE       # pending, no loop
    k = C.c_uint32()
    assert L.dyg_server_step(h, C.byref(k)) == 0 and k.value == 1
    buf = (dyg.ServerDone * 4)()
    assert L.dyg_server_poll(h, buf, 4, C.byref(k)) == 0 and k.value == 1
    d = buf[0]
    assert (d.tag, d.graph, d.op, d.n, d.status, d.first_update_id) == (9, 0, 1, 5, 0, 0)
    st = np.empty(5, np.int32)
    if d.n_rec:
        rx = np.empty(d.n_rec, np.uint32)
        assert L.dyg_server_fetch(h, 9, dyg._ptr(st), None, None, dyg._ptr(rx), None, None,
                                  d.n_rec - 1) == dyg.DYG_ERANGE   # kept
    assert L.dyg_server_fetch(h, 9, dyg._ptr(st), None, None, None, None, None, 0) == 0
    assert L.dyg_server_fetch(h, 9, None, None, None, None, None, None, 0) == dyg.DYG_EINVAL  # released
    assert L.dyg_server_step(h, C.byref(k)) == 0 and k.value == 0
    # bulk submission is all or nothing: a bad request or a repeated tag queues none
    tags = np.array([20, 21], np.uint64)
    graphs = np.array([0, 1], np.uint32)
    ops = np.array([1, 1], np.uint32)
    offs = np.array([0, 2, 4], np.uint64)
    bs = np.array([0, 1, 0, cases[1].n], np.uint32)
    bd = np.array([1, 2, 1, 0], np.uint32)
    args = lambda t, sr: (h, 2, dyg._ptr(t), dyg._ptr(graphs), dyg._ptr(ops), dyg._ptr(offs),
                          dyg._ptr(sr), dyg._ptr(bd), None)
    assert L.dyg_server_submit_many(*args(tags, bs)) == dyg.DYG_EINVAL
    assert b"request 1" in L.dyg_server_last_error(h) and L.dyg_server_pending(h) == 0
    bs[3] = 1
    assert L.dyg_server_submit_many(*args(np.array([20, 20], np.uint64), bs)) == dyg.DYG_EINVAL
    assert L.dyg_server_pending(h) == 0
    assert L.dyg_server_submit_many(*args(tags, bs)) == 0 and L.dyg_server_pending(h) == 2
    assert L.dyg_server_step(h, C.byref(k)) == 0 and k.value == 2      # one per graph, one step
    assert L.dyg_server_poll(h, buf, 4, C.byref(k)) == 0 and k.value == 2
    assert sorted((buf[i].tag, buf[i].graph, buf[i].first_update_id) for i in range(2)) == \
        [(20, 0, 5), (21, 1, 0)]
    for t in (20, 21):
        assert L.dyg_server_fetch(h, t, None, None, None, None, None, None, 0) == 0
    assert L.dyg_server_reset(h) == 0 and L.dyg_server_steps(h) == 0
    S.close()


def check_pool_against_plain(S, P, reqs, alone, n_graphs):
    for a, b in zip(reqs, alone):
        same_request(a, b)
    for k in range(n_graphs):
        for which, mine in (("H", P.H[k]), ("G", P.G[k])):
            want = mine.export()
            got = S.export(k, which)
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
            assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32))


@pytest.mark.parametrize("frac", [1.0, 0.4])
def test_pool_admission_matches_alone(dyg, frac):
    """Pool mode: graphs enter the device as their requests are scheduled.
    With a budget for all graphs each is admitted once; with 40 % of it
    graphs are evicted to host memory and admitted again as requests arrive
    (the loop thread, requests arriving meanwhile).  Every request still gets
    its result alone, and every graph ends with the rows of its own handles."""
    from dygrass_b200.serve import PlainServer, PoolServer, footprint_bytes, poisson_requests
    cases = mixed_cases()
    fps = [footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in cases]
    budget = int(max(frac * sum(fps), max(fps)) * 1.3)
    p = dyg.WalkParams.make(threshold=100.0, walkers=64)
    reqs = poisson_requests(cases, rate=3000.0, count=90, seed=6, size_hi=150)
    alone = [dataclasses.replace(r) for r in reqs]
    S = PoolServer(cases, p, p, hbm_budget=budget)
    st0 = S.stats()
    assert st0["graphs"] == len(cases) and st0["resident"] == 0
    done = S.serve(reqs)
    assert len(done) == len(reqs)
    st = S.stats()
    assert st["resident_bytes"] <= budget and st["pending"] == 0
    if frac < 1.0:
        assert st["evictions"] > 0 and st["admissions"] > len(cases)
    else:
        assert st["evictions"] == 0
    P = PlainServer(cases, p, p)
    P.serve(alone)
    check_pool_against_plain(S, P, reqs, alone, len(cases))
    infos = [S.graph_info(k) for k in range(len(cases))]
    assert [i["updates"] for i in infos] == [P.uid_next[k] for k in range(len(cases))]
    # the same replay after a reset: every graph back to its registered rows
    again = [dataclasses.replace(r, found_at=None, status=None, rec_src=None) for r in reqs]
    S.restore()
    assert S.stats()["resident"] == 0
    S.serve(again)
    for a, b in zip(again, alone):
        same_request(a, b)
    S.close()
    P.close()


def test_pool_stepwise_eviction_and_prefetch(dyg):
    """Stepping by hand with room for one graph at a time: a waiting graph
    evicts idle graphs only (a busy one only after it has waited 32 steps), so
    the resident graph runs its queue dry before the oldest waiting graph
    comes in; a prefetch evicts idle graphs only, and exports read evicted
    graphs from their host copies."""
    import ctypes as C
    from dygrass_b200.serve import PlainServer, PoolServer, Request, footprint_bytes
    cases = [W.grid_2d(20, 20, inserts=60, seed=s) for s in (31, 32, 33)]
    fps = [footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in cases]
    budget = int(max(fps) * 1.5)          # never two of these at once
    assert budget < 2 * min(fps)
    p = dyg.WalkParams.make(walkers=32)
    S = PoolServer(cases, p, p, hbm_budget=budget)
    P = PlainServer(cases, p, p)
    L, h = dyg.lib(), S._srv
    assert S.prefetch(0) and S.graph_info(0)["resident"] == 1
    assert S.prefetch(1) and S.graph_info(0)["resident"] == 0      # idle graph 0 evicted
    reqs = []
    for g in (2, 0, 1, 2):
        c = cases[g]
        k = len(reqs)
        reqs.append(Request(g, 0, c.ins_src[k * 5:k * 5 + 5], c.ins_dst[k * 5:k * 5 + 5],
                            c.ins_w[k * 5:k * 5 + 5]))
    alone = [dataclasses.replace(r) for r in reqs]
    S.submit_many(reqs)
    order = []
    k = C.c_uint32()
    while L.dyg_server_pending(h):
        assert L.dyg_server_step(h, C.byref(k)) == 0 and k.value == 1
        order.append([i for i in range(3) if S.graph_info(i)["resident"]])
    # graph 1 (resident, busy) first; then the oldest waiting graph (2) twice,
    # since it stays while its queue lasts; then graph 0
    assert order == [[1], [2], [2], [0]]
    done = S._collect()
    assert len(done) == 4
    for r in alone:
        P.run_one(r)
    check_pool_against_plain(S, P, reqs, alone, 3)
    S.close()
    P.close()


def test_pool_errors(dyg):
    import ctypes as C
    from dygrass_b200.serve import footprint_bytes
    c = mixed_cases()[0]
    p = dyg.WalkParams.make(walkers=32)
    L = dyg.lib()
    h = C.c_void_p()
    fp = footprint_bytes(c.n, len(c.g_src), len(c.h_src))
    assert L.dyg_server_create_pool(0, 1 << 20, C.byref(p), C.byref(p), -1, 0, None, C.byref(h)) == \
        dyg.DYG_EINVAL
    assert L.dyg_server_create_pool(c.n, fp // 2, C.byref(p), C.byref(p), -1, 0, None, C.byref(h)) == 0
    g = C.c_uint32()
    a = lambda x, t: np.ascontiguousarray(x, t)
    gs, gd, gw = a(c.g_src, np.uint32), a(c.g_dst, np.uint32), a(c.g_w, np.float32)
    hs, hd, hw = a(c.h_src, np.uint32), a(c.h_dst, np.uint32), a(c.h_w, np.float32)
    args = lambda n: (h, n, len(gs), dyg._ptr(gs), dyg._ptr(gd), dyg._ptr(gw), len(hs), dyg._ptr(hs),
                      dyg._ptr(hd), dyg._ptr(hw), C.byref(g))
    assert L.dyg_server_add_graph(*args(c.n)) == dyg.DYG_ENOMEM          # over the budget
    assert b"budget" in L.dyg_server_last_error(h)
    assert L.dyg_server_add_graph(*args(c.n - 1)) == dyg.DYG_EINVAL      # an id >= n
    assert L.dyg_server_reset(h) == dyg.DYG_EINVAL                       # registered rows not kept
    st = dyg.ServerStats()
    assert L.dyg_server_stats_read(h, C.byref(st)) == 0 and st.graphs == 0 and st.budget_bytes == fp // 2
    assert L.dyg_server_destroy(h) == 0
