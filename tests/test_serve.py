"""Continuous-batching server (dygrass_b200/serve.py): every request gets the
result it gets alone on its graph's own handles, and admission respects the
HBM budget."""
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


def test_mixed_requests_match_alone(dyg):
    import torch
    from dygrass_b200.serve import PlainServer, Server, poisson_requests
    cases = mixed_cases()
    p = dyg.WalkParams.make(threshold=100.0, walkers=128)
    reqs = poisson_requests(cases, rate=1e7, count=80, seed=3, size_hi=200)
    alone = [dataclasses.replace(r) for r in reqs]
    S = Server(cases, p, p)
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
