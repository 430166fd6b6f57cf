"""Many graphs in one launch per round (dygrass_b200/multi.py): the union
run gives every graph exactly what its own update loop gives, for every
launch shape the autotuner may pick."""
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


def per_graph(dyg, cases, p):
    out = []
    for c in cases:
        H = dyg.Graph.from_edges(c.n, c.h_src, c.h_dst, c.h_w)
        G = dyg.Graph.from_edges(c.n, c.g_src, c.g_dst, c.g_w)
        r = dyg.incremental_stream(H, c.ins_src, c.ins_dst, c.ins_w, p, G=G)
        out.append((r, H.export(), G.export()))
        H.close()
        G.close()
    return out


def check_same(M, plan, res, ref):
    pg = M.per_graph(plan, res)
    for g, (r, hx, gx) in enumerate(ref):
        fa, cd, ac = pg[g]
        assert np.array_equal(fa, r.found_at)
        assert np.array_equal(cd.view(np.uint32), r.conductance.view(np.uint32))
        assert np.array_equal(ac, r.accepted)
        for which, want in (("H", hx), ("G", gx)):
            got = M.graph_rows(which, g)
            assert np.array_equal(got[0], want[0])
            assert np.array_equal(got[1], want[1])
            assert np.array_equal(got[2].view(np.uint32), want[2].view(np.uint32))


def test_union_matches_per_graph_loops(dyg):
    from dygrass_b200.multi import ManyGraphs
    cases, p = W.rgg_many(k=7, n_lo=300, n_hi=6000, walkers=128)
    ref = per_graph(dyg, cases, p)
    M = ManyGraphs(cases)
    plan = M.plan()
    assert len(plan.rounds) == 10
    res = M.run(plan, p)
    check_same(M, plan, res, ref)
    assert sum(int(r.accepted.sum()) for r in res) > 0
    M.close()


@pytest.mark.parametrize("chunk,bpsm", [(64, 0), (128, 3), (32, 2)])
def test_launch_shape_does_not_change_results(dyg, chunk, bpsm):
    from dygrass_b200.multi import ManyGraphs
    cases, p = W.rgg_many(k=5, n_lo=300, n_hi=4000, walkers=128, seed=11)
    ref = per_graph(dyg, cases, p)
    dyg.tune_set(chunk, bpsm)
    try:
        M = ManyGraphs(cases)
        plan = M.plan()
        check_same(M, plan, M.run(plan, p), ref)
        M.close()
    finally:
        dyg.tune_set(0, 0)


def test_autotune(dyg):
    import torch
    from dygrass_b200.multi import autotune
    cases, p = W.rgg_many(k=6, n_lo=300, n_hi=3000, walkers=128, seed=5)
    try:
        best, trials = autotune(cases, params=p, chunks=(32, 64), blocks=(0, 4), walkers=(64,),
                                max_steps=(40,), kappa_graphs=2, repeats=1,
                                sync=torch.cuda.synchronize)
    finally:
        dyg.tune_set(0, 0)
    assert len(trials) >= 10 and best["seconds"] == min(t["seconds"] for t in trials
                                                        if t.get("kappa_ok", True))
    # every launch shape with both prune intervals (results do not depend on them)
    assert {t["prune_every"] for t in trials} == {1, 2}
    assert any("kappa" in t for t in trials)
    # the walk-length trial runs at the walker count chosen before it
    ms = [t for t in trials if t.get("max_steps") == 40]
    assert len(ms) == 1 and ms[0]["params"].max_steps == 40
    assert ms[0]["params"].walkers in (64, p.walkers)
    # the returned parameters are the best trial's
    assert best["params"].walkers == best["walkers"]
    assert best["params"].max_steps == best["max_steps"]


def test_decremental_ids_match_per_graph(dyg):
    """Deletions with per-edge update ids on a union of two meshes equal each
    mesh's own decremental batch."""
    wls = [W.mesh_3d(6, inserts=50, seed=3), W.mesh_3d(7, inserts=50, seed=4)]
    off = [0, wls[0].n]
    gs = np.concatenate([w.g_src + o for w, o in zip(wls, off)]).astype(np.uint32)
    gd = np.concatenate([w.g_dst + o for w, o in zip(wls, off)]).astype(np.uint32)
    gw = np.concatenate([w.g_w for w in wls])
    hs = np.concatenate([w.h_src + o for w, o in zip(wls, off)]).astype(np.uint32)
    hd = np.concatenate([w.h_dst + o for w, o in zip(wls, off)]).astype(np.uint32)
    hw = np.concatenate([w.h_w for w in wls])
    n = off[1] + wls[1].n
    Gu, Hu = dyg.Graph.from_edges(n, gs, gd, gw), dyg.Graph.from_edges(n, hs, hd, hw)
    p = dyg.WalkParams.make(walkers=64)
    k = [min(40, len(w.h_src)) for w in wls]
    ds = np.concatenate([w.h_src[:kk] + o for w, o, kk in zip(wls, off, k)]).astype(np.uint32)
    dd = np.concatenate([w.h_dst[:kk] + o for w, o, kk in zip(wls, off, k)]).astype(np.uint32)
    ids = np.concatenate([np.arange(kk, dtype=np.uint64) + 100 for kk in k])
    ru = dyg.decremental_batch_ids(Gu, Hu, ds, dd, ids, p)
    o = 0
    for w, of, kk in zip(wls, off, k):
        G = dyg.Graph.from_edges(w.n, w.g_src, w.g_dst, w.g_w)
        H = dyg.Graph.from_edges(w.n, w.h_src, w.h_dst, w.h_w)
        r = dyg.decremental_batch(G, H, w.h_src[:kk], w.h_dst[:kk], p, first_update_id=100)
        assert np.array_equal(ru.status[o:o + kk], r.status)
        assert np.array_equal(ru.conductance[o:o + kk].view(np.uint32), r.conductance.view(np.uint32))
        o += kk
        G.close()
        H.close()
    rp, col, wt = Hu.export()
    assert rp[-1] == sum(len(w.h_src) for w in wls) * 2 - 2 * sum(k) + 2 * len(ru.rec_src)
