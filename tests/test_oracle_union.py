"""The batched and serving modes' premise, checked on the oracle (no GPU):
graphs packed into one union graph at vertex offsets and updated round by
round, batch r of every graph in one batch whose edges carry their position
in their own graph's stream as update id, give every graph exactly the
found_at, conductance and accepted flags, and the final sparsifier rows, of
its own reference-style loop (ceil(n/10)-edge batches, first update id = the
batch's first position).  The same for the server's steps: the oldest
request of every graph per step, the step's insertions as one batch and its
deletions as another, each update with its graph's own update id.  The CUDA
path is held to the same property by tests/test_multi.py and
tests/test_serve.py."""
import os
import sys

import numpy as np

import dygrass_b200 as dyg
from dygrass_b200 import workloads as W
from dygrass_b200.multi import plan_rounds

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import pyoracle  # noqa: E402


def small_cases():
    cases, _ = W.rgg_many(k=3, n_lo=200, n_hi=1500, seed=31)
    cases += [W.grid_2d(12, 12, inserts=60, seed=32), W.mesh_3d(5, inserts=80, seed=33)]
    return cases


def union_graph(cases, offsets, which):
    cat = lambda xs, t: np.concatenate(xs).astype(t)
    s = cat([getattr(c, which + "_src") + o for c, o in zip(cases, offsets)], np.uint32)
    d = cat([getattr(c, which + "_dst") + o for c, o in zip(cases, offsets)], np.uint32)
    w = cat([getattr(c, which + "_w") for c in cases], np.float32)
    return pyoracle.OGraph(int(offsets[-1]), s, d, w)


def test_union_rounds_equal_each_graph_alone():
    cases = small_cases()
    p = dyg.WalkParams.make(threshold=50.0, walkers=64, max_steps=48)
    offsets = np.zeros(len(cases) + 1, np.int64)
    offsets[1:] = np.cumsum([c.n for c in cases])
    Hu, Gu = union_graph(cases, offsets, "h"), union_graph(cases, offsets, "g")
    streams = [(c.ins_src, c.ins_dst, c.ins_w) for c in cases]
    plan = plan_rounds(offsets, streams)
    alone = [(pyoracle.OGraph(c.n, c.h_src, c.h_dst, c.h_w), pyoracle.OGraph(c.n, c.g_src, c.g_dst, c.g_w))
             for c in cases]
    accepted = 0
    for rd in plan.rounds:
        fa, cd, ac = pyoracle.incremental_ids(Hu, rd.src, rd.dst, rd.w, rd.uid, p, G=Gu, threads=4)
        for g in np.unique(rd.graph):
            sel = rd.graph == g
            lo, hi = int(rd.pos[sel][0]), int(rd.pos[sel][-1]) + 1
            s, d, w = streams[g]
            Hg, Gg = alone[g]
            fa1, cd1, ac1, _ = pyoracle.incremental(Hg, s[lo:hi], d[lo:hi], w[lo:hi], p, G=Gg, threads=4,
                                                    first_uid=lo, single_batch=True)
            assert np.array_equal(fa[sel], fa1), g
            assert np.array_equal(cd[sel].view(np.uint32), cd1.view(np.uint32)), g
            assert np.array_equal(ac[sel], ac1), g
            accepted += int(ac1.sum())
    assert 0 < accepted < plan.n_edges            # both outcomes occur
    for which, u in (("H", Hu), ("G", Gu)):
        rp, col, w = u.export()
        for g, c in enumerate(cases):
            lo, hi = int(offsets[g]), int(offsets[g + 1])
            a, b = int(rp[lo]), int(rp[hi])
            rp1, col1, w1 = alone[g][0 if which == "H" else 1].export()
            assert np.array_equal(rp[lo:hi + 1] - rp[lo], rp1), (which, g)
            assert np.array_equal(col[a:b] - lo, col1), (which, g)
            assert np.array_equal(w[a:b].view(np.uint32), w1.view(np.uint32)), (which, g)


def test_update_ids_matter():
    """Control: the same union batch walked with the union's own positions as
    update ids (first id 0) differs from the per-graph loops, so the test above
    would notice ids that were not carried per graph."""
    cases = small_cases()
    p = dyg.WalkParams.make(threshold=50.0, walkers=64, max_steps=48)
    offsets = np.zeros(len(cases) + 1, np.int64)
    offsets[1:] = np.cumsum([c.n for c in cases])
    Hu, Hv = union_graph(cases, offsets, "h"), union_graph(cases, offsets, "h")
    rd = plan_rounds(offsets, [(c.ins_src, c.ins_dst, c.ins_w) for c in cases]).rounds[0]
    fa, cd, _ = pyoracle.incremental_ids(Hu, rd.src, rd.dst, rd.w, rd.uid, p, threads=4)
    fb, cb, _ = pyoracle.incremental_ids(Hv, rd.src, rd.dst, rd.w,
                                         np.arange(len(rd.src), dtype=np.uint64), p, threads=4)
    assert not (np.array_equal(fa, fb) and np.array_equal(cd.view(np.uint32), cb.view(np.uint32)))


def test_served_steps_equal_each_graph_alone():
    from dygrass_b200.serve import DELETE, INSERT, poisson_requests
    cases = small_cases()
    p = dyg.WalkParams.make(threshold=50.0, walkers=64, max_steps=48)
    offsets = np.zeros(len(cases) + 1, np.int64)
    offsets[1:] = np.cumsum([c.n for c in cases])
    reqs = poisson_requests(cases, rate=1e6, count=40, seed=9, size_hi=60)
    Hu, Gu = union_graph(cases, offsets, "h"), union_graph(cases, offsets, "g")
    queues = {g: [r for r in reqs if r.graph == g] for g in range(len(cases))}
    uid_next = [0] * len(cases)
    got = {}
    while any(queues.values()):
        heads = [queues[g].pop(0) for g in range(len(cases)) if queues[g]]
        for op in (INSERT, DELETE):
            sel = [r for r in heads if r.op == op and len(r.src)]
            if not sel:
                continue
            src = np.concatenate([r.src + offsets[r.graph] for r in sel]).astype(np.uint32)
            dst = np.concatenate([r.dst + offsets[r.graph] for r in sel]).astype(np.uint32)
            uid = np.concatenate([np.arange(len(r.src), dtype=np.uint64) + np.uint64(uid_next[r.graph])
                                  for r in sel])
            if op == INSERT:
                w = np.concatenate([r.w for r in sel]).astype(np.float32)
                out = pyoracle.incremental_ids(Hu, src, dst, w, uid, p, G=Gu, threads=4)
            else:
                st, cd, rx, ry, rk = pyoracle.decremental_ids(Gu, Hu, src, dst, uid, p, threads=4)
                owner = np.searchsorted(offsets, rx, side="right") - 1
                out = (st, cd)
            k = 0
            for r in sel:
                m = len(r.src)
                res = tuple(a[k:k + m] for a in out)
                if op == DELETE:
                    o = owner == r.graph
                    res += (list(zip((rx[o] - offsets[r.graph]).tolist(),
                                     (ry[o] - offsets[r.graph]).tolist(), rk[o].tolist())),)
                got[id(r)] = res
                k += m
        for r in heads:
            uid_next[r.graph] += len(r.src)
    alone = [(pyoracle.OGraph(c.n, c.h_src, c.h_dst, c.h_w), pyoracle.OGraph(c.n, c.g_src, c.g_dst, c.g_w))
             for c in cases]
    uid_alone = [0] * len(cases)
    n_rec = 0
    for r in reqs:
        Hg, Gg = alone[r.graph]
        u = uid_alone[r.graph]
        uid_alone[r.graph] += len(r.src)
        if not len(r.src):
            continue
        if r.op == INSERT:
            fa, cd, ac, _ = pyoracle.incremental(Hg, r.src, r.dst, r.w, p, G=Gg, threads=4, first_uid=u,
                                                 single_batch=True)
            gfa, gcd, gac = got[id(r)]
            assert np.array_equal(gfa, fa) and np.array_equal(gac, ac)
            assert np.array_equal(gcd.view(np.uint32), cd.view(np.uint32))
        else:
            st, cd, rx, ry, rk, _ = pyoracle.decremental(Gg, Hg, r.src, r.dst, p, threads=4, first_uid=u,
                                                         single_batch=True)
            gst, gcd, grec = got[id(r)]
            assert np.array_equal(gst, st)
            assert np.array_equal(gcd.view(np.uint32), cd.view(np.uint32))
            assert grec == list(zip(rx.tolist(), ry.tolist(), rk.tolist()))
            n_rec += len(grec)
    assert n_rec > 0                                  # deletions recovered edges
    for which, u in (("H", Hu), ("G", Gu)):
        rp, col, w = u.export()
        for g in range(len(cases)):
            lo, hi = int(offsets[g]), int(offsets[g + 1])
            a, b = int(rp[lo]), int(rp[hi])
            rp1, col1, w1 = alone[g][0 if which == "H" else 1].export()
            assert np.array_equal(rp[lo:hi + 1] - rp[lo], rp1), (which, g)
            assert np.array_equal(col[a:b] - lo, col1), (which, g)
            assert np.array_equal(w[a:b].view(np.uint32), w1.view(np.uint32)), (which, g)
