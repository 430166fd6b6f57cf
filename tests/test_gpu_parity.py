"""CUDA path (through the C ABI) against the CPU oracle: bit-exact.

Integer results (found_at, accepted flags, statuses, recovered edges and
their order, every row of the final graphs) must be identical; conductances
are compared as bit patterns (both sides compute 1/R with single IEEE
binary32 operations, no contraction).
"""
import numpy as np
import pytest

import kat_cases
from helpers import decr_inputs, incr_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dyg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import dygrass_b200
    dygrass_b200.lib()
    return dygrass_b200


def same_graph(g_dev, g_orc):
    rp1, c1, w1 = g_dev.export()
    rp2, c2, w2 = g_orc.export()
    assert np.array_equal(rp1, rp2)
    assert np.array_equal(c1, c2)
    assert np.array_equal(w1.view(np.uint32), w2.view(np.uint32))


def run_incr_both(dyg, oracle, n, hs, hd, hw, es, ed, ew, params, batch_size=0, with_g=None):
    H = dyg.Graph.from_edges(n, hs, hd, hw)
    Ho = oracle.OGraph(n, hs, hd, hw)
    G = Go = None
    if with_g is not None:
        gs, gd, gw = with_g
        G = dyg.Graph.from_edges(n, gs, gd, gw)
        Go = oracle.OGraph(n, gs, gd, gw)
    r = dyg.incremental_stream(H, es, ed, ew, params, batch_size=batch_size, G=G)
    fa, cd, ac, mv = oracle.incremental(Ho, es, ed, ew, params, batch_size=batch_size, G=Go)
    assert np.array_equal(r.found_at, fa)
    assert np.array_equal(r.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(r.accepted, ac)
    same_graph(H, Ho)
    if G is not None:
        same_graph(G, Go)
    return H, Ho, r, mv


@pytest.mark.parametrize("name", sorted(kat_cases.INCREMENTAL))
def test_kat_incremental(dyg, oracle, name):
    case = kat_cases.INCREMENTAL[name]
    n, hs, hd, hw, es, ed, ew = incr_inputs(case)
    p = dyg.WalkParams.make(threshold=case["threshold"], walkers=case["walkers"])
    _, _, r, _ = run_incr_both(dyg, oracle, n, hs, hd, hw, es, ed, ew, p)
    assert list(r.accepted) == case["expect_added"]


@pytest.mark.parametrize("name", sorted(kat_cases.DECREMENTAL))
def test_kat_decremental(dyg, oracle, name):
    case = kat_cases.DECREMENTAL[name]
    n, gs, gd, gw, hs, hd, hw, ds, dd = decr_inputs(case)
    p = dyg.WalkParams.make()
    G, H = dyg.Graph.from_edges(n, gs, gd, gw), dyg.Graph.from_edges(n, hs, hd, hw)
    Go, Ho = oracle.OGraph(n, gs, gd, gw), oracle.OGraph(n, hs, hd, hw)
    r = dyg.decremental_stream(G, H, ds, dd, p)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, ds, dd, p)
    assert np.array_equal(r.status, st)
    assert np.array_equal(r.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(r.rec_src, rx) and np.array_equal(r.rec_dst, ry)
    assert np.array_equal(r.rec_kind, rk)
    same_graph(G, Go)
    same_graph(H, Ho)
    got = sorted((min(a, b) + 1, max(a, b) + 1) for a, b in zip(r.rec_src, r.rec_dst))
    assert got == sorted(case["expect_added"])


def test_grid_100x100_full(dyg, oracle):
    """The 2-D grid configuration at full size: 10,000 vertices, 1,000
    insertions, 512 walkers, max_steps 64, threshold 10."""
    import dygrass_b200.workloads as wl
    W = wl.grid_2d()
    H, Ho, r, mv = run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst,
                                 W.ins_w, W.params, with_g=(W.g_src, W.g_dst, W.g_w))
    moves, walks = H.counters()
    assert walks == len(W.ins_src) * W.params.walkers
    assert 0 < moves < mv          # pruned walkers stop early; results are unchanged
    assert 0 < r.accepted.sum() < len(r.accepted)
    # exhaustive mode executes exactly the oracle's walker moves
    pe = dyg.WalkParams.make(threshold=W.params.threshold, walkers=W.params.walkers,
                             max_steps=W.params.max_steps, seed=W.params.seed,
                             flags=dyg.FLAG_EXHAUSTIVE)
    H2, _, r2, mv2 = run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst,
                                   W.ins_w, pe)
    assert H2.counters()[0] == mv2 == mv
    assert np.array_equal(r2.accepted, r.accepted)


@pytest.mark.parametrize("walkers", [32, 96, 160, 1024])
def test_walker_counts(dyg, oracle, walkers):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(40, 40, inserts=300)
    p = dyg.WalkParams.make(threshold=10.0, walkers=walkers, max_steps=64)
    run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst, W.ins_w, p)


@pytest.mark.parametrize("batch", [1, 7, 0, 1000])
def test_batch_sizes(dyg, oracle, batch):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(30, 30, inserts=200)
    run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst, W.ins_w,
                  W.params, batch_size=batch)


def test_weighted_transition(dyg, oracle):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(40, 40, inserts=300)
    p = dyg.WalkParams.make(threshold=10.0, walkers=128, max_steps=64, transition=1)
    run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst, W.ins_w, p)


def test_batch_api_matches_stream(dyg, oracle):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(30, 30, inserts=95)
    H1 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    H2 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    r1 = dyg.incremental_stream(H1, W.ins_src, W.ins_dst, W.ins_w, W.params)
    B = dyg.reference_batch_size(len(W.ins_src))
    acc = []
    for b0 in range(0, len(W.ins_src), B):
        r = dyg.incremental_batch(H2, W.ins_src[b0:b0 + B], W.ins_dst[b0:b0 + B],
                                  W.ins_w[b0:b0 + B], W.params, first_update_id=b0)
        acc.append(r.accepted)
    assert np.array_equal(np.concatenate(acc), r1.accepted)
    assert np.array_equal(H1.export()[1], H2.export()[1])


def test_device_pointers(dyg, oracle):
    import torch
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(30, 30, inserts=200)
    H1 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    H2 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    r1 = dyg.incremental_stream(H1, W.ins_src, W.ins_dst, W.ins_w, W.params)
    dev = torch.device("cuda:0")
    s = torch.from_numpy(W.ins_src.view(np.int32)).to(dev)
    d = torch.from_numpy(W.ins_dst.view(np.int32)).to(dev)
    w = torch.from_numpy(W.ins_w).to(dev)
    out = dyg.IncrementalResult(torch.empty(len(s), dtype=torch.int32, device=dev),
                                torch.empty(len(s), dtype=torch.float32, device=dev),
                                torch.empty(len(s), dtype=torch.uint8, device=dev))
    dyg.incremental_stream(H2, s, d, w, W.params, out=out)
    torch.cuda.synchronize()
    assert np.array_equal(out.accepted.cpu().numpy(), r1.accepted)
    assert np.array_equal(out.found_at.cpu().numpy(), r1.found_at)
    assert np.array_equal(H1.export()[1], H2.export()[1])


def small_mesh(k=12, inserts=400):
    import dygrass_b200.workloads as wl
    return wl.mesh_3d(k=k, inserts=inserts)


def test_mesh_incremental_then_decremental(dyg, oracle):
    """Insert stream (updating H and G), then the deletion stream, on a
    12^3 mesh: every status, recovered edge (in order) and row identical."""
    W = small_mesh()
    H, Ho, r, _ = run_incr_both(dyg, oracle, W.n, W.h_src, W.h_dst, W.h_w, W.ins_src, W.ins_dst,
                                W.ins_w, W.params, with_g=None)
    G = dyg.Graph.from_edges(W.n, np.concatenate([W.g_src, W.ins_src]),
                             np.concatenate([W.g_dst, W.ins_dst]), np.concatenate([W.g_w, W.ins_w]))
    Go = oracle.OGraph(W.n, np.concatenate([W.g_src, W.ins_src]),
                       np.concatenate([W.g_dst, W.ins_dst]), np.concatenate([W.g_w, W.ins_w]))
    rd = dyg.decremental_stream(G, H, W.del_src, W.del_dst, W.dparams)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, W.del_src, W.del_dst, W.dparams)
    assert np.array_equal(rd.status, st)
    assert np.array_equal(rd.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(rd.rec_src, rx) and np.array_equal(rd.rec_dst, ry)
    assert np.array_equal(rd.rec_kind, rk)
    same_graph(G, Go)
    same_graph(H, Ho)
    assert (st > 0).sum() > 0 and (st == -2).sum() > 0


@pytest.mark.parametrize("slack,headroom", [(0, 0.0), (1, 0.05)])
def test_tight_arenas_resume(dyg, oracle, slack, headroom):
    """Arenas with no room: appends halt the stream, the host grows the arena
    and resumes; recovered-edge records overflow their first buffer the same
    way.  Results must not change."""
    W = small_mesh(k=10, inserts=300)
    gs = np.concatenate([W.g_src, W.ins_src])
    gd = np.concatenate([W.g_dst, W.ins_dst])
    gw = np.concatenate([W.g_w, W.ins_w])
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w, slack_per_row=slack,
                             arena_headroom=headroom)
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w, slack_per_row=slack,
                             arena_headroom=headroom)
    Ho = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    Go = oracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w)
    r = dyg.incremental_stream(H, W.ins_src, W.ins_dst, W.ins_w, W.params, G=G)
    fa, cd, ac, _ = oracle.incremental(Ho, W.ins_src, W.ins_dst, W.ins_w, W.params, G=Go)
    assert np.array_equal(r.accepted, ac) and np.array_equal(r.found_at, fa)
    same_graph(H, Ho)
    same_graph(G, Go)
    d = dyg.decremental_stream(G, H, W.del_src, W.del_dst, W.dparams)
    st, cd2, rx, ry, rk, _ = oracle.decremental(Go, Ho, W.del_src, W.del_dst, W.dparams)
    assert np.array_equal(d.status, st)
    assert np.array_equal(d.rec_src, rx) and np.array_equal(d.rec_dst, ry)
    assert np.array_equal(d.rec_kind, rk)
    assert len(rx) > 4 * len(W.del_src) // 10    # more than one record buffer's worth per batch
    same_graph(G, Go)
    same_graph(H, Ho)


def test_mesh_exhaustive_and_pruned_agree(dyg, oracle):
    """Pruning changes only how many moves run, never a result."""
    W = small_mesh(k=10, inserts=300)
    outs = []
    for flags in (0, dyg.FLAG_EXHAUSTIVE):
        p = dyg.WalkParams.make(threshold=W.params.threshold, walkers=W.params.walkers,
                                max_steps=W.params.max_steps, seed=W.params.seed, flags=flags)
        dp = dyg.WalkParams.make(walkers=W.dparams.walkers, max_steps=W.dparams.max_steps,
                                 seed=W.dparams.seed, flags=flags)
        H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
        G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
        r = dyg.incremental_stream(H, W.ins_src, W.ins_dst, W.ins_w, p, G=G)
        d = dyg.decremental_stream(G, H, W.del_src, W.del_dst, dp)
        outs.append((r.found_at.tobytes(), r.conductance.tobytes(), d.status.tobytes(),
                     d.conductance.tobytes(), d.rec_src.tobytes(), d.rec_dst.tobytes(),
                     H.export()[1].tobytes(), G.export()[1].tobytes(),
                     H.counters()[0] + G.counters()[0]))
    assert outs[0][:-1] == outs[1][:-1]
    assert outs[0][-1] < outs[1][-1]


def test_decremental_fallback_path(dyg, oracle):
    """Deleting every edge of a vertex's H-and-G neighbourhood leaves edges
    without a path: the 2-step fallback walks run and match the oracle."""
    n = 30
    src = np.array([i for i in range(n - 1)] + [0, 5, 10], np.uint32)
    dst = np.array([i + 1 for i in range(n - 1)] + [10, 20, 25], np.uint32)
    w = np.linspace(0.5, 2.0, len(src)).astype(np.float32)
    dels_s = np.array([3, 26, 14], np.uint32)   # (26, 27) is a bridge: no path
    dels_d = np.array([4, 27, 15], np.uint32)
    p = dyg.WalkParams.make(walkers=64, max_steps=20, heuristic_walkers=16)
    G, H = dyg.Graph.from_edges(n, src, dst, w), dyg.Graph.from_edges(n, src, dst, w)
    Go, Ho = oracle.OGraph(n, src, dst, w), oracle.OGraph(n, src, dst, w)
    rd = dyg.decremental_stream(G, H, dels_s, dels_d, p)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, dels_s, dels_d, p)
    assert np.array_equal(rd.status, st)
    assert np.array_equal(rd.rec_src, rx) and np.array_equal(rd.rec_dst, ry)
    assert np.array_equal(rd.rec_kind, rk)
    same_graph(H, Ho)
    assert (st == -1).any()


def test_decremental_edge_cases(dyg, oracle):
    """Deletions absent from G, present in G only, duplicated within a batch."""
    W = small_mesh(k=8, inserts=50)
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    Go = oracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w)
    Ho = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    ds = np.array([W.g_src[0], W.g_src[0], W.ins_src[0], W.g_dst[5], W.h_src[3]], np.uint32)
    dd = np.array([W.g_dst[0], W.g_dst[0], W.ins_dst[0], W.g_src[5], W.h_dst[3]], np.uint32)
    rd = dyg.decremental_batch(G, H, ds, dd, W.dparams, first_update_id=77)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, ds, dd, W.dparams, first_uid=77,
                                               single_batch=True)
    assert np.array_equal(rd.status, st)
    assert st[1] == -3 and st[2] == -3
    assert np.array_equal(rd.rec_src, rx) and np.array_equal(rd.rec_dst, ry)
    same_graph(G, Go)
    same_graph(H, Ho)


def test_invalid_arguments(dyg):
    H = dyg.Graph.from_edges(4, np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32),
                             np.ones(3, np.float32))
    p = dyg.WalkParams.make(walkers=48)
    with pytest.raises(dyg.DygError) as e:
        dyg.incremental_stream(H, [0], [3], [1.0], p)
    assert e.value.status == 1
    p = dyg.WalkParams.make()
    with pytest.raises(dyg.DygError) as e:
        dyg.incremental_stream(H, [0], [7], [1.0], p)
    assert e.value.status == 1
    with pytest.raises(dyg.DygError):
        dyg.incremental_stream(H, [0], [2], [0.0], p)
    with pytest.raises(dyg.DygError):
        dyg.Graph.from_edges(3, np.array([0], np.uint32), np.array([5], np.uint32),
                             np.ones(1, np.float32))


def test_compaction_and_snapshots(dyg, oracle):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(40, 40, inserts=600)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w, slack_per_row=0, arena_headroom=0.0)
    H0 = H.clone()
    Ho = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    half = 300
    r1 = dyg.incremental_stream(H, W.ins_src[:half], W.ins_dst[:half], W.ins_w[:half], W.params)
    oracle.incremental(Ho, W.ins_src[:half], W.ins_dst[:half], W.ins_w[:half], W.params)
    before = H.info()
    H.compact()
    after = H.info()
    assert after["arena_used"] <= before["arena_used"]
    same_graph(H, Ho)
    dyg.incremental_stream(H, W.ins_src[half:], W.ins_dst[half:], W.ins_w[half:], W.params)
    oracle.incremental(Ho, W.ins_src[half:], W.ins_dst[half:], W.ins_w[half:], W.params)
    same_graph(H, Ho)
    # restoring the snapshot and replaying the first half reproduces it
    H.copy_from(H0)
    r2 = dyg.incremental_stream(H, W.ins_src[:half], W.ins_dst[:half], W.ins_w[:half], W.params)
    assert np.array_equal(r1.accepted, r2.accepted)


def test_compaction_long_rows(dyg, oracle):
    """Compaction moves each row with one warp, 128 slots per pass: a hub row
    of 9,000 slots (71 passes) and rows of 1 to 3 slots keep their contents
    and order, and later updates agree with the oracle."""
    n, gs, gd, gw, hs, hd, hw, es, ed, ew = hub_graph(9000, 21)
    G = dyg.Graph.from_edges(n, gs, gd, gw, slack_per_row=3, arena_headroom=0.5)
    Go = oracle.OGraph(n, gs, gd, gw)
    H = dyg.Graph.from_edges(n, hs, hd, hw)
    Ho = oracle.OGraph(n, hs, hd, hw)
    before = G.export()
    G.compact()
    after = G.export()
    for a, b in zip(before, after):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert G.info()["arena_used"] <= sum(len(x) for x in before[1:2]) + 3 * n
    # deletions of hub edges on the compacted G (walks through the hub)
    rng = np.random.default_rng(8)
    k = rng.choice(9000, 30, replace=False)
    ds, dd = np.zeros(30, np.uint32), (k + 1).astype(np.uint32)
    pd = dyg.WalkParams.make(walkers=64, max_steps=20)
    d = dyg.decremental_stream(G, H, ds, dd, pd)
    st, _, rx, ry, _, _ = oracle.decremental(Go, Ho, ds, dd, pd)
    assert np.array_equal(d.status, st)
    assert np.array_equal(d.rec_src, rx) and np.array_equal(d.rec_dst, ry)
    same_graph(G, Go)
    same_graph(H, Ho)


def hub_graph(n_leaves, seed, huge=0):
    """A hub joined to every leaf, plus a ring through the leaves; weights
    U[0.5, 2] except the hub edges to the first 50 leaves (100; the first
    `huge` of them 5e9, whose fixed-point weights saturate, so row sums wrap
    past 2^64).  H = the star + every 10th ring edge.  Insertions: 20 pairs
    of heavy leaves (walkers reach them through the hub) and 20 random
    pairs."""
    rng = np.random.default_rng(seed)
    leaves = np.arange(1, n_leaves + 1, dtype=np.uint32)
    ring = np.roll(leaves, -1)
    gs = np.concatenate([np.zeros(n_leaves, np.uint32), leaves])
    gd = np.concatenate([leaves, ring])
    gw = rng.uniform(0.5, 2.0, len(gs)).astype(np.float32)
    gw[:50] = 100.0
    gw[:huge] = 5e9
    h = np.concatenate([np.arange(n_leaves), n_leaves + np.arange(0, n_leaves, 10)])
    ins = np.concatenate([rng.choice(leaves[:50], size=(20, 2)), rng.choice(leaves, size=(20, 2))])
    ins = ins[ins[:, 0] != ins[:, 1]]
    iw = rng.uniform(0.5, 2.0, len(ins)).astype(np.float32)
    return (n_leaves + 1, gs, gd, gw, gs[h], gd[h], gw[h], ins[:, 0].copy(), ins[:, 1].copy(), iw)


@pytest.mark.parametrize("leaves,huge", [(200, 0), (9000, 0), (9000, 3)])
def test_weighted_long_rows(dyg, oracle, leaves, huge):
    """Weighted walks through a hub row: 200 slots (one warp pass), 9,000
    slots (71 tiles of 128, segments of two tiles), and 9,000 slots whose
    sums wrap past 2^64 (the whole row is scanned in order); insertions with
    G, then deletions of hub edges in H (walks on G through the hub)."""
    n, gs, gd, gw, hs, hd, hw, es, ed, ew = hub_graph(leaves, 11 + huge, huge)
    p = dyg.WalkParams.make(threshold=10.0, walkers=32, max_steps=20, transition=1)
    H, Ho, r, _ = run_incr_both(dyg, oracle, n, hs, hd, hw, es, ed, ew, p, with_g=(gs, gd, gw))
    assert 0 < r.accepted.sum() < len(r.accepted)
    G = dyg.Graph.from_edges(n, np.concatenate([gs, es]), np.concatenate([gd, ed]),
                             np.concatenate([gw, ew]))
    Go = oracle.OGraph(n, np.concatenate([gs, es]), np.concatenate([gd, ed]), np.concatenate([gw, ew]))
    rng = np.random.default_rng(5)
    k = rng.choice(leaves, 24, replace=False)
    ds, dd = np.zeros(24, np.uint32), (k + 1).astype(np.uint32)
    pd = dyg.WalkParams.make(walkers=32, max_steps=20, transition=1)
    d = dyg.decremental_stream(G, H, ds, dd, pd)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, ds, dd, pd)
    assert np.array_equal(d.status, st)
    assert np.array_equal(d.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(d.rec_src, rx) and np.array_equal(d.rec_dst, ry)
    same_graph(G, Go)
    same_graph(H, Ho)


def medium_rows_graph(seed):
    """A hub joined to 600 leaves (a row longer than 256 slots, which turns
    the long-row paths on), 40 vertices with 60..199 random neighbours each
    (rows of 33..256 slots, which such graphs edit one warp per row inside
    the long-row launch), and a ring through every vertex but the hub.
    H = the star, the ring and every other edge of the 40 vertices."""
    rng = np.random.default_rng(seed)
    n = 1001
    edges = {(0, v) for v in range(1, 601)}
    edges |= {(v, v + 1) for v in range(1, n - 1)} | {(1, n - 1)}
    mids = rng.choice(np.arange(601, n), 40, replace=False)
    mid_edges = set()
    for m in mids:
        for u in rng.choice(np.arange(1, n), int(rng.integers(60, 200)), replace=False):
            if u != m:
                mid_edges.add((int(min(m, u)), int(max(m, u))))
    mid_edges -= edges
    mid_list = sorted(mid_edges)
    e = np.array(sorted(edges) + mid_list, np.uint32)
    gw = rng.uniform(0.5, 2.0, len(e)).astype(np.float32)
    in_h = np.zeros(len(e), bool)
    in_h[:len(edges)] = True
    in_h[len(edges)::2] = True
    return n, e[:, 0].copy(), e[:, 1].copy(), gw, in_h, np.array(mid_list, np.uint32), rng


@pytest.mark.parametrize("seed", [3, 4])
def test_medium_rows_with_hub(dyg, oracle, seed):
    """Deletions on graphs with a hub row: rows of 33..256 slots with many
    deletions each, duplicates, pairs absent from G, hub edges and edges of
    G only, in one batch and in the reference's batches; statuses,
    recovered edges and every row of G and H equal the oracle's."""
    n, gs, gd, gw, in_h, mid, rng = medium_rows_graph(seed)
    hs, hd, hw = gs[in_h], gd[in_h], gw[in_h]
    pick = mid[rng.choice(len(mid), 300, replace=False)]
    dup = pick[rng.choice(300, 20, replace=False)]
    absent = []
    have = set(zip(gs.tolist(), gd.tolist()))
    while len(absent) < 10:
        a, b = sorted(rng.choice(np.arange(1, n), 2, replace=False).tolist())
        if (a, b) not in have:
            absent.append((a, b))
    hub = np.stack([np.zeros(10, np.uint32), rng.choice(np.arange(1, 601), 10, replace=False)], 1)
    dl = np.concatenate([pick, dup, np.array(absent, np.uint32), hub.astype(np.uint32)])
    dl = dl[rng.permutation(len(dl))]
    flip = rng.random(len(dl)) < 0.5
    ds = np.where(flip, dl[:, 1], dl[:, 0]).astype(np.uint32)
    dd = np.where(flip, dl[:, 0], dl[:, 1]).astype(np.uint32)
    p = dyg.WalkParams.make(walkers=64, max_steps=24, heuristic_walkers=8)
    for single in (True, False):
        G, H = dyg.Graph.from_edges(n, gs, gd, gw), dyg.Graph.from_edges(n, hs, hd, hw)
        Go, Ho = oracle.OGraph(n, gs, gd, gw), oracle.OGraph(n, hs, hd, hw)
        if single:
            rd = dyg.decremental_batch(G, H, ds, dd, p, first_update_id=5)
            st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, ds, dd, p, first_uid=5,
                                                       single_batch=True)
        else:
            rd = dyg.decremental_stream(G, H, ds, dd, p)
            st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, ds, dd, p)
        assert np.array_equal(rd.status, st)
        assert np.array_equal(rd.conductance.view(np.uint32), cd.view(np.uint32))
        assert np.array_equal(rd.rec_src, rx) and np.array_equal(rd.rec_dst, ry)
        assert np.array_equal(rd.rec_kind, rk)
        same_graph(G, Go)
        same_graph(H, Ho)
        assert (st == -3).sum() >= 20   # the duplicates' second copies and the absent pairs
