"""Stream files of the mixed updater (dynamic_update): oracle known-answer
cases and CUDA-vs-oracle parity.

The known-answer cases are worked out by hand from the reference's
preprocessing and commit rules (dynamic_update/gpu_graph.cuh:361-465,
620-723) on graphs where every walk is forced (each vertex has at most one
non-backtracking continuation), so the answers do not depend on the random
numbers.
"""
import numpy as np
import pytest

from dygrass_b200 import workloads as W

INS, DEL = 0, 1
MERGED, SELF_LOOP = -4, -5


def params(threshold=100.0, walkers=64, max_steps=100, hw=16):
    import dygrass_b200
    return dygrass_b200.WalkParams.make(threshold=threshold, walkers=walkers, max_steps=max_steps,
                                        heuristic_walkers=hw, seed=7)


def rows(g_export):
    rp, col, w = g_export
    return [[(int(col[j]), float(w[j])) for j in range(int(rp[v]), int(rp[v + 1]))]
            for v in range(len(rp) - 1)]


# path 0-1-2-3 (unit weights) as both G and H
PATH = (4, np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32),
        np.ones(3, np.float32))
# e0 re-inserts (0,1): merge; e1 new (0,2); e2 repeats it: merge into G only;
# e3 self-loop; e4 new (0,3); e5 new (1,3)
INS_FILE = (np.array([1, 0, 2, 3, 0, 1], np.uint32), np.array([0, 2, 0, 3, 3, 3], np.uint32),
            np.array([0.5, 2.0, 1.0, 1.0, 4.0, 4.0], np.float32))


def expect_insert(chunk):
    """Threshold 5; found_at counts the edges walked.  H after the merge:
    w01 = 1.5.  e1 (0->2, w 2): R = 1/1.5 + 1 = 1.667 at vertex 2, R*w = 3.3 < 5:
    found at step 2, rejected.  e4 (0->3, w 4): R*w = 6.7 >= 5 at vertex 2: no
    path, accepted.  e5 (1->3, w 4): via 2 R*w = 8 >= 5 fails; via 0 it needs
    H's new edge (0,3) (R = 0.667 + 0.25, R*w = 3.7): found at step 2 iff e4
    was committed in an earlier chunk."""
    e5_found = chunk == 1 or chunk == 2   # e1 | e4 | e5  or  e1 e4 | e5
    status = [MERGED, 2, MERGED, SELF_LOOP, -1, 2 if e5_found else -1]
    g_rows = [[(1, 1.5), (2, 3.0), (3, 4.0)], [(0, 1.5), (2, 1.0), (3, 4.0)],
              [(1, 1.0), (3, 1.0), (0, 3.0)], [(2, 1.0), (0, 4.0), (1, 4.0)]]
    h_rows = [[(1, 1.5), (3, 4.0)], [(0, 1.5), (2, 1.0)], [(1, 1.0), (3, 1.0)], [(2, 1.0), (0, 4.0)]]
    if not e5_found:
        h_rows[1].append((3, 4.0))
        h_rows[3].append((1, 4.0))
    return status, g_rows, h_rows


# G = square 0-1-2-3-0 plus chord (0,2); H = path 0-1-2-3
SQUARE_G = (4, np.array([0, 1, 2, 3, 0], np.uint32), np.array([1, 2, 3, 0, 2], np.uint32),
            np.array([1, 1, 1, 2, 1], np.float32))
SQUARE_H = (np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32), np.ones(3, np.float32))
# (1,0): in G and H, walked 1 -> 0; (0,2): G only; (1,3): not in G
DEL_FILE = (np.array([1, 0, 1], np.uint32), np.array([0, 2, 3], np.uint32))


def expect_delete():
    """After deleting (0,1) and (0,2), G is the path 1-2-3-0: the walk 1 -> 2 ->
    3 -> 0 has length 3; (1,2), (2,3) are in H, (3,0) is recovered in walk
    order with G's weight 2."""
    status = [3, -2, -3]
    recs = [(3, 0, 0)]
    h_rows = [[(3, 2.0)], [(2, 1.0)], [(1, 1.0), (3, 1.0)], [(2, 1.0), (0, 2.0)]]
    return status, recs, h_rows


@pytest.mark.parametrize("chunk", [1, 2, 3, 0])
def test_oracle_insert_kat(oracle, chunk):
    n, gs, gd, gw = PATH
    G, H = oracle.OGraph(n, gs, gd, gw), oracle.OGraph(n, gs, gd, gw)
    st, cd, _, _, _, _ = oracle.stream_file(G, H, INS, *INS_FILE, params(threshold=5.0),
                                            chunk=chunk)
    status, g_rows, h_rows = expect_insert(chunk)
    assert list(st) == status
    assert rows(G.export()) == g_rows
    assert rows(H.export()) == h_rows
    assert cd[1] == np.float32(1.0) / (np.float32(1.0) / np.float32(1.5) + np.float32(1.0))


def test_oracle_delete_kat(oracle):
    n, gs, gd, gw = SQUARE_G
    G, H = oracle.OGraph(n, gs, gd, gw), oracle.OGraph(n, *SQUARE_H)
    st, cd, rx, ry, rk, _ = oracle.stream_file(G, H, DEL, *DEL_FILE, None, params(), chunk=0)
    status, recs, h_rows = expect_delete()
    assert list(st) == status
    assert list(zip(rx.tolist(), ry.tolist(), rk.tolist())) == recs
    assert rows(H.export()) == h_rows
    assert rows(G.export()) == [[(3, 2.0)], [(2, 1.0)], [(1, 1.0), (3, 1.0)], [(2, 1.0), (0, 2.0)]]


def test_oracle_default_chunk(oracle):
    assert oracle.stream_default_chunk(1000) == 10000
    assert oracle.stream_default_chunk(1_000_000) == 50000
    assert oracle.stream_default_chunk(645_911) == 32295


# ------------------------------------------------------------------ GPU

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


def both(dyg, oracle, n, g, h, slack=2, headroom=0.5):
    G = dyg.Graph.from_edges(n, *g, slack_per_row=slack, arena_headroom=headroom)
    H = dyg.Graph.from_edges(n, *h, slack_per_row=slack, arena_headroom=headroom)
    return G, H, oracle.OGraph(n, *g), oracle.OGraph(n, *h)


def apply_both(dyg, oracle, G, H, Go, Ho, op, src, dst, w, p, uid0=0, chunk=0):
    r = dyg.stream_file(G, H, op, src, dst, w, p, first_update_id=uid0, chunk=chunk)
    st, cd, rx, ry, rk, _ = oracle.stream_file(Go, Ho, op, src, dst, w, p, first_uid=uid0,
                                               chunk=chunk)
    assert np.array_equal(r.status, st)
    assert np.array_equal(r.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(r.rec_src, rx)
    assert np.array_equal(r.rec_dst, ry)
    assert np.array_equal(r.rec_kind, rk)
    same_graph(G, Go)
    same_graph(H, Ho)
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [1, 2, 3, 0])
def test_gpu_insert_kat(dyg, oracle, chunk):
    n, gs, gd, gw = PATH
    G, H, Go, Ho = both(dyg, oracle, n, (gs, gd, gw), (gs, gd, gw))
    r = apply_both(dyg, oracle, G, H, Go, Ho, INS, *INS_FILE, params(threshold=5.0), chunk=chunk)
    status, g_rows, h_rows = expect_insert(chunk)
    assert list(r.status) == status
    assert rows(G.export()) == g_rows
    assert rows(H.export()) == h_rows


@pytest.mark.gpu
def test_gpu_delete_kat(dyg, oracle):
    n, gs, gd, gw = SQUARE_G
    G, H, Go, Ho = both(dyg, oracle, n, (gs, gd, gw), SQUARE_H)
    r = apply_both(dyg, oracle, G, H, Go, Ho, DEL, *DEL_FILE, None, params())
    status, recs, h_rows = expect_delete()
    assert list(r.status) == status
    assert list(zip(r.rec_src.tolist(), r.rec_dst.tolist(), r.rec_kind.tolist())) == recs
    assert rows(H.export()) == h_rows


def insert_file(wl, rng, n_new):
    """New lattice edges, re-inserted existing edges, repeats with other
    weights and self-loops, shuffled."""
    ex = rng.choice(len(wl.g_src), 60, replace=False)
    s = np.concatenate([wl.ins_src[:n_new], wl.g_src[ex], wl.g_dst[ex[:10]]])
    d = np.concatenate([wl.ins_dst[:n_new], wl.g_dst[ex], wl.g_src[ex[:10]]])
    w = np.concatenate([wl.ins_w[:n_new], rng.uniform(0.5, 2, 70).astype(np.float32)])
    rep = rng.choice(n_new, 40, replace=True)
    s = np.concatenate([s, wl.ins_dst[rep], np.arange(5, dtype=np.uint32)])
    d = np.concatenate([d, wl.ins_src[rep], np.arange(5, dtype=np.uint32)])
    w = np.concatenate([w, rng.uniform(0.5, 2, 45).astype(np.float32)])
    perm = rng.permutation(len(s))
    return s[perm].astype(np.uint32), d[perm].astype(np.uint32), w[perm].astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [0, 37])
def test_gpu_insert_file_parity(dyg, oracle, chunk):
    wl = W.grid_2d(24, 24, inserts=300)
    rng = np.random.default_rng(11)
    G, H, Go, Ho = both(dyg, oracle, wl.n, (wl.g_src, wl.g_dst, wl.g_w),
                        (wl.h_src, wl.h_dst, wl.h_w))
    s, d, w = insert_file(wl, rng, 300)
    r = apply_both(dyg, oracle, G, H, Go, Ho, INS, s, d, w, wl.params, uid0=1000, chunk=chunk)
    assert (r.status == MERGED).sum() >= 100
    assert (r.status == SELF_LOOP).sum() == 5
    assert (r.status == -1).sum() > 0 and (r.status >= 0).sum() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("n_file", [8192, 9000])
def test_gpu_insert_file_sizes(dyg, oracle, n_file):
    """Files of up to 8,192 edges are grouped by a one-block sort in shared
    memory, larger ones by a radix sort: both must give the oracle's merges,
    walks and rows (a file of exactly 8,192 edges fills the one-block sort)."""
    n_new = n_file - 115   # insert_file adds 115 repeats, merges and self-loops
    wl = W.grid_2d(150, 150, inserts=n_new, walkers=64)
    rng = np.random.default_rng(13)
    G, H, Go, Ho = both(dyg, oracle, wl.n, (wl.g_src, wl.g_dst, wl.g_w),
                        (wl.h_src, wl.h_dst, wl.h_w))
    s, d, w = insert_file(wl, rng, n_new)
    assert len(s) == n_file
    r = apply_both(dyg, oracle, G, H, Go, Ho, INS, s, d, w, wl.params, uid0=77)
    assert (r.status == MERGED).sum() >= 100
    assert (r.status == SELF_LOOP).sum() == 5


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [0, 41])
def test_gpu_delete_file_parity(dyg, oracle, chunk):
    wl = W.mesh_3d(10, inserts=500)
    rng = np.random.default_rng(12)
    gs = np.concatenate([wl.g_src, wl.ins_src])
    gd = np.concatenate([wl.g_dst, wl.ins_dst])
    gw = np.concatenate([wl.g_w, wl.ins_w])
    G, H, Go, Ho = both(dyg, oracle, wl.n, (gs, gd, gw), (wl.h_src, wl.h_dst, wl.h_w))
    pick = rng.choice(len(gs), 400, replace=False)
    hi = rng.choice(len(wl.h_src), 150, replace=False)   # make sure H edges are hit
    s = np.concatenate([gs[pick], wl.h_dst[hi], gs[pick[:20]], np.array([0, 1], np.uint32)])
    d = np.concatenate([gd[pick], wl.h_src[hi], gd[pick[:20]], np.array([999, 998], np.uint32)])
    r = apply_both(dyg, oracle, G, H, Go, Ho, DEL, s.astype(np.uint32), d.astype(np.uint32),
                   None, wl.dparams, uid0=5000, chunk=chunk)
    assert (r.status >= 1).sum() > 0 and (r.status == -3).sum() >= 20
    assert len(r.rec_src) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("slack,headroom,chunk", [(2, 0.5, 700), (0, 0.0, 300)])
def test_gpu_rmat_mixed_sequence(dyg, oracle, slack, headroom, chunk):
    """A mixed R-MAT stream file by file; tight arenas force the halt/resume
    path on both the G append and the per-chunk H appends."""
    wl = W.rmat_mixed(scale=11, n_updates=9000, file_size=1500, walkers=64)
    G, H, Go, Ho = both(dyg, oracle, wl.n, (wl.g_src, wl.g_dst, wl.g_w),
                        (wl.h_src, wl.h_dst, wl.h_w), slack=slack, headroom=headroom)
    uid = 0
    for op, s, d, w in wl.files:
        p = wl.dparams if op else wl.iparams
        apply_both(dyg, oracle, G, H, Go, Ho, op, s, d, w, p, uid0=uid, chunk=chunk)
        uid += len(s)


def two_hubs(N=600):
    """Hubs 0 and 1 joined to every leaf 2..N-1 (weight 1) in G and H; the
    hub-hub edge (0,1) (weight 100) in G only.  Every hub row is longer than
    the one-thread limit, so deletions, probes, moves and H-membership tests
    on them take the block-cooperative paths."""
    leaves = np.arange(2, N, dtype=np.uint32)
    hs = np.concatenate([np.zeros(N - 2, np.uint32), np.ones(N - 2, np.uint32)])
    hd = np.concatenate([leaves, leaves])
    hw = np.ones(len(hs), np.float32)
    gs = np.concatenate([hs, np.array([0], np.uint32)])
    gd = np.concatenate([hd, np.array([1], np.uint32)])
    gw = np.concatenate([hw, np.array([100.0], np.float32)])
    return N, (gs, gd, gw), (hs, hd, hw)


@pytest.mark.gpu
def test_gpu_long_rows(dyg, oracle):
    N, g, h = two_hubs()
    G, H, Go, Ho = both(dyg, oracle, N, g, h, slack=0, headroom=0.02)
    rng = np.random.default_rng(5)
    a = np.arange(2, 202, dtype=np.uint32)
    # deletions of hub edges: walks a -> 0 go through hub 1; a walker that
    # steps 1 -> 0 makes (1,0) a recovery candidate with two long H rows
    r = apply_both(dyg, oracle, G, H, Go, Ho, DEL, a, np.zeros(200, np.uint32), None,
                   params(walkers=64), uid0=0)
    assert (r.status >= 1).all()
    assert any((x, y) in ((0, 1), (1, 0)) for x, y in zip(r.rec_src, r.rec_dst))
    # insertions: the deleted hub edges come back (new in G: long-row G append),
    # existing hub edges merge (long-row probes), repeats fold; a low
    # threshold makes the walks fail so the hub row of H grows past its
    # capacity (long-row move)
    s = np.concatenate([a[:100], np.full(50, 1, np.uint32), a[:20]])
    d = np.concatenate([np.zeros(100, np.uint32), a[100:150], np.zeros(20, np.uint32)])
    w = rng.uniform(0.5, 2.0, len(s)).astype(np.float32)
    perm = rng.permutation(len(s))
    r = apply_both(dyg, oracle, G, H, Go, Ho, INS, s[perm], d[perm], w[perm],
                   params(threshold=0.5, walkers=64), uid0=1000, chunk=64)
    assert (r.status == -1).sum() >= 50 and (r.status == MERGED).sum() >= 70
    # the standalone decremental batch on the same long rows
    db = dyg.decremental_batch(G, H, a[100:180], np.zeros(80, np.uint32), params(walkers=64),
                               first_update_id=5000)
    st, cd, rx, ry, rk, _ = oracle.decremental(Go, Ho, a[100:180], np.zeros(80, np.uint32),
                                               params(walkers=64), first_uid=5000,
                                               single_batch=True)
    assert np.array_equal(db.status, st)
    assert np.array_equal(db.rec_src, rx) and np.array_equal(db.rec_dst, ry)
    same_graph(G, Go)
    same_graph(H, Ho)


@pytest.mark.gpu
@pytest.mark.parametrize("slack", [0, 2])
def test_gpu_long_tails(dyg, oracle, slack):
    """Appends of 100 and 300 edges to one row in one batch: the new tail is
    ordered by a warp (100) and by the leader alone (300); a threshold this
    low rejects every path longer than one step, so all are accepted."""
    N = 420
    ps = np.arange(N - 1, dtype=np.uint32)
    pd = ps + 1
    pw = np.ones(N - 1, np.float32)
    H = dyg.Graph.from_edges(N, ps, pd, pw, slack_per_row=slack, arena_headroom=0.1)
    Ho = oracle.OGraph(N, ps, pd, pw)
    p = params(threshold=1e-3, walkers=32)
    uid = 0
    for s, d in [(np.zeros(100, np.uint32), np.arange(2, 102, dtype=np.uint32)),
                 (np.arange(102, 402, dtype=np.uint32), np.zeros(300, np.uint32)),
                 (np.full(36, 1, np.uint32), np.arange(404, 440, dtype=np.uint32) % N),
                 (np.full(6, 3, np.uint32), np.arange(300, 306, dtype=np.uint32))]:
        w = np.linspace(0.5, 2.0, len(s)).astype(np.float32)
        r = dyg.incremental_batch(H, s, d, w, p, first_update_id=uid)
        fa, cd, ac, _ = oracle.incremental(Ho, s, d, w, p, first_uid=uid, single_batch=True)
        assert np.array_equal(r.found_at, fa) and np.array_equal(r.accepted, ac)
        same_graph(H, Ho)
        uid += len(s)
    assert rows(H.export())[0][0] == (1, 1.0) and len(rows(H.export())[0]) == 401
