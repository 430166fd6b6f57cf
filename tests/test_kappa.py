"""kappa(L_G, L_H), density and PCG iterations (include/dyg_eval.h) against
scipy's generalized eigensolvers, and the final-graph reconstruction of the
reference's decremental evaluation (dyGRASS.jl:467-541)."""
import numpy as np
import pytest
import scipy.linalg as sl
import scipy.sparse as sp
import scipy.sparse.linalg as sla

import dygrass_b200 as dyg
from dygrass_b200 import workloads as W
from dygrass_b200.evaluate import reconstruct_final


def lap(n, s, d, w, off=1e-6, dense=True):
    m = s != d
    s, d, w = s[m], d[m], np.asarray(w, np.float64)[m]
    A = sp.coo_matrix((np.concatenate([w, w]), (np.concatenate([s, d]), np.concatenate([d, s]))),
                      shape=(n, n)).tocsr()
    L = sp.diags(np.asarray(A.sum(axis=1)).ravel() + off) - A
    return L.toarray() if dense else L.tocsc()


def test_grid_matches_dense_eigensolver():
    wl = W.grid_2d(12, 12, inserts=10)
    A = lap(wl.n, wl.g_src, wl.g_dst, wl.g_w)
    B = lap(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    want = sl.eigh(A, B, eigvals_only=True).max()
    r = dyg.kappa(wl.n, wl.g_src, wl.g_dst, wl.g_w, wl.h_src, wl.h_dst, wl.h_w)
    assert r["kappa"] == pytest.approx(want, rel=1e-9)
    assert r["density"] == pytest.approx(len(wl.h_src) / wl.n)
    assert r["pcg_relres"] <= 1e-8 and 0 < r["pcg_iters"] < 200


def test_random_graph_tree_sparsifier():
    rng = np.random.default_rng(3)
    n = 300
    s = rng.integers(0, n, 2000).astype(np.uint32)
    d = rng.integers(0, n, 2000).astype(np.uint32)
    s = np.concatenate([s, np.arange(n - 1, dtype=np.uint32)])
    d = np.concatenate([d, np.arange(1, n, dtype=np.uint32)])   # connected
    w = rng.uniform(0.1, 10, len(s)).astype(np.float32)
    idx = W.sparsifier(n, s, d, w, 0.02, 5)
    A = lap(n, s, d, w)
    B = lap(n, s[idx], d[idx], w[idx])
    want = sl.eigh(A, B, eigvals_only=True).max()
    r = dyg.kappa(n, s, d, w, s[idx], d[idx], w[idx])
    assert r["kappa"] == pytest.approx(want, rel=1e-9)


def test_mesh_matches_sparse_eigsh():
    wl = W.mesh_3d(14, inserts=200)
    A = lap(wl.n, wl.g_src, wl.g_dst, wl.g_w, dense=False)
    B = lap(wl.n, wl.h_src, wl.h_dst, wl.h_w, dense=False)
    want = sla.eigsh(A, k=1, M=B, which="LA", tol=1e-12)[0][0]
    r = dyg.kappa(wl.n, wl.g_src, wl.g_dst, wl.g_w, wl.h_src, wl.h_dst, wl.h_w)
    assert r["kappa"] == pytest.approx(want, rel=1e-7)


def test_identical_graphs():
    wl = W.grid_2d(10, 10, inserts=5)
    r = dyg.kappa(wl.n, wl.g_src, wl.g_dst, wl.g_w, wl.g_src, wl.g_dst, wl.g_w)
    assert r["kappa"] == pytest.approx(1.0, rel=1e-9)
    assert r["pcg_iters"] <= 2


def test_bad_input():
    s = np.array([0, 1], np.uint32)
    d = np.array([1, 5], np.uint32)
    w = np.ones(2, np.float32)
    with pytest.raises(dyg.DygError):
        dyg.kappa(3, s, d, w, s[:1], d[:1], w[:1])
    with pytest.raises(dyg.DygError):
        dyg.kappa(3, s[:1], d[:1], -w[:1], s[:1], d[:1], w[:1])


def test_reconstruct_final():
    """dyGRASS.jl:478-541: deletions leave G and H; added edges enter H with
    their weight in G; an added edge missing from G is skipped."""
    g = (np.array([0, 1, 2, 0], np.uint32), np.array([1, 2, 3, 3], np.uint32),
         np.array([1.0, 2.0, 3.0, 4.0], np.float32))
    h = (np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32),
         np.array([1.0, 2.0, 3.0], np.float32))
    dl = (np.array([1], np.uint32), np.array([0], np.uint32))
    ad = (np.array([3, 1], np.uint32), np.array([0, 0], np.uint32))
    (gs, gd, gw), (hs, hd, hw) = reconstruct_final(g, h, dl, ad)
    assert sorted(zip(gs.tolist(), gd.tolist(), gw.tolist())) == [(0, 3, 4.0), (1, 2, 2.0),
                                                                 (2, 3, 3.0)]
    assert sorted(zip(hs.tolist(), hd.tolist(), hw.tolist())) == [(0, 3, 4.0), (1, 2, 2.0),
                                                                 (2, 3, 3.0)]
