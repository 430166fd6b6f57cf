"""Evaluation of an updated sparsifier, replacing the reference's Julia
driver (dyGRASS.jl:279-370 incremental_test, 467-549 decremental_test):
condition number kappa(L_G, L_H) and density |E_H| / |V|, computed by the
native dyg_kappa (include/dyg_eval.h).

The reference's decremental updater writes only the edges it added
(added_edges.mtx), so its driver rebuilds the final graphs from the files
(dyGRASS.jl:467-541): final G = updated dense graph minus the deletions,
final H = updated sparsifier minus the deletions plus the added edges, each
with its weight in the final G.  `reconstruct_final` restates that.

    python -m dygrass_b200.evaluate incremental <graph> [--dataset-dir ../dataset]
    python -m dygrass_b200.evaluate decremental <graph> [--dataset-dir ../dataset]
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import DygError, kappa, lib


def _read(path: str, offset: int, weighted: bool):
    """An edge file with the reference's per-file index base (dyg_mtx_read)."""
    import ctypes as C
    m = C.c_uint64()
    ps, pd, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    mx = C.c_uint32()
    st = lib().dyg_mtx_read(os.fsencode(path), offset, 1 if weighted else 0, C.byref(m),
                            C.byref(ps), C.byref(pd), C.byref(pw) if weighted else None,
                            C.byref(mx))
    if st != 0:
        raise DygError(st, "dyg_mtx_read", lib().dyg_last_error_string().decode())
    k = m.value
    try:
        s = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        d = np.ctypeslib.as_array(C.cast(pd, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        w = (np.ctypeslib.as_array(C.cast(pw, C.POINTER(C.c_float)), (max(k, 1),))[:k].copy()
             if weighted else np.ones(k, np.float32))
    finally:
        for p in (ps, pd, pw):
            if p:
                lib().dyg_mtx_free(p)
    return s, d, w


def _keyed(s, d, w) -> dict:
    """Edge -> weight, keyed (min, max); a later line overrides an earlier one
    (Julia's Dict comprehension)."""
    return {(min(int(a), int(b)), max(int(a), int(b))): np.float32(x) for a, b, x in zip(s, d, w)}


def _arrays(dct: dict):
    if not dct:
        return np.empty(0, np.uint32), np.empty(0, np.uint32), np.empty(0, np.float32)
    k = np.array(list(dct.keys()), np.uint32)
    return k[:, 0].copy(), k[:, 1].copy(), np.array(list(dct.values()), np.float32)


def reconstruct_final(g_edges, h_edges, del_edges, added_edges):
    """Final G and H after a decremental run (dyGRASS.jl:478-541).  Each
    argument is (src, dst[, w]); returns ((gs, gd, gw), (hs, hd, hw)).
    Deletions absent from G or H are skipped; an added edge takes its weight
    in the final G and is skipped if G lacks it."""
    G = _keyed(*g_edges)
    H = _keyed(*h_edges)
    for a, b in zip(*del_edges[:2]):
        k = (min(int(a), int(b)), max(int(a), int(b)))
        G.pop(k, None)
        H.pop(k, None)
    for a, b in zip(*added_edges[:2]):
        k = (min(int(a), int(b)), max(int(a), int(b)))
        if k in G:
            H[k] = G[k]
    return _arrays(G), _arrays(H)


def _nv(*edge_lists) -> int:
    m = 0
    for s, d, *_ in edge_lists:
        if len(s):
            m = max(m, int(s.max()) + 1, int(d.max()) + 1)
    return m


def incremental_eval(dataset_dir: str, graph: str, **opts) -> dict:
    """kappa and density of updated_adj_sparse.mtx against dense.mtx + ext.mtx
    (dyGRASS.jl:294-370): adj_sparse.mtx is 0-based, the others 1-based."""
    base = os.path.join(dataset_dir, graph)
    h0 = _read(os.path.join(base, "adj_sparse.mtx"), 0, True)
    g0 = _read(os.path.join(base, "dense.mtx"), 1, True)
    ext = _read(os.path.join(base, "ext.mtx"), 1, True)
    hu = _read(os.path.join(base, "updated_adj_sparse.mtx"), 1, True)
    g = tuple(np.concatenate([a, b]) for a, b in zip(g0, ext))
    n = _nv(h0, g, hu)
    out = {"vertices": n, "original": kappa(n, *g0, *h0, **opts),
           "updated": kappa(n, *g, *hu, **opts)}
    return out


def decremental_eval(dataset_dir: str, graph: str, **opts) -> dict:
    """kappa and density of the final sparsifier rebuilt from
    updated_dense.mtx, updated_adj_sparse.mtx, del.mtx and added_edges.mtx
    (dyGRASS.jl:467-549; all 1-based)."""
    base = os.path.join(dataset_dir, graph)
    g = _read(os.path.join(base, "updated_dense.mtx"), 1, True)
    h = _read(os.path.join(base, "updated_adj_sparse.mtx"), 1, True)
    dl = _read(os.path.join(base, "del.mtx"), 1, False)
    ad = _read(os.path.join(base, "added_edges.mtx"), 1, False)
    (gs, gd, gw), (hs, hd, hw) = reconstruct_final(g, h, dl, ad)
    n = _nv(g, h)
    return {"vertices": n, "final": kappa(n, gs, gd, gw, hs, hd, hw, **opts),
            "final_h_edges": len(hs)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("mode", choices=["incremental", "decremental"])
    ap.add_argument("graph")
    ap.add_argument("--dataset-dir", default="../dataset")
    a = ap.parse_args(argv)
    fn = incremental_eval if a.mode == "incremental" else decremental_eval
    print(json.dumps(fn(a.dataset_dir, a.graph)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
