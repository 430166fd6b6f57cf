"""Shared helpers for the tests: case loading in the reference's file
conventions and the reference's output-file format."""
from __future__ import annotations

import numpy as np


def incr_inputs(case):
    """(n, H0 src/dst/w 0-based in file order, ext src/dst/w 0-based)."""
    from kat_cases import n_vertices_incremental
    n = n_vertices_incremental(case)
    h = np.array([(a, b) for a, b, _ in case["adj_sparse"]], np.uint32).reshape(-1, 2)
    hw = np.array([w for _, _, w in case["adj_sparse"]], np.float32)
    # ext.mtx is 1-based (random_walk_incremental/functions.cpp:319, 328)
    e = np.array([(a - 1, b - 1) for a, b, _ in case["ext"]], np.uint32).reshape(-1, 2)
    ew = np.array([w for _, _, w in case["ext"]], np.float32)
    return n, h[:, 0].copy(), h[:, 1].copy(), hw, e[:, 0].copy(), e[:, 1].copy(), ew


def decr_inputs(case):
    from kat_cases import n_vertices_decremental
    n = n_vertices_decremental(case)
    g = np.array([(a - 1, b - 1) for a, b, _ in case["updated_dense"]], np.uint32)
    gw = np.array([w for _, _, w in case["updated_dense"]], np.float32)
    h = np.array([(a - 1, b - 1) for a, b, _ in case["updated_adj_sparse"]], np.uint32)
    hw = np.array([w for _, _, w in case["updated_adj_sparse"]], np.float32)
    d = np.array([(a - 1, b - 1) for a, b in case["del"]], np.uint32).reshape(-1, 2)
    return (n, g[:, 0].copy(), g[:, 1].copy(), gw, h[:, 0].copy(), h[:, 1].copy(), hw,
            d[:, 0].copy(), d[:, 1].copy())


def updated_sparse_text(h_src, h_dst, h_w, e_src, e_dst, e_w, accepted) -> str:
    """updated_adj_sparse.mtx as the reference writes it: the original lines,
    then the added edges in input order, ids + 1, weights in ostream's
    default format (random_walk_incremental/gpu_graph.cuh:433-446)."""
    out = [f"{a + 1} {b + 1} {float(w):g}" for a, b, w in zip(h_src, h_dst, h_w)]
    out += [f"{a + 1} {b + 1} {float(w):g}" for a, b, w, k in zip(e_src, e_dst, e_w, accepted) if k]
    return "\n".join(out) + ("\n" if out else "")


def edge_set(src, dst):
    return {(min(int(a), int(b)), max(int(a), int(b))) for a, b in zip(src, dst)}
