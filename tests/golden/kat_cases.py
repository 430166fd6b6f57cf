"""Known-answer cases for the update path.

Each case is a tiny dataset in the reference's file layout whose outcome does
not depend on the random stream: walkers start at a leaf or move on vertices
of degree 2, where the non-backtracking rule leaves one choice
(random_walk_incremental/main.cu:126-137), or every random choice leads to
the same decision with overwhelming probability (both directions of a cycle
are taken by ~256 of 512 walkers each).  So the same decisions must come out
of the reference's cuRAND updater, the Philox oracle and the CUDA path.

Incremental case = (adj_sparse lines 0-based, ext lines 1-based, threshold,
walkers); decremental case = (updated_dense, updated_adj_sparse, del lines,
all 1-based).  `expect` holds the decisions derived by hand from the
reference's stop rules.
"""
from __future__ import annotations


def _path(n, w=1.0, base=0, off=0):
    return [(off + i + base, off + i + 1 + base, w) for i in range(n - 1)]


def _cycle(n, w=1.0, base=0, off=0):
    return [(off + i + base, off + (i + 1) % n + base, w) for i in range(n)]


INCREMENTAL = {
    # distortion boundary: the walk fails when R * w_e >= threshold
    # (main.cu:144), checked before the target test (main.cu:149).
    "path_threshold": {
        "adj_sparse": _path(12),
        "ext": [(1, 5, 2.0), (1, 6, 2.0), (12, 7, 2.0), (12, 8, 2.4)],
        "threshold": 10.0, "walkers": 512,
        # 4 edges -> batches of 1.  (0,4): R=4, 8 < 10 found at step 4.
        # (0,5): R=5, 10 >= 10 fails -> added.  (11,6): R=5 -> added.
        # (11,7): found; the best walker uses the edge (11,6) added one batch
        # earlier: 11 -> 6 -> 7, R = 0.5 + 1, found at step 2.
        "expect_added": [0, 1, 1, 0],
        "expect_found_at": [4, -1, -1, 2],
    },
    # max_steps = 100: the loop runs while step < 100 (main.cu:116), so a
    # target 99 hops away is found and one 100 hops away is not.
    "path_max_steps": {
        "adj_sparse": _path(102),
        "ext": [(1, 100, 1.0), (1, 101, 1.0)],
        "threshold": 1e30, "walkers": 512,
        "expect_added": [0, 1],
        "expect_found_at": [99, -1],
    },
    # both directions of a cycle; the second edge duplicates the first one,
    # which the first batch added, so it is found at step 1.
    "cycle_two_ways": {
        "adj_sparse": _cycle(10),
        "ext": [(1, 6, 1.25), (1, 6, 1.0)],
        "threshold": 6.0, "walkers": 512,
        "expect_added": [1, 0],
        "expect_found_at": [-1, 1],
    },
    # snapshot semantics: 12 edges -> batches of 2.  (0,15) and (0,16) are in
    # the same batch and both fail (R reaches 12 first), so both are added
    # even though (0,16) would be found through (0,15) if batches were
    # sequential; (0,17) in the next batch is found through them.  The rest
    # are existing edges on a second path, found at step 1.
    "snapshot": {
        "adj_sparse": _path(21) + _path(20, off=21),
        "ext": [(1, 16, 1.0), (1, 17, 1.0), (1, 18, 1.0)] + [(22 + i, 23 + i, 1.0) for i in range(9)],
        "threshold": 12.0, "walkers": 512,
        "expect_added": [1, 1, 0] + [0] * 9,
    },
    # walkers counts that are not powers of two are reduced correctly
    # (the reference's tree is only correct for powers of two, main.cu:183;
    # with 96 walkers at a leaf every walker succeeds, so it still agrees).
    "walkers_96": {
        "adj_sparse": _path(12),
        "ext": [(1, 5, 2.0), (12, 8, 2.4)],
        "threshold": 10.0, "walkers": 96,
        "expect_added": [0, 0],
    },
}


def _decr_cycles(k, n, base=1):
    """k disjoint cycles of n vertices; H = each cycle minus its edge (n-1, 0)."""
    dense, sparse = [], []
    for c in range(k):
        cyc = _cycle(n, base=base, off=c * n)
        dense += cyc
        sparse += cyc[:-1]
    return dense, sparse


def _with_guard(dense, sparse):
    """Adds a disconnected edge on the two largest ids (the reference sizes its
    decremental arrays by the largest 0-based id, which drops the last vertex,
    random_walk_decremental/functions.cpp:123; a vertex nothing walks to keeps
    its runs in bounds).  The largest 0-based id is kept != 2 mod 4."""
    top = max(max(a, b) for a, b, _ in dense + sparse)
    a = top + 1
    while (a + 1 - 1) % 4 == 2:
        a += 1
    g = (a, a + 1, 1.0)
    return dense + [g], sparse + [g]


_d1, _s1 = _with_guard(*_decr_cycles(1, 12))
_d2, _s2 = _with_guard(*_decr_cycles(12, 8))

DECREMENTAL = {
    # deleting (1,2) of a 12-cycle whose sparsifier lacks (12,1): the only
    # path 1 -> 12 -> 11 ... -> 2 uses (12,1), which is recovered.
    "cycle_recover": {
        "updated_dense": _d1, "updated_adj_sparse": _s1,
        "del": [(1, 2)],
        "expect_added": [(1, 12)],
    },
    # 12 cycles, one deletion each -> batches of 2; each recovers its
    # cycle's missing edge.
    "cycles_batches": {
        "updated_dense": _d2, "updated_adj_sparse": _s2,
        "del": [(c * 8 + 2, c * 8 + 3) for c in range(12)],
        "expect_added": [(c * 8 + 1, c * 8 + 8) for c in range(12)],
    },
}


def write_incremental(case: dict, dirpath: str) -> None:
    import os
    os.makedirs(dirpath, exist_ok=True)
    with open(os.path.join(dirpath, "adj_sparse.mtx"), "w") as f:
        for a, b, w in case["adj_sparse"]:
            f.write(f"{a} {b} {w:g}\n")
    with open(os.path.join(dirpath, "ext.mtx"), "w") as f:
        for a, b, w in case["ext"]:
            f.write(f"{a} {b} {w:g}\n")


def write_decremental(case: dict, dirpath: str) -> None:
    import os
    os.makedirs(dirpath, exist_ok=True)
    for key in ("updated_dense", "updated_adj_sparse"):
        with open(os.path.join(dirpath, key + ".mtx"), "w") as f:
            for a, b, w in case[key]:
                f.write(f"{a} {b} {w:g}\n")
    with open(os.path.join(dirpath, "del.mtx"), "w") as f:
        for a, b in case["del"]:
            f.write(f"{a} {b}\n")


def n_vertices_incremental(case: dict) -> int:
    m = max(max(a, b) for a, b, _ in case["adj_sparse"]) + 1
    e = max(max(a, b) for a, b, _ in case["ext"])   # 1-based
    return max(m, e)


def n_vertices_decremental(case: dict) -> int:
    return max(max(a, b) for a, b, _ in case["updated_dense"] + case["updated_adj_sparse"])
