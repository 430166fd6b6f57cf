"""Agreement with the reference's own updaters (built from their sources into
oracle/_ref by `make -C oracle ref-gpu`) on the same input files.

The reference draws its walks from cuRAND and this implementation from
Philox, so single decisions differ; what must agree is the outcome: the
number of edges added, their overlap, and the condition number
kappa(L_G, L_H) of the updated sparsifier (computed by dyg_kappa for both).
kappa is a maximum over edges, set by the few heaviest edges a run happens to
leave out, so one run is one sample: this implementation runs with three
seeds and its median is compared (e.g. the 30^3 mesh below gives 99.65 for
six seeds through the library and 140.6 for the command-line default seed;
the reference gives 99.65).  Stated tolerance: added-edge counts within 15 %,
kappa of the reference within 10 % of the median of ours.

The inputs are the grid configuration (100x100, 1,000 insertions, threshold
10) and a 30^3 mesh with 6,000 insertions (threshold 100), both inside the
reference's room for grown rows: it allocates edge_count * 4 * 2 floats and
moves a row into the second half each time it grows
(random_walk_incremental/gpu_graph.cuh:210, 357-384), with no bound check, so
past a few thousand accepted edges on the mesh its rows are written beyond the
allocation and its device copy misses them (its teardown then aborts in
munmap_chunk).  Deletions run on
a 20^3 mesh with 2,000 insertions in G: 1,000 sparsifier edges, ten batches
of 100.  Every deletion is a sparsifier edge because the reference's walk
kernel reads a batch's targets at (block + number of walked edges) while they
are stored at (block + batch size) (random_walk_decremental/main.cu:94,
417-420; gpu_graph.cuh:453-454), which agree only when every deletion of the
batch is walked; with dense-only deletions mixed in it stops on its own
assertion after its first batch.  Its added_edges.mtx holds path edges only
(gpu_graph.cuh:533-538; fallback edges are not kept), so ours runs with
--path-edges-only.  Which sparsifier edges come back varies from run to run as
much between two seeds of ours as between ours and the reference, and so
does kappa (one run of each is one sample of a maximum), so the deletion
test runs nine seeds and asks that the reference's overlap with ours be at
least 0.85 of the median overlap between our seeds and that its kappa lie
within the range of ours.  The reference's decremental
vertex count leaves out the largest id (random_walk_decremental/
functions.cpp:123), so an extra isolated pair of vertices, never walked,
takes the largest ids.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from dygrass_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
OURS = os.path.join(ROOT, "dygrass_b200", "bin")


def need(name):
    path = os.path.join(REF, name)
    if not os.path.exists(path):
        pytest.skip(f"the reference's {name} is not built (make -C oracle ref-gpu)")
    return path


def write(path, s, d, w=None, base=1):
    with open(path, "w") as f:
        for i in range(len(s)):
            f.write(f"{s[i] + base} {d[i] + base}" + ("" if w is None else f" {float(w[i]):.9g}") + "\n")


def read_lines(path):
    out = []
    for ln in open(path):
        p = ln.split()
        if len(p) >= 2:
            out.append((int(p[0]), int(p[1]), float(p[2]) if len(p) > 2 else 1.0))
    return out


def run(binary, args, cwd):
    cp = subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=600)
    return cp


def key(a, b):
    return (min(a, b), max(a, b))


def kappa_of(n, g, h):
    import dygrass_b200 as dyg
    arr = lambda e: (np.array([x[0] for x in e], np.uint32), np.array([x[1] for x in e], np.uint32),
                     np.array([x[2] for x in e], np.float32))
    return dyg.kappa(n, *arr(g), *arr(h))["kappa"]


@pytest.mark.parametrize("case", ["grid", "mesh"])
def test_incremental_agrees_with_reference(tmp_path, case):
    binary = need("incremental_update")
    if case == "grid":
        wl = W.grid_2d(100, 100, inserts=1000)
        thr, walkers = 10.0, 512
    else:
        wl = W.mesh_3d(30, inserts=6000)
        thr, walkers = 100.0, 512
    added = {}
    runs = [("ref", binary, [])] + [(f"ours{k}", os.path.join(OURS, "incremental_update"),
                                     [f"--seed={sd}"]) for k, sd in enumerate((20251203, 1, 2))]
    for who, exe, extra in runs:
        ds = tmp_path / who / "dataset" / case
        ds.mkdir(parents=True)
        write(ds / "adj_sparse.mtx", wl.h_src, wl.h_dst, wl.h_w, base=0)
        write(ds / "ext.mtx", wl.ins_src, wl.ins_dst, wl.ins_w, base=1)
        rd = tmp_path / who / "run"
        rd.mkdir()
        cp = run(exe, [case, repr(thr), str(walkers)] + extra, rd)
        # the reference's teardown can abort after its work is done and its
        # file written (munmap_chunk in the gpu_graph destructor)
        assert cp.returncode == 0 or (who == "ref" and "completed successfully" in cp.stdout), \
            (who, cp.stdout[-500:], cp.stderr[-500:])
        lines = read_lines(ds / "updated_adj_sparse.mtx")
        assert len(lines) >= len(wl.h_src)
        added[who] = lines[len(wl.h_src):]
    g = [(a, b, float(x)) for a, b, x in zip(np.concatenate([wl.g_src, wl.ins_src]),
                                               np.concatenate([wl.g_dst, wl.ins_dst]),
                                               np.concatenate([wl.g_w, wl.ins_w]))]
    h0 = list(zip(wl.h_src.tolist(), wl.h_dst.tolist(), wl.h_w.astype(float).tolist()))
    to0 = lambda e: [(a - 1, b - 1, w) for a, b, w in e]
    ra = {key(a, b) for a, b, _ in added["ref"]}
    assert len(ra) > 0
    k_ref = kappa_of(wl.n, g, h0 + to0(added["ref"]))
    ks, jacs = [], []
    for who in ("ours0", "ours1", "ours2"):
        oa = {key(a, b) for a, b, _ in added[who]}
        assert abs(len(oa) - len(ra)) <= 0.15 * len(ra), (who, len(oa), len(ra))
        jacs.append(len(ra & oa) / len(ra | oa))
        ks.append(kappa_of(wl.n, g, h0 + to0(added[who])))
    k_med = float(np.median(ks))
    print(f"\n{case}: added ref {len(ra)} ours {[len(added[w]) for w in ('ours0', 'ours1', 'ours2')]} "
          f"jaccard {np.round(jacs, 3).tolist()} kappa ref {k_ref:.3f} ours {np.round(ks, 3).tolist()}")
    assert min(jacs) >= 0.5, jacs
    assert abs(k_med - k_ref) <= 0.10 * k_ref, (ks, k_ref)


def test_decremental_agrees_with_reference(tmp_path):
    import dygrass_b200 as dyg
    from dygrass_b200.evaluate import reconstruct_final
    binary = need("decremental_update")
    wl = W.mesh_3d(20, inserts=2000)
    gs = np.concatenate([wl.g_src, wl.ins_src, [wl.n]]).astype(np.uint32)
    gd = np.concatenate([wl.g_dst, wl.ins_dst, [wl.n + 1]]).astype(np.uint32)
    gw = np.concatenate([wl.g_w, wl.ins_w, [1.0]]).astype(np.float32)
    hs = np.concatenate([wl.h_src, [wl.n]]).astype(np.uint32)
    hd = np.concatenate([wl.h_dst, [wl.n + 1]]).astype(np.uint32)
    hw = np.concatenate([wl.h_w, [1.0]]).astype(np.float32)
    pick = np.random.default_rng(8).choice(len(wl.h_src), 1000, replace=False)
    del_s, del_d = wl.h_src[pick].astype(np.uint32), wl.h_dst[pick].astype(np.uint32)
    added = {}
    runs = [("ref", binary, [])] + [(f"ours{k}", os.path.join(OURS, "decremental_update"),
                                     ["--path-edges-only", f"--seed={sd}"])
                                    for k, sd in enumerate((20251203,) + tuple(range(1, 9)))]
    for who, exe, extra in runs:
        ds = tmp_path / who / "dataset" / "mesh20"
        ds.mkdir(parents=True)
        write(ds / "updated_dense.mtx", gs, gd, gw)
        write(ds / "updated_adj_sparse.mtx", hs, hd, hw)
        write(ds / "del.mtx", del_s, del_d)
        rd = tmp_path / who / "run"
        rd.mkdir()
        cp = run(exe, ["mesh20"] + extra, rd)
        assert "Added edges saved to" in cp.stdout and (cp.returncode == 0 or who == "ref"), \
            (who, cp.stdout[-500:], cp.stderr[-500:])
        added[who] = {key(a - 1, b - 1) for a, b, _ in read_lines(ds / "added_edges.mtx")}
    n = wl.n + 2
    ks = {}
    for who, e in added.items():
        ed = sorted(e)
        (g1, h1) = reconstruct_final((gs, gd, gw), (hs, hd, hw), (del_s, del_d),
                                     (np.array([x for x, _ in ed], np.uint32),
                                      np.array([y for _, y in ed], np.uint32)))
        ks[who] = dyg.kappa(n, *g1, *h1)["kappa"]
    seeds = [w for w in added if w != "ref"]
    jac = lambda x, y: len(x & y) / len(x | y)
    j_ref = [jac(added[w], added["ref"]) for w in seeds]
    j_own = [jac(added[x], added[y]) for i, x in enumerate(seeds) for y in seeds[i + 1:]]
    ours = sorted(ks[w] for w in seeds)
    print(f"\ndecremental: added ref {len(added['ref'])} ours {[len(added[w]) for w in seeds]} "
          f"jaccard vs ref median {np.median(j_ref):.3f}, between seeds median {np.median(j_own):.3f} "
          f"kappa ref {ks['ref']:.1f} ours {np.round(ours, 1).tolist()}")
    assert len(added["ref"]) > 0
    for w in seeds:
        assert abs(len(added[w]) - len(added["ref"])) <= 0.15 * len(added["ref"]), (w, len(added[w]))
    assert np.median(j_ref) >= 0.85 * np.median(j_own), (j_ref, j_own)
    assert ours[0] <= ks["ref"] <= ours[-1], (ours, ks["ref"])
