"""Bit-exact parity at the benchmarked sizes.

The 3-D mesh at 100^3 (1,000,000 vertices, 2,970,000 edges): the whole
benchmark step, 200,000 insertions in 10 batches of 20,000 (walking H, every
insertion also entering G) and then all 317,000 deletions in 10 batches of
31,700, through the C ABI against the CPU oracle: found_at, conductance bits,
accepted flags, deletion statuses, recovered edges in commit order, and every
row of the final G and H (ids and weight bits).  Row order after thousands of
arena moves and 31,700-edge deletion batches is where a scale-dependent
defect would show.

R-MAT scale 20 (645,911 vertices after the largest component, hub rows of up
to 64,772 slots): the first four files of the mixed stream (three insertion
files with weight merges, then a deletion file), file by file, with the same
comparisons.  Hub rows drive the block-cooperative row kernels.
"""
import time

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


def same_graph(g_dev, g_orc, what):
    rp1, c1, w1 = g_dev.export()
    rp2, c2, w2 = g_orc.export()
    assert np.array_equal(rp1, rp2), f"{what}: row lengths differ"
    assert np.array_equal(c1, c2), f"{what}: row contents or order differ"
    assert np.array_equal(w1.view(np.uint32), w2.view(np.uint32)), f"{what}: weights differ"


def test_mesh100_full_step(dyg, oracle):
    wl = W.mesh_3d(100)
    assert (wl.n, len(wl.g_src), len(wl.ins_src), len(wl.del_src)) == (1_000_000, 2_970_000,
                                                                         200_000, 317_000)
    H = dyg.Graph.from_edges(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    G = dyg.Graph.from_edges(wl.n, wl.g_src, wl.g_dst, wl.g_w)
    Ho = oracle.OGraph(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    Go = oracle.OGraph(wl.n, wl.g_src, wl.g_dst, wl.g_w)

    t0 = time.time()
    r = dyg.incremental_stream(H, wl.ins_src, wl.ins_dst, wl.ins_w, wl.params, G=G)
    fa, cd, ac, _ = oracle.incremental(Ho, wl.ins_src, wl.ins_dst, wl.ins_w, wl.params, G=Go)
    assert np.array_equal(r.found_at, fa)
    assert np.array_equal(r.conductance.view(np.uint32), cd.view(np.uint32))
    assert np.array_equal(r.accepted, ac)
    assert 100_000 < int(ac.sum()) < 160_000
    same_graph(H, Ho, "H after insertions")
    same_graph(G, Go, "G after insertions")

    d = dyg.decremental_stream(G, H, wl.del_src, wl.del_dst, wl.dparams)
    st, cd2, rx, ry, rk, _ = oracle.decremental(Go, Ho, wl.del_src, wl.del_dst, wl.dparams)
    assert np.array_equal(d.status, st)
    assert np.array_equal(d.conductance.view(np.uint32), cd2.view(np.uint32))
    assert np.array_equal(d.rec_src, rx) and np.array_equal(d.rec_dst, ry)
    assert np.array_equal(d.rec_kind, rk)
    assert int((st > 0).sum()) > 50_000 and len(rx) > 100_000
    same_graph(H, Ho, "H after deletions")
    same_graph(G, Go, "G after deletions")
    print(f"mesh 100^3 full step: {int(ac.sum())} insertions added, {int((st > 0).sum())} "
          f"deletions walked, {len(rx)} edges recovered ({time.time() - t0:.1f} s)")


def test_rmat20_first_files(dyg, oracle):
    wl = W.rmat_mixed(scale=20, n_updates=4 * 4096)
    ops = [f[0] for f in wl.files]
    assert ops == [dyg.STREAM_INSERT] * 3 + [dyg.STREAM_DELETE]
    deg = np.bincount(np.concatenate([wl.g_src, wl.g_dst]))
    assert deg.max() > 60_000
    G = dyg.Graph.from_edges(wl.n, wl.g_src, wl.g_dst, wl.g_w)
    H = dyg.Graph.from_edges(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    Go = oracle.OGraph(wl.n, wl.g_src, wl.g_dst, wl.g_w)
    Ho = oracle.OGraph(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    uid = 0
    for i, (op, s, d, w) in enumerate(wl.files):
        p = wl.iparams if op == dyg.STREAM_INSERT else wl.dparams
        r = dyg.stream_file(G, H, op, s, d, w, p, first_update_id=uid)
        st, cd, rx, ry, rk, _ = oracle.stream_file(Go, Ho, op, s, d, w, p, first_uid=uid)
        assert np.array_equal(r.status, st), f"file {i}: statuses differ"
        assert np.array_equal(r.conductance.view(np.uint32), cd.view(np.uint32))
        assert np.array_equal(r.rec_src, rx) and np.array_equal(r.rec_dst, ry)
        assert np.array_equal(r.rec_kind, rk)
        uid += len(s)
    same_graph(G, Go, "G after four files")
    same_graph(H, Ho, "H after four files")
