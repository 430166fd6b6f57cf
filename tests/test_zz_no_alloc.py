"""dyg_incremental_walk_noalloc: the incremental walk decision for callers
that cannot allocate device memory (a serving loop that reserves its memory
at start-up and forbids cudaMalloc afterwards, or a plugin whose host
framework owns all device allocations).  Called through the C ABI, twice in
a row, its outputs must equal those of dyg_incremental_batch on the same
sparsifier snapshot and update ids, bit for bit (the tolerance every parity
test here uses).  Collected last so that a failure here comes after every
other test has run; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_incremental_batch_twice():
    import torch
    import dygrass_b200 as dyg
    import dygrass_b200.workloads as wl

    assert torch.cuda.is_available()
    W = wl.grid_2d()                       # 100x100 grid, 1,000 insertions
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    dev = torch.device("cuda:0")
    L = dyg.lib()
    for call, (b0, b1) in enumerate([(0, 400), (400, 1000)]):
        s = torch.from_numpy(W.ins_src[b0:b1].view(np.int32)).to(dev)
        d = torch.from_numpy(W.ins_dst[b0:b1].view(np.int32)).to(dev)
        w = torch.from_numpy(W.ins_w[b0:b1]).to(dev)
        n = b1 - b0
        fa = torch.full((n,), -7, dtype=torch.int32, device=dev)
        cd = torch.full((n,), -7.0, dtype=torch.float32, device=dev)
        ac = torch.full((n,), 7, dtype=torch.uint8, device=dev)
        rc = L.dyg_incremental_walk_noalloc(H.handle, s.data_ptr(), d.data_ptr(), w.data_ptr(), n,
                                            b0, C.byref(W.params), fa.data_ptr(), cd.data_ptr(),
                                            ac.data_ptr(), None)
        assert rc == 0, L.dyg_last_error_string()
        torch.cuda.synchronize()
        # the existing entry point on a copy of the same snapshot
        Hc = H.clone()
        ref = dyg.incremental_batch(Hc, W.ins_src[b0:b1], W.ins_dst[b0:b1], W.ins_w[b0:b1],
                                    W.params, first_update_id=b0)
        Hc.close()
        assert np.array_equal(fa.cpu().numpy(), ref.found_at), call
        assert np.array_equal(cd.cpu().numpy().view(np.uint32), ref.conductance.view(np.uint32)), call
        assert np.array_equal(ac.cpu().numpy(), ref.accepted), call
        assert 0 < int(ref.accepted.sum()) < n


def test_noalloc_rejects_oversized_and_host_buffers():
    import torch
    import dygrass_b200 as dyg

    H = dyg.Graph.from_edges(4, np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32),
                             np.ones(3, np.float32))
    L = dyg.lib()
    p = dyg.WalkParams.make()
    n = 65536 + 1
    dev = torch.device("cuda:0")
    s = torch.zeros(n, dtype=torch.int32, device=dev)
    w = torch.ones(n, dtype=torch.float32, device=dev)
    o = torch.empty(n, dtype=torch.int32, device=dev)
    rc = L.dyg_incremental_walk_noalloc(H.handle, s.data_ptr(), s.data_ptr(), w.data_ptr(), n, 0,
                                        C.byref(p), o.data_ptr(), None, None, None)
    assert rc == 1 and b"exceeds the maximum" in L.dyg_last_error_string()
    hs = np.zeros(4, np.uint32)
    hw = np.ones(4, np.float32)
    rc = L.dyg_incremental_walk_noalloc(H.handle, hs.ctypes.data, hs.ctypes.data, hw.ctypes.data, 4,
                                        0, C.byref(p), None, None, None, None)
    assert rc == 1 and b"device pointers" in L.dyg_last_error_string()


@pytest.mark.parametrize("transition,flags", [(1, 0), (0, 1)])
def test_noalloc_other_walk_modes(transition, flags):
    """The weighted transition and exhaustive walkers (every walker to its
    natural end) go through other kernel instances; the no-allocation entry
    point must equal dyg_incremental_batch there too."""
    import torch
    import dygrass_b200 as dyg
    import dygrass_b200.workloads as wl

    W = wl.grid_2d(40, 40, inserts=300)
    p = dyg.WalkParams.make(threshold=10.0, walkers=128, max_steps=64, transition=transition,
                            flags=flags)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    dev = torch.device("cuda:0")
    L = dyg.lib()
    n = len(W.ins_src)
    s = torch.from_numpy(W.ins_src.view(np.int32)).to(dev)
    d = torch.from_numpy(W.ins_dst.view(np.int32)).to(dev)
    w = torch.from_numpy(W.ins_w).to(dev)
    fa = torch.empty(n, dtype=torch.int32, device=dev)
    cd = torch.empty(n, dtype=torch.float32, device=dev)
    ac = torch.empty(n, dtype=torch.uint8, device=dev)
    rc = L.dyg_incremental_walk_noalloc(H.handle, s.data_ptr(), d.data_ptr(), w.data_ptr(), n, 0,
                                        C.byref(p), fa.data_ptr(), cd.data_ptr(), ac.data_ptr(), None)
    assert rc == 0, L.dyg_last_error_string()
    torch.cuda.synchronize()
    ref = dyg.incremental_batch(H.clone(), W.ins_src, W.ins_dst, W.ins_w, p)
    assert np.array_equal(fa.cpu().numpy(), ref.found_at)
    assert np.array_equal(cd.cpu().numpy().view(np.uint32), ref.conductance.view(np.uint32))
    assert np.array_equal(ac.cpu().numpy(), ref.accepted)


def test_noalloc_marks_endpoints_outside_the_graph():
    """An edge naming a vertex >= |V| gets found_at = -2 (its walkers do not
    run) and the other edges their usual results."""
    import torch
    import dygrass_b200 as dyg
    import dygrass_b200.workloads as wl

    W = wl.grid_2d(30, 30, inserts=64)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    dev = torch.device("cuda:0")
    L = dyg.lib()
    src = W.ins_src.copy()
    src[5] = W.n
    n = len(src)
    s = torch.from_numpy(src.view(np.int32)).to(dev)
    d = torch.from_numpy(W.ins_dst.view(np.int32)).to(dev)
    w = torch.from_numpy(W.ins_w).to(dev)
    fa = torch.empty(n, dtype=torch.int32, device=dev)
    ac = torch.empty(n, dtype=torch.uint8, device=dev)
    rc = L.dyg_incremental_walk_noalloc(H.handle, s.data_ptr(), d.data_ptr(), w.data_ptr(), n, 0,
                                        C.byref(W.params), fa.data_ptr(), None, ac.data_ptr(), None)
    assert rc == 0, L.dyg_last_error_string()
    got = fa.cpu().numpy()
    assert got[5] == -2 and ac.cpu().numpy()[5] == 0
    keep = np.arange(n) != 5
    ids = np.arange(n, dtype=np.uint64)[keep]
    ref = dyg.incremental_batch_ids(H.clone(), W.ins_src[keep], W.ins_dst[keep], W.ins_w[keep], ids,
                                    W.params)
    assert np.array_equal(got[keep], ref.found_at)
