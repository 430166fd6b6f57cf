"""Inputs that are not a valid batch, given in DEVICE memory, are rejected
before anything changes: the call returns DYG_EINVAL and G and H export
byte-identical to before.  Host batches get the same answer from the host
check; device batches are checked by a kernel at the start of the call, which
halts every later kernel of the call.

Each test compares the exports right after the bad call, before anything
walks the graphs again, and only then runs a valid call, which must match the
oracle (so the halt and the error bits were cleared)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dyg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import dygrass_b200
    dygrass_b200.lib()
    return dygrass_b200


def dev(a, view=None):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a if view is None else a.view(view)).cuda()


def snapshot(*gs):
    out = []
    for g in gs:
        rp, c, w = g.export()
        out.append((rp.copy(), c.copy(), w.view(np.uint32).copy()))
    return out


def assert_same(before, after):
    for (r1, c1, w1), (r2, c2, w2) in zip(before, after):
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2) and np.array_equal(w1, w2)


def expect_einval(dyg, fn):
    with pytest.raises(dyg.DygError) as e:
        fn()
    assert e.value.status == dyg.DYG_EINVAL
    return str(e.value)


def small(seed=3):
    import dygrass_b200.workloads as wl
    return wl.mesh_3d(k=8, inserts=240, seed=seed)


@pytest.mark.parametrize("bad", ["src", "dst", "w0", "wneg", "wnan", "winf"])
def test_incremental_device_batch_rejected(dyg, oracle, bad):
    W = small()
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    s, d, w = W.ins_src.copy(), W.ins_dst.copy(), W.ins_w.copy()
    k = len(s) - 7   # in the last batch: earlier batches would commit first without the check
    if bad == "src":
        s[k] = W.n
    elif bad == "dst":
        d[k] = W.n + 5
    else:
        w[k] = {"w0": 0.0, "wneg": -1.0, "wnan": np.nan, "winf": np.inf}[bad]
    before = snapshot(H, G)
    msg = expect_einval(dyg, lambda: dyg.incremental_stream(
        H, dev(s, np.int32), dev(d, np.int32), dev(w), W.params, G=G))
    assert "changed nothing" in msg
    assert_same(before, snapshot(H, G))
    # the handles still work: the valid stream matches the oracle
    Ho = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    r = dyg.incremental_stream(H, dev(W.ins_src, np.int32), dev(W.ins_dst, np.int32), dev(W.ins_w),
                               W.params)
    fa, cd, ac, _ = oracle.incremental(Ho, W.ins_src, W.ins_dst, W.ins_w, W.params)
    assert np.array_equal(r.found_at, fa) and np.array_equal(r.accepted, ac)
    assert np.array_equal(H.export()[1], Ho.export()[1])


def test_incremental_batch_ids_device_rejected(dyg):
    W = small()
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    s = W.ins_src.copy()
    s[3] = 0xFFFFFFFF
    ids = np.arange(len(s), dtype=np.uint64)
    before = snapshot(H)
    expect_einval(dyg, lambda: dyg.incremental_batch_ids(
        H, dev(s, np.int32), dev(W.ins_dst, np.int32), dev(W.ins_w), dev(ids, np.int64), W.params))
    assert_same(before, snapshot(H))


def test_decremental_device_batch_rejected(dyg, oracle):
    W = small()
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    s, d = W.del_src.copy(), W.del_dst.copy()
    d[len(d) - 2] = W.n
    before = snapshot(G, H)
    expect_einval(dyg, lambda: dyg.decremental_stream(G, H, dev(s, np.int32), dev(d, np.int32),
                                                      W.dparams))
    assert_same(before, snapshot(G, H))
    Go, Ho = oracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w), oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    r = dyg.decremental_stream(G, H, dev(W.del_src, np.int32), dev(W.del_dst, np.int32), W.dparams)
    st, _, rx, ry, rk, _ = oracle.decremental(Go, Ho, W.del_src, W.del_dst, W.dparams)
    assert np.array_equal(r.status, st)
    assert np.array_equal(r.rec_src, rx) and np.array_equal(r.rec_dst, ry)
    assert np.array_equal(r.rec_kind, rk)


@pytest.mark.parametrize("op", ["insert", "delete"])
def test_stream_file_device_rejected(dyg, op):
    W = small()
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    if op == "insert":
        s, d, w = W.ins_src.copy(), W.ins_dst.copy(), W.ins_w.copy()
        w[11] = np.nan
        code, args = dyg.STREAM_INSERT, (dev(s, np.int32), dev(d, np.int32), dev(w))
    else:
        s, d = W.del_src.copy(), W.del_dst.copy()
        s[0] = W.n
        code, args = dyg.STREAM_DELETE, (dev(s, np.int32), dev(d, np.int32), None)
    before = snapshot(G, H)
    expect_einval(dyg, lambda: dyg.stream_file(G, H, code, *args, W.params, chunk=50))
    assert_same(before, snapshot(G, H))


def test_sharded_calls_reject_device_batches(dyg):
    import torch
    from dygrass_b200.shard import GpuBackend
    W = small()
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    back = GpuBackend(torch.device("cuda", 0))
    s = W.ins_src[:50].copy()
    s[20] = W.n
    ds, dd, dw = dev(s, np.int32), dev(W.ins_dst[:50], np.int32), dev(W.ins_w[:50])
    before = snapshot(H, G)
    keys = back.zeros_keys(50)
    expect_einval(dyg, lambda: back.walk_keys(H, ds, dd, dw, 0, 0, 50, W.params, keys))
    expect_einval(dyg, lambda: back.incr_commit(H, G, ds, dd, dw, keys))
    x = W.del_src[:30].copy()
    x[29] = W.n
    expect_einval(dyg, lambda: back.decr_delete(G, H, dev(x, np.int32),
                                                dev(W.del_dst[:30], np.int32), 0))
    assert_same(before, snapshot(H, G))


def test_recovered_read_ranges(dyg, oracle):
    """The default decremental wrapper passes no record buffers and reads the
    records afterwards; both forms give the oracle's records."""
    W = small(seed=8)
    G = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w)
    H = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
    Go, Ho = oracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w), oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    r = dyg.decremental_stream(G, H, W.del_src, W.del_dst, W.dparams)
    st, _, rx, ry, rk, _ = oracle.decremental(Go, Ho, W.del_src, W.del_dst, W.dparams)
    assert len(rx) > 4
    assert np.array_equal(r.rec_src, rx) and np.array_equal(r.rec_dst, ry)
    a, b, c = dyg.recovered_read(G, 3, first=2)
    assert np.array_equal(a, rx[2:5]) and np.array_equal(b, ry[2:5]) and np.array_equal(c, rk[2:5])
    with pytest.raises(dyg.DygError) as e:
        dyg.recovered_read(G, 2, first=len(rx) - 1)
    assert e.value.status == dyg.DYG_ERANGE
