"""The split ABI of a sharded batch on one GPU: two replicas play two ranks
(each walks its range, the key arrays are combined by max, both commit); both
replicas end equal to a third that ran the whole batches.  Nothing here waits
on another rank: the replicas run one after the other."""
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


def same_graph(a, b):
    ea, eb = a.export(), b.export()
    assert np.array_equal(ea[0], eb[0]) and np.array_equal(ea[1], eb[1])
    assert np.array_equal(ea[2].view(np.uint32), eb[2].view(np.uint32))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_equals_whole(dyg, world):
    import torch
    from dygrass_b200.shard import GpuBackend, split
    wl = W.mesh_3d(9, inserts=700, seed=5)
    p = dyg.WalkParams.make(threshold=100.0, walkers=64, max_steps=100, seed=5)
    mk = lambda: (dyg.Graph.from_edges(wl.n, wl.h_src, wl.h_dst, wl.h_w, slack_per_row=0,
                                       arena_headroom=0.0),
                  dyg.Graph.from_edges(wl.n, wl.g_src, wl.g_dst, wl.g_w, slack_per_row=0,
                                       arena_headroom=0.0))
    reps = [mk() for _ in range(world)]
    Hw, Gw = mk()
    back = GpuBackend(torch.device("cuda", 0))
    t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a if dt is None else a.view(dt))).cuda()
    B = 175
    for b0 in range(0, len(wl.ins_src), B):
        s, d, w = (x[b0:b0 + B] for x in (wl.ins_src, wl.ins_dst, wl.ins_w))
        ds, dd, dw = t(s, np.int32), t(d, np.int32), t(w)
        parts = []
        for r, (H, G) in enumerate(reps):
            k = back.zeros_keys(len(s))
            lo, hi = split(len(s), r, world)
            back.walk_keys(H, ds, dd, dw, b0, lo, hi, p, k)
            parts.append(k)
        keys = torch.stack(parts).max(dim=0).values.contiguous()
        outs = [back.incr_commit(H, G, ds, dd, dw, keys.clone()) for H, G in reps]
        ref = dyg.incremental_batch(Hw, s, d, w, p, first_update_id=b0, G=Gw)
        for o in outs:
            assert np.array_equal(o[0].cpu().numpy(), ref.found_at)
            assert np.array_equal(o[1].cpu().numpy().view(np.uint32), ref.conductance.view(np.uint32))
            assert np.array_equal(o[2].cpu().numpy(), ref.accepted)
    rng = np.random.default_rng(6)
    pick = rng.choice(len(wl.h_src), 160, replace=False)
    for b0 in range(0, 160, 40):
        s, d = wl.h_src[pick[b0:b0 + 40]], wl.h_dst[pick[b0:b0 + 40]]
        ds, dd = t(s, np.int32), t(d, np.int32)
        states = [back.decr_delete(G, H, ds, dd, 5000 + b0) for H, G in reps]
        nw = states[0][0]
        assert all(x[0] == nw for x in states)
        parts = []
        for r, (H, G) in enumerate(reps):
            k = back.zeros_keys(nw)
            lo, hi = split(nw, r, world)
            back.decr_walk_keys(G, lo, hi, p, k)
            parts.append(k)
        keys = torch.stack(parts).max(dim=0).values.contiguous()
        outs = [back.decr_commit(G, H, p, keys.clone(), nw, st, 40 * 200)
                for (H, G), (_, st) in zip(reps, states)]
        ref = dyg.decremental_batch(Gw, Hw, s, d, p, first_update_id=5000 + b0)
        for st, cd, rx, ry, rk in outs:
            assert np.array_equal(st.cpu().numpy()[:len(s)], ref.status)
            assert np.array_equal(rx, ref.rec_src) and np.array_equal(ry, ref.rec_dst)
            assert np.array_equal(rk, ref.rec_kind)
    for H, G in reps:
        same_graph(H, Hw)
        same_graph(G, Gw)
