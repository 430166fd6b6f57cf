"""A batch sharded over processes (gloo, world size 2 and 3, CPU): the driver
of dygrass_b200.shard with the oracle as its compute gives every rank the
whole-batch result, insertions and deletions, over several batches."""
import json
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (root, os.path.join(root, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    import pyoracle as O
    from dygrass_b200 import WalkParams
    from dygrass_b200 import workloads as W
    from dygrass_b200.shard import allreduce_max, decremental_sharded, incremental_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    ok, why = True, ""
    try:
        wl = W.mesh_3d(8, inserts=600, seed=9)
        p = WalkParams.make(threshold=100.0, walkers=64, max_steps=100, seed=9)
        back = O.ShardBackend(threads=2)
        comb = allreduce_max()
        Hs, Gs = O.OGraph(wl.n, wl.h_src, wl.h_dst, wl.h_w), O.OGraph(wl.n, wl.g_src, wl.g_dst, wl.g_w)
        Hr, Gr = O.OGraph(wl.n, wl.h_src, wl.h_dst, wl.h_w), O.OGraph(wl.n, wl.g_src, wl.g_dst, wl.g_w)
        B = 150
        for b0 in range(0, len(wl.ins_src), B):
            s, d, w = (x[b0:b0 + B] for x in (wl.ins_src, wl.ins_dst, wl.ins_w))
            fa, cd, ac = incremental_sharded(back, Hs, Gs, s, d, w, b0, p, rank, world, comb)
            fa2, cd2, ac2, _ = O.incremental(Hr, s, d, w, p, G=Gr, first_uid=b0, single_batch=True,
                                             threads=2)
            ok &= bool(np.array_equal(fa, fa2) and np.array_equal(cd.view(np.uint32), cd2.view(np.uint32))
                       and np.array_equal(ac, ac2))
        rng = np.random.default_rng(4)
        pick = rng.choice(len(wl.h_src), 120, replace=False)
        ds, dd = wl.h_src[pick], wl.h_dst[pick]
        for b0 in range(0, len(ds), 40):
            s, d = ds[b0:b0 + 40], dd[b0:b0 + 40]
            st, cd, rx, ry, rk = decremental_sharded(back, Gs, Hs, s, d, 1000 + b0, p, rank, world, comb)
            st2, cd2, rx2, ry2, rk2, _ = O.decremental(Gr, Hr, s, d, p, first_uid=1000 + b0,
                                                       single_batch=True, threads=2)
            ok &= bool(np.array_equal(st, st2) and np.array_equal(rx, rx2) and np.array_equal(ry, ry2)
                       and np.array_equal(rk, rk2))
        for a, b in ((Hs, Hr), (Gs, Gr)):
            ea, eb = a.export(), b.export()
            ok &= all(np.array_equal(x.view(np.uint32) if x.dtype == np.float32 else x,
                                     y.view(np.uint32) if y.dtype == np.float32 else y)
                      for x, y in zip(ea, eb))
    except Exception as e:   # reported to the parent
        ok, why = False, repr(e)
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ok": bool(ok), "why": why}, f)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batches_match_whole_batches(tmp_path, world):
    """world 3 splits the batches and walk lists into uneven rank ranges."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        res = json.load(open(tmp_path / f"rank{r}.json"))
        assert res["ok"], res["why"]
