"""Host-side logic of the batched and serving modes, on the CPU: the rounds
that carry batch r of every graph (multi.plan_rounds), the request generator,
latency statistics and footprint estimate of the server (serve.py)."""
from types import SimpleNamespace

import numpy as np

from dygrass_b200.multi import plan_rounds
from dygrass_b200.serve import DELETE, INSERT, Request, footprint_bytes, latency_stats, poisson_requests


def streams_of(lengths, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for m in lengths:
        out.append((rng.integers(0, 50, m).astype(np.uint32), rng.integers(0, 50, m).astype(np.uint32),
                    rng.uniform(0.5, 2.0, m).astype(np.float32)))
    return out


def check_plan(plan, offsets, streams, sizes):
    # every graph's edges appear once, batch r of graph g in round r, in stream
    # order, with global ids, update id = position in the graph's stream
    assert plan.counts == [len(s) for s, _, _ in streams]
    assert plan.n_edges == sum(plan.counts)
    seen = {g: [] for g in range(len(streams))}
    for r, rd in enumerate(plan.rounds):
        for g in np.unique(rd.graph):
            sel = rd.graph == g
            pos = rd.pos[sel]
            B = sizes[g]
            assert np.array_equal(pos, np.arange(r * B, min((r + 1) * B, len(streams[g][0]))))
            s, d, w = streams[g]
            assert np.array_equal(rd.src[sel], s[pos] + offsets[g])
            assert np.array_equal(rd.dst[sel], d[pos] + offsets[g])
            assert np.array_equal(rd.w[sel].view(np.uint32), w[pos].view(np.uint32))
            assert np.array_equal(rd.uid[sel], pos.astype(np.uint64))
            seen[g] += pos.tolist()
        # graphs appear in index order within a round
        assert np.all(np.diff(rd.graph) >= 0)
    for g, (s, _, _) in enumerate(streams):
        assert seen[g] == list(range(len(s)))
    assert len(plan.rounds) == max(-(-len(s) // sizes[g]) for g, (s, _, _) in enumerate(streams) if len(s))


def test_plan_reference_batches():
    lengths = [0, 7, 25, 100, 1]
    streams = streams_of(lengths)
    offsets = np.array([0, 50, 100, 150, 200, 250], np.int64)
    plan = plan_rounds(offsets, streams)
    sizes = [max(1, -(-m // 10)) for m in lengths]     # ceil(m/10)
    check_plan(plan, offsets, streams, sizes)
    assert len(plan.rounds) == 10


def test_plan_given_batch_sizes():
    lengths = [13, 4, 9]
    streams = streams_of(lengths, seed=1)
    offsets = np.array([0, 50, 100, 150], np.int64)
    sizes = [5, 1, 9]
    plan = plan_rounds(offsets, streams, sizes)
    check_plan(plan, offsets, streams, sizes)
    assert len(plan.rounds) == 4


def test_plan_empty():
    plan = plan_rounds(np.array([0, 10], np.int64), streams_of([0]))
    assert plan.rounds == [] and plan.n_edges == 0


def fake_cases(k=3, n=40, seed=2):
    rng = np.random.default_rng(seed)
    cases = []
    for g in range(k):
        m = 60 + 10 * g
        iu, ju = np.triu_indices(n, 1)                  # distinct pairs
        pick = rng.choice(len(iu), m, replace=False)
        src, dst = iu[pick].astype(np.uint32), ju[pick].astype(np.uint32)
        cases.append(SimpleNamespace(n=n, g_src=src, g_dst=dst, h_src=src[:10], h_dst=dst[:10],
                                     ins_src=rng.integers(0, n, 300).astype(np.uint32),
                                     ins_dst=rng.integers(0, n, 300).astype(np.uint32),
                                     ins_w=rng.uniform(1, 2, 300).astype(np.float32)))
    return cases


def test_poisson_requests():
    cases = fake_cases()
    a = poisson_requests(cases, rate=1000.0, count=200, seed=7, size_hi=40)
    b = poisson_requests(cases, rate=1000.0, count=200, seed=7, size_hi=40)
    assert [(r.graph, r.op, r.arrival, r.src.tolist()) for r in a] == \
        [(r.graph, r.op, r.arrival, r.src.tolist()) for r in b]            # seeded
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert 0.1 < arr[-1] < 0.4                                            # mean gap 1/rate
    ins = {g: 0 for g in range(len(cases))}
    dels = {g: set() for g in range(len(cases))}
    for r in a:
        c = cases[r.graph]
        assert len(r.src) == len(r.dst) <= 40
        if r.op == INSERT:
            # the next edges of the graph's insertion pool, in order
            k = ins[r.graph]
            assert np.array_equal(r.src, c.ins_src[k:k + len(r.src)])
            assert np.array_equal(r.w, c.ins_w[k:k + len(r.src)])
            ins[r.graph] += len(r.src)
        else:
            assert r.op == DELETE and r.w is None
            pairs = set(zip(r.src.tolist(), r.dst.tolist()))
            g_pairs = set(zip(c.g_src.tolist(), c.g_dst.tolist()))
            assert pairs <= g_pairs
            # deletions of a graph never repeat an edge of its dense graph
            idx = [i for i in range(len(c.g_src)) if (c.g_src[i], c.g_dst[i]) in pairs]
            assert not (dels[r.graph] & set(idx))
            dels[r.graph] |= set(idx)
    assert any(r.op == INSERT for r in a) and any(r.op == DELETE for r in a)


def test_latency_stats_and_recovered():
    reqs = []
    for i in range(100):
        r = Request(0, INSERT, np.arange(i % 5 + 1, dtype=np.uint32), np.arange(i % 5 + 1, dtype=np.uint32),
                    arrival=0.01 * i)
        r.done = r.arrival + 0.001 * (i + 1)
        reqs.append(r)
    refused = Request(1, DELETE, np.zeros(3, np.uint32), np.ones(3, np.uint32))
    refused.done = -1.0
    st = latency_stats(reqs + [refused])
    assert st["requests"] == 100
    assert st["updates"] == sum(i % 5 + 1 for i in range(100))
    assert abs(st["p50_ms"] - np.percentile(np.arange(1, 101), 50)) < 1e-9
    assert abs(st["p99_ms"] - np.percentile(np.arange(1, 101), 99)) < 1e-9
    r = Request(0, DELETE, np.zeros(1, np.uint32), np.ones(1, np.uint32))
    assert r.recovered == []
    r.rec_src = np.array([3, 4], np.uint32)
    r.rec_dst = np.array([5, 6], np.uint32)
    r.rec_kind = np.array([0, 1], np.uint8)
    assert r.recovered == [(3, 5, 0), (4, 6, 1)]


def test_footprint_grows_with_the_graph():
    base = footprint_bytes(1000, 4000, 1500)
    assert base > 0
    assert footprint_bytes(2000, 4000, 1500) > base
    assert footprint_bytes(1000, 8000, 1500) > base
    assert footprint_bytes(1000, 4000, 3000) > base
    # slots (12 B each) of both graphs with headroom, plus descriptors
    assert base >= 12 * 2 * (4000 + 1500)


def test_server_needs_an_admitted_graph():
    import pytest
    from dygrass_b200.serve import Server
    cases = fake_cases(k=2)
    with pytest.raises(ValueError, match="HBM budget"):
        Server(cases, None, None, hbm_budget=10.0)


def test_partition_by_footprint():
    """Graphs over ranks by footprint: every graph once, largest first onto
    the least loaded rank, loads within the largest graph of each other."""
    from dygrass_b200.shard import partition_by_footprint
    rng = np.random.default_rng(3)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(1e3), np.log(2e5), 256))]
    for world in (1, 2, 3, 8):
        parts = partition_by_footprint(sizes, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)
    assert partition_by_footprint([5, 1, 4, 2], 2) == [[0, 1], [2, 3]]


def test_bench_split_modes():
    """bench.py's N > 1 defaults: the mesh shards one graph's batches, the
    many-graph and serving workloads partition their graphs, the mixed
    stream runs replicas; N = 1 is a single replica."""
    import argparse
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    ns = lambda **kw: argparse.Namespace(**{"shard": False, "split": "auto", **kw})
    assert bench.resolve_split(ns(workload="mesh"), 1) == "replicas"
    assert bench.resolve_split(ns(workload="mesh"), 4) == "shard"
    assert bench.resolve_split(ns(workload="rgg_many"), 4) == "partition"
    assert bench.resolve_split(ns(workload="serve"), 2) == "partition"
    assert bench.resolve_split(ns(workload="rmat"), 8) == "replicas"
    assert bench.resolve_split(ns(workload="mesh", split="replicas"), 8) == "replicas"
    assert bench.resolve_split(ns(workload="rmat", shard=True), 2) == "shard"


def test_serving_mix_threads_agree():
    """The serving mix's graphs are built by a thread pool: each graph comes
    from its own seeds and the sizes are drawn in order first, so any number
    of workers gives the same graphs in the same order."""
    from dygrass_b200 import workloads as wl
    one, p1, d1 = wl.serving_mix(k=7, seed=11, threads=1)
    many, p2, d2 = wl.serving_mix(k=7, seed=11, threads=4)
    assert len(one) == len(many) == 7
    fields = ("g_src", "g_dst", "g_w", "h_src", "h_dst", "h_w", "ins_src", "ins_dst", "ins_w")
    for a, b in zip(one, many):
        assert a.n == b.n
        for f in fields:
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert bytes(p1) == bytes(p2) and bytes(d1) == bytes(d2)


def test_bench_default_steps(monkeypatch):
    """20 timed steps by default (several clock samples inside the timed
    region); 5 for the reference arm, whose step is the whole workload on
    the host cores; an explicit --steps wins."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    for argv, want in ((["bench.py"], 20), (["bench.py", "--impl", "reference"], 5),
                       (["bench.py", "--steps", "7"], 7),
                       (["bench.py", "--impl", "reference", "--steps", "2"], 2)):
        monkeypatch.setattr(sys, "argv", argv)
        assert bench.parse().steps == want
