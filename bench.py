#!/usr/bin/env python
"""Benchmark of the dyGRASS update path on B200.

Workload (default "mesh"): the plain incremental + decremental configuration
at scale -- 3-D 7-point mesh 100x100x100 (1,000,000 vertices, 2,970,000
edges) with FP32 log-uniform weights over [1e-2, 1e2], sparsifier =
spanning tree + 5% off-tree edges, 200,000 insertions at hop distance
2..10 (10 batches, threshold 100, 512 walkers, max_steps 100), then deletion
of 10% of the dense graph's edges (317,000, 10 batches) recovered through
walks on the updated dense graph.  Synthetic, seeded (dygrass_b200/workloads.py).

One step = the whole update stream (insertions then deletions) from the
initial graphs, which are restored (untimed) before every step together
with an L2 flush (a 256 MB write).  value = edge updates (insertions +
deletions) per second over all ranks; the device-resident run keeps inputs
and outputs in HBM, e2e passes host (pinned) buffers through the C ABI.

Workload "rmat": the mixed-stream configuration -- R-MAT scale 20 (edge
factor 16, a=0.57, b=c=0.19), symmetrised, deduplicated, largest connected
component (645,911 vertices, 15.7 M edges at the default seed), weights
U[0.1, 10], sparsifier = spanning tree + 5% off-tree; 500,000 updates in
stream files of 4,096 (70% insertion files, 30% deletion files), threshold
50, 256 walkers, max_steps 128.  One step = every file in order through
dyg_stream_file from the initial graphs.

Workload "rgg_many": the batched many-graph configuration -- 256 random
geometric graphs (n log-uniform in [1e3, 2e5], mean degree 8, weights
1/distance), each with sparsifier = spanning tree + 10% off-tree and 0.05 n
insertions; threshold 100, 512 walkers, max_steps 100.  The graphs form one
union graph and a step is the 10 rounds that carry batch r of every graph
(dygrass_b200/multi.py), after an autotune of the walk launch shape.  The
plain per-graph loop on the same updates is timed beside it.

Workload "serve": the serving configuration -- 80 graphs mixed from the
mesh, R-MAT and random-geometric generators (--serve-mix large: about 10.8 GB
of footprint), update requests of log-uniform size in [1, 4096], 60%
insertions / 40% deletions.  value = the continuous-batching pool server's
throughput (the native scheduler of include/dyg_serve.h, driven by
dygrass_b200/serve.py) replaying a fixed request set that is all pending at
once (saturation), timed with CUDA events with every graph resident; then
p50/p99 latency at Poisson arrival rates swept around that capacity, for the
server and for the plain sequential path (every request alone on its graph's
own handles), and the same replay with a budget of half the footprint, where
graphs are admitted and evicted while requests run.

N > 1 (torchrun): every rank runs an independent replica of the workload
(weak scaling, no data-path collective); times are the max over ranks.

--impl reference: the reference has no CPU implementation of this path, so
the reference arm times the CPU port of its update loop (oracle/, all host
threads) on the whole workload per step (serve: the first 300 requests).

Workload "refgpu": the reference's own CUDA updaters (built unmodified for
sm_100a in oracle/_ref) against this library on identical input files.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_MOVE = 64   # two 32-byte sectors: row descriptor + chosen slot


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 20; 5 for --impl reference, whose step is the "
                         "whole workload on the host cores)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--refgpu-repeats", type=int, default=10)
    ap.add_argument("--workload", choices=["mesh", "grid", "rmat", "rgg_many", "serve", "refgpu"],
                    default="mesh")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-mix", choices=["small", "large"], default="large",
                    help="serving graphs: large = meshes 60^3..100^3, R-MAT scales 17..20, "
                         "random geometric graphs (about 10.8 GB at 80 graphs); small = the "
                         "quick mix")
    ap.add_argument("--serve-graphs", type=int, default=80)
    ap.add_argument("--rgg-graphs", type=int, default=256)
    ap.add_argument("--rgg-n-hi", type=int, default=200_000)
    ap.add_argument("--tune-walkers", action="store_true",
                    help="let the autotuner lower the walker count and the walk length at equal "
                         "kappa (within 5 %% of the workload's own parameters on sample graphs)")
    ap.add_argument("--rmat-scale", type=int, default=20)
    ap.add_argument("--rmat-updates", type=int, default=500_000)
    ap.add_argument("--mesh-k", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--split", choices=["auto", "replicas", "shard", "partition"], default="auto",
                    help="how N > 1 ranks share the work (see resolve_split)")
    ap.add_argument("--shard", action="store_true",
                    help="mesh: one graph, every batch split over the ranks (keys all-reduced), "
                         "strong scaling; default N > 1 runs independent replicas")
    ap.add_argument("--no-plain", action="store_true",
                    help="rgg_many: skip timing the plain per-graph loop")
    ap.add_argument("--transition", choices=["uniform", "weighted"], default="uniform",
                    help="walk transition: uniform (the reference's) or the opt-in weighted mode")
    ap.add_argument("--no-exhaustive-leg", action="store_true",
                    help="skip the extra timed pass with every walker run to its end")
    ap.add_argument("--exhaustive", action="store_true",
                    help="run every walker to its natural end (no pruning)")
    ap.add_argument("--profile-only", action="store_true",
                    help="one short device-resident step (for profilers)")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 5 if args.impl == "reference" else 20
    return args


def resolve_split(args, world):
    """How N > 1 ranks share the work: "shard" (one graph, each batch's
    walks split over the ranks, winner keys all-reduced), "partition"
    (independent graphs divided by footprint) or "replicas" (each rank its
    own copy of the workload).  auto: shard for the mesh and grid, partition
    for the many-graph and serving workloads, replicas for the mixed stream
    (stream files have no split entry points)."""
    if world == 1:
        return "replicas"
    if args.shard:
        return "shard"
    if args.split != "auto":
        return args.split
    return {"mesh": "shard", "grid": "shard", "rgg_many": "partition",
            "serve": "partition"}.get(args.workload, "replicas")


def _my_graphs(args, cases, rank, world):
    """This rank's graphs when the graphs are partitioned, else all."""
    if args.split_mode != "partition":
        return list(range(len(cases)))
    from dygrass_b200.serve import footprint_bytes
    from dygrass_b200.shard import partition_by_footprint
    fps = [footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in cases]
    return partition_by_footprint(fps, world)[rank]


def make_workload(args, rank, world=1):
    import dygrass_b200.workloads as wl
    # replicas draw their own inputs; a sharded or partitioned job is one workload
    seed = wl.MASTER_SEED + (1000 * rank if args.split_mode == "replicas" else 0)
    if args.workload == "serve":
        from dygrass_b200.serve import Request, footprint_bytes, poisson_requests
        cases, ip, dp = wl.serving_mix(k=args.serve_graphs, seed=seed,
                                        large=args.serve_mix == "large")
        reqs = poisson_requests(cases, 1.0, args.serve_requests, seed + 5)
        job = sum(len(r.src) for r in reqs)
        mine = _my_graphs(args, cases, rank, world)
        if len(mine) != len(cases):
            slot = {g: k for k, g in enumerate(mine)}
            cases = [cases[g] for g in mine]
            reqs = [Request(slot[r.graph], r.op, r.src, r.dst, r.w, arrival=r.arrival)
                    for r in reqs if r.graph in slot]

        class Serve:
            pass
        W = Serve()
        W.cases, W.params, W.dparams = cases, ip, dp
        W.requests = reqs
        W.n_updates = sum(len(r.src) for r in W.requests)
        W.job_updates = job
        W.n = sum(c.n for c in cases)
        W.footprint = sum(footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in cases)
        return W
    if args.workload == "rgg_many":
        cases, p = wl.rgg_many(k=args.rgg_graphs, n_hi=args.rgg_n_hi, seed=seed)
        job = sum(len(c.ins_src) for c in cases)
        cases = [cases[g] for g in _my_graphs(args, cases, rank, world)]

        class Many:
            pass
        W = Many()
        W.cases, W.params, W.dparams = cases, p, p
        W.n_updates = sum(len(c.ins_src) for c in cases)
        W.job_updates = job
        W.n = sum(c.n for c in cases)
        return W
    if args.workload == "rmat":
        W = wl.rmat_mixed(scale=args.rmat_scale, n_updates=args.rmat_updates, seed=seed)
        W.params = W.iparams
    elif args.workload == "grid":
        W = wl.grid_2d(seed=seed)
    else:
        W = wl.mesh_3d(k=args.mesh_k, seed=seed)
    if args.exhaustive:
        import dygrass_b200 as dyg
        W.params.flags |= dyg.FLAG_EXHAUSTIVE
        W.dparams.flags |= dyg.FLAG_EXHAUSTIVE
    if args.transition == "weighted":
        import dygrass_b200 as dyg
        W.params.transition = dyg.TRANSITION_WEIGHTED
        W.dparams.transition = dyg.TRANSITION_WEIGHTED
    return W


def workload_config(W, args):
    cfg = _workload_config(W, args)
    if args.transition == "weighted":
        cfg["workload"] += ", weighted transition (opt-in, not the reference's rule)"
        cfg["transition"] = "weighted"
    return cfg


def _workload_config(W, args):
    if args.workload == "serve":
        ins = sum(len(r.src) for r in W.requests if r.op == 0)
        mix = ("meshes 60^3..100^3, R-MAT scales 17..20, random geometric n <= 2e5"
               if args.serve_mix == "large" else "meshes 12^3..48^3, R-MAT scales 10..16, "
                                                 "random geometric n <= 2e5")
        return {"workload": f"serve {len(W.cases)} graphs ({mix}) in a native pool server, "
                            f"{len(W.requests)} requests of log-uniform size [1, 4096], 60% insert / "
                            f"40% delete, threshold 100, 512 walkers, max_steps 100",
                "graphs": len(W.cases), "vertices": W.n,
                "edges": int(sum(len(c.g_src) for c in W.cases)),
                "footprint_bytes_estimate": W.footprint, "requests": len(W.requests),
                "updates": W.n_updates, "insertions": ins, "deletions": W.n_updates - ins}
    if args.workload == "rgg_many":
        return {"workload": f"rgg_many {len(W.cases)} random geometric graphs, n log-uniform "
                            f"[1,000, {args.rgg_n_hi:,}], mean degree 8, 0.05 n insertions each, "
                            f"threshold 100, {W.params.walkers} walkers, max_steps 100, "
                            f"one launch per round over all graphs",
                "graphs": len(W.cases), "vertices": W.n,
                "edges": int(sum(len(c.g_src) for c in W.cases)),
                "sparsifier_edges": int(sum(len(c.h_src) for c in W.cases)),
                "insertions": W.n_updates}
    if args.workload == "rmat":
        nins = sum(len(f[1]) for f in W.files if f[0] == 0)
        return {"workload": f"rmat scale {args.rmat_scale} mixed stream, files of 4,096 (70% insert / "
                            f"30% delete), threshold 50, 256 walkers, max_steps 128",
                "vertices": W.n, "edges": int(len(W.g_src)), "sparsifier_edges": int(len(W.h_src)),
                "updates": W.n_updates, "insertions": nins, "deletions": W.n_updates - nins,
                "files": len(W.files)}
    if args.workload == "grid":
        return {"workload": "grid_2d 100x100, 1,000 insertions, threshold 10, 512 walkers, max_steps 64",
                "vertices": W.n, "edges": int(len(W.g_src)), "insertions": int(len(W.ins_src)),
                "deletions": 0}
    return {"workload": f"mesh_3d {args.mesh_k}^3 incremental+decremental, threshold 100, 512 walkers, max_steps 100",
            "vertices": W.n, "edges": int(len(W.g_src)), "sparsifier_edges": int(len(W.h_src)),
            "insertions": int(len(W.ins_src)), "deletions": int(len(W.del_src)),
            "batches": "10 insertion + 10 deletion (ceil(N/10) each)"}


# --------------------------------------------------------------- clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix=f"dyg_clocks{device_index}_", suffix=".csv")
        os.close(fd)

    def start(self):
        """Starts nvidia-smi and returns once its first sample is written, so
        that the samples after it fall inside the timed region."""
        self.n0 = 0
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            self.f.flush()
            with open(self.path) as g:
                n = sum(1 for _ in g)
            if n:
                self.n0 = n
                return
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = open(self.path).read().splitlines()
        inside = lines[self.n0:]
        for line in inside or lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax = float(parts[2].split()[0])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm) if inside else 0,
                "when": "during the timed region" if inside else "just before the timed region"}


# ------------------------------------------------------------- our arm

def dom_is_decr(prof):
    return prof["decr_walk_ms"] >= prof["incr_walk_ms"]


def dom_name(prof):
    return "k_walk<0,0>" if dom_is_decr(prof) else "k_walk<1,0>"


def dom_bytes(prof, incr_moves, decr_moves, steps):
    """Algorithmic bytes per launch of the dominant walk kernel."""
    if dom_is_decr(prof):
        return decr_moves * steps * BYTES_PER_MOVE / max(prof["decr_walk_launches"], 1)
    return incr_moves * steps * BYTES_PER_MOVE / max(prof["incr_walk_launches"], 1)


def dom_ms(prof):
    if dom_is_decr(prof):
        return prof["decr_walk_ms"] / max(prof["decr_walk_launches"], 1)
    return prof["incr_walk_ms"] / max(prof["incr_walk_launches"], 1)


KERNEL_DESC = {"k_walk<0,0>": "k_walk<0,0> (decremental walk on G)",
               "k_walk<1,0>": "k_walk<1,0> (incremental walk on H)"}


def run_ours(args, rank, world, local_rank):
    import torch
    import dygrass_b200 as dyg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = make_workload(args, rank, world)
    nin, ndel = len(W.ins_src), len(W.del_src)

    H0 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w, device=local_rank)
    G0 = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w, device=local_rank)
    H, G = H0.clone(), G0.clone()

    def t(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev) if dt is None else \
            torch.from_numpy(np.ascontiguousarray(a).view(dt)).to(dev)

    d_is, d_id, d_iw = t(W.ins_src, np.int32), t(W.ins_dst, np.int32), t(W.ins_w)
    d_ds, d_dd = t(W.del_src, np.int32), t(W.del_dst, np.int32)
    rec_cap = max(ndel, 1) * (W.dparams.max_steps + 4 * W.dparams.heuristic_walkers) // 8 + 1024
    o_inc = dyg.IncrementalResult(torch.empty(nin, dtype=torch.int32, device=dev),
                                  torch.empty(nin, dtype=torch.float32, device=dev),
                                  torch.empty(nin, dtype=torch.uint8, device=dev))
    o_st = torch.empty(max(ndel, 1), dtype=torch.int32, device=dev)
    o_cd = torch.empty(max(ndel, 1), dtype=torch.float32, device=dev)
    o_rx = torch.empty(rec_cap, dtype=torch.int32, device=dev)
    o_ry = torch.empty(rec_cap, dtype=torch.int32, device=dev)
    o_rk = torch.empty(rec_cap, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def reset():
        H.copy_from(H0, sp)
        G.copy_from(G0, sp)
        flush.fill_(rank + 1)

    shard_back = None
    if args.shard:
        from dygrass_b200.shard import GpuBackend, allreduce_max, decremental_sharded, incremental_sharded
        shard_back = GpuBackend(dev, stream=sp)
        combine = allreduce_max() if world > 1 else (lambda k: k)
        Bi, Bd = dyg.reference_batch_size(nin), dyg.reference_batch_size(max(ndel, 1))

    def step_sharded():
        for b0 in range(0, nin, Bi):
            sl = slice(b0, min(b0 + Bi, nin))
            fa, cd, ac = incremental_sharded(shard_back, H, G, d_is[sl], d_id[sl], d_iw[sl], b0,
                                             W.params, rank, world, combine)
            o_inc.accepted[sl] = ac
        nrec = 0
        for b0 in range(0, ndel, Bd):
            sl = slice(b0, min(b0 + Bd, ndel))
            st, cd, rx, ry, rk = decremental_sharded(shard_back, G, H, d_ds[sl], d_dd[sl], b0,
                                                     W.dparams, rank, world, combine)
            nrec += len(rx)
        return nrec

    def step_device():
        if shard_back is not None:
            return step_sharded()
        dyg.incremental_stream(H, d_is, d_id, d_iw, W.params, G=G, stream=sp, out=o_inc)
        nrec = 0
        if ndel:
            nrec = dyg.decremental_stream_into(G, H, d_ds, d_dd, W.dparams, o_st, o_cd, o_rx, o_ry,
                                               o_rk, rec_cap, stream=sp)
        return nrec

    if args.profile_only:
        reset()
        step_device()
        torch.cuda.synchronize()
        return None

    for _ in range(args.warmup):
        reset()
        step_device()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # ---- device-resident timed region
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    m0 = (H.counters()[0], G.counters()[0])
    launches0 = dyg.kernel_launches()
    dyg.profile_reset()
    dyg.profile_enable(True)
    times = []
    nrec = 0
    for _ in range(args.steps):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nrec = step_device()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    dyg.profile_enable(False)
    prof = dyg.profile_read()
    launches = dyg.kernel_launches() - launches0
    m1 = (H.counters()[0], G.counters()[0])
    clk = clocks.stop()
    barrier()
    ms = float(np.mean(times))
    ms_max = ms
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
    incr_moves = (m1[0] - m0[0]) / args.steps
    decr_moves = (m1[1] - m0[1]) / args.steps
    accepted = int(o_inc.accepted.sum().item())

    # ---- end-to-end through host buffers (pinned), copies inside the region
    e2e = None
    if not args.no_e2e and not args.shard:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        h_is, h_id, h_iw = pin(W.ins_src), pin(W.ins_dst), pin(W.ins_w)
        h_ds, h_dd = pin(W.del_src), pin(W.del_dst)
        h_out = dyg.IncrementalResult(pin(np.empty(nin, np.int32)), pin(np.empty(nin, np.float32)),
                                      pin(np.empty(nin, np.uint8)))
        h_st, h_cd = pin(np.empty(max(ndel, 1), np.int32)), pin(np.empty(max(ndel, 1), np.float32))
        h_rx, h_ry = pin(np.empty(rec_cap, np.uint32)), pin(np.empty(rec_cap, np.uint32))
        h_rk = pin(np.empty(rec_cap, np.uint8))
        barrier()
        torch.cuda.synchronize()
        et = []
        nrec_h = 0
        for _ in range(max(1, args.steps)):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dyg.incremental_stream(H, h_is, h_id, h_iw, W.params, G=G, stream=sp, out=h_out)
            if ndel:
                nrec_h = dyg.decremental_stream_into(G, H, h_ds, h_dd, W.dparams, h_st, h_cd, h_rx,
                                                     h_ry, h_rk, rec_cap, stream=sp)
            e1.record(stream)
            e1.synchronize()
            et.append(e0.elapsed_time(e1))
        barrier()
        ems = float(np.mean(et))
        if world > 1:
            import torch.distributed as dist
            tt = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        assert np.array_equal(h_out.accepted, o_inc.accepted.cpu().numpy())
        e2e = {"value": world * (nin + ndel) / (ems / 1e3), "unit": "edge_updates/s",
               "ms_per_step": ems,
               "h2d_bytes_per_step": int(nin * 12 + ndel * 8),
               "d2h_bytes_per_step": int(nin * 9 + ndel * 8 + nrec_h * 9)}

    # ---- the same step with every walker run to its natural end (as the
    # reference's and the CPU port's walkers run): separates the pruning
    # saving from the hardware's
    exh = None
    if not args.exhaustive and not args.shard and not args.no_exhaustive_leg:
        pe = type(W.params).from_buffer_copy(W.params)
        pde = type(W.dparams).from_buffer_copy(W.dparams)
        pe.flags |= dyg.FLAG_EXHAUSTIVE
        pde.flags |= dyg.FLAG_EXHAUSTIVE
        barrier()
        torch.cuda.synchronize()
        xm0 = (H.counters()[0], G.counters()[0])
        xt = []
        for _ in range(max(1, args.steps)):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dyg.incremental_stream(H, d_is, d_id, d_iw, pe, G=G, stream=sp, out=o_inc)
            if ndel:
                dyg.decremental_stream_into(G, H, d_ds, d_dd, pde, o_st, o_cd, o_rx, o_ry, o_rk,
                                            rec_cap, stream=sp)
            e1.record(stream)
            e1.synchronize()
            xt.append(e0.elapsed_time(e1))
        xm1 = (H.counters()[0], G.counters()[0])
        barrier()
        xms = float(np.mean(xt))
        if world > 1:
            import torch.distributed as dist
            tt = torch.tensor([xms], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            xms = float(tt.item())
        assert int(o_inc.accepted.sum().item()) == accepted   # pruning changes no result
        n_x = max(1, args.steps)
        exh = {"value": world * (nin + ndel) / (xms / 1e3), "unit": "edge_updates/s",
               "ms_per_step": xms, "incr_walker_moves": (xm1[0] - xm0[0]) / n_x,
               "decr_walker_moves": (xm1[1] - xm0[1]) / n_x}

    walk_ms = prof["incr_walk_ms"] + prof["decr_walk_ms"]
    walk_launches = prof["incr_walk_launches"] + prof["decr_walk_launches"]
    moves_total = (incr_moves + decr_moves) * args.steps
    res = {
        "ms_per_step": ms_max, "steps_ms": times, "nin": nin, "ndel": ndel, "accepted": accepted,
        "recovered": nrec, "incr_moves": incr_moves, "decr_moves": decr_moves,
        "walk_ms_per_step": walk_ms / args.steps, "walk_launches": walk_launches,
        "prof": prof, "launches_per_step": launches / args.steps, "clocks": clk, "e2e": e2e,
        "exhaustive": exh,
        "walk_bytes_per_launch": moves_total * BYTES_PER_MOVE / max(walk_launches, 1),
        "walk_ms_per_launch": walk_ms / max(walk_launches, 1),
        # dominant kernel: the walk kernel with the larger measured time
        "dom_kernel": dom_name(prof),
        "dom_bytes_per_launch": dom_bytes(prof, incr_moves, decr_moves, args.steps),
        "dom_ms_per_launch": dom_ms(prof),
        "W": W,
    }
    for g in (H, G, H0, G0):
        g.close()
    return res


def run_mixed(args, rank, world, local_rank):
    """The mixed-stream workload: every stream file in order per step."""
    import torch
    import dygrass_b200 as dyg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = make_workload(args, rank, world)
    H0 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w, device=local_rank)
    G0 = dyg.Graph.from_edges(W.n, W.g_src, W.g_dst, W.g_w, device=local_rank)
    H, G = H0.clone(), G0.clone()
    nmax = max(len(f[1]) for f in W.files)
    rec_cap = nmax * (W.dparams.max_steps + 4 * W.dparams.heuristic_walkers) + 1024

    def t(a, dt=None):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev) if dt is None else \
            torch.from_numpy(np.ascontiguousarray(a).view(dt)).to(dev)

    dfiles = [(op, t(s_, np.int32), t(d_, np.int32), None if w_ is None else t(w_))
              for op, s_, d_, w_ in W.files]
    o_st = torch.empty(nmax, dtype=torch.int32, device=dev)
    o_cd = torch.empty(nmax, dtype=torch.float32, device=dev)
    o_rx = torch.empty(rec_cap, dtype=torch.int32, device=dev)
    o_ry = torch.empty(rec_cap, dtype=torch.int32, device=dev)
    o_rk = torch.empty(rec_cap, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    n_upd = W.n_updates

    def reset():
        H.copy_from(H0, sp)
        G.copy_from(G0, sp)
        flush.fill_(rank + 1)

    def apply(files, st, cd, rx, ry, rk):
        uid, acc, nrec = 0, 0, 0
        for op, s_, d_, w_ in files:
            p = W.dparams if op else W.iparams
            nrec += dyg.stream_file_into(G, H, op, s_, d_, w_, p, st, cd, rx, ry, rk, rec_cap,
                                         first_update_id=uid, stream=sp)
            uid += len(s_)
        return nrec

    if args.profile_only:
        reset()
        apply(dfiles, o_st, o_cd, o_rx, o_ry, o_rk)
        torch.cuda.synchronize()
        return None
    for _ in range(args.warmup):
        reset()
        apply(dfiles, o_st, o_cd, o_rx, o_ry, o_rk)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    m0 = (H.counters()[0], G.counters()[0])
    launches0 = dyg.kernel_launches()
    dyg.profile_reset()
    dyg.profile_enable(True)
    times, nrec = [], 0
    for _ in range(args.steps):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        nrec = apply(dfiles, o_st, o_cd, o_rx, o_ry, o_rk)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    dyg.profile_enable(False)
    prof = dyg.profile_read()
    launches = dyg.kernel_launches() - launches0
    m1 = (H.counters()[0], G.counters()[0])
    clk = clocks.stop()
    barrier()
    ms = float(np.mean(times))
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    incr_moves = (m1[0] - m0[0]) / args.steps
    decr_moves = (m1[1] - m0[1]) / args.steps

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        hfiles = [(op, pin(s_), pin(d_), None if w_ is None else pin(w_)) for op, s_, d_, w_ in W.files]
        h_st, h_cd = pin(np.empty(nmax, np.int32)), pin(np.empty(nmax, np.float32))
        h_rx, h_ry = pin(np.empty(rec_cap, np.uint32)), pin(np.empty(rec_cap, np.uint32))
        h_rk = pin(np.empty(rec_cap, np.uint8))
        barrier()
        torch.cuda.synchronize()
        et, nrec_h = [], 0
        for _ in range(max(1, args.steps)):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            nrec_h = apply(hfiles, h_st, h_cd, h_rx, h_ry, h_rk)
            e1.record(stream)
            e1.synchronize()
            et.append(e0.elapsed_time(e1))
        barrier()
        ems = float(np.mean(et))
        if world > 1:
            import torch.distributed as dist
            tt = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        nins = sum(len(f[1]) for f in W.files if f[0] == 0)
        e2e = {"value": world * n_upd / (ems / 1e3), "unit": "edge_updates/s", "ms_per_step": ems,
               "h2d_bytes_per_step": int(nins * 12 + (n_upd - nins) * 8),
               "d2h_bytes_per_step": int(n_upd * 8 + nrec_h * 9)}

    walk_ms = prof["incr_walk_ms"] + prof["decr_walk_ms"]
    walk_launches = prof["incr_walk_launches"] + prof["decr_walk_launches"]
    res = {
        "ms_per_step": ms, "steps_ms": times, "nin": n_upd, "ndel": 0, "accepted": None,
        "recovered": nrec, "incr_moves": incr_moves, "decr_moves": decr_moves,
        "walk_ms_per_step": walk_ms / args.steps, "walk_launches": walk_launches, "prof": prof,
        "launches_per_step": launches / args.steps, "clocks": clk, "e2e": e2e,
        "dom_kernel": dom_name(prof),
        "dom_bytes_per_launch": dom_bytes(prof, incr_moves, decr_moves, args.steps),
        "dom_ms_per_launch": dom_ms(prof),
        "W": W,
    }
    for g in (H, G, H0, G0):
        g.close()
    return res


def run_many(args, rank, world, local_rank):
    """Many graphs: union rounds (timed) and the plain per-graph loop."""
    import torch
    import dygrass_b200 as dyg
    from dygrass_b200.multi import ManyGraphs, autotune

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = make_workload(args, rank, world)
    p = W.params
    best, trials = autotune(W.cases, params=p, chunks=(32, 64), blocks=(0, 4),
                            walkers=(128, 256) if args.tune_walkers else (),
                            max_steps=(48, 64, 80) if args.tune_walkers else (), repeats=2,
                            device=local_rank, sync=torch.cuda.synchronize)
    p = best["params"]
    M = ManyGraphs(W.cases, device=local_rank)
    plan = M.plan()
    H0, G0 = M.H.clone(), M.G.clone()
    t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a if dt is None else a.view(dt))).to(dev)
    for rd in plan.rounds:
        rd.src, rd.dst, rd.w, rd.uid = (t(rd.src, np.int32), t(rd.dst, np.int32), t(rd.w),
                                        t(rd.uid, np.int64))
    outs = [dyg.IncrementalResult(torch.empty(len(rd.graph), dtype=torch.int32, device=dev),
                                  torch.empty(len(rd.graph), dtype=torch.float32, device=dev),
                                  torch.empty(len(rd.graph), dtype=torch.uint8, device=dev))
            for rd in plan.rounds]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def reset():
        M.H.copy_from(H0, sp)
        M.G.copy_from(G0, sp)
        flush.fill_(rank + 1)

    if args.profile_only:
        reset()
        M.run(plan, p, stream=sp, outs=outs)
        torch.cuda.synchronize()
        return None
    for _ in range(args.warmup):
        reset()
        M.run(plan, p, stream=sp, outs=outs)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    m0 = M.H.counters()[0]
    launches0 = dyg.kernel_launches()
    dyg.profile_reset()
    dyg.profile_enable(True)
    times = []
    for _ in range(args.steps):
        reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        M.run(plan, p, stream=sp, outs=outs)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    dyg.profile_enable(False)
    prof = dyg.profile_read()
    launches = dyg.kernel_launches() - launches0
    incr_moves = (M.H.counters()[0] - m0) / args.steps
    clk = clocks.stop()
    barrier()
    ms = float(np.mean(times))
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    accepted = int(sum(int(o.accepted.sum().item()) for o in outs))

    # the plain path: every graph its own handles and its own update loop
    plain_ms = None
    if not args.no_plain:
        per = []
        for c in W.cases:
            Hg = dyg.Graph.from_edges(c.n, c.h_src, c.h_dst, c.h_w, device=local_rank)
            Gg = dyg.Graph.from_edges(c.n, c.g_src, c.g_dst, c.g_w, device=local_rank)
            per.append((Hg, Gg, Hg.clone(), Gg.clone(), t(c.ins_src, np.int32), t(c.ins_dst, np.int32),
                        t(c.ins_w), dyg.IncrementalResult(
                            torch.empty(len(c.ins_src), dtype=torch.int32, device=dev),
                            torch.empty(len(c.ins_src), dtype=torch.float32, device=dev),
                            torch.empty(len(c.ins_src), dtype=torch.uint8, device=dev))))
        pt = []
        for it in range(2):
            for Hg, Gg, H0g, G0g, *_ in per:
                Hg.copy_from(H0g, sp)
                Gg.copy_from(G0g, sp)
            flush.fill_(rank + 2)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for Hg, Gg, _, _, s_, d_, w_, o_ in per:
                dyg.incremental_stream(Hg, s_, d_, w_, p, G=Gg, stream=sp, out=o_)
            e1.record(stream)
            e1.synchronize()
            if it:
                pt.append(e0.elapsed_time(e1))
        plain_ms = float(np.mean(pt))
        plain_acc = int(sum(int(x[-1].accepted.sum().item()) for x in per))
        assert plain_acc == accepted, "union rounds and per-graph loops disagree"
        for x in per:
            for g in x[:4]:
                g.close()

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        hplan = M.plan()
        for rd in hplan.rounds:
            rd.src, rd.dst, rd.w, rd.uid = pin(rd.src), pin(rd.dst), pin(rd.w), pin(rd.uid)
        houts = [dyg.IncrementalResult(pin(np.empty(len(rd.graph), np.int32)),
                                       pin(np.empty(len(rd.graph), np.float32)),
                                       pin(np.empty(len(rd.graph), np.uint8))) for rd in hplan.rounds]
        et = []
        for _ in range(max(1, args.steps)):
            reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            M.run(hplan, p, stream=sp, outs=houts)
            e1.record(stream)
            e1.synchronize()
            et.append(e0.elapsed_time(e1))
        ems = float(np.mean(et))
        if world > 1:
            import torch.distributed as dist
            tt = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ems = float(tt.item())
        units_e2e = W.job_updates if args.split_mode == "partition" else world * plan.n_edges
        e2e = {"value": units_e2e / (ems / 1e3), "unit": "edge_updates/s",
               "ms_per_step": ems, "h2d_bytes_per_step": int(plan.n_edges * 20),
               "d2h_bytes_per_step": int(plan.n_edges * 9)}

    res = {
        "ms_per_step": ms, "steps_ms": times, "nin": plan.n_edges, "ndel": 0,
        "accepted": accepted, "recovered": 0, "incr_moves": incr_moves, "decr_moves": 0.0,
        "walk_ms_per_step": prof["incr_walk_ms"] / args.steps,
        "walk_launches": prof["incr_walk_launches"], "prof": prof,
        "launches_per_step": launches / args.steps, "clocks": clk, "e2e": e2e,
        "dom_kernel": "k_walk<1,0>",
        "dom_bytes_per_launch": dom_bytes(prof, incr_moves, 0.0, args.steps),
        "dom_ms_per_launch": dom_ms(prof),
        "plain_ms_per_step": plain_ms,
        "tuned": {k: v for k, v in best.items() if k != "params"},
        "tune_trials": [{k: v for k, v in t.items() if k != "params"} for t in trials], "W": W,
    }
    for g in (H0, G0):
        g.close()
    M.close()
    return res


def _arrive(reqs, rate):
    """Copies of the requests with Poisson arrival times at `rate` per
    second (the request set's own exponential draws, rescaled; rate None:
    all pending at once)."""
    import dataclasses
    out = [dataclasses.replace(r) for r in reqs]
    for r in out:
        r.arrival = 0.0 if rate is None else r.arrival / rate
    return out


def run_serve(args, rank, world, local_rank):
    """The serving workload through the native pool server.  Steady state:
    before every replay (untimed) the server is reset to the registered graphs
    and every graph is prefetched, then the requests are replayed at
    saturation (all pending at once) or at Poisson rates, device-timed, each
    request getting the result it gets alone.  Oversubscribed: the same replay
    with a budget of half the mix's footprint, starting with no graph
    resident, so graphs are admitted and evicted while requests run.  The
    plain path is every graph on its own handles, requests one at a time."""
    import torch
    import dygrass_b200 as dyg
    from dygrass_b200.serve import PlainServer, PoolServer, footprint_bytes, latency_stats

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = make_workload(args, rank, world)
    fp_total = sum(footprint_bytes(c.n, len(c.g_src), len(c.h_src)) for c in W.cases)
    S = PoolServer(W.cases, W.params, W.dparams, hbm_budget=int(fp_total * 1.5), device=local_rank)
    stream = torch.cuda.current_stream(dev)
    sync = torch.cuda.synchronize
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    n_upd = W.n_updates
    n_ins = sum(len(r.src) for r in W.requests if r.op == 0)

    def warm(server):
        server.restore()
        if isinstance(server, PoolServer):
            for g in range(len(W.cases)):
                assert server.prefetch(g)

    def replay(server, rate, reset=warm):
        reset(server)
        flush.fill_(rank + 1)
        sync()
        return server.serve(_arrive(W.requests, rate), sync=sync)

    if args.profile_only:
        replay(S, None)
        return None
    for _ in range(args.warmup):
        replay(S, None)
    sync()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = dyg.kernel_launches()
    dyg.profile_reset()
    times, steps, moves = [], 0, [0, 0]
    phases = {k: 0.0 for k in ("admit", "stage", "insert", "delete", "fetch", "split")}
    nrec = 0
    for _ in range(args.steps):
        warm(S)
        flush.fill_(rank + 1)
        sync()
        m0 = S.counters()
        reqs = _arrive(W.requests, None)
        dyg.profile_enable(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done = S.serve(reqs)
        e1.record(stream)
        e1.synchronize()
        dyg.profile_enable(False)
        times.append(e0.elapsed_time(e1))
        m1 = S.counters()
        moves[0] += m1[0] - m0[0]
        moves[1] += m1[1] - m0[1]
        st = S.stats()   # the replay's own (warm() resets the server)
        steps = st["steps"]
        for k in phases:
            phases[k] += st["ns_" + k] / 1e6 / args.steps
        nrec = sum(len(r.rec_src) for r in done if r.op == 1 and r.rec_src is not None)
    prof = dyg.profile_read()
    launches = dyg.kernel_launches() - launches0
    clk = clocks.stop()
    ms = float(np.mean(times))
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    incr_moves, decr_moves = moves[0] / args.steps, moves[1] / args.steps
    capacity = len(W.requests) / (ms / 1e3)      # requests per second at saturation

    # latency at swept arrival rates, server and plain path
    P = PlainServer(W.cases, W.params, W.dparams, device=local_rank)
    P.snapshot()
    sweep = []
    for frac in (0.25, 0.5, 0.9):
        rate = capacity * frac
        row = {"rate_req_per_s": rate, "fraction_of_capacity": frac,
               "server": latency_stats(replay(S, rate))}
        row["plain"] = latency_stats(replay(P, rate))
        sweep.append(row)
    sync()
    plain_sat = latency_stats(replay(P, None))
    P.close()
    S.close()
    # oversubscribed: half the footprint, no graph resident at the start
    S2 = PoolServer(W.cases, W.params, W.dparams, hbm_budget=int(fp_total * 0.5), device=local_rank)
    over = []
    for _ in range(2):
        S2.restore()
        flush.fill_(rank + 1)
        sync()
        reqs = _arrive(W.requests, None)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done2 = S2.serve(reqs)
        e1.record(stream)
        e1.synchronize()
        st2 = S2.stats()
        row = {"ms_per_replay": e0.elapsed_time(e1), "admissions": st2["admissions"],
               "evictions": st2["evictions"], "steps": st2["steps"]}
        row.update({k: v for k, v in latency_stats(done2).items() if k != "throughput_updates_per_s"})
        row["updates_per_s"] = n_upd / (row["ms_per_replay"] / 1e3)
        over.append(row)
    S2.close()
    plain_ups = plain_sat["throughput_updates_per_s"]
    res = {
        "ms_per_step": ms, "steps_ms": times, "nin": n_upd, "ndel": 0, "accepted": None,
        "recovered": nrec, "incr_moves": incr_moves, "decr_moves": decr_moves,
        "walk_ms_per_step": (prof["incr_walk_ms"] + prof["decr_walk_ms"]) / args.steps,
        "walk_launches": prof["incr_walk_launches"] + prof["decr_walk_launches"], "prof": prof,
        "launches_per_step": launches / args.steps, "clocks": clk,
        "e2e": {"value": (W.job_updates if args.split_mode == "partition" else world * n_upd)
                         / (ms / 1e3), "unit": "edge_updates/s", "ms_per_step": ms,
                "h2d_bytes_per_step": int(sum(len(r.src) * (20 if r.op == 0 else 16)
                                              for r in W.requests)),
                "d2h_bytes_per_step": int(sum(len(r.src) * (9 if r.op == 0 else 8)
                                              for r in W.requests)),
                "note": "the server takes host arrays: its device-timed run is end to end"},
        "dom_kernel": dom_name(prof),
        "dom_bytes_per_launch": dom_bytes(prof, incr_moves, decr_moves, args.steps),
        "dom_ms_per_launch": dom_ms(prof),
        "serving": {"server_steps_per_replay": steps, "capacity_req_per_s": capacity,
                    "insertions_per_replay": n_ins, "deletions_per_replay": n_upd - n_ins,
                    "footprint_bytes": fp_total, "budget_bytes": int(fp_total * 1.5),
                    "host_phase_ms_per_replay": phases,
                    "phase_note": "host wall time of the server's steps: admission, staging, the "
                                  "insertion and deletion runs (device work and synchronize "
                                  "included), result fetch, per-request split",
                    "sweep": sweep, "plain_saturated": plain_sat,
                    "speedup_vs_plain": (n_upd / (ms / 1e3)) / plain_ups if plain_ups else None,
                    "oversubscribed": {"budget_bytes": int(fp_total * 0.5), "replays": over},
                    "scheduler": "native pool server (include/dyg_serve.h): loop thread, pinned "
                                 "staging, admission by footprint, eviction to host memory"},
        "W": W,
    }
    return res


# --------------------------------------------------------- CPU baseline

def cpu_baseline_serve(W, threads=None, max_requests=300):
    """The oracle applying the first requests one by one on their graphs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    th = threads or pyoracle.max_threads()
    reqs = W.requests[:max_requests]
    gs, uid = {}, {}
    for r in reqs:
        if r.graph not in gs:
            c = W.cases[r.graph]
            gs[r.graph] = (pyoracle.OGraph(c.n, c.g_src, c.g_dst, c.g_w),
                           pyoracle.OGraph(c.n, c.h_src, c.h_dst, c.h_w))
            uid[r.graph] = 0
    t0 = time.perf_counter()
    for r in reqs:
        Go, Ho = gs[r.graph]
        if r.op == 0:
            pyoracle.incremental(Ho, r.src, r.dst, r.w, W.params, G=Go, threads=th,
                                 first_uid=uid[r.graph], single_batch=True)
        else:
            pyoracle.decremental(Go, Ho, r.src, r.dst, W.dparams, threads=th,
                                 first_uid=uid[r.graph], single_batch=True)
        uid[r.graph] += len(r.src)
    dt = time.perf_counter() - t0
    nu = sum(len(r.src) for r in reqs)
    return {"value": nu / dt, "unit": "edge_updates/s", "cores": th, "kind": "port", "seconds": dt,
            "sample": f"oracle (C/OpenMP, {th} threads): the first {len(reqs)} requests ({nu} "
                      f"updates) one by one on their graphs (graph loading not timed)"}


def cpu_baseline_many(W, threads=None):
    """The oracle's per-graph update loop over every graph of the workload,
    measured end to end (graph loading not timed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    th = threads or pyoracle.max_threads()
    gs = [(pyoracle.OGraph(c.n, c.h_src, c.h_dst, c.h_w), pyoracle.OGraph(c.n, c.g_src, c.g_dst, c.g_w))
          for c in W.cases]
    t0 = time.perf_counter()
    for c, (Ho, Go) in zip(W.cases, gs):
        pyoracle.incremental(Ho, c.ins_src, c.ins_dst, c.ins_w, W.params, G=Go, threads=th)
    dt = time.perf_counter() - t0
    return {"value": W.n_updates / dt, "unit": "edge_updates/s", "cores": th, "kind": "port",
            "seconds": dt,
            "sample": f"oracle (C/OpenMP, {th} threads): the whole workload, every graph's update "
                      f"loop ({len(W.cases)} graphs, {W.n_updates} insertions), measured; walkers "
                      f"run to their natural end as the reference's do"}


def _one_core(pyoracle, th, runs):
    """Times each (label, fn(threads)) of `runs` at 1 thread and at `th`
    threads; fn gets fresh identical state each time.  Returns the rates."""
    out = {}
    tot = [0, 0.0, 0.0]
    for label, n_upd, fn in runs:
        t1 = fn(1)
        tn = fn(th)
        out[label] = {"updates": n_upd, "seconds_1_core": t1, f"seconds_{th}_cores": tn,
                      "value_1_core": n_upd / t1, f"value_{th}_cores": n_upd / tn}
        tot[0] += n_upd
        tot[1] += t1
        tot[2] += tn
    # the samples together: updates over the summed measured times
    out["samples_together"] = {"updates": tot[0], "value_1_core": tot[0] / tot[1],
                               f"value_{th}_cores": tot[0] / tot[2]}
    return out


def cpu_baseline_mixed(W, threads=None, one_core=True):
    """The oracle on the whole mixed stream, file by file in stream order,
    measured end to end.  With one_core: the first insertion file and the
    first deletion file, each from identical cloned state, at 1 thread and at
    all threads (measured rates of that sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    th = threads or pyoracle.max_threads()
    Ho = pyoracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    Go = pyoracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w)
    snaps = {}
    uid, dt = 0, 0.0
    for op, s_, d_, w_ in W.files:
        if one_core and op not in snaps:
            snaps[op] = (Go.clone(), Ho.clone(), uid, s_, d_, w_)
        p = W.dparams if op else W.iparams
        t0 = time.perf_counter()
        pyoracle.stream_file(Go, Ho, op, s_, d_, w_, p, first_uid=uid, threads=th)
        dt += time.perf_counter() - t0
        uid += len(s_)
    nins = sum(len(f[1]) for f in W.files if f[0] == 0)
    out = {"value": W.n_updates / dt, "unit": "edge_updates/s", "cores": th, "kind": "port",
           "seconds": dt,
           "sample": f"oracle (C/OpenMP, {th} threads): the whole stream ({len(W.files)} files, "
                     f"{nins} insertions, {W.n_updates - nins} deletions) in order, measured; "
                     f"walkers run to their natural end as the reference's do"}
    if one_core:
        runs = []
        for op, (g0, h0, u0, s_, d_, w_) in sorted(snaps.items()):
            p = W.dparams if op else W.iparams

            def fn(t, g0=g0, h0=h0, u0=u0, s_=s_, d_=d_, w_=w_, op=op, p=p):
                g, h = g0.clone(), h0.clone()
                t0 = time.perf_counter()
                pyoracle.stream_file(g, h, op, s_, d_, w_, p, first_uid=u0, threads=t)
                return time.perf_counter() - t0
            runs.append(("first_delete_file" if op else "first_insert_file", len(s_), fn))
        out["one_core"] = _one_core(pyoracle, th, runs)
    return out


def cpu_baseline(W, threads=None, one_core=True):
    """The oracle (the reference's update loop restated in C; OpenMP over the
    (edge, walker) pairs of a batch) on the whole workload, measured end to
    end: the insertion stream in the reference's ceil(N/10) batches, every
    insertion also entering G, then the deletion stream in ceil(N/10)
    batches.  Walkers run to their natural end, as the reference's do.
    With one_core: two samples, each timed at 1 thread and at all threads
    from identical cloned state -- the first insertion batch on the initial
    graphs, and the first tenth of the first deletion batch (as one batch) on
    the graphs the insertions left."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    th = threads or pyoracle.max_threads()
    nin, ndel = len(W.ins_src), len(W.del_src)
    Ho = pyoracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    Go = pyoracle.OGraph(W.n, W.g_src, W.g_dst, W.g_w)
    h_init, g_init = (Ho.clone(), Go.clone()) if one_core else (None, None)
    from dygrass_b200 import reference_batch_size
    B = reference_batch_size(nin)
    t0 = time.perf_counter()
    pyoracle.incremental(Ho, W.ins_src, W.ins_dst, W.ins_w, W.params, batch_size=B, G=Go, threads=th)
    t_in = time.perf_counter() - t0
    h_mid, g_mid = (Ho.clone(), Go.clone()) if (one_core and ndel) else (None, None)
    t_de = 0.0
    if ndel:
        Bd = reference_batch_size(ndel)
        t0 = time.perf_counter()
        pyoracle.decremental(Go, Ho, W.del_src, W.del_dst, W.dparams, batch_size=Bd, threads=th)
        t_de = time.perf_counter() - t0
    out = {"value": (nin + ndel) / (t_in + t_de), "unit": "edge_updates/s", "cores": th,
           "kind": "port", "seconds": t_in + t_de,
           "seconds_insertions": t_in, "seconds_deletions": t_de,
           "sample": f"oracle (C/OpenMP, {th} threads): the whole workload, {nin} insertions in "
                     f"batches of {B}" + (f" then {ndel} deletions in batches of "
                                          f"{reference_batch_size(ndel)}" if ndel else "")
                     + ", measured; walkers run to their natural end as the reference's do"}
    if one_core:
        runs = []

        def f_ins(t):
            h, g = h_init.clone(), g_init.clone()
            t0 = time.perf_counter()
            pyoracle.incremental(h, W.ins_src[:B], W.ins_dst[:B], W.ins_w[:B], W.params, G=g,
                                 threads=t, first_uid=0, single_batch=True)
            return time.perf_counter() - t0
        runs.append(("first_insertion_batch", B, f_ins))
        if ndel:
            nd = max(1, reference_batch_size(ndel) // 10)

            def f_del(t):
                g, h = g_mid.clone(), h_mid.clone()
                t0 = time.perf_counter()
                pyoracle.decremental(g, h, W.del_src[:nd], W.del_dst[:nd], W.dparams, threads=t,
                                     first_uid=0, single_batch=True)
                return time.perf_counter() - t0
            runs.append(("first_deletions_as_one_batch", nd, f_del))
        out["one_core"] = _one_core(pyoracle, th, runs)
    return out


# ------------------------------------------------- the reference's GPU updater

_TIME_RE = None


def _time_taken(stdout):
    """The "Time taken: N milliseconds" line both updaters print."""
    import re
    global _TIME_RE
    _TIME_RE = _TIME_RE or re.compile(r"Time taken: (\d+) milliseconds")
    m = _TIME_RE.search(stdout)
    return int(m.group(1)) if m else None


def _write_mtx(path, s, d, w=None, base=1):
    with open(path, "w") as f:
        for i in range(len(s)):
            f.write(f"{int(s[i]) + base} {int(d[i]) + base}"
                    + ("" if w is None else f" {float(w[i]):.9g}") + "\n")


def run_refgpu(args):
    """The reference's own CUDA updaters (unmodified sources built for sm_100a
    into oracle/_ref) against this library on identical input files, on one
    B200.  Cases are those the reference runs correctly: the 100x100 grid
    with 1,000 insertions, a 30^3 mesh with 6,000 insertions (inside the room
    its grown rows have), and 1,000 sparsifier deletions on a 20^3 mesh (every
    deletion in H, which its batch indexing needs).  Each binary prints its
    own "Time taken" (ms resolution, the span of
    random_walk_incremental/main.cu:297-344 and
    random_walk_decremental/main.cu:388-449); each runs `repeats` times and
    the median counts.  This library is timed three ways on the same inputs
    with max_steps 100 (the reference's compile-time value): the drop-in
    executables (same print, same span), the library call with host arrays
    (copies included; CUDA events), and the library call on device-resident
    arrays, each with pruned and with exhaustive walkers."""
    import shutil
    import torch
    import dygrass_b200 as dyg
    import dygrass_b200.workloads as wl
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    our_dir = os.path.join(ROOT, "dygrass_b200", "bin")
    need = [os.path.join(ref_dir, b) for b in ("incremental_update", "decremental_update")]
    if not all(os.path.exists(x) for x in need):
        print(json.dumps({"workload": "refgpu", "unavailable": "the reference's updaters are not "
                          "built in oracle/_ref (make -C oracle ref-gpu where its sources are)"}))
        return 0
    torch.cuda.set_device(0)
    R = max(1, args.refgpu_repeats)
    tmp = tempfile.mkdtemp(prefix="dyg_refgpu_")
    cases = []

    def run_cli(exe, argv, cwd):
        cp = subprocess.run([exe] + argv, cwd=cwd, capture_output=True, text=True, timeout=600)
        return _time_taken(cp.stdout), cp

    def lib_times(fn, reps):
        ts = []
        for _ in range(reps):
            setup = fn(None)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            fn(setup)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return ts

    try:
        for name, kind, thr in (("grid 100x100, 1,000 insertions, threshold 10, 512 walkers", "incr", 10.0),
                                ("mesh 30^3, 6,000 insertions, threshold 100, 512 walkers", "incr", 100.0),
                                ("mesh 20^3 + 2,000 insertions, 1,000 sparsifier deletions, 512 walkers",
                                 "decr", 100.0)):
            case = {"case": name}
            if kind == "incr":
                W = wl.grid_2d(100, 100, inserts=1000) if "grid" in name else wl.mesh_3d(30, inserts=6000)
                n_upd = len(W.ins_src)
                files = lambda ds: (_write_mtx(os.path.join(ds, "adj_sparse.mtx"), W.h_src, W.h_dst,
                                               W.h_w, base=0),
                                    _write_mtx(os.path.join(ds, "ext.mtx"), W.ins_src, W.ins_dst,
                                               W.ins_w, base=1))
                argv = lambda g: [g, repr(thr), "512"]
                exe_ref, exe_our = need[0], os.path.join(our_dir, "incremental_update")
                p = dyg.WalkParams.make(threshold=thr, walkers=512, max_steps=100)
                H0 = dyg.Graph.from_edges(W.n, W.h_src, W.h_dst, W.h_w)
                H = H0.clone()
                dev = [torch.from_numpy(np.ascontiguousarray(a).view(np.int32 if a.dtype == np.uint32
                                                                      else a.dtype)).cuda()
                       for a in (W.ins_src, W.ins_dst, W.ins_w)]

                def lib_call(pp, arrays):
                    def fn(setup):
                        if setup is None:
                            H.copy_from(H0)
                            return True
                        dyg.incremental_stream(H, *arrays, pp)
                    return fn
                host = (W.ins_src, W.ins_dst, W.ins_w)
            else:
                W = wl.mesh_3d(20, inserts=2000)
                gs = np.concatenate([W.g_src, W.ins_src, [W.n]]).astype(np.uint32)
                gd = np.concatenate([W.g_dst, W.ins_dst, [W.n + 1]]).astype(np.uint32)
                gw = np.concatenate([W.g_w, W.ins_w, [1.0]]).astype(np.float32)
                hs = np.concatenate([W.h_src, [W.n]]).astype(np.uint32)
                hd = np.concatenate([W.h_dst, [W.n + 1]]).astype(np.uint32)
                hw = np.concatenate([W.h_w, [1.0]]).astype(np.float32)
                pick = np.random.default_rng(8).choice(len(W.h_src), 1000, replace=False)
                ds_, dd_ = W.h_src[pick].astype(np.uint32), W.h_dst[pick].astype(np.uint32)
                n_upd = len(ds_)
                files = lambda ds: (_write_mtx(os.path.join(ds, "updated_dense.mtx"), gs, gd, gw),
                                    _write_mtx(os.path.join(ds, "updated_adj_sparse.mtx"), hs, hd, hw),
                                    _write_mtx(os.path.join(ds, "del.mtx"), ds_, dd_))
                argv = lambda g: [g]
                exe_ref, exe_our = need[1], os.path.join(our_dir, "decremental_update")
                p = dyg.WalkParams.make(walkers=512, max_steps=100)
                nv = W.n + 2
                G0, H0 = dyg.Graph.from_edges(nv, gs, gd, gw), dyg.Graph.from_edges(nv, hs, hd, hw)
                G, H = G0.clone(), H0.clone()
                dev = [torch.from_numpy(a.view(np.int32)).cuda() for a in (ds_, dd_)]

                def lib_call(pp, arrays):
                    def fn(setup):
                        if setup is None:
                            G.copy_from(G0)
                            H.copy_from(H0)
                            return True
                        dyg.decremental_stream(G, H, *arrays, pp)
                    return fn
                host = (ds_, dd_)
            case["updates"] = n_upd
            for who, exe in (("reference", exe_ref), ("ours_cli", exe_our)):
                ms = []
                for r in range(R):
                    root = os.path.join(tmp, f"{who}{r}")
                    ds = os.path.join(root, "dataset", "g")
                    os.makedirs(ds)
                    os.makedirs(os.path.join(root, "run"))
                    files(ds)
                    t, cp = run_cli(exe, argv("g"), os.path.join(root, "run"))
                    if t is None:
                        raise RuntimeError(f"{who} printed no time: {cp.stdout[-300:]} {cp.stderr[-300:]}")
                    ms.append(t)
                    shutil.rmtree(root, ignore_errors=True)
                case[f"{who}_ms"] = {"median": float(np.median(ms)), "runs": ms,
                                     "resolution": "1 ms (the binary's own print)"}
            pe = type(p).from_buffer_copy(p)
            pe.flags |= dyg.FLAG_EXHAUSTIVE
            for label, pp, arrays in (("ours_lib_device", p, dev), ("ours_lib_device_exhaustive", pe, dev),
                                      ("ours_lib_host", p, host), ("ours_lib_host_exhaustive", pe, host)):
                lib_times(lib_call(pp, arrays), 2)   # warm-up
                ts = lib_times(lib_call(pp, arrays), R)
                case[f"{label}_ms"] = {"median": float(np.median(ts)), "runs": ts,
                                       "resolution": "CUDA events"}
            ref_ms = case["reference_ms"]["median"]
            for label in ("ours_cli", "ours_lib_device", "ours_lib_device_exhaustive", "ours_lib_host",
                          "ours_lib_host_exhaustive"):
                m = case[f"{label}_ms"]["median"]
                case[f"{label}_updates_per_s"] = n_upd / (m / 1e3) if m > 0 else None
                case[f"speedup_{label}_vs_reference"] = ref_ms / m if m > 0 else None
            case["reference_updates_per_s"] = n_upd / (ref_ms / 1e3) if ref_ms > 0 else None
            cases.append(case)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print(json.dumps({"metric": "edge updates/sec, the reference's CUDA updater vs this library",
                      "workload": "refgpu", "unit": "edge_updates/s", "n_gpus": 1, "repeats": R,
                      "data": "synthetic (seeded generators, dygrass_b200/workloads.py), written as "
                              "the reference's .mtx files", "cases": cases}))
    return 0


# ---------------------------------------------------------------- main

def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    args.split_mode = resolve_split(args, world) if args.impl != "reference" else "replicas"
    if args.split_mode == "shard":
        args.shard = True

    if args.workload == "refgpu":   # one line holding both updaters' times
        return run_refgpu(args) if rank == 0 else 0
    if args.impl == "reference":
        if rank != 0:
            return 0
        W = make_workload(args, 0)
        base = {"rmat": cpu_baseline_mixed, "rgg_many": cpu_baseline_many,
                "serve": cpu_baseline_serve}.get(args.workload, cpu_baseline)
        vals = []
        for i in range(args.warmup + args.steps):
            r = base(W, one_core=False) if base is not cpu_baseline_many and \
                base is not cpu_baseline_serve else base(W)
            if i >= args.warmup:
                vals.append(r)
        # a step's time is the measured time of its sample (the whole workload,
        # except for serve)
        v = float(np.mean([r["value"] for r in vals]))
        out = {"metric": "edge updates/sec (incr+decr)", "value": v, "unit": "edge_updates/s",
               "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": float(np.mean([r["seconds"] for r in vals])) * 1e3,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded)", "config": workload_config(W, args),
               "cpu_baseline": {k: vals[-1][k] for k in ("value", "unit", "cores", "kind", "sample")},
               "e2e": {"value": v, "unit": "edge_updates/s", "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}}
        out["cpu_baseline"]["value"] = v
        print(json.dumps(out))
        return 0

    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    runner = {"rmat": run_mixed, "rgg_many": run_many, "serve": run_serve}.get(args.workload,
                                                                                run_ours)
    res = runner(args, rank, world, local_rank)
    if res is None:
        return 0
    W = res.pop("W")
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    peak_note = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = res["dom_bytes_per_launch"] / (res["dom_ms_per_launch"] / 1e3) / 1e9
    traffic, traffic_src, l2_bytes = None, None, None
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tpath):
        for t in json.load(open(tpath)).get("entries", []):
            opts = ("mesh_k", "rgg_graphs", "rgg_n_hi", "rmat_scale", "rmat_updates", "serve_requests")
            if t.get("workload") == args.workload and t.get("kernel") == res["dom_kernel"] \
                    and t.get("exhaustive", False) == args.exhaustive \
                    and all(t[o] == getattr(args, o) for o in opts if o in t):
                traffic = t.get("dram_bytes_per_launch")
                l2_bytes = t.get("l2_bytes_per_launch")
                traffic_src = "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch " \
                              "(profiles/roofline_traffic.json)"
    nin, ndel = res["nin"], res["ndel"]
    ms = res["ms_per_step"]
    if args.split_mode == "shard":
        units = nin + ndel                  # one workload, split over the ranks
    elif args.split_mode == "partition":
        units = W.job_updates               # the graphs divided over the ranks
    else:
        units = world * (nin + ndel)        # one replica per rank
    value = units / (ms / 1e3)
    moves = res["incr_moves"] + res["decr_moves"]
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        cpu = {"rmat": cpu_baseline_mixed, "rgg_many": cpu_baseline_many,
               "serve": cpu_baseline_serve}.get(args.workload, cpu_baseline)(W)
    out = {
        "metric": "edge updates/sec (incr+decr)",
        "value": value, "unit": "edge_updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators, dygrass_b200/workloads.py)",
        **({"scaling": "strong"} if args.split_mode in ("shard", "partition") else {}),
        "config": dict(workload_config(W, args), l2="flushed between steps (256 MB write)",
                       parallelism={"shard": f"one graph, batches sharded x{world} (winner keys "
                                                      f"all-reduced)",
                                    "partition": f"graphs partitioned by footprint x{world}",
                                    "replicas": f"replicas x{world}"}[args.split_mode]),
        "walker_steps_per_s": world * moves / (ms / 1e3),
        "breakdown": {"insertions_added": res["accepted"], "edges_recovered": res["recovered"],
                      "incr_walker_moves": res["incr_moves"], "decr_walker_moves": res["decr_moves"],
                      "walk_kernel_ms_per_step": res["walk_ms_per_step"],
                      "walk_launches_per_step": res["walk_launches"] / args.steps,
                      "launches_per_step": res["launches_per_step"],
                      "steps_ms": res["steps_ms"],
                      **({"exhaustive": res["exhaustive"]} if res.get("exhaustive") else {})},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "peak_source": f"{peak_note} hbm_gbs (MEASURED_PEAKS.json)",
                     "kernel": KERNEL_DESC[res["dom_kernel"]], "traffic_source": traffic_src,
                     "bytes_model": f"{BYTES_PER_MOVE} B per walker move (row descriptor sector + slot sector)",
                     "algorithmic_bytes_per_launch": res["dom_bytes_per_launch"],
                     "ms_per_launch": res["dom_ms_per_launch"],
                     "useful_bytes_per_move": 16,
                     "sector_efficiency": 16 / BYTES_PER_MOVE,
                     # payload bytes only (8 B descriptor + 8 B slot per move)
                     "sector_efficient_frac": achieved * 16 / BYTES_PER_MOVE / hbm,
                     # L2 bytes per launch (ncu lts__t_bytes.sum) over the live launch time
                     "l2_bytes_per_launch": l2_bytes,
                     "l2_gbs": (l2_bytes / (res["dom_ms_per_launch"] / 1e3) / 1e9) if l2_bytes else None,
                     "note": "the graphs are largely L2-resident: traffic (ncu DRAM bytes per launch) "
                             "is well below the algorithmic bytes, so frac is an equivalent-bandwidth "
                             "figure (l2_gbs is the L2 rate); the walk is bound by instruction issue "
                             "and gather latency (ncu counters of the walk kernel under profiles/); "
                             "of each move's two sectors, 16 B (descriptor + slot) are payload"},
        "clocks": res["clocks"],
        "e2e": res["e2e"],
        "gpu_launches": int(round(res["launches_per_step"] * args.steps)),
        "pruning": not args.exhaustive,
        **({"serving": res["serving"]} if args.workload == "serve" else {}),
        **({"batched": {"plain_per_graph_ms_per_step": res["plain_ms_per_step"],
                        "speedup_vs_plain": (res["plain_ms_per_step"] / ms
                                             if res["plain_ms_per_step"] else None),
                        "tuned": res["tuned"], "rounds": 10}}
           if args.workload == "rgg_many" else {}),
        "cpu_baseline": cpu,
    }
    print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
