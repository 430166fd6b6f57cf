"""Many independent graphs updated in one launch per round.

The graphs are packed into one union graph, each at its own vertex offset.
Walks never leave a graph, rows only receive their own graph's edges, and
each edge carries its own update id (its position in its graph's stream), so
one dyg_incremental_batch_ids call over batch r of every graph gives each
graph exactly what its own reference loop (ceil(n/10)-edge batches,
random_walk_incremental/gpu_graph.cuh:135) gives for batch r.  A whole
stream of every graph is therefore max_g(#batches) launches of the update
pipeline instead of sum_g(#batches).

`autotune` picks the walk kernel's launch shape (walkers per warp fetch,
blocks per SM) by timing the rounds; the results do not depend on it.
Optionally it also lowers the walker count, keeping the fastest setting
whose kappa(L_G, L_H) on sample graphs stays within a tolerance of the
given walker count's.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import Graph, IncrementalResult, WalkParams, incremental_batch_ids, kappa, reference_batch_size, tune_set


@dataclass
class Round:
    src: object            # global ids (numpy or device tensor)
    dst: object
    w: object
    uid: object            # per-edge update ids
    graph: np.ndarray      # graph index of each edge (host)
    pos: np.ndarray        # position of each edge in its graph's stream (host)


@dataclass
class Plan:
    rounds: list
    n_edges: int
    counts: list = field(default_factory=list)   # insertions per graph


def plan_rounds(offsets, streams, batch_sizes=None) -> Plan:
    """Rounds over graphs at vertex offsets[g]: round r holds batch r of every
    graph's stream (src, dst, w local ids), with global ids, the edge's
    position in its graph's stream as its update id, and its graph index.
    Batch sizes are ceil(n_g/10) (random_walk_incremental/gpu_graph.cuh:135)
    unless given per graph."""
    per = []
    for g, (s, d, w) in enumerate(streams):
        m = len(s)
        B = (batch_sizes[g] if batch_sizes else reference_batch_size(m)) or 1
        per.append((g, np.asarray(s, np.uint32), np.asarray(d, np.uint32),
                    np.asarray(w, np.float32), m, B))
    nrounds = max((-(-m // B) for *_, m, B in per if m), default=0)
    rounds = []
    for r in range(nrounds):
        cs, cd, cw, cu, cg, cp = [], [], [], [], [], []
        for g, s, d, w, m, B in per:
            lo, hi = r * B, min((r + 1) * B, m)
            if lo >= hi:
                continue
            off = offsets[g]
            cs.append(s[lo:hi] + off)
            cd.append(d[lo:hi] + off)
            cw.append(w[lo:hi])
            cu.append(np.arange(lo, hi, dtype=np.uint64))
            cg.append(np.full(hi - lo, g, np.int32))
            cp.append(np.arange(lo, hi, dtype=np.int64))
        rounds.append(Round(np.concatenate(cs).astype(np.uint32), np.concatenate(cd).astype(np.uint32),
                            np.concatenate(cw), np.concatenate(cu), np.concatenate(cg),
                            np.concatenate(cp)))
    return Plan(rounds, sum(m for *_, m, _ in per), [m for *_, m, _ in per])


class ManyGraphs:
    """Union of independent graphs: H (and optionally G) on the device."""

    def __init__(self, cases, with_g: bool = True, device: int = -1, slack_per_row: int = 2):
        self.cases = cases
        self.offsets = np.zeros(len(cases) + 1, np.int64)
        self.offsets[1:] = np.cumsum([c.n for c in cases])
        self.n = int(self.offsets[-1])
        if self.n >= 2 ** 32:
            raise ValueError("too many vertices for one union graph")
        hs, hd, hw, gs, gd, gw = [], [], [], [], [], []
        for off, c in zip(self.offsets[:-1], cases):
            hs.append(c.h_src + off)
            hd.append(c.h_dst + off)
            hw.append(c.h_w)
            if with_g:
                gs.append(c.g_src + off)
                gd.append(c.g_dst + off)
                gw.append(c.g_w)
        cat = lambda a, t: np.concatenate(a).astype(t) if a else np.empty(0, t)
        self.H = Graph.from_edges(self.n, cat(hs, np.uint32), cat(hd, np.uint32), cat(hw, np.float32),
                                  slack_per_row=slack_per_row, device=device)
        self.G = (Graph.from_edges(self.n, cat(gs, np.uint32), cat(gd, np.uint32),
                                   cat(gw, np.float32), slack_per_row=slack_per_row, device=device)
                  if with_g else None)

    def plan(self, streams=None, batch_sizes=None) -> Plan:
        """Rounds of the insertion streams (default: each case's ins_*):
        round r holds batch r of every graph, batch sizes ceil(n_g/10) unless
        given."""
        if streams is None:
            streams = [(c.ins_src, c.ins_dst, c.ins_w) for c in self.cases]
        return plan_rounds(self.offsets, streams, batch_sizes)

    def run(self, plan: Plan, params: WalkParams, stream: int | None = None, outs=None):
        """Applies every round; returns the per-round IncrementalResults."""
        res = []
        for i, rd in enumerate(plan.rounds):
            out = outs[i] if outs else None
            res.append(incremental_batch_ids(self.H, rd.src, rd.dst, rd.w, rd.uid, params, G=self.G,
                                             stream=stream, out=out))
        return res

    def per_graph(self, plan: Plan, results):
        """Scatters round results back: a list of (found_at, cond, accepted)
        per graph, in stream order."""
        out = [(np.empty(m, np.int32), np.empty(m, np.float32), np.empty(m, np.uint8))
               for m in plan.counts]
        for rd, r in zip(plan.rounds, results):
            fa = np.asarray(r.found_at if isinstance(r.found_at, np.ndarray) else r.found_at.cpu())
            cd = np.asarray(r.conductance if isinstance(r.conductance, np.ndarray) else r.conductance.cpu())
            ac = np.asarray(r.accepted if isinstance(r.accepted, np.ndarray) else r.accepted.cpu())
            for g in np.unique(rd.graph):
                sel = rd.graph == g
                out[g][0][rd.pos[sel]] = fa[sel]
                out[g][1][rd.pos[sel]] = cd[sel]
                out[g][2][rd.pos[sel]] = ac[sel]
        return out

    def graph_rows(self, which: str, g: int):
        """(row_ptr, col, w) of graph g's part of H or G, local ids."""
        rp, col, w = (self.H if which == "H" else self.G).export()
        lo, hi = int(self.offsets[g]), int(self.offsets[g + 1])
        a, b = int(rp[lo]), int(rp[hi])
        return rp[lo:hi + 1] - rp[lo], col[a:b] - lo, w[a:b]

    def close(self):
        for x in (self.H, self.G):
            if x is not None:
                x.close()


def _timed(fn, sync):
    sync()
    t0 = time.perf_counter()
    fn()
    sync()
    return time.perf_counter() - t0


def autotune(cases, plan_streams=None, params: WalkParams | None = None,
             chunks=(32, 64, 128), blocks=(0, 5, 4), prune_every=(1, 2), walkers=(), max_steps=(),
             kappa_graphs: int = 4, kappa_tol: float = 0.05, repeats: int = 2, device: int = -1,
             sync=lambda: None):
    """Times the rounds of the cases' streams for each launch shape and prune
    interval (tune_set), then each walker count in `walkers` and each walk
    length in `max_steps` (below the parameters' own), each accepted only if
    the mean kappa of the
    `kappa_graphs` smallest graphs stays within kappa_tol of the value at the
    parameters' own walker count and walk length.  Returns (best dict, list of
    all measurements); the best dict's "params" are the walk parameters to
    use.  Leaves the best launch shape set (tune_set)."""
    params = params or WalkParams.make()
    trials = []
    M = ManyGraphs(cases, device=device)
    pl = M.plan(plan_streams)
    H0, G0 = M.H.clone(), M.G.clone()

    tune_set(0, 0)   # one untimed pass first: no trial pays the warm-up
    M.run(pl, params)
    sync()

    def measure(p, chunk, bpsm, pe=1):
        tune_set(chunk, bpsm, pe)
        t = []
        for _ in range(repeats):
            M.H.copy_from(H0)
            M.G.copy_from(G0)
            t.append(_timed(lambda: M.run(pl, p), sync))
        return min(t)

    for chunk in chunks:
        if params.walkers % chunk:
            continue
        for b in blocks:
            for pe in prune_every:
                trials.append({"walkers": params.walkers, "chunk": chunk, "blocks_per_sm": b,
                               "prune_every": pe, "seconds": measure(params, chunk, b, pe)})
    best = min(trials, key=lambda t: t["seconds"])
    best["params"] = params
    best["max_steps"] = params.max_steps
    if walkers or max_steps:
        small = sorted(range(len(cases)), key=lambda i: cases[i].n)[:kappa_graphs]

        def mean_kappa(p):
            M = ManyGraphs([cases[i] for i in small], device=device)
            pl = M.plan([(cases[i].ins_src, cases[i].ins_dst, cases[i].ins_w) for i in small])
            M.run(pl, p)
            ks = []
            for j, i in enumerate(small):
                c = cases[i]
                rp, col, w = M.graph_rows("H", j)
                rows = np.repeat(np.arange(c.n, dtype=np.uint32), np.diff(rp).astype(np.int64))
                keep = col >= rows
                gs = np.concatenate([c.g_src, c.ins_src])
                gd = np.concatenate([c.g_dst, c.ins_dst])
                gw = np.concatenate([c.g_w, c.ins_w])
                ks.append(kappa(c.n, gs, gd, gw, rows[keep], col[keep], w[keep])["kappa"])
            M.close()
            return float(np.mean(ks))

        k_ref = mean_kappa(params)
        best["kappa"] = k_ref
        # walker counts at the full walk length, then walk lengths at the
        # walker count chosen so far
        options = [(wk, params.max_steps) for wk in walkers
                   if wk < params.walkers and wk % 32 == 0]
        options += [(None, ms) for ms in max_steps if 0 < ms < params.max_steps]
        for wk, ms in options:
            wk = best["walkers"] if wk is None else wk
            p = WalkParams.make(threshold=params.threshold, walkers=wk, max_steps=ms,
                                heuristic_walkers=params.heuristic_walkers,
                                transition=params.transition, flags=params.flags,
                                seed=params.seed)
            k = mean_kappa(p)
            chunk = best["chunk"] if wk % best["chunk"] == 0 else 32
            t = {"walkers": wk, "max_steps": ms, "chunk": chunk,
                 "blocks_per_sm": best["blocks_per_sm"], "prune_every": best["prune_every"],
                 "kappa": k, "kappa_ok": abs(k - k_ref) <= kappa_tol * k_ref, "params": p}
            t["seconds"] = measure(p, chunk, best["blocks_per_sm"], best["prune_every"])
            trials.append(t)
            if t["kappa_ok"] and t["seconds"] < best["seconds"]:
                best = t
    for x in (H0, G0):
        x.close()
    M.close()
    tune_set(best["chunk"], best["blocks_per_sm"], best["prune_every"])
    return best, trials
