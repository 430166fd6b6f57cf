"""Serving many resident graphs with continuous batching.

Requests are update batches for one graph (insertions or deletions, any
size).  The server keeps every admitted graph resident in one union graph
(each at its own vertex offset, as in multi.py) with its own update counter,
so a graph's random streams depend only on its own history.  Each scheduler
step takes the oldest pending request of every graph that has one, runs all
insertion requests of the step as one incremental batch and all deletion
requests as one decremental batch, and completes them; requests that arrive
meanwhile join the next step.  Graphs are disjoint and a graph's requests run
in arrival order, one per step, so every request gets exactly the result it
gets when run alone on its graph's own handles (tested).

The scheduler is native (include/dyg_serve.h, csrc/server.cu): requests are
copied into its per-graph queues, its loop thread runs a step whenever one is
pending, stages each step through page-locked memory and splits the results
per request, and this module submits, polls and fetches.  Server(native=False)
runs the same steps from Python over dyg_incremental_batch_ids /
dyg_decremental_batch_ids (kept to measure the scheduler against).

Admission (Server): graphs are admitted in the given order while their
estimated device footprint (dense graph and sparsifier arenas and
descriptors) fits the HBM budget; requests for other graphs are refused.
PoolServer admits graphs as their requests are scheduled and evicts
resident ones to host memory to make room, within the same budget.
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

from . import (DygError, Graph, ServerDone, ServerGraphInfo, ServerStats, WalkParams, _check, _ptr,
               decremental_batch_ids, incremental_batch_ids, lib)

INSERT, DELETE = 0, 1


@dataclass
class Request:
    graph: int
    op: int                       # INSERT or DELETE
    src: np.ndarray               # local vertex ids
    dst: np.ndarray
    w: np.ndarray | None = None   # insertions only
    arrival: float = 0.0          # seconds on the server's clock
    # filled on completion
    done: float = 0.0
    first_update_id: int = 0
    found_at: np.ndarray | None = None      # insertions
    conductance: np.ndarray | None = None
    accepted: np.ndarray | None = None
    status: np.ndarray | None = None        # deletions
    rec_src: np.ndarray | None = None       # recovered edges, local ids, commit order
    rec_dst: np.ndarray | None = None
    rec_kind: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival

    @property
    def recovered(self) -> list:
        """[(x, y, kind), ...] of the recovered edges."""
        if self.rec_src is None:
            return []
        return list(zip(self.rec_src.tolist(), self.rec_dst.tolist(), self.rec_kind.tolist()))


def footprint_bytes(n: int, g_edges: int, h_edges: int, headroom: float = 0.5,
                    slack: int = 2) -> int:
    """Estimated device bytes of one graph in the union: per slot 12 B
    (slot + weight) with arena headroom, per vertex 12 B (descriptor +
    capacity) for G and H each."""
    slots = lambda m: (2 * m + slack * n) * (1 + headroom)
    return int(12 * (slots(g_edges) + slots(h_edges)) + 24 * n)


class Server:
    def __init__(self, cases, iparams: WalkParams, dparams: WalkParams,
                 hbm_budget: float = float("inf"), device: int = -1, native: bool = True):
        self.iparams, self.dparams = iparams, dparams
        self.admitted, offs, used = [], [0], 0
        for i, c in enumerate(cases):
            fp = footprint_bytes(c.n, len(c.g_src), len(c.h_src))
            if used + fp > hbm_budget:
                continue
            used += fp
            self.admitted.append(i)
            offs.append(offs[-1] + c.n)
        if not self.admitted:
            raise ValueError("no graph fits the HBM budget")
        self.footprint = used
        self.slot = {g: k for k, g in enumerate(self.admitted)}
        self.offsets = np.array(offs, np.int64)
        cat = lambda xs, t: np.concatenate(xs).astype(t) if xs else np.empty(0, t)
        sel = [cases[g] for g in self.admitted]
        n = int(self.offsets[-1])
        self.H = Graph.from_edges(n, cat([c.h_src + o for c, o in zip(sel, offs)], np.uint32),
                                  cat([c.h_dst + o for c, o in zip(sel, offs)], np.uint32),
                                  cat([c.h_w for c in sel], np.float32), device=device)
        self.G = Graph.from_edges(n, cat([c.g_src + o for c, o in zip(sel, offs)], np.uint32),
                                  cat([c.g_dst + o for c, o in zip(sel, offs)], np.uint32),
                                  cat([c.g_w for c in sel], np.float32), device=device)
        self.native = native
        self._srv = None
        if native:
            h = C.c_void_p()
            o32 = np.ascontiguousarray(self.offsets, np.uint32)
            _check(lib().dyg_server_create(self.G.handle, self.H.handle, len(self.admitted), _ptr(o32),
                                           C.byref(iparams), C.byref(dparams), None, C.byref(h)),
                   "dyg_server_create")
            self._srv = h
            self._tags = {}          # tag -> Request, submitted and not yet collected
            self._next_tag = 0
            self._poll = (ServerDone * 1024)()
            self._t0_ns = 0
        else:
            self.queues = {g: deque() for g in self.admitted}
            self.uid_next = {g: 0 for g in self.admitted}
            self._steps = 0
        self.t0 = time.perf_counter()

    @property
    def steps(self) -> int:
        return int(lib().dyg_server_steps(self._srv)) if self.native else self._steps

    def now(self) -> float:
        if self.native:
            return (lib().dyg_server_now_ns(self._srv) - self._t0_ns) * 1e-9
        return time.perf_counter() - self.t0

    def snapshot(self):
        """Keeps a device copy of the graphs for restore()."""
        self._snap = (self.H.clone(), self.G.clone())

    def restore(self, stream: int | None = None):
        """Back to the snapshot: graphs, update counters, empty queues."""
        self.H.copy_from(self._snap[0], stream)
        self.G.copy_from(self._snap[1], stream)
        if self.native:
            _check(lib().dyg_server_reset(self._srv), "dyg_server_reset")
            self._tags.clear()
        else:
            self.uid_next = {g: 0 for g in self.admitted}
            for q in self.queues.values():
                q.clear()
            self._steps = 0

    def submit(self, r: Request) -> bool:
        """Queues a request; False if its graph was not admitted."""
        if r.graph not in self.slot:
            return False
        if not self.native:
            self.queues[r.graph].append(r)
            return True
        src = np.ascontiguousarray(r.src, np.uint32)
        dst = np.ascontiguousarray(r.dst, np.uint32)
        w = np.ascontiguousarray(r.w, np.float32) if r.op == INSERT else None
        tag = self._next_tag
        self._next_tag += 1
        _check(lib().dyg_server_submit(self._srv, tag, self.slot[r.graph], r.op, _ptr(src), _ptr(dst),
                                       _ptr(w), len(src)), "dyg_server_submit")
        self._tags[tag] = r
        return True

    def submit_many(self, reqs) -> None:
        """Queues requests in order, with one call for the native server;
        requests of graphs not admitted get done = -1."""
        ok = []
        for r in reqs:
            if r.graph in self.slot:
                ok.append(r)
            else:
                r.done = -1.0
        if not self.native:
            for r in ok:
                self.queues[r.graph].append(r)
            return
        if not ok:
            return
        lens = np.fromiter((len(r.src) for r in ok), np.uint64, len(ok))
        offs = np.zeros(len(ok) + 1, np.uint64)
        np.cumsum(lens, out=offs[1:])
        src = np.concatenate([np.asarray(r.src, np.uint32) for r in ok])
        dst = np.concatenate([np.asarray(r.dst, np.uint32) for r in ok])
        w = np.concatenate([np.asarray(r.w, np.float32) if r.op == INSERT
                            else np.zeros(len(r.src), np.float32) for r in ok])
        tags = np.arange(self._next_tag, self._next_tag + len(ok), dtype=np.uint64)
        graphs = np.fromiter((self.slot[r.graph] for r in ok), np.uint32, len(ok))
        ops = np.fromiter((r.op for r in ok), np.uint32, len(ok))
        _check(lib().dyg_server_submit_many(self._srv, len(ok), _ptr(tags), _ptr(graphs), _ptr(ops),
                                            _ptr(offs), _ptr(src), _ptr(dst), _ptr(w)),
               "dyg_server_submit_many")
        self._next_tag += len(ok)
        for t, r in zip(tags.tolist(), ok):
            self._tags[t] = r

    def pending(self) -> bool:
        if self.native:
            return lib().dyg_server_pending(self._srv) > 0
        return any(self.queues.values())

    def _collect(self) -> list:
        """Completed requests of the native server, with their results."""
        L = lib()
        out = []
        while True:
            k = C.c_uint32()
            _check(L.dyg_server_poll(self._srv, self._poll, len(self._poll), C.byref(k)),
                   "dyg_server_poll")
            for i in range(k.value):
                d = self._poll[i]
                r = self._tags.pop(d.tag)
                if d.status != 0:
                    raise DygError(d.status, "server step", L.dyg_server_last_error(self._srv).decode())
                m = d.n
                r.first_update_id = d.first_update_id
                r.done = (d.t_done_ns - self._t0_ns) * 1e-9
                cd = np.empty(m, np.float32)
                if r.op == INSERT:
                    fa, ac = np.empty(m, np.int32), np.empty(m, np.uint8)
                    _check(L.dyg_server_fetch(self._srv, d.tag, _ptr(fa), _ptr(cd), _ptr(ac), None, None,
                                              None, 0), "dyg_server_fetch")
                    r.found_at, r.conductance, r.accepted = fa, cd, ac
                else:
                    st = np.empty(m, np.int32)
                    nr = d.n_rec
                    rx, ry, rk = np.empty(nr, np.uint32), np.empty(nr, np.uint32), np.empty(nr, np.uint8)
                    _check(L.dyg_server_fetch(self._srv, d.tag, _ptr(st), _ptr(cd), None, _ptr(rx),
                                              _ptr(ry), _ptr(rk), nr), "dyg_server_fetch")
                    r.status, r.conductance = st, cd
                    r.rec_src, r.rec_dst, r.rec_kind = rx, ry, rk
                out.append(r)
            if k.value < len(self._poll):
                return out

    def _batch(self, reqs):
        src, dst, w, uid = [], [], [], []
        for r in reqs:
            off = self.offsets[self.slot[r.graph]]
            r.first_update_id = self.uid_next[r.graph]
            src.append(np.asarray(r.src, np.int64) + off)
            dst.append(np.asarray(r.dst, np.int64) + off)
            if r.op == INSERT:
                w.append(np.asarray(r.w, np.float32))
            uid.append(np.arange(len(r.src), dtype=np.uint64) + np.uint64(r.first_update_id))
            self.uid_next[r.graph] += len(r.src)
        return (np.concatenate(src).astype(np.uint32), np.concatenate(dst).astype(np.uint32),
                np.concatenate(w) if w else None, np.concatenate(uid))

    def step(self) -> list:
        """Runs the oldest pending request of every graph; returns them."""
        if self.native:
            _check(lib().dyg_server_step(self._srv, None), "dyg_server_step")
            return self._collect()
        heads = [q.popleft() for q in self.queues.values() if q]
        for r in heads:
            r.first_update_id = self.uid_next[r.graph]
        ins = [r for r in heads if r.op == INSERT and len(r.src)]
        dels = [r for r in heads if r.op == DELETE and len(r.src)]
        if ins:
            s, d, w, u = self._batch(ins)
            res = incremental_batch_ids(self.H, s, d, w, u, self.iparams, G=self.G)
            k = 0
            for r in ins:
                m = len(r.src)
                r.found_at = res.found_at[k:k + m].copy()
                r.conductance = res.conductance[k:k + m].copy()
                r.accepted = res.accepted[k:k + m].copy()
                k += m
        if dels:
            s, d, _, u = self._batch(dels)
            res = decremental_batch_ids(self.G, self.H, s, d, u, self.dparams)
            k = 0
            # recovered edges come in commit order: edge by edge, so each
            # belongs to the request whose vertex range holds it
            owner = np.searchsorted(self.offsets, res.rec_src, side="right") - 1
            for r in dels:
                m = len(r.src)
                r.status = res.status[k:k + m].copy()
                r.conductance = res.conductance[k:k + m].copy()
                k += m
                sl = self.slot[r.graph]
                sel = owner == sl
                off = self.offsets[sl]
                r.rec_src = (res.rec_src[sel] - off).astype(np.uint32)
                r.rec_dst = (res.rec_dst[sel] - off).astype(np.uint32)
                r.rec_kind = res.rec_kind[sel].copy()
        t = self.now()
        for r in heads:
            r.done = t
            if r.op == INSERT and r.found_at is None:
                r.found_at = np.empty(0, np.int32)
                r.conductance = np.empty(0, np.float32)
                r.accepted = np.empty(0, np.uint8)
            if r.op == DELETE and r.status is None:
                r.status = np.empty(0, np.int32)
                r.conductance = np.empty(0, np.float32)
                r.rec_src = r.rec_dst = np.empty(0, np.uint32)
                r.rec_kind = np.empty(0, np.uint8)
        self._steps += 1
        return heads

    def serve(self, requests, sync=lambda: None) -> list:
        """Replays requests at their arrival times (seconds from now) with
        continuous batching; returns the completed requests."""
        order = sorted(requests, key=lambda r: r.arrival)
        if self.native:
            return self._serve_native(order, sync)
        self.t0 = time.perf_counter()
        i, done = 0, []
        while i < len(order) or self.pending():
            t = self.now()
            while i < len(order) and order[i].arrival <= t:
                if not self.submit(order[i]):
                    order[i].done = -1.0
                i += 1
            if self.pending():
                done += self.step()
                sync()
            elif i < len(order):
                time.sleep(max(0.0, min(order[i].arrival - self.now(), 0.001)))
        return done

    def _serve_native(self, order, sync) -> list:
        L = lib()
        self._t0_ns = L.dyg_server_now_ns(self._srv)
        i = 0
        while i < len(order) and order[i].arrival <= 0.0:   # pending at once
            i += 1
        # Requests pending at once go in chunks (each one checked and queued
        # as a whole), the loop starting after the first: steps run on the
        # device while the client still builds the later chunks' arrays.
        chunk = 128
        self.submit_many(order[:min(i, chunk)])
        done = []
        _check(L.dyg_server_start(self._srv), "dyg_server_start")
        try:
            for k in range(chunk, i, chunk):
                self.submit_many(order[k:min(i, k + chunk)])
            while i < len(order):
                t = self.now()
                j = i
                while j < len(order) and order[j].arrival <= t:
                    j += 1
                if j > i:
                    self.submit_many(order[i:j])
                    i = j
                done += self._collect()
                if i < len(order):
                    time.sleep(max(0.0, min(order[i].arrival - self.now(), 0.001)))
            # results are fetched while the last steps run
            while L.dyg_server_drain(self._srv, 0.001) != 0:
                done += self._collect()
        finally:
            _check(L.dyg_server_stop(self._srv), "dyg_server_stop")
        done += self._collect()
        sync()
        return done

    def close(self):
        if self._srv is not None:
            lib().dyg_server_destroy(self._srv)
            self._srv = None
        for x in (self.H, self.G) + tuple(getattr(self, "_snap", ())):
            x.close()


class PoolServer(Server):
    """The native server in pool mode (dyg_server_create_pool): it owns its
    union graphs and admits the registered graphs by footprint within
    `hbm_budget` bytes as their requests are scheduled, evicting resident
    graphs to host memory to make room (idle ones least recently used first).
    Results equal each graph's requests run alone on its own handles."""

    def __init__(self, cases, iparams: WalkParams, dparams: WalkParams, hbm_budget: float,
                 vertex_capacity: int | None = None, device: int = -1, keep_initial: bool = True):
        self.iparams, self.dparams = iparams, dparams
        self.native = True
        self.admitted = list(range(len(cases)))     # every graph is registered
        self.slot = {g: g for g in self.admitted}
        self.H = self.G = None
        self._srv = None
        L = lib()
        vcap = int(vertex_capacity or sum(c.n for c in cases))
        h = C.c_void_p()
        _check(L.dyg_server_create_pool(vcap, int(hbm_budget), C.byref(iparams), C.byref(dparams),
                                        int(device), 1 if keep_initial else 0, None, C.byref(h)),
               "dyg_server_create_pool")
        self._srv = h
        a = lambda x, t: np.ascontiguousarray(x, t)
        for c in cases:
            gid = C.c_uint32()
            gs, gd, gw = a(c.g_src, np.uint32), a(c.g_dst, np.uint32), a(c.g_w, np.float32)
            hs, hd, hw = a(c.h_src, np.uint32), a(c.h_dst, np.uint32), a(c.h_w, np.float32)
            _check(L.dyg_server_add_graph(h, int(c.n), len(gs), _ptr(gs), _ptr(gd), _ptr(gw), len(hs),
                                          _ptr(hs), _ptr(hd), _ptr(hw), C.byref(gid)),
                   "dyg_server_add_graph")
        self._tags = {}
        self._next_tag = 0
        self._poll = (ServerDone * 1024)()
        self._t0_ns = 0
        self.t0 = time.perf_counter()

    @property
    def footprint(self) -> int:
        return self.stats()["resident_bytes"]

    def snapshot(self):
        """The registered graphs are kept by the server (keep_initial)."""

    def restore(self, stream: int | None = None):
        """Every graph back to its registered rows, none resident."""
        _check(lib().dyg_server_reset(self._srv), "dyg_server_reset")
        self._tags.clear()

    def prefetch(self, graph: int) -> bool:
        r = C.c_uint32()
        _check(lib().dyg_server_prefetch(self._srv, int(graph), C.byref(r)), "dyg_server_prefetch")
        return bool(r.value)

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().dyg_server_stats_read(self._srv, C.byref(st)), "dyg_server_stats_read")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def counters(self) -> tuple[int, int]:
        """Walker moves so far: (insertion walks on H, deletion walks on G)."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().dyg_server_counters(self._srv, C.byref(a), C.byref(b)), "dyg_server_counters")
        return a.value, b.value

    def graph_info(self, graph: int) -> dict:
        gi = ServerGraphInfo()
        _check(lib().dyg_server_graph_info_read(self._srv, int(graph), C.byref(gi)),
               "dyg_server_graph_info_read")
        return {k: getattr(gi, k) for k, _ in gi._fields_ if k != "pad"}

    def export(self, graph: int, which: str):
        """(row_ptr, col, w) of a graph's G or H, local ids."""
        n = self.graph_info(graph)["n_vertices"]
        rp = np.zeros(n + 1, np.uint64)
        k = 0 if which == "G" else 1
        _check(lib().dyg_server_graph_export(self._srv, int(graph), k, _ptr(rp), None, None, 0),
               "dyg_server_graph_export")
        m = int(rp[n])
        col, w = np.empty(max(m, 1), np.uint32), np.empty(max(m, 1), np.float32)
        _check(lib().dyg_server_graph_export(self._srv, int(graph), k, _ptr(rp), _ptr(col), _ptr(w), m),
               "dyg_server_graph_export")
        return rp, col[:m], w[:m]

    def close(self):
        if self._srv is not None:
            lib().dyg_server_destroy(self._srv)
            self._srv = None


class PlainServer:
    """The plain sequential path: every graph its own handles, requests one
    at a time in arrival order."""

    def __init__(self, cases, iparams: WalkParams, dparams: WalkParams, device: int = -1):
        self.iparams, self.dparams = iparams, dparams
        self.H = [Graph.from_edges(c.n, c.h_src, c.h_dst, c.h_w, device=device) for c in cases]
        self.G = [Graph.from_edges(c.n, c.g_src, c.g_dst, c.g_w, device=device) for c in cases]
        self.uid_next = [0] * len(cases)

    def snapshot(self):
        self._snap = ([h.clone() for h in self.H], [g.clone() for g in self.G])

    def restore(self, stream: int | None = None):
        for x, y in zip(self.H + self.G, self._snap[0] + self._snap[1]):
            x.copy_from(y, stream)
        self.uid_next = [0] * len(self.H)

    def run_one(self, r: Request):
        from . import decremental_batch, incremental_batch
        g = r.graph
        r.first_update_id = self.uid_next[g]
        if r.op == INSERT:
            res = incremental_batch(self.H[g], r.src, r.dst, r.w, self.iparams,
                                    first_update_id=r.first_update_id, G=self.G[g])
            r.found_at, r.conductance, r.accepted = res.found_at, res.conductance, res.accepted
        else:
            res = decremental_batch(self.G[g], self.H[g], r.src, r.dst, self.dparams,
                                    first_update_id=r.first_update_id)
            r.status, r.conductance = res.status, res.conductance
            r.rec_src, r.rec_dst, r.rec_kind = res.rec_src, res.rec_dst, res.rec_kind
        self.uid_next[g] += len(r.src)

    def serve(self, requests, sync=lambda: None) -> list:
        order = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        for r in order:
            wait = r.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            self.run_one(r)
            sync()
            r.done = time.perf_counter() - t0
        return order

    def close(self):
        snap = getattr(self, "_snap", ([], []))
        for x in self.H + self.G + snap[0] + snap[1]:
            x.close()


def poisson_requests(cases, rate: float, count: int, seed: int, ins_frac: float = 0.6,
                     size_lo: int = 1, size_hi: int = 4096):
    """Requests with exponential inter-arrival times (mean 1/rate), sizes
    log-uniform in [size_lo, size_hi], insertions with probability ins_frac.
    An insertion takes the next edges of its graph's insertion pool (the
    case's ins_*), a deletion edges of its dense graph not deleted before
    (uniform).  Sizes are capped by what the graph has left."""
    rng = np.random.default_rng(seed)
    nxt = [0] * len(cases)
    alive = [rng.permutation(len(c.g_src)) for c in cases]
    dpos = [0] * len(cases)
    t, out = 0.0, []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        g = int(rng.integers(len(cases)))
        c = cases[g]
        size = int(np.exp(rng.uniform(np.log(size_lo), np.log(size_hi + 1))))
        if rng.random() < ins_frac:
            k = min(size, len(c.ins_src) - nxt[g])
            sl = slice(nxt[g], nxt[g] + k)
            nxt[g] += k
            out.append(Request(g, INSERT, c.ins_src[sl], c.ins_dst[sl], c.ins_w[sl], arrival=t))
        else:
            k = min(size, len(alive[g]) - dpos[g])
            idx = alive[g][dpos[g]:dpos[g] + k]
            dpos[g] += k
            out.append(Request(g, DELETE, c.g_src[idx], c.g_dst[idx], arrival=t))
    return out


def latency_stats(done) -> dict:
    lat = np.array([r.latency for r in done if r.done >= 0]) * 1e3
    upd = sum(len(r.src) for r in done if r.done >= 0)
    span = max(r.done for r in done) if done else 0.0
    return {"requests": int(len(lat)), "updates": int(upd),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "throughput_updates_per_s": upd / span if span > 0 else None}
