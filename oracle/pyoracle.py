"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, as the checker or the timed host baseline.
Its API mirrors dygrass_b200's so that parity tests read alike.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class Params(C.Structure):
    _fields_ = [("threshold", C.c_float), ("walkers", C.c_uint32), ("max_steps", C.c_uint32),
                ("transition", C.c_uint32), ("heuristic_walkers", C.c_uint32),
                ("pad", C.c_uint32), ("seed", C.c_uint64)]

    @classmethod
    def from_walk_params(cls, p):
        return cls(p.threshold, p.walkers, p.max_steps, p.transition, p.heuristic_walkers, 0,
                   p.seed)


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "ORACLE_CC=gcc"], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        P = C.POINTER(Params)
        sig = {
            "orc_philox4x32_10": ([vp, vp, vp], None),
            "orc_draw": ([u64, u64, u32, u32, u32], u32),
            "orc_graph_from_edges": ([u32, u64, vp, vp, vp], vp),
            "orc_graph_free": ([vp], None),
            "orc_graph_clone": ([vp], vp),
            "orc_graph_num_vertices": ([vp], u32),
            "orc_graph_num_slots": ([vp], u64),
            "orc_graph_export": ([vp, vp, vp, vp], u64),
            "orc_graph_has_edge": ([vp, u32, u32], C.c_int),
            "orc_incremental_batch": ([vp, vp, vp, vp, vp, u32, u64, P, C.c_int, vp, vp, vp], u64),
            "orc_incremental_stream": ([vp, vp, vp, vp, vp, u32, u32, P, C.c_int, vp, vp, vp], u64),
            "orc_decremental_batch": ([vp, vp, vp, vp, u32, u64, P, C.c_int, vp, vp, vp, vp, vp, u64,
                                       C.POINTER(u64)], u64),
            "orc_decremental_stream": ([vp, vp, vp, vp, u32, u32, P, C.c_int, vp, vp, vp, vp, vp, u64,
                                        C.POINTER(u64)], u64),
            "orc_decremental_walk_path": ([vp, u32, u32, u64, u32, P, vp, C.POINTER(C.c_float)], C.c_int32),
            "orc_max_threads": ([], C.c_int),
            "orc_stream_default_chunk": ([u32], u32),
            "orc_walk_keys": ([vp, vp, vp, vp, u64, u32, u32, C.c_int, P, C.c_int, vp, vp], None),
            "orc_incremental_commit_keys": ([vp, vp, vp, vp, vp, u32, vp, vp, vp, vp], None),
            "orc_walk_keys_ids": ([vp, vp, vp, vp, vp, u32, P, C.c_int, vp, vp], None),
            "orc_decremental_batch_ids": ([vp, vp, vp, vp, vp, u32, P, C.c_int, vp, vp, vp, vp, vp, u64,
                                           C.POINTER(u64)], u64),
            "orc_decremental_delete": ([vp, vp, vp, vp, u32, vp, vp, vp], u32),
            "orc_decremental_walk_list_keys": ([vp, vp, vp, vp, u32, u32, u64, P, C.c_int, vp], None),
            "orc_decremental_commit_keys": ([vp, vp, vp, vp, vp, u32, u64, P, vp, vp, vp, vp, vp, vp,
                                             u64, C.POINTER(u64)], None),
            "orc_stream_file": ([vp, vp, u32, vp, vp, vp, u32, u64, u32, P, C.c_int, vp, vp, vp, vp,
                                 vp, u64, C.POINTER(u64)], u64),
        }
        for name, (a, r) in sig.items():
            f = getattr(L, name)
            f.argtypes = a
            f.restype = r
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(_p(c), _p(k), _p(out))
    return out


def draw(seed, uid, domain, walker, d) -> int:
    return int(lib().orc_draw(seed, uid, domain, walker, d))


def max_threads() -> int:
    return int(lib().orc_max_threads())


class OGraph:
    def __init__(self, n, src, dst, w):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        w = np.ascontiguousarray(w, np.float32)
        self.h = lib().orc_graph_from_edges(int(n), len(src), _p(src), _p(dst), _p(w))

    @classmethod
    def _wrap(cls, h):
        g = cls.__new__(cls)
        g.h = h
        return g

    def clone(self) -> "OGraph":
        return OGraph._wrap(lib().orc_graph_clone(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_graph_free(self.h)
            self.h = None

    def export(self):
        n = lib().orc_graph_num_vertices(self.h)
        s = lib().orc_graph_num_slots(self.h)
        rp = np.zeros(n + 1, np.uint64)
        col = np.zeros(max(s, 1), np.uint32)
        w = np.zeros(max(s, 1), np.float32)
        lib().orc_graph_export(self.h, _p(rp), _p(col), _p(w))
        return rp, col[:s], w[:s]

    def has_edge(self, a, b) -> bool:
        return bool(lib().orc_graph_has_edge(self.h, a, b))


def incremental(H: OGraph, src, dst, w, params, batch_size=0, G: OGraph | None = None,
                threads=None, first_uid=0, single_batch=False):
    """Returns (found_at, cond, accepted, walker_moves)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = np.ascontiguousarray(w, np.float32)
    n = len(src)
    fa = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    ac = np.empty(n, np.uint8)
    P = Params.from_walk_params(params)
    th = threads or max_threads()
    if single_batch:
        mv = lib().orc_incremental_batch(H.h, G.h if G else None, _p(src), _p(dst), _p(w), n,
                                         first_uid, C.byref(P), th, _p(fa), _p(cd), _p(ac))
    else:
        mv = lib().orc_incremental_stream(H.h, G.h if G else None, _p(src), _p(dst), _p(w), n,
                                          batch_size, C.byref(P), th, _p(fa), _p(cd), _p(ac))
    return fa, cd, ac, int(mv)


def incremental_ids(H: OGraph, src, dst, w, uids, params, G: OGraph | None = None, threads=None):
    """One incremental batch whose edge e walks with update id uids[e]
    (the batched many-graph mode).  Returns (found_at, cond, accepted)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = np.ascontiguousarray(w, np.float32)
    uids = np.ascontiguousarray(uids, np.uint64)
    n = len(src)
    keys = np.empty(max(n, 1), np.uint64)
    fa = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    ac = np.empty(n, np.uint8)
    P = Params.from_walk_params(params)
    th = threads or max_threads()
    lib().orc_walk_keys_ids(H.h, _p(src), _p(dst), _p(w), _p(uids), n, C.byref(P), th, _p(keys), None)
    lib().orc_incremental_commit_keys(H.h, G.h if G else None, _p(src), _p(dst), _p(w), n, _p(keys),
                                      _p(fa), _p(cd), _p(ac))
    return fa, cd, ac


def decremental(G: OGraph, H: OGraph, src, dst, params, batch_size=0, threads=None,
                first_uid=0, single_batch=False):
    """Returns (status, cond, rec_src, rec_dst, rec_kind, walker_moves)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    n = len(src)
    cap = n * (params.max_steps + 4 * params.heuristic_walkers) + 16
    st = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    rx = np.empty(cap, np.uint32)
    ry = np.empty(cap, np.uint32)
    rk = np.empty(cap, np.uint8)
    nr = C.c_uint64()
    P = Params.from_walk_params(params)
    th = threads or max_threads()
    if single_batch:
        mv = lib().orc_decremental_batch(G.h, H.h, _p(src), _p(dst), n, first_uid, C.byref(P), th,
                                         _p(st), _p(cd), _p(rx), _p(ry), _p(rk), cap, C.byref(nr))
    else:
        mv = lib().orc_decremental_stream(G.h, H.h, _p(src), _p(dst), n, batch_size, C.byref(P), th,
                                          _p(st), _p(cd), _p(rx), _p(ry), _p(rk), cap, C.byref(nr))
    k = nr.value
    return st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy(), int(mv)


def decremental_ids(G: OGraph, H: OGraph, src, dst, uids, params, threads=None):
    """One decremental batch whose deletion e uses update id uids[e].
    Returns (status, cond, rec_src, rec_dst, rec_kind)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    uids = np.ascontiguousarray(uids, np.uint64)
    n = len(src)
    cap = n * (params.max_steps + 4 * params.heuristic_walkers) + 16
    st, cd = np.empty(n, np.int32), np.empty(n, np.float32)
    rx, ry, rk = np.empty(cap, np.uint32), np.empty(cap, np.uint32), np.empty(cap, np.uint8)
    nr = C.c_uint64()
    P = Params.from_walk_params(params)
    lib().orc_decremental_batch_ids(G.h, H.h, _p(src), _p(dst), _p(uids), n, C.byref(P),
                                    threads or max_threads(), _p(st), _p(cd), _p(rx), _p(ry), _p(rk),
                                    cap, C.byref(nr))
    k = nr.value
    return st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy()


def stream_file(G: OGraph, H: OGraph, op, src, dst, w, params, first_uid=0, chunk=0,
                threads=None):
    """One stream file; returns (status, cond, rec_src, rec_dst, rec_kind, walker_moves)."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    w = None if w is None else np.ascontiguousarray(w, np.float32)
    n = len(src)
    cap = n * (params.max_steps + 4 * params.heuristic_walkers) + 16
    st = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    rx = np.empty(cap, np.uint32)
    ry = np.empty(cap, np.uint32)
    rk = np.empty(cap, np.uint8)
    nr = C.c_uint64()
    P = Params.from_walk_params(params)
    th = threads or max_threads()
    mv = lib().orc_stream_file(G.h, H.h, int(op), _p(src), _p(dst), _p(w), n, first_uid, chunk,
                               C.byref(P), th, _p(st), _p(cd), _p(rx), _p(ry), _p(rk), cap,
                               C.byref(nr))
    k = nr.value
    return st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy(), int(mv)


def stream_default_chunk(n_vertices) -> int:
    return int(lib().orc_stream_default_chunk(int(n_vertices)))


class ShardBackend:
    """The oracle behind dygrass_b200.shard's backend interface (keys are
    torch CPU int64 tensors, exchanged with gloo in tests)."""

    def __init__(self, threads=None):
        self.th = threads or max_threads()
        self._last = None

    def zeros_keys(self, n):
        import torch
        return torch.zeros(max(n, 1), dtype=torch.int64)

    @staticmethod
    def _u64(keys):
        return keys.numpy().view(np.uint64)

    def walk_keys(self, H, src, dst, w, first_uid, lo, hi, p, keys):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        w = np.ascontiguousarray(w, np.float32)
        P = Params.from_walk_params(p)
        lib().orc_walk_keys(H.h, _p(src), _p(dst), _p(w), first_uid, lo, hi, 1, C.byref(P), self.th,
                            _p(self._u64(keys)), None)

    def incr_commit(self, H, G, src, dst, w, keys):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        w = np.ascontiguousarray(w, np.float32)
        n = len(src)
        fa, cd, ac = np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.uint8)
        lib().orc_incremental_commit_keys(H.h, G.h if G else None, _p(src), _p(dst), _p(w), n,
                                          _p(self._u64(keys)), _p(fa), _p(cd), _p(ac))
        return fa, cd, ac

    def decr_delete(self, G, H, src, dst, first_uid):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        n = len(src)
        st, cd = np.empty(n, np.int32), np.empty(n, np.float32)
        wl = np.empty(max(n, 1), np.uint32)
        nf = lib().orc_decremental_delete(G.h, H.h, _p(src), _p(dst), n, _p(st), _p(cd), _p(wl))
        self._last = (src, dst, wl, first_uid)
        return nf, (st, cd)

    def decr_walk_keys(self, G, lo, hi, p, keys):
        src, dst, wl, first_uid = self._last
        P = Params.from_walk_params(p)
        lib().orc_decremental_walk_list_keys(G.h, _p(src), _p(dst), _p(wl), lo, hi, first_uid,
                                             C.byref(P), self.th, _p(self._u64(keys)))

    def decr_commit(self, G, H, p, keys, n_walk, state, rec_cap=None):
        src, dst, wl, first_uid = self._last
        st, cd = state
        if rec_cap is None:   # the bound of a batch: a path plus fallback edges per deletion
            rec_cap = len(src) * (p.max_steps + 4 * p.heuristic_walkers) + 16
        P = Params.from_walk_params(p)
        rx, ry, rk = (np.empty(max(rec_cap, 1), np.uint32), np.empty(max(rec_cap, 1), np.uint32),
                      np.empty(max(rec_cap, 1), np.uint8))
        nr = C.c_uint64()
        lib().orc_decremental_commit_keys(G.h, H.h, _p(src), _p(dst), _p(wl), n_walk, first_uid,
                                          C.byref(P), _p(self._u64(keys)), _p(st), _p(cd), _p(rx),
                                          _p(ry), _p(rk), rec_cap, C.byref(nr))
        k = nr.value
        return st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy()
