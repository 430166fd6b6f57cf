"""One graph's update batches sharded over processes (one per GPU).

Every rank holds a replica of G and H.  For each batch, rank r walks the
contiguous range [n*r/world, n*(r+1)/world) of the batch (for deletions: of
the batch's walk list, after every rank has applied the same deletions) and
writes the winner keys of that range into an array that is zero elsewhere;
an element-wise max over the ranks (all-reduce MAX of 8 bytes per edge over
NVLink) gives every rank the whole key array, and every rank commits the
batch the same way.  The result on every rank is the whole-batch result
(dyg_incremental_batch / dyg_decremental_batch with the same update ids):
the keys are the same numbers and the commit is the same code.

The driver is written against a small backend interface so that the same
code runs on GPUs (GpuBackend, over include/dyg.h) and in tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import WalkParams, _check, _ptr, lib, recovered_read


def split(n: int, rank: int, world: int):
    """The contiguous range of rank `rank`."""
    return n * rank // world, n * (rank + 1) // world


def partition_by_footprint(sizes, world: int) -> list:
    """Independent graphs over `world` ranks by device footprint: largest
    first, each to the rank holding the least so far (ties to the lower
    rank).  Returns one ascending index list per rank."""
    parts = [[] for _ in range(world)]
    load = [0] * world
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


class GpuBackend:
    """Replicas on one GPU per process; keys and outputs are torch tensors."""

    def __init__(self, device, stream: int | None = None):
        import torch
        self.torch = torch
        self.dev = device
        self.stream = stream
        L = lib()
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        P = C.POINTER(WalkParams)
        for name, args in {
            "dyg_walk_keys": [vp, vp, vp, vp, vp, u64, u32, u32, u32, u32, P, vp, vp],
            "dyg_incremental_commit_keys": [vp, vp, vp, vp, vp, u32, vp, vp, vp, vp, vp],
            "dyg_decremental_delete": [vp, vp, vp, vp, vp, u64, u32, vp, vp, C.POINTER(u32), vp],
            "dyg_decremental_walk_keys": [vp, u32, u32, P, vp, vp],
            "dyg_decremental_commit_keys": [vp, vp, P, vp, u32, vp, vp, vp, vp, vp, u64,
                                            C.POINTER(u64), vp],
        }.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        self.L = L

    def zeros_keys(self, n):
        return self.torch.zeros(max(n, 1), dtype=self.torch.int64, device=self.dev)

    def walk_keys(self, H, src, dst, w, first_uid, lo, hi, p, keys):
        _check(self.L.dyg_walk_keys(H.handle, _ptr(src), _ptr(dst), _ptr(w), None, int(first_uid),
                                    len(src), lo, hi, 1, C.byref(p), _ptr(keys), self.stream),
               "dyg_walk_keys")

    def incr_commit(self, H, G, src, dst, w, keys):
        n = len(src)
        t = self.torch
        out = (t.empty(n, dtype=t.int32, device=self.dev), t.empty(n, dtype=t.float32, device=self.dev),
               t.empty(n, dtype=t.uint8, device=self.dev))
        _check(self.L.dyg_incremental_commit_keys(H.handle, G.handle if G else None, _ptr(src),
                                                  _ptr(dst), _ptr(w), n, _ptr(keys), _ptr(out[0]),
                                                  _ptr(out[1]), _ptr(out[2]), self.stream),
               "dyg_incremental_commit_keys")
        return out

    def decr_delete(self, G, H, src, dst, first_uid):
        n = len(src)
        t = self.torch
        st = t.empty(max(n, 1), dtype=t.int32, device=self.dev)
        cd = t.empty(max(n, 1), dtype=t.float32, device=self.dev)
        nw = C.c_uint32()
        _check(self.L.dyg_decremental_delete(G.handle, H.handle, _ptr(src), _ptr(dst), None,
                                             int(first_uid), n, _ptr(st), _ptr(cd), C.byref(nw),
                                             self.stream), "dyg_decremental_delete")
        return nw.value, (st, cd)

    def decr_walk_keys(self, G, lo, hi, p, keys):
        _check(self.L.dyg_decremental_walk_keys(G.handle, lo, hi, C.byref(p), _ptr(keys),
                                                self.stream), "dyg_decremental_walk_keys")

    def decr_commit(self, G, H, p, keys, n_walk, state, rec_cap=None):
        """rec_cap None: no record buffers are passed; the total comes back
        from the commit and exactly that many records are read afterwards."""
        st, cd = state
        nr = C.c_uint64()
        if rec_cap is None:
            _check(self.L.dyg_decremental_commit_keys(G.handle, H.handle, C.byref(p), _ptr(keys),
                                                      n_walk, _ptr(st), _ptr(cd), None, None, None,
                                                      0, C.byref(nr), self.stream),
                   "dyg_decremental_commit_keys")
            return (st, cd) + tuple(recovered_read(G, nr.value))
        rx = np.empty(max(rec_cap, 1), np.uint32)
        ry = np.empty(max(rec_cap, 1), np.uint32)
        rk = np.empty(max(rec_cap, 1), np.uint8)
        _check(self.L.dyg_decremental_commit_keys(G.handle, H.handle, C.byref(p), _ptr(keys), n_walk,
                                                  _ptr(st), _ptr(cd), _ptr(rx), _ptr(ry), _ptr(rk),
                                                  rec_cap, C.byref(nr), self.stream),
               "dyg_decremental_commit_keys")
        k = nr.value
        return st, cd, rx[:k], ry[:k], rk[:k]


def incremental_sharded(backend, H, G, src, dst, w, first_uid, p, rank, world, combine):
    """One incremental batch over `world` ranks; combine(keys) must return the
    element-wise max of every rank's keys (all-reduce MAX).  Returns
    (found_at, conductance, accepted)."""
    n = len(src)
    keys = backend.zeros_keys(n)
    lo, hi = split(n, rank, world)
    backend.walk_keys(H, src, dst, w, first_uid, lo, hi, p, keys)
    keys = combine(keys)
    return backend.incr_commit(H, G, src, dst, w, keys)


def decremental_sharded(backend, G, H, src, dst, first_uid, p, rank, world, combine,
                        rec_cap: int | None = None):
    """One decremental batch over `world` ranks.  Returns (status,
    conductance, rec_src, rec_dst, rec_kind)."""
    n_walk, state = backend.decr_delete(G, H, src, dst, first_uid)
    keys = backend.zeros_keys(n_walk)
    lo, hi = split(n_walk, rank, world)
    backend.decr_walk_keys(G, lo, hi, p, keys)
    keys = combine(keys)
    return backend.decr_commit(G, H, p, keys, n_walk, state, rec_cap)


def allreduce_max(group=None):
    """combine() over torch.distributed (NCCL for GPU tensors, gloo for CPU)."""
    import torch.distributed as dist

    def f(keys):
        dist.all_reduce(keys, op=dist.ReduceOp.MAX, group=group)
        return keys
    return f
