"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference's datasets are not available (they are downloaded from a
private drive by datasetdownload.py), so every workload here is generated:

  grid_2d   -- 2-D grid, FP32 weights U[0.5, 2.0], sparsifier = maximum-weight
               spanning tree + 10% of the off-tree edges, insertions at grid
               hop distance 2..8 with weights U[0.5, 2.0]; threshold 10,
               512 walkers, max_steps 64.  At 100x100: 10,000 vertices,
               19,800 edges, 1,000 insertions.
  mesh_3d   -- 3-D 7-point mesh, FP32 weights log-uniform [1e-2, 1e2],
               sparsifier = spanning tree + 5% off-tree, insertions at hop
               distance 2..10 with the same weight law, then deletion of 10%
               of the dense graph's edges (after insertions), uniform;
               threshold 100, 512 walkers, max_steps 100.  At 100^3:
               1,000,000 vertices, 2,970,000 edges, 200,000 insertions,
               317,000 deletions.
  rmat_mixed -- R-MAT (a, b, c) = (0.57, 0.19, 0.19), edge factor 16,
               symmetrised, deduplicated, largest connected component,
               FP32 weights U[0.1, 10]; sparsifier = spanning tree + 5%
               off-tree; a mixed stream of insert / delete files of 4,096
               updates, 70% insertions (further R-MAT pairs; existing edges
               merge their weight) and 30% deletions (uniform over the edges
               present); threshold 50, 256 walkers, max_steps 128.  At
               scale 20: 2^20 ids, 500,000 updates in 123 files.
  rgg_many   -- independent random geometric graphs in the unit square (n
               log-uniform, radius for mean degree 8, weights 1/distance,
               largest component), each with sparsifier = maximum spanning tree
               + 10% off-tree and 0.05 n insertions at distance [r, 3r);
               threshold 100 (the configuration leaves it open; 100 is the
               reference's example bound), 512 walkers, max_steps 100.  The
               full configuration is 256 graphs with n in [1e3, 2e5].
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import WalkParams, _ptr, lib

MASTER_SEED = 20251203
W_UNIFORM = 0
W_LOGUNIFORM = 1


def lattice(nx: int, ny: int, nz: int, wdist: int, lo: float, hi: float, seed: int):
    m = int(lib().dyg_synth_lattice_edges(nx, ny, nz))
    src = np.empty(m, np.uint32)
    dst = np.empty(m, np.uint32)
    w = np.empty(m, np.float32)
    lib().dyg_synth_lattice(nx, ny, nz, wdist, lo, hi, seed, _ptr(src), _ptr(dst), _ptr(w))
    return src, dst, w


def sparsifier(n: int, src, dst, w, frac: float, seed: int) -> np.ndarray:
    idx = np.empty(len(src), np.uint64)
    k = lib().dyg_synth_sparsifier(n, len(src), _ptr(src), _ptr(dst), _ptr(w), frac, seed, _ptr(idx))
    return idx[:k]


def lattice_inserts(nx, ny, nz, src, dst, count, hop_lo, hop_hi, wdist, lo, hi, seed):
    os_ = np.empty(count, np.uint32)
    od = np.empty(count, np.uint32)
    ow = np.empty(count, np.float32)
    k = lib().dyg_synth_lattice_inserts(nx, ny, nz, len(src), _ptr(src), _ptr(dst), count, hop_lo,
                                        hop_hi, wdist, lo, hi, seed, _ptr(os_), _ptr(od), _ptr(ow))
    return os_[:k], od[:k], ow[:k]


def sample(m: int, k: int, seed: int) -> np.ndarray:
    out = np.empty(k, np.uint64)
    lib().dyg_synth_sample(m, k, seed, _ptr(out))
    return out


def rmat(scale: int, edge_factor: int, a: float, b: float, c: float, wlo: float, whi: float,
         seed: int):
    """Returns (n, src, dst, w, id_map) of the R-MAT graph's largest component."""
    n = C.c_uint32()
    ps, pd, pw, pm = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    m = int(lib().dyg_synth_rmat(scale, edge_factor, a, b, c, wlo, whi, seed, C.byref(n),
                                 C.byref(ps), C.byref(pd), C.byref(pw), C.byref(pm)))
    try:
        src = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_uint32)), (max(m, 1),))[:m].copy()
        dst = np.ctypeslib.as_array(C.cast(pd, C.POINTER(C.c_uint32)), (max(m, 1),))[:m].copy()
        w = np.ctypeslib.as_array(C.cast(pw, C.POINTER(C.c_float)), (max(m, 1),))[:m].copy()
        idm = np.ctypeslib.as_array(C.cast(pm, C.POINTER(C.c_uint32)), (1 << scale,)).copy()
    finally:
        for p in (ps, pd, pw, pm):
            lib().dyg_mtx_free(p)
    return int(n.value), src, dst, w, idm


def rmat_stream(scale, a, b, c, id_map, src, dst, n_updates, file_size, del_frac, wlo, whi,
                seed):
    """Returns a list of (op, src, dst, w) stream files (op 0 insert, 1 delete)."""
    nf = (n_updates + file_size - 1) // file_size
    ops = np.zeros(max(nf, 1), np.uint8)
    os_ = np.empty(max(n_updates, 1), np.uint32)
    od = np.empty(max(n_updates, 1), np.uint32)
    ow = np.empty(max(n_updates, 1), np.float32)
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    nf = int(lib().dyg_synth_rmat_stream(scale, a, b, c, _ptr(id_map), len(src), _ptr(src),
                                         _ptr(dst), n_updates, file_size, del_frac, wlo, whi,
                                         seed, _ptr(ops), _ptr(os_), _ptr(od), _ptr(ow)))
    files = []
    for f in range(nf):
        lo, hi = f * file_size, min((f + 1) * file_size, n_updates)
        files.append((int(ops[f]), os_[lo:hi].copy(), od[lo:hi].copy(),
                      None if ops[f] else ow[lo:hi].copy()))
    return files


def rgg(n: int, avg_deg: float, n_ins: int, seed: int):
    """Returns (n, src, dst, w, ins_src, ins_dst, ins_w)."""
    no, ni = C.c_uint32(), C.c_uint32()
    ptrs = [C.c_void_p() for _ in range(6)]
    m = int(lib().dyg_synth_rgg(int(n), float(avg_deg), int(n_ins), int(seed), C.byref(no),
                                C.byref(ptrs[0]), C.byref(ptrs[1]), C.byref(ptrs[2]), C.byref(ni),
                                C.byref(ptrs[3]), C.byref(ptrs[4]), C.byref(ptrs[5])))
    k = ni.value
    try:
        def arr(p, cnt, t):
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), (max(cnt, 1),))[:cnt].copy()
        out = (int(no.value), arr(ptrs[0], m, C.c_uint32), arr(ptrs[1], m, C.c_uint32),
               arr(ptrs[2], m, C.c_float), arr(ptrs[3], k, C.c_uint32), arr(ptrs[4], k, C.c_uint32),
               arr(ptrs[5], k, C.c_float))
    finally:
        for p in ptrs:
            lib().dyg_mtx_free(p)
    return out


@dataclass
class GraphCase:
    n: int
    g_src: np.ndarray
    g_dst: np.ndarray
    g_w: np.ndarray
    h_src: np.ndarray
    h_dst: np.ndarray
    h_w: np.ndarray
    ins_src: np.ndarray
    ins_dst: np.ndarray
    ins_w: np.ndarray


def rgg_many(k: int = 256, n_lo: int = 1000, n_hi: int = 200_000, seed: int = MASTER_SEED,
             walkers: int = 512, max_steps: int = 100, threshold: float = 100.0):
    """Returns (list of GraphCase, WalkParams)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), k)).astype(np.int64)
    cases = []
    for i, n0 in enumerate(sizes):
        n, s, d, w, is_, id_, iw = rgg(int(n0), 8.0, int(0.05 * n0), seed + 101 + i)
        idx = sparsifier(n, s, d, w, 0.10, seed + 7001 + i)
        cases.append(GraphCase(n, s, d, w, s[idx], d[idx], w[idx], is_, id_, iw))
    return cases, WalkParams.make(threshold=threshold, walkers=walkers, max_steps=max_steps,
                                  seed=seed)


def rmat_case(scale: int, seed: int, n_ins: int, edge_factor: int = 16) -> GraphCase:
    """An R-MAT graph (largest component, weights U[0.1, 10]) with sparsifier
    = spanning tree + 5% off-tree and n_ins further R-MAT pairs inside the
    component (repeats of existing edges included)."""
    a, b, c = 0.57, 0.19, 0.19
    n, s, d, w, idm = rmat(scale, edge_factor, a, b, c, 0.1, 10.0, seed)
    idx = sparsifier(n, s, d, w, 0.05, seed + 1)
    ps = np.empty(n_ins * 4, np.uint32)
    pd = np.empty(n_ins * 4, np.uint32)
    lib().dyg_synth_rmat_pairs(scale, n_ins * 4, a, b, c, seed + 2, _ptr(ps), _ptr(pd))
    u, v = idm[ps], idm[pd]
    ok = (u != 0xFFFFFFFF) & (v != 0xFFFFFFFF) & (u != v)
    u, v = u[ok][:n_ins], v[ok][:n_ins]
    rng = np.random.default_rng(seed + 3)
    iw = rng.uniform(0.1, 10.0, len(u)).astype(np.float32)
    return GraphCase(n, s, d, w, s[idx], d[idx], w[idx], u.astype(np.uint32), v.astype(np.uint32), iw)


def serving_mix(k: int = 64, seed: int = MASTER_SEED, large: bool = False, threads: int = 0):
    """k resident graphs drawn in turn from the three generators: 3-D meshes
    (k^3, k in [12, 48]), R-MAT (scale 10..16) and random geometric graphs
    (n log-uniform in [1e3, 2e5]); each with an insertion pool of 0.5 n edges
    (at most 20,000).  large: meshes 60^3..100^3 and R-MAT scales 17..20 (about
    8.3 GB of footprint for 64 graphs, 10.8 GB for 80).  The sizes are drawn
    in order from one generator seeded with seed, and each graph from its own
    seeds, so the graphs are built by `threads` workers (0: one per core; the
    native generators release the GIL) with the same result as one by one.
    Returns (cases, insertion params, deletion params): threshold 100, 512
    walkers, max_steps 100."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(seed)
    m_lo, m_hi, sc_lo, sc_hi = (60, 101, 17, 21) if large else (12, 49, 10, 17)
    specs = []
    for i in range(k):
        kind = i % 3
        if kind == 0:
            specs.append((0, int(rng.integers(m_lo, m_hi)), seed + 31 * i))
        elif kind == 1:
            specs.append((1, int(rng.integers(sc_lo, sc_hi)), seed + 31 * i))
        else:
            specs.append((2, int(np.exp(rng.uniform(np.log(1e3), np.log(2e5)))), seed + 31 * i))

    def build(spec):
        kind, size, sd = spec
        if kind == 0:
            wl = mesh_3d(size, inserts=min(20_000, max(1, size ** 3 // 2)), seed=sd)
            return GraphCase(wl.n, wl.g_src, wl.g_dst, wl.g_w, wl.h_src, wl.h_dst, wl.h_w,
                             wl.ins_src, wl.ins_dst, wl.ins_w)
        if kind == 1:
            return rmat_case(size, sd, n_ins=min(20_000, (1 << size) // 2))
        n, s, d, w, is_, id_, iw = rgg(size, 8.0, size // 2, sd)
        idx = sparsifier(n, s, d, w, 0.10, sd + 1)
        return GraphCase(n, s, d, w, s[idx], d[idx], w[idx], is_, id_, iw)

    workers = max(1, min(threads or os.cpu_count() or 1, len(specs)))
    with ThreadPoolExecutor(workers) as ex:
        cases = list(ex.map(build, specs))
    p = WalkParams.make(threshold=100.0, walkers=512, max_steps=100, seed=seed)
    return cases, p, WalkParams.make(walkers=512, max_steps=100, seed=seed)


@dataclass
class MixedWorkload:
    name: str
    n: int
    g_src: np.ndarray
    g_dst: np.ndarray
    g_w: np.ndarray
    h_src: np.ndarray
    h_dst: np.ndarray
    h_w: np.ndarray
    files: list                 # (op, src, dst, w or None) in stream order
    iparams: WalkParams = None  # insert files
    dparams: WalkParams = None  # delete files
    meta: dict = field(default_factory=dict)

    @property
    def n_updates(self) -> int:
        return sum(len(f[1]) for f in self.files)


def rmat_mixed(scale: int = 20, edge_factor: int = 16, n_updates: int = 500_000,
               file_size: int = 4096, del_frac: float = 0.30, seed: int = MASTER_SEED,
               walkers: int = 256, max_steps: int = 128, threshold: float = 50.0) -> MixedWorkload:
    a, b, c = 0.57, 0.19, 0.19
    n, src, dst, w, idm = rmat(scale, edge_factor, a, b, c, 0.1, 10.0, seed + 11)
    idx = sparsifier(n, src, dst, w, 0.05, seed + 12)
    files = rmat_stream(scale, a, b, c, idm, src, dst, n_updates, file_size, del_frac, 0.1, 10.0,
                        seed + 13)
    ip = WalkParams.make(threshold=threshold, walkers=walkers, max_steps=max_steps, seed=seed)
    dp = WalkParams.make(walkers=walkers, max_steps=max_steps, seed=seed)
    return MixedWorkload(f"rmat_{scale}", n, src, dst, w, src[idx], dst[idx], w[idx], files,
                         iparams=ip, dparams=dp,
                         meta={"scale": scale, "edge_factor": edge_factor, "seed": seed,
                               "file_size": file_size, "del_frac": del_frac})


@dataclass
class Workload:
    name: str
    n: int
    g_src: np.ndarray          # dense graph G0 (file order)
    g_dst: np.ndarray
    g_w: np.ndarray
    h_src: np.ndarray          # sparsifier H0 (file order)
    h_dst: np.ndarray
    h_w: np.ndarray
    ins_src: np.ndarray        # insertion stream
    ins_dst: np.ndarray
    ins_w: np.ndarray
    del_src: np.ndarray = field(default_factory=lambda: np.empty(0, np.uint32))
    del_dst: np.ndarray = field(default_factory=lambda: np.empty(0, np.uint32))
    params: WalkParams = None   # incremental
    dparams: WalkParams = None  # decremental
    meta: dict = field(default_factory=dict)


def grid_2d(nx: int = 100, ny: int = 100, inserts: int = 1000, seed: int = MASTER_SEED,
            walkers: int = 512, max_steps: int = 64, threshold: float = 10.0) -> Workload:
    src, dst, w = lattice(nx, ny, 1, W_UNIFORM, 0.5, 2.0, seed + 1)
    n = nx * ny
    idx = sparsifier(n, src, dst, w, 0.10, seed + 2)
    isrc, idst, iw = lattice_inserts(nx, ny, 1, src, dst, inserts, 2, 8, W_UNIFORM, 0.5, 2.0, seed + 3)
    p = WalkParams.make(threshold=threshold, walkers=walkers, max_steps=max_steps, seed=seed)
    return Workload(f"grid_{nx}x{ny}", n, src, dst, w, src[idx], dst[idx], w[idx], isrc, idst, iw,
                    params=p, dparams=WalkParams.make(walkers=walkers, max_steps=100, seed=seed),
                    meta={"nx": nx, "ny": ny, "seed": seed})


def mesh_3d(k: int = 100, inserts: int = 200_000, del_frac: float = 0.10,
            seed: int = MASTER_SEED, walkers: int = 512, max_steps: int = 100,
            threshold: float = 100.0) -> Workload:
    src, dst, w = lattice(k, k, k, W_LOGUNIFORM, 1e-2, 1e2, seed + 1)
    n = k * k * k
    idx = sparsifier(n, src, dst, w, 0.05, seed + 2)
    isrc, idst, iw = lattice_inserts(k, k, k, src, dst, inserts, 2, 10, W_LOGUNIFORM, 1e-2, 1e2,
                                     seed + 3)
    gs = np.concatenate([src, isrc])
    gd = np.concatenate([dst, idst])
    nd = int(np.floor(del_frac * len(gs)))
    di = sample(len(gs), nd, seed + 4)
    p = WalkParams.make(threshold=threshold, walkers=walkers, max_steps=max_steps, seed=seed)
    dp = WalkParams.make(walkers=walkers, max_steps=max_steps, seed=seed)
    return Workload(f"mesh_{k}^3", n, src, dst, w, src[idx], dst[idx], w[idx], isrc, idst, iw,
                    gs[di], gd[di], params=p, dparams=dp, meta={"k": k, "seed": seed})
