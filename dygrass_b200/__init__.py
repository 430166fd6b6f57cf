"""dygrass_b200 -- B200 (sm_100a) implementation of the dyGRASS update path.

The product is the C ABI in include/dyg.h, implemented by the in-tree
libdygrass.so (CUDA kernels + host runtime).  This module is a thin ctypes
mirror of that ABI for Python callers, tests and the benchmark: numpy arrays
are passed as host pointers, torch CUDA tensors as device pointers.  There is
no CPU fallback: if the library is missing, importing fails.

The reference's interface is two executables (incremental_update,
decremental_update); dygrass_b200/bin holds drop-ins built on this ABI.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libdygrass.so")

DYG_OK = 0
DYG_EINVAL, DYG_ENOMEM, DYG_ECUDA, DYG_ERANGE, DYG_ESTATE = 1, 2, 3, 4, 5
STATUS_NAMES = {0: "DYG_OK", 1: "DYG_EINVAL", 2: "DYG_ENOMEM", 3: "DYG_ECUDA", 4: "DYG_ERANGE",
                5: "DYG_ESTATE", 6: "DYG_ENOTSUP", 7: "DYG_EIO"}
TRANSITION_UNIFORM = 0
TRANSITION_WEIGHTED = 1
FLAG_EXHAUSTIVE = 1
DEL_NOT_IN_G = -3
DEL_NOT_IN_H = -2
DEL_NO_PATH = -1
REC_PATH = 0
REC_FALLBACK = 1
STREAM_INSERT = 0
STREAM_DELETE = 1
INS_MERGED = -4
INS_SELF_LOOP = -5


class MtxInfo(C.Structure):
    """dyg_mtx_info: the mixed updater's format detection of a graph file."""
    _fields_ = [("skip_lines", C.c_int64), ("has_header", C.c_int32),
                ("has_dimensions", C.c_int32), ("weighted", C.c_int32), ("laplacian", C.c_int32),
                ("triangular", C.c_int32), ("base", C.c_int32), ("v_max", C.c_uint32),
                ("v_min", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class KappaOpts(C.Structure):
    """Mirror of dyg_kappa_opts (include/dyg_eval.h)."""
    _fields_ = [("offset", C.c_double), ("tol", C.c_double), ("max_iter", C.c_uint32),
                ("pcg_max_iter", C.c_uint32), ("pcg_rtol", C.c_double), ("seed", C.c_uint64)]


class KappaResult(C.Structure):
    """Mirror of dyg_kappa_result (include/dyg_eval.h)."""
    _fields_ = [("kappa", C.c_double), ("density", C.c_double), ("lanczos_iters", C.c_uint32),
                ("pcg_iters", C.c_uint32), ("pcg_relres", C.c_double), ("factor_nnz", C.c_uint64)]


class DygError(RuntimeError):
    def __init__(self, status: int, what: str, msg: str):
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class WalkParams(C.Structure):
    """Mirror of dyg_walk_params (include/dyg.h)."""
    _fields_ = [("threshold", C.c_float), ("walkers", C.c_uint32), ("max_steps", C.c_uint32),
                ("transition", C.c_uint32), ("heuristic_walkers", C.c_uint32),
                ("flags", C.c_uint32), ("seed", C.c_uint64)]

    @classmethod
    def make(cls, threshold=100.0, walkers=512, max_steps=100, transition=TRANSITION_UNIFORM,
             heuristic_walkers=16, seed=20251203, flags=0):
        return cls(float(threshold), int(walkers), int(max_steps), int(transition),
                   int(heuristic_walkers), int(flags), int(seed))


class Profile(C.Structure):
    """Mirror of dyg_profile (include/dyg.h)."""
    _fields_ = [("incr_walk_ms", C.c_double), ("decr_walk_ms", C.c_double),
                ("other_walk_ms", C.c_double), ("incr_walk_launches", C.c_uint64),
                ("decr_walk_launches", C.c_uint64), ("other_walk_launches", C.c_uint64)]


class ServerDone(C.Structure):
    """A completed server request (dyg_server_done, include/dyg_serve.h)."""
    _fields_ = [("tag", C.c_uint64), ("graph", C.c_uint32), ("op", C.c_uint32), ("n", C.c_uint32),
                ("status", C.c_int32), ("first_update_id", C.c_uint64), ("n_rec", C.c_uint64),
                ("step", C.c_uint64), ("t_submit_ns", C.c_uint64), ("t_start_ns", C.c_uint64),
                ("t_done_ns", C.c_uint64)]


class ServerStats(C.Structure):
    """Mirror of dyg_server_stats (include/dyg_serve.h)."""
    _fields_ = [("graphs", C.c_uint32), ("resident", C.c_uint32), ("waiting", C.c_uint32),
                ("pending", C.c_uint32), ("resident_bytes", C.c_uint64), ("budget_bytes", C.c_uint64),
                ("admissions", C.c_uint64), ("evictions", C.c_uint64), ("steps", C.c_uint64),
                ("ns_admit", C.c_uint64), ("ns_stage", C.c_uint64), ("ns_insert", C.c_uint64),
                ("ns_delete", C.c_uint64), ("ns_fetch", C.c_uint64), ("ns_split", C.c_uint64)]


class ServerGraphInfo(C.Structure):
    """Mirror of dyg_server_graph_info (include/dyg_serve.h)."""
    _fields_ = [("n_vertices", C.c_uint32), ("resident", C.c_uint32), ("vertex_offset", C.c_uint32),
                ("pad", C.c_uint32), ("footprint_bytes", C.c_uint64), ("updates", C.c_uint64),
                ("admissions", C.c_uint64), ("evictions", C.c_uint64), ("pending", C.c_uint64)]


class GraphOpts(C.Structure):
    _fields_ = [("slack_per_row", C.c_uint32), ("reserved", C.c_uint32),
                ("arena_headroom", C.c_double), ("device", C.c_int32), ("pad", C.c_int32)]


_lib = None


def lib() -> C.CDLL:
    """Load libdygrass.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m dygrass_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32
    sig = {
        "dyg_version": ([], C.c_char_p),
        "dyg_last_error_string": ([], C.c_char_p),
        "dyg_walk_params_default": ([C.POINTER(WalkParams)], None),
        "dyg_graph_opts_default": ([C.POINTER(GraphOpts)], None),
        "dyg_reference_batch_size": ([u32], u32),
        "dyg_graph_create_from_edges": ([u32, u64, vp, vp, vp, C.POINTER(GraphOpts), C.POINTER(vp)], C.c_int),
        "dyg_graph_create_from_csr": ([u32, vp, vp, vp, C.POINTER(GraphOpts), C.POINTER(vp)], C.c_int),
        "dyg_graph_clone": ([vp, C.POINTER(vp)], C.c_int),
        "dyg_graph_copy_from": ([vp, vp, vp], C.c_int),
        "dyg_graph_destroy": ([vp], C.c_int),
        "dyg_graph_info": ([vp, C.POINTER(u32), C.POINTER(u64), C.POINTER(u64), C.POINTER(u64)], C.c_int),
        "dyg_graph_export": ([vp, vp, vp, vp, u64], C.c_int),
        "dyg_graph_compact": ([vp, vp], C.c_int),
        "dyg_graph_counters": ([vp, C.POINTER(u64), C.POINTER(u64)], C.c_int),
        "dyg_incremental_batch": ([vp, vp, vp, vp, vp, u32, u64, C.POINTER(WalkParams), vp, vp, vp, vp], C.c_int),
        "dyg_incremental_stream": ([vp, vp, vp, vp, vp, u32, u32, C.POINTER(WalkParams), vp, vp, vp, vp], C.c_int),
        "dyg_decremental_batch": ([vp, vp, vp, vp, u32, u64, C.POINTER(WalkParams), vp, vp, vp, vp, vp, u64,
                                   C.POINTER(u64), vp], C.c_int),
        "dyg_decremental_stream": ([vp, vp, vp, vp, u32, u32, C.POINTER(WalkParams), vp, vp, vp, vp, vp, u64,
                                    C.POINTER(u64), vp], C.c_int),
        "dyg_stream_default_chunk": ([u32], u32),
        "dyg_recovered_read": ([vp, u64, u64, vp, vp, vp], C.c_int),
        "dyg_stream_file": ([vp, vp, u32, vp, vp, vp, u32, u64, u32, C.POINTER(WalkParams), vp, vp, vp,
                             vp, vp, u64, C.POINTER(u64), vp], C.c_int),
        "dyg_synth_rmat": ([u32, u32, C.c_double, C.c_double, C.c_double, C.c_float, C.c_float, u64,
                            C.POINTER(u32), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                            C.POINTER(vp)], u64),
        "dyg_synth_rmat_pairs": ([u32, u64, C.c_double, C.c_double, C.c_double, u64, vp, vp], None),
        "dyg_synth_rmat_stream": ([u32, C.c_double, C.c_double, C.c_double, vp, u64, vp, vp, u64, u32,
                                   C.c_double, C.c_float, C.c_float, u64, vp, vp, vp, vp], u64),
        "dyg_mtx_read": ([C.c_char_p, u32, C.c_int, C.POINTER(u64), C.POINTER(vp), C.POINTER(vp),
                          C.POINTER(vp), C.POINTER(u32)], C.c_int),
        "dyg_mtx_free": ([vp], None),
        "dyg_mtx_detect": ([C.c_char_p, C.POINTER(MtxInfo)], C.c_int),
        "dyg_stream_read": ([C.c_char_p, u32, C.POINTER(u64), C.POINTER(vp), C.POINTER(vp),
                             C.POINTER(vp), C.POINTER(C.c_int32)], C.c_int),
        "dyg_stream_op_from_name": ([C.c_char_p, u32], u32),
        "dyg_kappa_opts_default": ([C.POINTER(KappaOpts)], None),
        "dyg_synth_rgg": ([u32, C.c_double, u32, u64, C.POINTER(u32), C.POINTER(vp), C.POINTER(vp),
                           C.POINTER(vp), C.POINTER(u32), C.POINTER(vp), C.POINTER(vp),
                           C.POINTER(vp)], u64),
        "dyg_incremental_batch_ids": ([vp, vp, vp, vp, vp, vp, u32, C.POINTER(WalkParams), vp, vp,
                                       vp, vp], C.c_int),
        "dyg_decremental_batch_ids": ([vp, vp, vp, vp, vp, u32, C.POINTER(WalkParams), vp, vp, vp,
                                       vp, vp, u64, C.POINTER(u64), vp], C.c_int),
        "dyg_tune_set": ([u32, u32], None),
        "dyg_tune_set_prune_interval": ([u32], None),
        "dyg_kappa": ([u32, u64, vp, vp, vp, u64, vp, vp, vp, C.POINTER(KappaOpts),
                       C.POINTER(KappaResult)], C.c_int),
        "dyg_mtx_read_auto": ([C.c_char_p, C.POINTER(MtxInfo), C.POINTER(u64), C.POINTER(vp),
                               C.POINTER(vp), C.POINTER(vp)], C.c_int),
        "dyg_mtx_write": ([C.c_char_p, C.c_int, u64, vp, vp, vp, u32], C.c_int),
        "dyg_synth_lattice_edges": ([u32, u32, u32], u64),
        "dyg_synth_lattice": ([u32, u32, u32, u32, C.c_float, C.c_float, u64, vp, vp, vp], None),
        "dyg_synth_sparsifier": ([u32, u64, vp, vp, vp, C.c_double, u64, vp], u64),
        "dyg_synth_lattice_inserts": ([u32, u32, u32, u64, vp, vp, u64, u32, u32, u32, C.c_float, C.c_float,
                                       u64, vp, vp, vp], u64),
        "dyg_synth_sample": ([u64, u64, u64, vp], None),
        "dyg_profile_enable": ([C.c_int], C.c_int),
        "dyg_profile_reset": ([], C.c_int),
        "dyg_profile_read": ([C.POINTER(Profile)], C.c_int),
        "dyg_kernel_launches": ([], u64),
        "dyg_incremental_walk_noalloc": ([vp, vp, vp, vp, u32, u64, C.POINTER(WalkParams), vp, vp, vp, vp],
                                         C.c_int),
        "dyg_server_create": ([vp, vp, u32, vp, C.POINTER(WalkParams), C.POINTER(WalkParams), vp,
                               C.POINTER(vp)], C.c_int),
        "dyg_server_destroy": ([vp], C.c_int),
        "dyg_server_submit": ([vp, u64, u32, u32, vp, vp, vp, u32], C.c_int),
        "dyg_server_submit_many": ([vp, u32, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "dyg_server_step": ([vp, C.POINTER(u32)], C.c_int),
        "dyg_server_start": ([vp], C.c_int),
        "dyg_server_stop": ([vp], C.c_int),
        "dyg_server_drain": ([vp, C.c_double], C.c_int),
        "dyg_server_pending": ([vp], u32),
        "dyg_server_poll": ([vp, C.POINTER(ServerDone), u32, C.POINTER(u32)], C.c_int),
        "dyg_server_fetch": ([vp, u64, vp, vp, vp, vp, vp, vp, u64], C.c_int),
        "dyg_server_reset": ([vp], C.c_int),
        "dyg_server_steps": ([vp], u64),
        "dyg_server_now_ns": ([vp], u64),
        "dyg_server_last_error": ([vp], C.c_char_p),
        "dyg_server_create_pool": ([u32, u64, C.POINTER(WalkParams), C.POINTER(WalkParams), C.c_int, u32,
                                    vp, C.POINTER(vp)], C.c_int),
        "dyg_server_add_graph": ([vp, u32, u64, vp, vp, vp, u64, vp, vp, vp, C.POINTER(u32)], C.c_int),
        "dyg_server_prefetch": ([vp, u32, C.POINTER(u32)], C.c_int),
        "dyg_server_stats_read": ([vp, C.POINTER(ServerStats)], C.c_int),
        "dyg_server_graph_info_read": ([vp, u32, C.POINTER(ServerGraphInfo)], C.c_int),
        "dyg_server_graph_export": ([vp, u32, u32, vp, vp, vp, u64], C.c_int),
        "dyg_server_counters": ([vp, C.POINTER(u64), C.POINTER(u64)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(status: int, what: str) -> None:
    if status != DYG_OK:
        raise DygError(status, what, lib().dyg_last_error_string().decode())


def _ptr(a):
    """Pointer of a numpy array (host) or a torch tensor (host or device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous()
        return a.data_ptr()
    raise TypeError(type(a))


def _as(a, dtype):
    if a is None or hasattr(a, "data_ptr"):
        return a
    return np.ascontiguousarray(a, dtype=dtype)


def profile_enable(on: bool = True) -> None:
    _check(lib().dyg_profile_enable(1 if on else 0), "dyg_profile_enable")


def profile_reset() -> None:
    _check(lib().dyg_profile_reset(), "dyg_profile_reset")


def profile_read() -> dict:
    p = Profile()
    _check(lib().dyg_profile_read(C.byref(p)), "dyg_profile_read")
    return {f: getattr(p, f) for f, _ in Profile._fields_}


def kernel_launches() -> int:
    return int(lib().dyg_kernel_launches())


def version() -> str:
    return lib().dyg_version().decode()


def reference_batch_size(n: int) -> int:
    return int(lib().dyg_reference_batch_size(int(n)))


class Graph:
    """A device-resident dynamic CSR (dyg_graph handle)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_edges(cls, n_vertices: int, src, dst, w, slack_per_row: int = 2,
                   arena_headroom: float = 0.5, device: int = -1) -> "Graph":
        src = _as(src, np.uint32)
        dst = _as(dst, np.uint32)
        w = _as(w, np.float32)
        opts = GraphOpts(int(slack_per_row), 0, float(arena_headroom), int(device), 0)
        h = C.c_void_p()
        _check(lib().dyg_graph_create_from_edges(int(n_vertices), len(src), _ptr(src), _ptr(dst),
                                                 _ptr(w), C.byref(opts), C.byref(h)),
               "dyg_graph_create_from_edges")
        return cls(h.value)

    @classmethod
    def from_csr(cls, n_vertices: int, row_ptr, col, w, slack_per_row: int = 2,
                 arena_headroom: float = 0.5, device: int = -1) -> "Graph":
        """Rows as given (no reverse slots added)."""
        rp = np.ascontiguousarray(row_ptr, np.uint64)
        col = _as(col, np.uint32)
        w = _as(w, np.float32)
        opts = GraphOpts(int(slack_per_row), 0, float(arena_headroom), int(device), 0)
        h = C.c_void_p()
        _check(lib().dyg_graph_create_from_csr(int(n_vertices), _ptr(rp), _ptr(col), _ptr(w),
                                               C.byref(opts), C.byref(h)),
               "dyg_graph_create_from_csr")
        return cls(h.value)

    def clone(self) -> "Graph":
        h = C.c_void_p()
        _check(lib().dyg_graph_clone(self._h, C.byref(h)), "dyg_graph_clone")
        return Graph(h.value)

    def copy_from(self, other: "Graph", stream: int | None = None) -> None:
        _check(lib().dyg_graph_copy_from(self._h, other._h, stream), "dyg_graph_copy_from")

    def close(self) -> None:
        if self._h is not None and self._h.value:
            lib().dyg_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def info(self) -> dict:
        n = C.c_uint32()
        s, u, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib().dyg_graph_info(self._h, C.byref(n), C.byref(s), C.byref(u), C.byref(c)),
               "dyg_graph_info")
        return {"n_vertices": n.value, "n_slots": s.value, "arena_used": u.value,
                "arena_cap": c.value}

    def export(self):
        """(row_ptr[n+1] u64, col u32, w f32) in row order."""
        inf = self.info()
        n, s = inf["n_vertices"], inf["n_slots"]
        rp = np.zeros(n + 1, np.uint64)
        col = np.zeros(max(s, 1), np.uint32)
        w = np.zeros(max(s, 1), np.float32)
        _check(lib().dyg_graph_export(self._h, _ptr(rp), _ptr(col), _ptr(w), s), "dyg_graph_export")
        return rp, col[:s], w[:s]

    def compact(self, stream: int | None = None) -> None:
        _check(lib().dyg_graph_compact(self._h, stream), "dyg_graph_compact")

    def counters(self) -> tuple[int, int]:
        m, k = C.c_uint64(), C.c_uint64()
        _check(lib().dyg_graph_counters(self._h, C.byref(m), C.byref(k)), "dyg_graph_counters")
        return m.value, k.value


@dataclass
class IncrementalResult:
    found_at: np.ndarray   # i32: winner's step count or -1
    conductance: np.ndarray  # f32: winner's 1/R (0 if none)
    accepted: np.ndarray   # u8: 1 iff the edge was added to H


def incremental_batch(H: Graph, src, dst, w, params: WalkParams, first_update_id: int = 0,
                      G: Graph | None = None, stream: int | None = None) -> IncrementalResult:
    src, dst, w = _as(src, np.uint32), _as(dst, np.uint32), _as(w, np.float32)
    n = len(src)
    out = IncrementalResult(np.empty(n, np.int32), np.empty(n, np.float32), np.empty(n, np.uint8))
    _check(lib().dyg_incremental_batch(H.handle, G.handle if G else None, _ptr(src), _ptr(dst),
                                       _ptr(w), n, int(first_update_id), C.byref(params),
                                       _ptr(out.found_at), _ptr(out.conductance),
                                       _ptr(out.accepted), stream), "dyg_incremental_batch")
    return out


def incremental_stream(H: Graph, src, dst, w, params: WalkParams, batch_size: int = 0,
                       G: Graph | None = None, stream: int | None = None,
                       out: IncrementalResult | None = None) -> IncrementalResult:
    """The reference's update loop: batches of ceil(n/10) unless batch_size."""
    src, dst, w = _as(src, np.uint32), _as(dst, np.uint32), _as(w, np.float32)
    n = len(src)
    if out is None:
        out = IncrementalResult(np.empty(n, np.int32), np.empty(n, np.float32),
                                np.empty(n, np.uint8))
    _check(lib().dyg_incremental_stream(H.handle, G.handle if G else None, _ptr(src), _ptr(dst),
                                        _ptr(w), n, int(batch_size), C.byref(params),
                                        _ptr(out.found_at), _ptr(out.conductance),
                                        _ptr(out.accepted), stream), "dyg_incremental_stream")
    return out


@dataclass
class DecrementalResult:
    status: np.ndarray      # i32: path length or DEL_* code
    conductance: np.ndarray  # f32
    rec_src: np.ndarray     # u32 recovered edges, commit order
    rec_dst: np.ndarray
    rec_kind: np.ndarray    # u8: REC_PATH / REC_FALLBACK


def recovered_read(G: Graph, count: int, first: int = 0):
    """Recovered edges [first, first + count) of the last decremental call on
    G (dyg_recovered_read): (rec_src, rec_dst, rec_kind) as numpy arrays."""
    rx = np.empty(max(count, 1), np.uint32)
    ry = np.empty(max(count, 1), np.uint32)
    rk = np.empty(max(count, 1), np.uint8)
    _check(lib().dyg_recovered_read(G.handle, int(first), int(count), _ptr(rx), _ptr(ry), _ptr(rk)),
           "dyg_recovered_read")
    return rx[:count], ry[:count], rk[:count]


def _decremental(fn, G, H, src, dst, params, arg, stream, rec_cap):
    """With rec_cap None the call records no edges into caller buffers; the
    total comes back in n_rec and exactly that many are read afterwards."""
    src, dst = _as(src, np.uint32), _as(dst, np.uint32)
    n = len(src)
    st = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    nrec = C.c_uint64()
    if rec_cap is None:
        _check(fn(G.handle, H.handle, _ptr(src), _ptr(dst), n, int(arg), C.byref(params), _ptr(st),
                  _ptr(cd), None, None, None, 0, C.byref(nrec), stream), fn.__name__)
        return DecrementalResult(st, cd, *recovered_read(G, nrec.value))
    rx = np.empty(max(rec_cap, 1), np.uint32)
    ry = np.empty(max(rec_cap, 1), np.uint32)
    rk = np.empty(max(rec_cap, 1), np.uint8)
    _check(fn(G.handle, H.handle, _ptr(src), _ptr(dst), n, int(arg), C.byref(params), _ptr(st),
              _ptr(cd), _ptr(rx), _ptr(ry), _ptr(rk), rec_cap, C.byref(nrec), stream),
           fn.__name__)
    k = nrec.value
    return DecrementalResult(st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy())


def decremental_stream_into(G: Graph, H: Graph, src, dst, params: WalkParams, status, conductance,
                            rec_src, rec_dst, rec_kind, rec_cap: int, batch_size: int = 0,
                            stream: int | None = None) -> int:
    """decremental_stream writing into caller buffers (numpy or torch, host or
    device); returns the number of recovered edges."""
    src, dst = _as(src, np.uint32), _as(dst, np.uint32)
    nrec = C.c_uint64()
    _check(lib().dyg_decremental_stream(G.handle, H.handle, _ptr(src), _ptr(dst), len(src),
                                        int(batch_size), C.byref(params), _ptr(status),
                                        _ptr(conductance), _ptr(rec_src), _ptr(rec_dst),
                                        _ptr(rec_kind), int(rec_cap), C.byref(nrec), stream),
           "dyg_decremental_stream")
    return nrec.value


def decremental_batch(G: Graph, H: Graph, src, dst, params: WalkParams, first_update_id: int = 0,
                      stream: int | None = None, rec_cap: int | None = None) -> DecrementalResult:
    return _decremental(lib().dyg_decremental_batch, G, H, src, dst, params, first_update_id,
                        stream, rec_cap)


def decremental_stream(G: Graph, H: Graph, src, dst, params: WalkParams, batch_size: int = 0,
                       stream: int | None = None, rec_cap: int | None = None) -> DecrementalResult:
    return _decremental(lib().dyg_decremental_stream, G, H, src, dst, params, batch_size, stream,
                        rec_cap)


def mtx_detect(path: str) -> dict:
    """Format detection of a graph file with the mixed updater's rules."""
    info = MtxInfo()
    _check(lib().dyg_mtx_detect(os.fsencode(path), C.byref(info)), "dyg_mtx_detect")
    return info.as_dict()


def mtx_read_auto(path: str):
    """Returns (info dict, src, dst, w): the records as the mixed updater's
    graph loader reads them (0-based)."""
    info = MtxInfo()
    m = C.c_uint64()
    ps, pd, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _check(lib().dyg_mtx_read_auto(os.fsencode(path), C.byref(info), C.byref(m), C.byref(ps),
                                   C.byref(pd), C.byref(pw)), "dyg_mtx_read_auto")
    k = m.value
    try:
        src = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        dst = np.ctypeslib.as_array(C.cast(pd, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        w = np.ctypeslib.as_array(C.cast(pw, C.POINTER(C.c_float)), (max(k, 1),))[:k].copy()
    finally:
        for p in (ps, pd, pw):
            lib().dyg_mtx_free(p)
    return info.as_dict(), src, dst, w


def stream_read(path: str, base: int):
    """Returns (src, dst, w, weighted) of one stream file, ids minus base."""
    m = C.c_uint64()
    ps, pd, pw = C.c_void_p(), C.c_void_p(), C.c_void_p()
    wt = C.c_int32()
    _check(lib().dyg_stream_read(os.fsencode(path), int(base), C.byref(m), C.byref(ps),
                                 C.byref(pd), C.byref(pw), C.byref(wt)), "dyg_stream_read")
    k = m.value
    try:
        src = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        dst = np.ctypeslib.as_array(C.cast(pd, C.POINTER(C.c_uint32)), (max(k, 1),))[:k].copy()
        w = np.ctypeslib.as_array(C.cast(pw, C.POINTER(C.c_float)), (max(k, 1),))[:k].copy()
    finally:
        for p in (ps, pd, pw):
            lib().dyg_mtx_free(p)
    return src, dst, w, bool(wt.value)


def stream_op_from_name(name: str, prev_op: int = 0) -> int:
    return int(lib().dyg_stream_op_from_name(os.fsencode(name), int(prev_op)))


def kappa(n: int, g_src, g_dst, g_w, h_src, h_dst, h_w, **opts) -> dict:
    """kappa(L_G, L_H), density and the PCG iteration count (dyg_kappa).
    Edge lists give each undirected edge once; opts override dyg_kappa_opts."""
    o = KappaOpts()
    lib().dyg_kappa_opts_default(C.byref(o))
    for k, v in opts.items():
        setattr(o, k, v)
    gs, gd, gw = (np.ascontiguousarray(a, t) for a, t in
                  ((g_src, np.uint32), (g_dst, np.uint32), (g_w, np.float32)))
    hs, hd, hw = (np.ascontiguousarray(a, t) for a, t in
                  ((h_src, np.uint32), (h_dst, np.uint32), (h_w, np.float32)))
    r = KappaResult()
    _check(lib().dyg_kappa(int(n), len(gs), _ptr(gs), _ptr(gd), _ptr(gw), len(hs), _ptr(hs),
                           _ptr(hd), _ptr(hw), C.byref(o), C.byref(r)), "dyg_kappa")
    return {k: getattr(r, k) for k, _ in r._fields_}


def graph_edges(g: "Graph"):
    """(src, dst, w) of a device graph, each undirected edge once (u <= v,
    the weight of u's first slot holding v)."""
    rp, col, w = g.export()
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.uint32), np.diff(rp).astype(np.int64))
    keep = col >= rows
    u, v, x = rows[keep], col[keep], w[keep]
    key = u.astype(np.uint64) << np.uint64(32) | v.astype(np.uint64)
    _, first = np.unique(key, return_index=True)
    first.sort()
    return u[first], v[first], x[first]


def incremental_batch_ids(H: Graph, src, dst, w, update_ids, params: WalkParams,
                          G: Graph | None = None, stream: int | None = None,
                          out: IncrementalResult | None = None) -> IncrementalResult:
    """One incremental batch with an update id per edge (dyg_incremental_batch_ids)."""
    src, dst, w = _as(src, np.uint32), _as(dst, np.uint32), _as(w, np.float32)
    ids = _as(update_ids, np.uint64)
    n = len(src)
    if out is None:
        out = IncrementalResult(np.empty(n, np.int32), np.empty(n, np.float32),
                                np.empty(n, np.uint8))
    _check(lib().dyg_incremental_batch_ids(H.handle, G.handle if G else None, _ptr(src), _ptr(dst),
                                           _ptr(w), _ptr(ids), n, C.byref(params),
                                           _ptr(out.found_at), _ptr(out.conductance),
                                           _ptr(out.accepted), stream),
           "dyg_incremental_batch_ids")
    return out


def decremental_batch_ids(G: Graph, H: Graph, src, dst, update_ids, params: WalkParams,
                          stream: int | None = None, rec_cap: int | None = None) -> DecrementalResult:
    """One decremental batch with an update id per edge (dyg_decremental_batch_ids)."""
    src, dst = _as(src, np.uint32), _as(dst, np.uint32)
    ids = _as(update_ids, np.uint64)
    n = len(src)
    if rec_cap is None:
        rec_cap = n * (params.max_steps + 4 * params.heuristic_walkers) + 16
    st = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    rx = np.empty(max(rec_cap, 1), np.uint32)
    ry = np.empty(max(rec_cap, 1), np.uint32)
    rk = np.empty(max(rec_cap, 1), np.uint8)
    nrec = C.c_uint64()
    _check(lib().dyg_decremental_batch_ids(G.handle, H.handle, _ptr(src), _ptr(dst), _ptr(ids), n,
                                           C.byref(params), _ptr(st), _ptr(cd), _ptr(rx), _ptr(ry),
                                           _ptr(rk), rec_cap, C.byref(nrec), stream),
           "dyg_decremental_batch_ids")
    k = nrec.value
    return DecrementalResult(st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy())


def tune_set(walk_chunk: int = 0, blocks_per_sm: int = 0, prune_every: int = 0) -> None:
    """Walk-kernel launch shape for this process and the iterations between a
    walker's reads of its edge's best result (results do not depend on them;
    0 = default)."""
    lib().dyg_tune_set(int(walk_chunk), int(blocks_per_sm))
    lib().dyg_tune_set_prune_interval(int(prune_every))


def stream_default_chunk(n_vertices: int) -> int:
    """Walk-list chunk of the mixed updater: 5% of |V|, at least 10000."""
    return int(lib().dyg_stream_default_chunk(int(n_vertices)))


def stream_file(G: Graph, H: Graph, op: int, src, dst, w, params: WalkParams,
                first_update_id: int = 0, chunk: int = 0, stream: int | None = None,
                rec_cap: int | None = None) -> DecrementalResult:
    """One file of the mixed insert/delete stream (dyg_stream_file).

    op STREAM_INSERT: status = found_at / -1 (accepted) / INS_MERGED /
    INS_SELF_LOOP; op STREAM_DELETE: status = path length / DEL_* codes, plus
    the recovered edges.  w may be None for delete files."""
    src, dst = _as(src, np.uint32), _as(dst, np.uint32)
    w = None if w is None else _as(w, np.float32)
    n = len(src)
    st = np.empty(n, np.int32)
    cd = np.empty(n, np.float32)
    if rec_cap is None:
        nrec = C.c_uint64()
        _check(lib().dyg_stream_file(G.handle, H.handle, int(op), _ptr(src), _ptr(dst), _ptr(w), n,
                                     int(first_update_id), int(chunk), C.byref(params), _ptr(st),
                                     _ptr(cd), None, None, None, 0, C.byref(nrec), stream),
               "dyg_stream_file")
        recs = recovered_read(G, nrec.value) if op != STREAM_INSERT else recovered_read(G, 0)
        return DecrementalResult(st, cd, *recs)
    rx = np.empty(max(rec_cap, 1), np.uint32)
    ry = np.empty(max(rec_cap, 1), np.uint32)
    rk = np.empty(max(rec_cap, 1), np.uint8)
    nrec = C.c_uint64()
    _check(lib().dyg_stream_file(G.handle, H.handle, int(op), _ptr(src), _ptr(dst), _ptr(w), n,
                                 int(first_update_id), int(chunk), C.byref(params), _ptr(st),
                                 _ptr(cd), _ptr(rx), _ptr(ry), _ptr(rk), int(rec_cap),
                                 C.byref(nrec), stream), "dyg_stream_file")
    k = nrec.value
    return DecrementalResult(st, cd, rx[:k].copy(), ry[:k].copy(), rk[:k].copy())


def stream_file_into(G: Graph, H: Graph, op: int, src, dst, w, params: WalkParams, status,
                     conductance, rec_src, rec_dst, rec_kind, rec_cap: int,
                     first_update_id: int = 0, chunk: int = 0, stream: int | None = None) -> int:
    """stream_file writing into caller buffers (numpy or torch, host or
    device); returns the number of recovered edges."""
    src, dst = _as(src, np.uint32), _as(dst, np.uint32)
    w = None if w is None else _as(w, np.float32)
    nrec = C.c_uint64()
    _check(lib().dyg_stream_file(G.handle, H.handle, int(op), _ptr(src), _ptr(dst), _ptr(w), len(src),
                                 int(first_update_id), int(chunk), C.byref(params), _ptr(status),
                                 _ptr(conductance), _ptr(rec_src), _ptr(rec_dst), _ptr(rec_kind),
                                 int(rec_cap), C.byref(nrec), stream), "dyg_stream_file")
    return nrec.value


__all__ = ["Graph", "WalkParams", "GraphOpts", "DygError", "incremental_batch",
           "incremental_stream", "decremental_batch", "decremental_stream", "lib", "version",
           "reference_batch_size", "IncrementalResult", "DecrementalResult", "stream_file",
           "stream_file_into", "stream_default_chunk", "kappa", "graph_edges", "recovered_read"]
