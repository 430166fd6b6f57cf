"""Host-side checks of the C ABI library (no GPU needed): it loads, exports
every symbol its headers declare, and its host-only parts work."""
import os
import re

import numpy as np

import dygrass_b200 as dyg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dyg_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol():
    import ctypes
    L = ctypes.CDLL(dyg.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_defaults():
    assert "sm_100a" in dyg.version()
    p = dyg.WalkParams()
    dyg.lib().dyg_walk_params_default(p)
    assert (p.walkers, p.max_steps, p.heuristic_walkers) == (512, 100, 16)


def test_reference_batch_size():
    # ceil(n/10) (random_walk_incremental/gpu_graph.cuh:135)
    for n, b in [(1, 1), (9, 1), (10, 1), (11, 2), (95, 10), (1000, 100), (200000, 20000),
                 (317000, 31700)]:
        assert dyg.reference_batch_size(n) == b


def test_no_cpu_fallback_without_gpu():
    import torch
    if torch.cuda.is_available():
        return
    with np.testing.assert_raises(dyg.DygError):
        dyg.Graph.from_edges(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32),
                             np.ones(2, np.float32))


def test_mtx_roundtrip(tmp_path):
    import ctypes as C
    p = tmp_path / "a.mtx"
    p.write_text("%%MatrixMarket comment\n1 2 0.5\n2 3\t2.25\n\n3 1 1e-05\n")
    L = dyg.lib()
    n = C.c_uint64()
    s, d, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    mx = C.c_uint32()
    assert L.dyg_mtx_read(str(p).encode(), 1, 1, C.byref(n), C.byref(s), C.byref(d), C.byref(w),
                          C.byref(mx)) == 0
    assert n.value == 3 and mx.value == 2
    src = np.ctypeslib.as_array(C.cast(s, C.POINTER(C.c_uint32)), (3,)).copy()
    wt = np.ctypeslib.as_array(C.cast(w, C.POINTER(C.c_float)), (3,)).copy()
    assert list(src) == [0, 1, 2]
    assert wt[2] == np.float32(1e-05)
    q = tmp_path / "b.mtx"
    assert L.dyg_mtx_write(str(q).encode(), 0, 3, s, d, w, 1) == 0
    # ostream default formatting: %g, 6 significant digits
    assert q.read_text() == "1 2 0.5\n2 3 2.25\n3 1 1e-05\n"
    for x in (s, d, w):
        L.dyg_mtx_free(x)
