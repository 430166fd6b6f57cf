"""The drop-in executables on the reference's file contract: same argv,
same ../dataset/<graph>/ layout, same output files (compared with the
oracle's decisions written in the reference's format)."""
import os
import subprocess

import numpy as np
import pytest

import kat_cases
from helpers import decr_inputs, incr_inputs, updated_sparse_text

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dygrass_b200", "bin")


@pytest.mark.parametrize("name", sorted(kat_cases.INCREMENTAL))
def test_incremental_cli(tmp_path, oracle, name):
    case = kat_cases.INCREMENTAL[name]
    kat_cases.write_incremental(case, str(tmp_path / "dataset" / name))
    run = tmp_path / "run"
    run.mkdir()
    cp = subprocess.run([os.path.join(BIN, "incremental_update"), name, repr(case["threshold"]),
                         str(case["walkers"])], cwd=run, capture_output=True, text=True, timeout=120)
    assert cp.returncode == 0, cp.stderr
    assert "Time taken:" in cp.stdout
    n, hs, hd, hw, es, ed, ew = incr_inputs(case)
    class P: pass
    p = P()
    p.threshold, p.walkers, p.max_steps, p.transition = case["threshold"], case["walkers"], 100, 0
    p.heuristic_walkers, p.seed = 16, 20251203
    H = oracle.OGraph(n, hs, hd, hw)
    _, _, ac, _ = oracle.incremental(H, es, ed, ew, p)
    got = (tmp_path / "dataset" / name / "updated_adj_sparse.mtx").read_text()
    assert got == updated_sparse_text(hs, hd, hw, es, ed, ew, ac)
    assert f"Edges added: {int(ac.sum())} out of {len(ac)} samples" in cp.stdout


@pytest.mark.parametrize("name", sorted(kat_cases.DECREMENTAL))
def test_decremental_cli(tmp_path, name):
    case = kat_cases.DECREMENTAL[name]
    kat_cases.write_decremental(case, str(tmp_path / "dataset" / name))
    run = tmp_path / "run"
    run.mkdir()
    cp = subprocess.run([os.path.join(BIN, "decremental_update"), name], cwd=run,
                        capture_output=True, text=True, timeout=120)
    assert cp.returncode == 0, cp.stderr
    lines = (tmp_path / "dataset" / name / "added_edges.mtx").read_text().split("\n")
    got = sorted(tuple(int(x) for x in ln.split()) for ln in lines if ln.strip())
    assert got == sorted(case["expect_added"])


def _write_graph(path, n, s, d, w):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n% written by the test\n")
        f.write(f"{n} {n} {len(s)}\n")
        for a, b, x in zip(s, d, w):
            f.write(f"{a + 1} {b + 1} {float(x):.9g}\n")


def _graph_lines(g, oracle_graph):
    rp, col, w = oracle_graph.export()
    out = []
    for u in range(len(rp) - 1):
        for j in range(int(rp[u]), int(rp[u + 1])):
            if int(col[j]) >= u:
                out.append((u, int(col[j]), float(w[j])))
    out.sort(key=lambda t: (t[0], t[1]))
    lines, last = [], None
    for u, v, x in out:
        if (u, v) != last:
            lines.append(f"{u + 1} {v + 1} {x:g}")
        last = (u, v)
    return lines


def test_dynamic_update_cli(tmp_path, oracle):
    """dynamic_update on a folder of insertion and deletion stream files:
    both output graphs equal the oracle's after the same files."""
    import dygrass_b200 as dyg
    from dygrass_b200 import workloads as W
    wl = W.rmat_mixed(scale=10, n_updates=4000, file_size=700, walkers=64)
    ds = tmp_path / "dataset" / "rmat10"
    (ds / "stream_edges" / "sub").mkdir(parents=True)
    _write_graph(ds / "new_adj_dense.mtx", wl.n, wl.g_src, wl.g_dst, wl.g_w)
    _write_graph(ds / "new_adj_sparse.mtx", wl.n, wl.h_src, wl.h_dst, wl.h_w)
    (ds / "stream_edges" / "notes.txt").write_text("not a stream file\n")
    for i, (op, s, d, w) in enumerate(wl.files):
        kind = "decremental" if op else "incremental"
        with open(ds / "stream_edges" / f"stream_{i:04d}_{kind}.mtx", "w") as f:
            for k in range(len(s)):
                f.write(f"{s[k] + 1} {d[k] + 1}" + ("\n" if op else f" {float(w[k]):.9g}\n"))
    cp = subprocess.run([os.path.join(BIN, "dynamic_update"), "rmat10", "50", "128", "128", "64",
                         "64", "--timestamp=T"], cwd=tmp_path, capture_output=True, text=True,
                        timeout=300)
    assert cp.returncode == 0, cp.stdout[-2000:] + cp.stderr
    assert f"Found {len(wl.files)} stream updates files" in cp.stdout

    info, gs, gd, gw = dyg.mtx_read_auto(str(ds / "new_adj_dense.mtx"))
    _, hs, hd, hw = dyg.mtx_read_auto(str(ds / "new_adj_sparse.mtx"))
    assert info["triangular"] and info["has_dimensions"] and info["base"] == 1
    G, H = oracle.OGraph(wl.n, gs, gd, gw), oracle.OGraph(wl.n, hs, hd, hw)
    ip = dyg.WalkParams.make(threshold=50.0, walkers=64, max_steps=128)
    dp = dyg.WalkParams.make(threshold=50.0, walkers=64, max_steps=128)
    names = sorted(os.listdir(ds / "stream_edges"))
    uid, op = 0, 0
    for nm in names:
        if not (nm.startswith("stream_") and ".mtx" in nm):
            continue
        op = dyg.stream_op_from_name(nm, op)
        s, d, w, _ = dyg.stream_read(str(ds / "stream_edges" / nm), 1)
        oracle.stream_file(G, H, op, s, d, w if op == 0 else None, dp if op else ip, first_uid=uid)
        uid += len(s)
    out = tmp_path / "output" / "rmat10" / "T"
    assert (out / "adj_dense.mtx").read_text().split("\n")[:-1] == _graph_lines(None, G)
    assert (out / "adj_sparse.mtx").read_text().split("\n")[:-1] == _graph_lines(None, H)


def test_decremental_snapshot_matches_reconstruction(tmp_path):
    """The final H that the reference's evaluation rebuilds from the files
    (updated graphs minus del.mtx plus added_edges.mtx, dyGRASS.jl:478-541)
    is the device H that decremental_update snapshots."""
    from dygrass_b200 import workloads as W
    from dygrass_b200.evaluate import _read, reconstruct_final
    wl = W.mesh_3d(10, inserts=400)
    gs = np.concatenate([wl.g_src, wl.ins_src])
    gd = np.concatenate([wl.g_dst, wl.ins_dst])
    gw = np.concatenate([wl.g_w, wl.ins_w])
    ds = tmp_path / "dataset" / "mesh10"
    ds.mkdir(parents=True)
    for name, (s, d, w) in (("updated_dense.mtx", (gs, gd, gw)),
                            ("updated_adj_sparse.mtx", (wl.h_src, wl.h_dst, wl.h_w))):
        (ds / name).write_text("".join(f"{a + 1} {b + 1} {float(x):.9g}\n" for a, b, x in zip(s, d, w)))
    (ds / "del.mtx").write_text("".join(f"{a + 1} {b + 1}\n" for a, b in zip(wl.del_src, wl.del_dst)))
    snap = tmp_path / "snap"
    snap.mkdir()
    run = tmp_path / "run"
    run.mkdir()
    cp = subprocess.run([os.path.join(BIN, "decremental_update"), "mesh10", f"--snapshot-dir={snap}"],
                        cwd=run, capture_output=True, text=True, timeout=300)
    assert cp.returncode == 0, cp.stderr
    g = _read(str(ds / "updated_dense.mtx"), 1, True)
    h = _read(str(ds / "updated_adj_sparse.mtx"), 1, True)
    dl = _read(str(ds / "del.mtx"), 1, False)
    ad = _read(str(ds / "added_edges.mtx"), 1, False)
    assert len(ad[0]) > 0
    (fgs, fgd, fgw), (fhs, fhd, fhw) = reconstruct_final(g, h, dl, ad)

    def lines(s, d, w):
        return sorted(f"{min(a, b) + 1} {max(a, b) + 1} {float(x):g}"
                      for a, b, x in zip(s.tolist(), d.tolist(), w.tolist()))
    assert sorted((snap / "adj_sparse.mtx").read_text().split("\n")[:-1]) == lines(fhs, fhd, fhw)
    assert sorted((snap / "adj_dense.mtx").read_text().split("\n")[:-1]) == lines(fgs, fgd, fgw)
