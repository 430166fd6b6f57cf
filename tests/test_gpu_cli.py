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
