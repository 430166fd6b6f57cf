"""Command-line tools without a GPU: the usage line and exit code 0 without
arguments (random_walk_incremental/main.cu:243, random_walk_decremental/
main.cu:323, dynamic_update/main.cu:28), exit code 2 for an unknown option, and
exit code 1 with the missing file named when the dataset is absent -- all
before any device work."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "dygrass_b200", "bin")

TOOLS = {
    "incremental_update": (["g", "1.0", "32"], "adj_sparse.mtx"),
    "decremental_update": (["g"], "updated_dense.mtx"),
    "dynamic_update": (["g", "1.0", "1", "1", "32", "32"], ".mtx"),
}


def run(tool, args, cwd):
    exe = os.path.join(BIN, tool)
    if not os.path.exists(exe):
        pytest.skip(f"{tool} is not built")
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("tool", sorted(TOOLS))
def test_usage_without_arguments(tool, tmp_path):
    cp = run(tool, [], tmp_path)
    assert cp.returncode == 0
    assert cp.stdout.startswith("Input:") and "graph name" in cp.stdout


@pytest.mark.parametrize("tool", sorted(TOOLS))
def test_unknown_option(tool, tmp_path):
    args, _ = TOOLS[tool]
    cp = run(tool, args + ["--no-such-option"], tmp_path)
    assert cp.returncode == 2
    assert "unknown option" in cp.stderr


@pytest.mark.parametrize("tool", sorted(TOOLS))
def test_missing_dataset(tool, tmp_path):
    args, fname = TOOLS[tool]
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    cp = run(tool, args, run_dir)
    assert cp.returncode == 1
    assert fname in cp.stderr and "g" in cp.stderr
