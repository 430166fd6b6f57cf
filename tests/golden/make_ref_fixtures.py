"""Generates tests/golden/ref_kat.json: outputs of the reference's own
updaters on the known-answer cases of kat_cases.py.

The reference (random_walk_incremental/, random_walk_decremental/) is built
unmodified from its sources by `make -C oracle ref-gpu` into oracle/_ref/;
it needs a GPU, so this script runs on a machine with a B200:

    python tests/golden/make_ref_fixtures.py out/ref_kat.json

It writes each case as ../dataset/<case>/ (the reference's fixed relative
layout, main.cu:247-249, 326-329) under a scratch directory, runs the
binary from a sibling directory, and records updated_adj_sparse.mtx /
added_edges.mtx and the binaries' summary lines.
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import kat_cases  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def main(out_path):
    scratch = tempfile.mkdtemp(prefix="dyg_ref_")
    ds = os.path.join(scratch, "dataset")
    run = os.path.join(scratch, "run")
    os.makedirs(run)
    result = {"incremental": {}, "decremental": {}, "generator": "tests/golden/make_ref_fixtures.py"}
    for name, case in kat_cases.INCREMENTAL.items():
        d = os.path.join(ds, name)
        kat_cases.write_incremental(case, d)
        cp = subprocess.run([os.path.join(REF, "incremental_update"), name, repr(case["threshold"]),
                             str(case["walkers"])], cwd=run, capture_output=True, text=True,
                            timeout=120)
        out = open(os.path.join(d, "updated_adj_sparse.mtx")).read() if cp.returncode == 0 else None
        lines = [ln for ln in cp.stdout.splitlines() if ln.startswith(("No path", "Edges added"))]
        result["incremental"][name] = {"returncode": cp.returncode, "updated_adj_sparse": out,
                                       "summary": lines, "stderr_tail": cp.stderr[-400:]}
        print(name, cp.returncode, lines, flush=True)
    for name, case in kat_cases.DECREMENTAL.items():
        d = os.path.join(ds, name)
        kat_cases.write_decremental(case, d)
        cp = subprocess.run([os.path.join(REF, "decremental_update"), name], cwd=run,
                            capture_output=True, text=True, timeout=120)
        # The reference writes added_edges.mtx and prints "Added edges saved
        # to" before its teardown; its teardown can abort (heap damage from the
        # out-of-range degree[v_max] write, random_walk_decremental/
        # functions.cpp:123, 169), so the file is kept when it was completed.
        edges = None
        path = os.path.join(d, "added_edges.mtx")
        if "Added edges saved to" in cp.stdout and os.path.exists(path):
            edges = sorted([int(x) for x in ln.split()[:2]] for ln in open(path) if ln.strip())
        lines = [ln for ln in cp.stdout.splitlines() if ln.startswith(("Increased", "Density", "No path count"))]
        result["decremental"][name] = {"returncode": cp.returncode, "added_edges": edges,
                                       "summary": lines, "stderr_tail": cp.stderr[-400:]}
        print(name, cp.returncode, edges, lines, flush=True)
    shutil.rmtree(scratch, ignore_errors=True)
    with open(out_path, "w") as f:
        json.dump(result, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_kat.json"))
