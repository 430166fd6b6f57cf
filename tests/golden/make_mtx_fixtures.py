"""Generates tests/golden/mtx_detect.json: the reference's own MTX format
detection (auto_detect_graph_info, dynamic_update/functions.cpp:35-291) on
its test inputs.

The inputs are the twelve files the reference's detection test writes
(dynamic_update/test.cpp:53-178, read here from that file's
create_test_file calls), its fixture dynamic_update/test_matrix.mtx, and a
few more cases written below.  The reference's detector is built from its
sources by `make -C oracle ref` into oracle/_ref/ref_detect (host C++, no
GPU needed):

    make -C oracle ref && python tests/golden/make_mtx_fixtures.py
"""
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _reference_root() -> str:
    """$REF, else the default of oracle/Makefile's REF."""
    if os.environ.get("REF"):
        return os.environ["REF"]
    with open(os.path.join(ROOT, "oracle", "Makefile")) as f:
        for line in f:
            if line.startswith("REF ?="):
                return line.split("?=", 1)[1].strip()
    raise RuntimeError("set REF to the reference's source tree")


REF_SRC = os.path.join(_reference_root(), "dynamic_update")
DETECT = os.path.join(ROOT, "oracle", "_ref", "ref_detect")

FIELDS = ["skip_lines", "has_header", "has_dimensions", "weighted", "laplacian", "triangular",
          "base", "v_max", "v_min"]

# Cases beyond the reference's own: written for this fixture.
EXTRA = {
    "zero_based_dims": "% zero-based with a dimensions line\n5 5 4\n0 1 1.5\n1 2 2.5\n2 3 0.5\n3 4 1.0\n",
    "unweighted_raw": "1 2\n2 3\n3 1\n",
    "lower_laplacian": "%%MatrixMarket matrix coordinate real symmetric\n3 3 5\n1 1 2.0\n2 1 -1.0\n"
                       "2 2 2.0\n3 2 -1.0\n3 3 1.0\n",
    "full_late_reverse": "1 2 1.0\n2 3 1.0\n3 4 1.0\n4 5 1.0\n2 1 1.0\n",
    "dims_mismatch": "6 6 5\n1 2 1.0\n2 3 1.0\n3 4 1.0\n",
    "crlf_free_blank_lines": "1 2 1.0\n\n2 3 2.0\n\n3 1 3.0\n",
}


def c_string_literals(text):
    """The concatenated C string literals of `text` (\\n, \\t, \\\\ and \\" decoded)."""
    out = []
    for m in re.finditer(r'"((?:[^"\\]|\\.)*)"', text):
        out.append(m.group(1).encode().decode("unicode_escape"))
    return "".join(out)


def reference_cases():
    src = open(os.path.join(REF_SRC, "test.cpp")).read()
    cases = []
    for m in re.finditer(r'create_test_file\(test_dir \+ "/([^"]+)",(.*?)\);', src, re.S):
        cases.append((m.group(1), c_string_literals(m.group(2))))
    cases.append(("test_matrix.mtx", open(os.path.join(REF_SRC, "test_matrix.mtx")).read()))
    return cases


def detect(path):
    out = subprocess.run([DETECT, path], capture_output=True, text=True, check=True).stdout
    vals = [int(x) for x in out.strip().split("\n")[-1].split()]
    return dict(zip(FIELDS, vals))


def main(out_path):
    cases = reference_cases() + sorted(EXTRA.items())
    assert len(cases) >= 13, "expected the reference's twelve test files and its fixture"
    tmp = tempfile.mkdtemp(prefix="dyg_mtx_")
    rows = []
    for name, content in cases:
        p = os.path.join(tmp, name if name.endswith(".mtx") else name + ".mtx")
        with open(p, "w") as f:
            f.write(content)
        rows.append({"name": name, "content": content, "expect": detect(p)})
    json.dump({"generator": "tests/golden/make_mtx_fixtures.py", "fields": FIELDS, "cases": rows},
              open(out_path, "w"), indent=1)
    print(f"wrote {len(rows)} cases to {out_path}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "mtx_detect.json"))
