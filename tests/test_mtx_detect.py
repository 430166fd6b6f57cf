"""MTX format detection and the auto-detecting reader (the mixed updater's
graph loading, dynamic_update/functions.cpp:35-587) against the reference's
own detector: tests/golden/mtx_detect.json holds its results on the twelve
files of its detection test (dynamic_update/test.cpp:53-178), its fixture
test_matrix.mtx and a few more cases (tests/golden/make_mtx_fixtures.py)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "mtx_detect.json")))
MAP = {"skip_lines": "skip_lines", "has_header": "has_header", "has_dimensions": "has_dimensions",
       "weighted": "weighted", "laplacian": "laplacian", "triangular": "triangular",
       "base": "base", "v_max": "v_max", "v_min": "v_min"}


@pytest.mark.parametrize("case", FIX["cases"], ids=[c["name"] for c in FIX["cases"]])
def test_detect_matches_reference(tmp_path, case):
    import dygrass_b200 as dyg
    p = tmp_path / "g.mtx"
    p.write_text(case["content"])
    got = dyg.mtx_detect(str(p))
    assert {k: got[MAP[k]] for k in FIX["fields"]} == case["expect"]


def test_fixture_covers_reference_cases():
    names = {c["name"] for c in FIX["cases"]}
    assert len([n for n in names if n.startswith("test") and n[4].isdigit()]) == 12
    assert "test_matrix.mtx" in names


def read(tmp_path, text):
    import dygrass_b200 as dyg
    p = tmp_path / "g.mtx"
    p.write_text(text)
    return dyg.mtx_read_auto(str(p))


def test_read_auto_triangular_weighted(tmp_path):
    info, s, d, w = read(tmp_path, "%%MatrixMarket\n% c\n4 4 3\n1 2 0.5\n2 3 1.0\n3 4 0.8\n")
    assert info["triangular"] and info["base"] == 1 and info["skip_lines"] == 3
    assert s.tolist() == [0, 1, 2] and d.tolist() == [1, 2, 3]
    assert w.tolist() == [np.float32(0.5), 1.0, np.float32(0.8)]


def test_read_auto_laplacian(tmp_path):
    """Diagonal records dropped, off-diagonal weights negated."""
    info, s, d, w = read(tmp_path, "3 3 5\n1 1 2.0\n2 1 -1.0\n2 2 2.0\n3 2 -1.5\n3 3 1.0\n")
    assert info["laplacian"] and info["triangular"]
    assert list(zip(s.tolist(), d.tolist(), w.tolist())) == [(1, 0, 1.0), (2, 1, 1.5)]


def test_read_auto_unweighted_zero_based(tmp_path):
    info, s, d, w = read(tmp_path, "0 1\n1 2\n2 0\n")
    assert info["base"] == 0 and not info["weighted"]
    assert s.tolist() == [0, 1, 2] and d.tolist() == [1, 2, 0] and (w == 1.0).all()


def test_read_auto_full(tmp_path):
    info, s, d, w = read(tmp_path, "1 2 1.0\n1 3 2.0\n2 1 1.0\n2 3 3.0\n3 1 2.0\n3 2 3.0\n")
    assert info["triangular"] == 0 and len(s) == 6


def test_detect_errors(tmp_path):
    import dygrass_b200 as dyg
    p = tmp_path / "bad.mtx"
    p.write_text("3 4 5\n7 8 9 10 11\n")
    with pytest.raises(dyg.DygError):
        dyg.mtx_detect(str(p))
    p.write_text("2 3 1.0\n3 4 1.0\n")
    with pytest.raises(dyg.DygError):   # ids neither 0- nor 1-based
        dyg.mtx_detect(str(p))
