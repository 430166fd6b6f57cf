"""The CPU oracle against published Philox vectors and known-answer cases.

Philox4x32-10 vectors: Random123 known-answer tests (Salmon et al., SC'11).
Known-answer cases: tests/golden/kat_cases.py (decisions derived from the
reference's stop rules); when tests/golden/ref_kat.json exists (outputs of
the reference's own updaters run on a B200), the oracle's output files must
match it byte for byte (incremental) / as sets (decremental).
"""
import json
import os

import numpy as np
import pytest

import kat_cases
from helpers import decr_inputs, incr_inputs, updated_sparse_text

HERE = os.path.dirname(os.path.abspath(__file__))
REF_KAT = os.path.join(HERE, "golden", "ref_kat.json")


class P:  # walk params with the fields pyoracle reads
    def __init__(self, threshold=100.0, walkers=512, max_steps=100, transition=0,
                 heuristic_walkers=16, seed=20251203):
        self.threshold, self.walkers, self.max_steps = threshold, walkers, max_steps
        self.transition, self.heuristic_walkers, self.seed = transition, heuristic_walkers, seed


@pytest.mark.parametrize("ctr,key,out", [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
])
def test_philox_kat(oracle, ctr, key, out):
    assert list(oracle.philox(ctr, key)) == out


def test_draw_counter_layout(oracle):
    seed, uid, dom, walker = 0x1234_5678_9ABC_DEF0, (7 << 32) | 99, 1, 33
    for d in range(9):
        block = oracle.philox([d >> 2, walker, uid & 0xFFFFFFFF, ((uid >> 32) & 0xFFFFFF) | (dom << 24)],
                              [seed & 0xFFFFFFFF, seed >> 32])
        assert oracle.draw(seed, uid, dom, walker, d) == block[d & 3]


@pytest.mark.parametrize("name", sorted(kat_cases.INCREMENTAL))
def test_incremental_known_answers(oracle, name):
    case = kat_cases.INCREMENTAL[name]
    n, hs, hd, hw, es, ed, ew = incr_inputs(case)
    H = oracle.OGraph(n, hs, hd, hw)
    p = P(threshold=case["threshold"], walkers=case["walkers"])
    fa, cd, ac, _ = oracle.incremental(H, es, ed, ew, p)
    assert list(ac) == case["expect_added"]
    if "expect_found_at" in case:
        assert list(fa) == case["expect_found_at"]
    # found_at > 0 <=> not added; conductance is 1/R of the winner
    assert all((f > 0) == (a == 0) for f, a in zip(fa, ac))
    assert all((c > 0) == (a == 0) for c, a in zip(cd, ac))


def test_incremental_threshold_conductance(oracle):
    case = kat_cases.INCREMENTAL["path_threshold"]
    n, hs, hd, hw, es, ed, ew = incr_inputs(case)
    H = oracle.OGraph(n, hs, hd, hw)
    fa, cd, ac, _ = oracle.incremental(H, es, ed, ew, P(threshold=10.0))
    assert cd[0] == np.float32(0.25)                      # R = 4 over unit weights
    assert cd[3] == np.float32(1.0) / np.float32(1.5)     # 11 -> 6 (w 2) -> 7


@pytest.mark.parametrize("name", sorted(kat_cases.DECREMENTAL))
def test_decremental_known_answers(oracle, name):
    case = kat_cases.DECREMENTAL[name]
    n, gs, gd, gw, hs, hd, hw, ds, dd = decr_inputs(case)
    G = oracle.OGraph(n, gs, gd, gw)
    H = oracle.OGraph(n, hs, hd, hw)
    st, cd, rx, ry, rk, _ = oracle.decremental(G, H, ds, dd, P())
    got = sorted((min(a, b) + 1, max(a, b) + 1) for a, b, k in zip(rx, ry, rk) if k == 0)
    assert got == sorted(case["expect_added"])
    assert all(s > 0 for s in st)
    for a, b in case["expect_added"]:
        assert H.has_edge(a - 1, b - 1)
    for a, b in zip(ds, dd):
        assert not G.has_edge(a, b) and not H.has_edge(a, b)


@pytest.mark.skipif(not os.path.exists(REF_KAT), reason="no reference outputs recorded")
def test_oracle_matches_reference_outputs(oracle):
    ref = json.load(open(REF_KAT))
    n_checked = 0
    for name, rec in ref["incremental"].items():
        if rec.get("updated_adj_sparse") is None:
            continue
        n_checked += 1
        case = kat_cases.INCREMENTAL[name]
        n, hs, hd, hw, es, ed, ew = incr_inputs(case)
        H = oracle.OGraph(n, hs, hd, hw)
        _, _, ac, _ = oracle.incremental(H, es, ed, ew, P(threshold=case["threshold"],
                                                           walkers=case["walkers"]))
        assert updated_sparse_text(hs, hd, hw, es, ed, ew, ac) == rec["updated_adj_sparse"], name
    for name, rec in ref["decremental"].items():
        if rec.get("added_edges") is None:
            continue
        n_checked += 1
        case = kat_cases.DECREMENTAL[name]
        n, gs, gd, gw, hs, hd, hw, ds, dd = decr_inputs(case)
        G = oracle.OGraph(n, gs, gd, gw)
        H = oracle.OGraph(n, hs, hd, hw)
        _, _, rx, ry, rk, _ = oracle.decremental(G, H, ds, dd, P())
        got = sorted((int(min(a, b)) + 1, int(max(a, b)) + 1) for a, b, k in zip(rx, ry, rk) if k == 0)
        assert got == sorted(tuple(e) for e in rec["added_edges"]), name
    assert n_checked >= len(kat_cases.INCREMENTAL)


def test_snapshot_vs_sequential(oracle):
    """Batch size 1 (sequential) finds (0,16) through (0,15); the reference's
    batches of 2 do not."""
    case = kat_cases.INCREMENTAL["snapshot"]
    n, hs, hd, hw, es, ed, ew = incr_inputs(case)
    H = oracle.OGraph(n, hs, hd, hw)
    _, _, ac, _ = oracle.incremental(H, es, ed, ew, P(threshold=12.0), batch_size=1)
    assert list(ac[:3]) == [1, 0, 0]


def test_oracle_threads_do_not_change_results(oracle):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(30, 30, inserts=200)
    outs = []
    for th in (1, 4):
        H = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
        fa, cd, ac, mv = oracle.incremental(H, W.ins_src, W.ins_dst, W.ins_w, W.params, threads=th)
        outs.append((fa.tobytes(), cd.tobytes(), ac.tobytes(), mv, H.export()[1].tobytes()))
    assert outs[0] == outs[1]


def test_weighted_transition_oracle_runs(oracle):
    import dygrass_b200.workloads as wl
    W = wl.grid_2d(20, 20, inserts=100)
    H = oracle.OGraph(W.n, W.h_src, W.h_dst, W.h_w)
    p = P(threshold=10.0, max_steps=64, transition=1)
    fa, cd, ac, mv = oracle.incremental(H, W.ins_src, W.ins_dst, W.ins_w, p)
    assert mv > 0 and 0 < ac.sum() < len(ac)
