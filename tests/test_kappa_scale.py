"""Spectral quality at scale: kappa(L_G, L_H) of a 3-D mesh before and
after the benchmark's update pattern -- insertions of 20 % of |V| in 10
batches, then deletions of 10 % of the updated G in 10 batches (the 100^3
benchmark's proportions).

The final graphs come from the CPU oracle, which the GPU path matches bit
for bit (tests/test_gpu_scale.py at 100^3), so this is the kappa of the GPU's
result.  kappa is the FP64 Lanczos estimate of dyg_kappa, whose factorisation
of L_H fills in on a 3-D sparsifier, and more after the recovered paths
close long cycles: at 40^3 (64,000 vertices) the final estimate takes about
7 minutes, at 60^3 over half an hour and at 100^3 hours, so the size is
DYG_KAPPA_K (default 40).  The test is skipped unless DYG_KAPPA_SCALE=1:

    DYG_KAPPA_SCALE=1 python -m pytest tests/test_kappa_scale.py -s
"""
import os
import time

import numpy as np
import pytest

from dygrass_b200 import workloads as W

pytestmark = pytest.mark.skipif(os.environ.get("DYG_KAPPA_SCALE") != "1",
                                reason="minutes of CPU: set DYG_KAPPA_SCALE=1")


def undirected(g):
    rp, c, w = g.export()
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.uint32), np.diff(rp).astype(np.int64))
    keep = c > rows
    return rows[keep], c[keep], w[keep]


def test_kappa_mesh_step(oracle):
    import dygrass_b200 as dyg
    t0 = time.time()
    k = int(os.environ.get("DYG_KAPPA_K", "40"))
    wl = W.mesh_3d(k, inserts=k ** 3 // 5)
    Ho = oracle.OGraph(wl.n, wl.h_src, wl.h_dst, wl.h_w)
    Go = oracle.OGraph(wl.n, wl.g_src, wl.g_dst, wl.g_w)
    _, _, ac, _ = oracle.incremental(Ho, wl.ins_src, wl.ins_dst, wl.ins_w, wl.params, G=Go)
    _, _, rx, _, _, _ = oracle.decremental(Go, Ho, wl.del_src, wl.del_dst, wl.dparams)
    k_final = dyg.kappa(wl.n, *undirected(Go), *undirected(Ho))
    k_init = dyg.kappa(wl.n, wl.g_src, wl.g_dst, wl.g_w, wl.h_src, wl.h_dst, wl.h_w)
    print(f"\nmesh {k}^3: {int(ac.sum())} insertions added, {len(rx)} edges recovered; "
          f"kappa {k_init['kappa']:.2f} -> {k_final['kappa']:.2f}, density "
          f"{k_init['density']:.4f} -> {k_final['density']:.4f}, PCG iterations "
          f"{k_init['pcg_iters']} -> {k_final['pcg_iters']} ({time.time() - t0:.0f} s)")
    # Deleting sparsifier edges raises kappa and the recovered paths only
    # partly bring it back; the reference's own decremental updater does the
    # same (tests/test_reference_agreement.py compares its kappa after
    # deletions with this updater's over several seeds).  At 40^3 the step
    # takes kappa from 130.3 to 461.4 and PCG from 91 to 120 iterations.  The
    # bounds catch a sparsifier that lost its quality.
    assert 1.0 <= k_init["kappa"] and np.isfinite(k_final["kappa"])
    assert k_final["kappa"] <= 10.0 * k_init["kappa"]
    assert k_final["pcg_iters"] <= 3 * k_init["pcg_iters"]
