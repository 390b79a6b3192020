"""Partition quality of the default mode (north star D4), on the CPU through
the oracle, whose default mode the GPU reproduces bit for bit
(test_gpu_parity.py, test_gpu_quality.py):

* balance: every part weight <= (1 + eps) W / k;
* cut: over 10 seeds, the mean ratio to the cut of the reference's own
  configuration (reference mode, METIS on the coarsest graph) is <= 1.02.

The circuit-like graph whose giant component the reference's coarsening
collapses into one vertex (METIS then cannot split the coarsest graph) must
still come out balanced."""
import numpy as np
import pytest

SEEDS = range(1, 11)


def gggp(orc, gen):
    return lambda x, a, w, vw, k: orc.init_partition(gen.Csr(x, a, w, vw), k)


@pytest.mark.parametrize("n,k", [(1 << 14, 8), (1 << 15, 64)])
def test_default_mode_cut_within_2pct_of_reference(orc, gen, n, k):
    if not orc.has_metis():
        pytest.skip("the reference's METIS library is not available")
    ratios = []
    for seed in SEEDS:
        g = gen.delaunay(n, seed)
        _, ref = orc.partition(g, k)
        part, dm = orc.partition(g, k, init=gggp(orc, gen), enforce_balance=True)
        W = int(g.vwgt.sum())
        pw = np.bincount(part, weights=g.vwgt, minlength=k)
        assert pw.max() <= 1.03 * W / k
        assert dm["cut"] == orc.cut(g, part)
        ratios.append(dm["cut"] / ref["cut"])
    assert np.mean(ratios) <= 1.02, ratios


def test_collapsed_component_is_balanced(orc, gen):
    g = gen.circuit(60000, seed=4, levels=60, hub_max=2000)
    k = 8
    part, dm = orc.partition(g, k, init=gggp(orc, gen), enforce_balance=True)
    W = int(g.vwgt.sum())
    assert np.bincount(part, weights=g.vwgt, minlength=k).max() <= 1.03 * W / k
    # without the coarse-vertex stop the giant component becomes one vertex
    _, bad = orc.partition(g, k, init=gggp(orc, gen), enforce_balance=True, coarse_vertex_frac=0)
    assert bad["max_part_weight"] > 2 * W / k
