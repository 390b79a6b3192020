"""Hierarchy reuse across k: one graph partitioned for several k over one
coarsening (gkw_partition_multi_k) gives, for every k, exactly the part
vector and cut that gkw_partition gives for that k alone (integer work:
exact)."""
import numpy as np
import pytest

from graphs import star_graph, two_components, weighted

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["default", "reference"])
def test_multi_k_matches_alone(pkg, gen, mode):
    o = pkg.default_options() if mode == "default" else pkg.default_options(enforce_balance=0)
    graphs = [gen.delaunay(20000, 5), gen.circuit(30000, seed=2, levels=60, hub_max=3000),
              weighted(gen, gen.delaunay(8000, 9), seed=4), two_components(gen, 21), star_graph(gen, 3000),
              gen.grid27(12, 11, 10)]
    ks = [2, 3, 8, 64, 256, 1]
    h = pkg.Handle(0)
    for gi, g in enumerate(graphs):
        parts, cuts = h.partition_multi_k(g.xadj, g.adjncy, g.adjwgt, g.vwgt, ks, o)
        assert parts.shape == (len(ks), g.n)
        for q, k in enumerate(ks):
            p, c, _ = h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, o)
            assert np.array_equal(parts[q], p), (gi, k)
            assert cuts[q] == c, (gi, k)
    h.close()


def test_multi_k_edge_cases(pkg, gen):
    h = pkg.Handle(0)
    g = gen.delaunay(3000, 3)
    parts, cuts = h.partition_multi_k(g.xadj, g.adjncy, g.adjwgt, g.vwgt, [])
    assert parts.shape == (0, g.n) and cuts.shape == (0,)
    e = gen.from_edges(0, np.zeros(0, np.int64), np.zeros(0, np.int64))
    parts, cuts = h.partition_multi_k(e.xadj, e.adjncy, e.adjwgt, e.vwgt, [4, 2])
    assert parts.shape == (2, 0) and list(cuts) == [0, 0]
    with pytest.raises(pkg.GkwError):
        h.partition_multi_k(g.xadj, g.adjncy, g.adjwgt, g.vwgt, [4, 0])
    h.close()
