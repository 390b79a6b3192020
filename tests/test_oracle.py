"""The oracle: pinned against the reference's bundled METIS known answers and
hand-checked small cases of every reference rule it restates (CPU only)."""
import os

import numpy as np
import pytest

import oracle
from graphs import path_graph, star_graph, weighted


def csr(gen, n, edges, w=None, vw=None):
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    return gen.from_edges(n, e[:, 0], e[:, 1], w, vw)


# ---------------------------------------------------------------------------
# pins: the reference's bundled METIS on the reference's own fixture
# ---------------------------------------------------------------------------
needs_n11 = pytest.mark.skipif(not (os.path.exists(oracle.N11_PATH) and oracle.has_metis()),
                               reason="reference fixture or METIS not available")


@needs_n11
@pytest.mark.parametrize("k,cut,maxpw", [(8, 349, 261), (64, 2083, 33)])
def test_metis_known_answers_n11(k, cut, maxpw):
    g = oracle.read_metis_graph(oracle.N11_PATH)
    assert (g.n, g.m) == (2048, 12254)
    part, obj = oracle.metis_kway(g, k)
    assert obj == cut == oracle.cut(g, part)
    assert oracle.part_weights(g, part, k).max() == maxpw


@needs_n11
@pytest.mark.parametrize("k,cut,maxpw", [(8, 355, 257), (64, 1254, 33)])
def test_metis_recursive_known_answers_n11(k, cut, maxpw):
    # METIS_PartGraphRecursive, the recursive-bisection alternative init
    # (metis.h:185); answers measured here with the bundled METIS 5.2.1
    g = oracle.read_metis_graph(oracle.N11_PATH)
    part, obj = oracle.metis_recursive(g, k)
    assert obj == cut == oracle.cut(g, part)
    assert oracle.part_weights(g, part, k).max() == maxpw
    assert len(np.unique(part)) == k


@needs_n11
def test_partition_with_recursive_metis_init(gen):
    g = oracle.read_metis_graph(oracle.N11_PATH)

    def init(x, a, w, vw, kk):
        return oracle.metis_recursive(gen.Csr(x, a, w, vw), kk)[0]
    for k in (8, 64):
        part, info = oracle.partition(g, k, init=init)
        assert info["cut"] == oracle.cut(g, part)
        assert part.min() >= 0 and part.max() < k
        bal, binfo = oracle.partition(g, k, init=init, enforce_balance=True)
        assert oracle.part_weights(g, bal, k).max() <= oracle.balance_cap(int(g.vwgt.sum()), k)


# ---------------------------------------------------------------------------
# A3 heavy-edge candidate (coarsen.hpp:39-78)
# ---------------------------------------------------------------------------
def test_match_rules(gen):
    # 0 -- 1,2,3 with weights 2,2,2; deg(1)=3, deg(2)=1... build explicit graph
    edges = [(0, 1), (0, 2), (0, 3), (1, 4), (1, 5), (3, 6), (7, 8)]
    w = [2, 2, 2, 1, 1, 1, 0]
    g = csr(gen, 10, edges, w)
    cand = oracle.match(g)
    # vertex 0: neighbours 1 (deg 3), 2 (deg 1), 3 (deg 2), all weight 2 -> min degree = 2
    assert cand[0] == 2
    # vertex 1: neighbours 0 (w2) beats 4,5 (w1)
    assert cand[1] == 0
    # vertex 7 and 8: only a zero-weight edge -> themselves; 9 isolated -> itself
    assert cand[7] == 7 and cand[8] == 8 and cand[9] == 9
    # ties on weight and degree: the first in adjacency order
    g2 = csr(gen, 4, [(0, 1), (0, 2), (0, 3)])
    assert oracle.match(g2)[0] == 1


# ---------------------------------------------------------------------------
# A5 union-find, Jacobi schedule (coarsen.hpp:80-118, 461-469)
# ---------------------------------------------------------------------------
def test_union_find_path_distances(gen):
    n = 7
    g = path_graph(gen, n)
    cand = oracle.match(g)
    # interior vertices point to the smaller-id neighbour (equal degree, first in
    # the sorted row) except next to an end, where the degree-1 end wins
    assert list(cand) == [1, 0, 1, 2, 3, 6, 5]
    root, dist, launches = oracle.union_find(cand)
    assert list(root) == [4, 4, 4, 4, 4, 6, 6]
    assert list(dist) == [4, 3, 2, 1, 0, 1, 0]     # hop distance from the root
    assert launches == 5                              # 4 raising rounds + 1 quiet round


def test_union_find_components(gen):
    cand = np.array([1, 0, 3, 2, 2, 5], dtype=np.int32)   # {0,1}, {2,3,4}, {5}
    root, dist, launches = oracle.union_find(cand)
    assert list(root) == [1, 1, 4, 4, 4, 5]
    assert list(dist) == [1, 0, 1, 2, 0, 0]
    assert launches == 3


# ---------------------------------------------------------------------------
# A6/A7 group order and cap (coarsen.hpp:408-421, 120-155)
# ---------------------------------------------------------------------------
def test_group_map_chunks():
    root = np.array([9] * 10, dtype=np.int32)
    dist = np.array([3, 2, 2, 1, 1, 1, 2, 3, 1, 0], dtype=np.int32)
    cmap, nc, order = oracle.group_map(root, dist, 6)
    # sorted (dist, id): 9 | 3 4 5 8 | 1 2 6 | 0 7
    assert list(order) == [9, 3, 4, 5, 8, 1, 2, 6, 0, 7]
    assert nc == 2
    assert [cmap[v] for v in order] == [0] * 6 + [1] * 4
    # groups are numbered by root id; small groups are one chunk
    root2 = np.array([2, 2, 2, 5, 5, 5], dtype=np.int32)
    cmap2, nc2, _ = oracle.group_map(root2, np.array([1, 1, 0, 1, 2, 0], np.int32), 6)
    assert nc2 == 2 and list(cmap2) == [0, 0, 0, 1, 1, 1]


# ---------------------------------------------------------------------------
# A9 contraction (coarsen.hpp:302-349)
# ---------------------------------------------------------------------------
def test_contract_small(gen):
    # square 0-1-2-3-0 plus diagonal 0-2, weights 1..5; coarse: {0,1}->0, {2,3}->1
    g = csr(gen, 4, [(0, 1), (1, 2), (2, 3), (3, 0), (0, 2)], [1, 2, 3, 4, 5])
    cmap = np.array([0, 0, 1, 1], np.int32)
    cx, ca, cw = oracle.contract(g, cmap, 2)
    assert list(cx) == [0, 1, 2]
    assert list(ca) == [1, 0]
    assert list(cw) == [2 + 4 + 5, 2 + 4 + 5]   # 1-2, 3-0, 0-2 cross; 0-1 and 2-3 internal
    assert list(oracle.coarse_vwgt(np.array([1, 2, 3, 4], np.int32), cmap, 2)) == [3, 7]


def test_contract_properties(gen):
    g = weighted(gen, gen.delaunay(3000, 2), 5)
    r, d, _ = oracle.union_find(oracle.match(g))
    cmap, nc, _ = oracle.group_map(r, d, 6)
    cx, ca, cw = oracle.contract(g, cmap, nc)
    cg = gen.Csr(cx, ca, cw, oracle.coarse_vwgt(g.vwgt, cmap, nc))
    gen.check_csr(cg)   # symmetric, sorted-unique rows, no self loops
    for c in range(nc):
        row = ca[cx[c]:cx[c + 1]]
        assert np.all(np.diff(row) > 0)
    src = np.repeat(np.arange(g.n), np.diff(g.xadj))
    cross = cmap[src] != cmap[g.adjncy]
    assert cw.sum() == g.adjwgt[cross].sum()
    assert cg.vwgt.sum() == g.vwgt.sum()


# ---------------------------------------------------------------------------
# A13 gains with the unsigned comparison (uncoarsen.hpp:175-237)
# ---------------------------------------------------------------------------
def test_unsigned_gain_quirk(gen):
    # v=0 in part 0: own-part neighbours 1,2,3 (w 1 each -> id = 3),
    # neighbour 4 in part 1 (w 5 -> gain +2), neighbour 5 in part 2 (w 1 -> gain -2)
    g = csr(gen, 6, [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5)], [1, 1, 1, 5, 1])
    part = np.array([0, 0, 0, 0, 1, 2], np.int32)
    z = np.zeros(6, np.int32)
    upd = np.array([1, 0, 0, 0, 0, 0], np.int32)
    b, gain, t = oracle.update_vertex_info(g, 3, part, upd, z, z, z)
    # (unsigned)(-2) > 2: the reference keeps the negative gain and part 2
    assert b[0] == 1 and gain[0] == -2 and t[0] == 2
    # with vertex 5 in the own part (id = 4) only the positive gain 5 - 4 remains
    part2 = np.array([0, 0, 0, 0, 1, 0], np.int32)
    b, gain, t = oracle.update_vertex_info(g, 3, part2, upd, z, z, z)
    assert gain[0] == 1 and t[0] == 1
    # all gains zero -> gain 0, target = own part
    g3 = csr(gen, 3, [(0, 1), (0, 2)])
    b, gain, t = oracle.update_vertex_info(g3, 2, np.array([0, 0, 1], np.int32), np.array([1, 0, 0], np.int32),
                                           np.zeros(3, np.int32), np.zeros(3, np.int32), np.zeros(3, np.int32))
    assert b[0] == 1 and gain[0] == 0 and t[0] == 0


# ---------------------------------------------------------------------------
# A14-A19 refinement rounds (uncoarsen.hpp:427-506)
# ---------------------------------------------------------------------------
def test_refine_independent_set_and_cap(gen):
    # path 0..5 split [0,0,1,1,1,0]: vertex 5 wants part 1 (gain 1), vertex 2 wants 0
    g = path_graph(gen, 6)
    part = np.array([0, 0, 1, 1, 1, 0], np.int32)
    n = g.n
    pw = oracle.part_weights(g, part, 2)
    maxw = oracle.max_part_weight(6, 2)   # 3*1.03+1 = 4.09
    res = oracle.refine(g, 2, maxw, part, np.zeros(n, np.int32), np.zeros(n, np.int32), part.copy(),
                        np.ones(n, np.int32), pw, move_cap=1)
    assert res["moves"] >= 1
    assert oracle.cut(g, res["part"]) == oracle.cut(g, part) - res["gain_sum"]
    assert np.array_equal(res["pw"], oracle.part_weights(g, res["part"], 2))
    assert res["pw"].max() <= maxw


def test_refine_invariants_random(gen):
    g = weighted(gen, gen.delaunay(4000, 6), 1)
    rng = np.random.default_rng(3)
    k = 8
    part = np.minimum(np.arange(g.n) * k // g.n, k - 1).astype(np.int32)
    flip = rng.random(g.n) < 0.1
    part[flip] = rng.integers(0, k, flip.sum())
    pw = oracle.part_weights(g, part, k)
    maxw = oracle.max_part_weight(int(g.vwgt.sum()), k)
    n = g.n
    res = oracle.refine(g, k, maxw, part, np.zeros(n, np.int32), np.zeros(n, np.int32), part.copy(),
                        np.ones(n, np.int32), pw, move_cap=64)
    assert oracle.cut(g, res["part"]) == oracle.cut(g, part) - res["gain_sum"]
    assert res["gain_sum"] > 0
    assert np.array_equal(res["pw"], oracle.part_weights(g, res["part"], k))
    # no destination part was pushed above MAXW by refinement
    over = res["pw"] > maxw
    assert np.all(res["pw"][over] <= pw[over])


def test_max_part_weight_formula():
    # graph_partitioner.hpp:230 evaluated as float(double(float(W)/float(k)) * 1.03 + 1)
    for W, k in [(2048, 8), (1048576, 64), (12345, 7), (4000000, 256)]:
        q = np.float32(np.float32(W) / np.float32(k))
        assert oracle.max_part_weight(W, k) == np.float32(float(q) * (1.0 + 0.03) + 1.0)


def test_oracle_partition_properties(gen):
    g = weighted(gen, gen.delaunay(6000, 4), 2)
    for k in (4, 16):
        init = lambda x, a, w, vw, kk: oracle.init_partition(gen.Csr(x, a, w, vw), kk)
        part, info = oracle.partition(g, k, init=init)
        assert part.min() >= 0 and part.max() < k
        assert info["cut"] == oracle.cut(g, part)
        assert info["level_n"][0] == g.n and all(a > b for a, b in zip(info["level_n"], info["level_n"][1:]))
        assert info["level_n"][-1] <= 20 * k or len(info["level_n"]) >= 1
        part2, info2 = oracle.partition(g, k, init=init)
        assert np.array_equal(part, part2)


def test_no_coarsening_keeps_initial_partition(gen):
    # n <= 20k: the initial partition is the answer (no refinement at the coarsest level)
    g = gen.delaunay(100, 3)
    init = lambda x, a, w, vw, kk: oracle.init_partition(gen.Csr(x, a, w, vw), kk)
    part, info = oracle.partition(g, 8, init=init)
    assert info["n_levels"] == 1
    assert np.array_equal(part, oracle.init_partition(g, 8))


def test_star_and_path_hierarchies(gen):
    for g in (star_graph(gen, 3000), path_graph(gen, 900)):
        init = lambda x, a, w, vw, kk: oracle.init_partition(gen.Csr(x, a, w, vw), kk)
        part, info = oracle.partition(g, 4, init=init)
        assert info["cut"] == oracle.cut(g, part)


# ---------------------------------------------------------------------------
# hierarchy reuse across k: the levels do not depend on k except where the
# coarsening stops, so the hierarchies of two k share their common prefix
# (the premise of gkw_partition_multi_k)
# ---------------------------------------------------------------------------
def test_hierarchies_of_different_k_share_a_prefix(gen):
    from graphs import weighted
    init = lambda x, a, w, vw, kk: oracle.init_partition(gen.Csr(x, a, w, vw), kk)
    for g in (gen.delaunay(20000, 5), weighted(gen, gen.delaunay(8000, 9), seed=4),
              gen.circuit(30000, seed=2, levels=60, hub_max=3000)):
        for enforce in (False, True):
            levels = []
            for k in (2, 8, 64, 256):
                _, info = oracle.partition(g, k, init=init, enforce_balance=enforce)
                levels.append((info["level_n"], info["level_m"]))
            for (n1, m1) in levels:
                for (n2, m2) in levels:
                    L = min(len(n1), len(n2))
                    assert n1[:L] == n2[:L] and m1[:L] == m2[:L]
            # a larger k never coarsens deeper
            depths = [len(n) for n, _ in levels]
            assert depths == sorted(depths, reverse=True)
