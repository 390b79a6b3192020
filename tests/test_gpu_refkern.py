"""The oracle pinned against the reference's own kernels.

oracle/_ref/librefkern.so runs kernels copied unchanged out of the reference's
gkway/coarsen.hpp and gkway/uncoarsen.hpp (built by oracle/Makefile from a
reference tree; oracle/refkern.cu lists which ones and what runs on the host
instead).  Every rule the oracle restates is compared with the reference's
kernel on the same input, bit for bit, and so is the reference's whole
partitioner run on its kernels against the oracle in reference mode with METIS
on the coarsest graph.  k stays at most 64: the reference's update_vertex_info
keeps 128 * k counters in a 12000-word shared array (k <= 93)."""
import numpy as np
import pytest

from graphs import small_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rk():
    from oracle import refkern
    if not refkern.available():
        pytest.fail("oracle/_ref/librefkern.so is missing: build the oracle with REF=<reference root>")
    return refkern


@pytest.fixture(scope="module")
def cases(gen, orc):
    out = list(small_cases(gen))
    n11 = orc.read_metis_graph(orc.N11_PATH)
    out.append(("delaunay_n11", n11))
    return out


def test_matching_with_score(rk, orc, cases):
    for name, g in cases:
        assert np.array_equal(rk.match(g), orc.match(g)), name


def test_hec_union_find_labels(rk, orc, cases):
    """Labels (the component's largest id) are schedule-independent and equal;
    the reference's iteration stamps depend on its schedule and never exceed
    the canonical (Jacobi) ones."""
    for name, g in cases:
        cand = orc.match(g)
        keys, launches = rk.union_find(cand)
        root, dist, orc_launches = orc.union_find(cand)
        assert np.array_equal((keys >> np.uint64(32)).astype(np.int64) - 1, root), name
        assert np.all((keys & np.uint64(0xffffffff)).astype(np.int64) <= dist), name
        assert launches <= orc_launches, name


def test_group_kernels(rk, orc, cases):
    for name, g in cases:
        root, dist, _ = orc.union_find(orc.match(g))
        for cap in (6, 2, 40):
            cmap, nc = rk.group_map(root, dist, cap)
            c2, nc2, _ = orc.group_map(root, dist, cap)
            assert nc == nc2, (name, cap)
            assert np.array_equal(cmap, c2), (name, cap)


def test_coarse_vwgt_and_contraction(rk, orc, cases):
    for name, g in cases:
        root, dist, _ = orc.union_find(orc.match(g))
        cmap, nc, _ = orc.group_map(root, dist, 6)
        assert np.array_equal(rk.coarse_vwgt(g.vwgt, cmap, nc), orc.coarse_vwgt(g.vwgt, cmap, nc)), name
        got, want = rk.contract(g, cmap, nc), orc.contract(g, cmap, nc)
        for a, b in zip(got, want):
            assert np.array_equal(a, b), name


def test_expand_partition(rk, orc, cases):
    """expand_partition against the projection rule the oracle applies inline
    (part and boundary from the coarse vertex, gain 0, target = part,
    boundary vertices flagged)."""
    rng = np.random.default_rng(3)
    for name, g in cases:
        root, dist, _ = orc.union_find(orc.match(g))
        cmap, nc, _ = orc.group_map(root, dist, 6)
        part_c = rng.integers(0, 8, nc).astype(np.int32)
        bnd_c = rng.integers(0, 2, nc).astype(np.int32)
        part, bnd, gain, target, upd = rk.expand(cmap, part_c, bnd_c)
        assert np.array_equal(part, part_c[cmap]) and np.array_equal(bnd, bnd_c[cmap]), name
        assert not gain.any() and np.array_equal(target, part) and np.array_equal(upd, bnd), name


def _state(g, k, seed):
    rng = np.random.default_rng(seed)
    part = np.minimum((np.arange(g.n) * k) // max(g.n, 1), k - 1).astype(np.int32)
    flip = rng.random(g.n) < 0.05
    part[flip] = rng.integers(0, k, flip.sum())
    return part, rng


def test_update_vertex_info(rk, orc, cases):
    for name, g in cases:
        for k in (2, 7, 64):
            part, rng = _state(g, k, 5)
            updated = (rng.random(g.n) < 0.7).astype(np.int32)
            boundary = rng.integers(0, 2, g.n).astype(np.int32)
            gain = rng.integers(-3, 4, g.n).astype(np.int32)
            target = rng.integers(0, k, g.n).astype(np.int32)
            got = rk.update_vertex_info(g, k, part, updated, boundary, gain, target)
            want = orc.update_vertex_info(g, k, part, updated, boundary, gain, target)
            for a, b in zip(got, want):
                assert np.array_equal(a, b), (name, k)


def test_refinement_level(rk, orc, cases):
    """One level's refinement loop: the reference's find_mv_wgt_sequence,
    find_balance_sequence, apply_sequence_move and update_vertex_info kernels
    against the oracle's rounds (move caps 1024 and 64; tight and loose MAXW).
    Graphs above 10k vertices run only the loose k = 4 case: at k = 33 and 64
    they take thousands of rounds, each several launches and a host read on
    the reference's kernels (minutes of GPU time for no new rule)."""
    for name, g in cases:
        for k, cap, slack in ((4, 1024, 0.03), (33, 64, 0.03), (64, 1024, 0.0)):
            if g.n > 10000 and k > 4:
                continue
            part, _ = _state(g, k, 8)
            n = g.n
            pw = orc.part_weights(g, part, k)
            W = int(g.vwgt.astype(np.int64).sum())
            maxw = orc.max_part_weight(W, k, slack)
            args = (g, k, maxw, part, np.zeros(n, np.int32), np.zeros(n, np.int32), part.copy(),
                    np.ones(n, np.int32), pw)
            got = rk.refine(*args, move_cap=cap)
            want = orc.refine(*args, move_cap=cap)
            for key in ("rounds", "moves", "gain_sum"):
                assert got[key] == want[key], (name, k, key, got[key], want[key])
            for key in ("part", "boundary", "gain", "target", "pw"):
                assert np.array_equal(got[key], want[key]), (name, k, key)


def test_calculate_cutsize(rk, orc, cases):
    for name, g in cases:
        part, _ = _state(g, 16, 2)
        assert rk.cutsize(g, part) == orc.cut(g, part), name


@pytest.mark.parametrize("which,k", [("delaunay_n11", 8), ("delaunay_n11", 64), ("delaunay_20k", 64),
                                     ("grid27_12x11x10", 8), ("delaunay_w", 16), ("two_components", 32)])
def test_reference_partitioner_on_its_kernels(rk, orc, cases, which, k):
    """The reference's whole partitioner run on its kernels (METIS on the
    coarsest graph, the canonical union-find schedule) equals the oracle in
    reference mode: every level size, every level's refinement rounds, the
    part vector and the cut."""
    g = dict(cases)[which]
    metis = lambda x, a, w, vw, kk: orc.metis_kway(_csr(x, a, w, vw), kk)[0]
    uf = lambda cand: orc.union_find(cand)[:2]
    part, info = rk.partition(g, k, metis, uf)
    ref, oinfo = orc.partition(g, k, enforce_balance=False)
    assert info["level_n"] == oinfo["level_n"] and info["level_m"] == oinfo["level_m"]
    assert info["refine_rounds"] == oinfo["refine_rounds"]
    assert np.array_equal(part, ref)
    assert info["cut"] == oinfo["cut"] == orc.cut(g, part)


def _csr(x, a, w, vw):
    import __graft_entry__ as ge
    return ge.load_generators().Csr(x, a, w, vw)
