"""Bit-exact parity of the CUDA path against the oracle, phase by phase and end
to end.  Integer work: every comparison is exact equality."""
import numpy as np
import pytest

from conftest import to_dev
from graphs import small_cases, weighted

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases(gen):
    return small_cases(gen)


def _np(t):
    return t.cpu().numpy()


def test_match(handle, orc, cases):
    for name, g in cases:
        cand = _np(handle.match(to_dev(g)))
        assert np.array_equal(cand, orc.match(g)), name


def test_union_find(handle, orc, cases):
    import torch
    for name, g in cases:
        cand = orc.match(g)
        root, dist, rounds = handle.union_find(torch.from_numpy(cand).cuda())
        r2, d2, l2 = orc.union_find(cand)
        assert np.array_equal(_np(root), r2), name
        assert np.array_equal(_np(dist), d2), name
        assert rounds == l2, name


def test_group_map(handle, orc, cases):
    import torch
    for name, g in cases:
        r, d, _ = orc.union_find(orc.match(g))
        for cap in (6, 2, 40):
            cmap, nc = handle.group_map(torch.from_numpy(r).cuda(), torch.from_numpy(d).cuda(), cap)
            c2, nc2, _ = orc.group_map(r, d, cap)
            assert nc == nc2, (name, cap)
            assert np.array_equal(_np(cmap), c2), (name, cap)


def test_contract(handle, orc, cases):
    import torch
    for name, g in cases:
        r, d, _ = orc.union_find(orc.match(g))
        cmap, nc, _ = orc.group_map(r, d, 6)
        cx, ca, cw, cv = handle.contract(to_dev(g), torch.from_numpy(cmap).cuda(), nc)
        ox, oa, ow = orc.contract(g, cmap, nc)
        assert np.array_equal(_np(cx), ox), name
        assert np.array_equal(_np(ca), oa), name
        assert np.array_equal(_np(cw), ow), name
        assert np.array_equal(_np(cv), orc.coarse_vwgt(g.vwgt, cmap, nc)), name


def _random_state(g, k, seed):
    rng = np.random.default_rng(seed)
    # blocky parts so that most vertices are interior: contiguous id ranges
    part = np.minimum((np.arange(g.n) * k) // max(g.n, 1), k - 1).astype(np.int32)
    flip = rng.random(g.n) < 0.05
    part[flip] = rng.integers(0, k, flip.sum())
    updated = (rng.random(g.n) < 0.7).astype(np.int32)
    boundary = rng.integers(0, 2, g.n).astype(np.int32)
    gain = rng.integers(-3, 4, g.n).astype(np.int32)
    target = rng.integers(0, k, g.n).astype(np.int32)
    return part, updated, boundary, gain, target


def test_update_vertex_info(handle, orc, cases):
    import torch
    for name, g in cases:
        for k in (2, 7, 64):
            part, updated, boundary, gain, target = _random_state(g, k, 5)
            dv = [torch.from_numpy(a.copy()).cuda() for a in (part, updated, boundary, gain, target)]
            handle.update_vertex_info(to_dev(g), k, *dv)
            b2, g2, t2 = orc.update_vertex_info(g, k, part, updated, boundary, gain, target)
            assert np.array_equal(_np(dv[2]), b2), (name, k)
            assert np.array_equal(_np(dv[3]), g2), (name, k)
            assert np.array_equal(_np(dv[4]), t2), (name, k)


def test_refine_level(handle, orc, cases):
    import torch
    for name, g in cases:
        for k, cap in ((4, 1024), (33, 64), (64, 2048)):
            part, _, _, _, _ = _random_state(g, k, 8)
            n = g.n
            updated = np.ones(n, np.int32)
            boundary = np.zeros(n, np.int32)
            gain = np.zeros(n, np.int32)
            target = part.copy()
            pw = orc.part_weights(g, part, k)
            W = int(g.vwgt.astype(np.int64).sum())
            maxw = orc.max_part_weight(W, k)
            ref = orc.refine(g, k, maxw, part, boundary, gain, target, updated, pw, move_cap=cap)
            dv = [torch.from_numpy(a.copy()).cuda() for a in (part, boundary, gain, target, updated)]
            dpw = torch.from_numpy(pw.astype(np.int32)).cuda()
            rounds, moves = handle.refine(to_dev(g), k, maxw, cap, dv[0], dv[1], dv[2], dv[3], dv[4], dpw)
            assert rounds == ref["rounds"] and moves == ref["moves"], (name, k, rounds, ref["rounds"])
            assert np.array_equal(_np(dv[0]), ref["part"]), (name, k)
            assert np.array_equal(_np(dv[1]), ref["boundary"]), (name, k)
            assert np.array_equal(_np(dv[2]), ref["gain"]), (name, k)
            assert np.array_equal(_np(dv[3]), ref["target"]), (name, k)
            assert np.array_equal(_np(dpw).astype(np.int64), ref["pw"]), (name, k)


def test_init_partition(handle, orc, cases):
    for name, g in cases:
        if g.n > 8000:
            continue
        for k in (2, 8, 13, 64):
            for seed in (1, 5):
                p = _np(handle.init_partition(to_dev(g), k, seed=seed))
                assert np.array_equal(p, orc.init_partition(g, k, seed=seed)), (name, k, seed)


def _gggp(orc, gen):
    return lambda x, a, w, vw, kk: orc.init_partition(gen.Csr(x, a, w, vw), kk)


def _exact_boundary(g, part):
    src = np.repeat(np.arange(g.n), np.diff(g.xadj))
    diff = part[src] != part[g.adjncy]
    b = np.zeros(g.n, np.int32)
    np.logical_or.at(b, src[diff], True)
    return b.astype(np.int32)


def test_balance_level(handle, orc, pkg, cases):
    import torch
    rng = np.random.default_rng(12)
    for name, g in cases:
        for k in (4, 32):
            part = np.minimum((np.arange(g.n) * k) // max(g.n, 1), k - 1).astype(np.int32)
            # overload: move a block of part 1 into part 0 and a random 10% into part k-1
            part[(part == 1) & (rng.random(g.n) < 0.5)] = 0
            part[rng.random(g.n) < 0.1] = k - 1
            bnd = _exact_boundary(g, part)
            gain = np.zeros(g.n, np.int32)
            target = part.copy()
            pw = orc.part_weights(g, part, k)
            cap = orc.balance_cap(int(g.vwgt.astype(np.int64).sum()), k)
            assert cap == pkg.balance_cap(int(g.vwgt.astype(np.int64).sum()), k)
            for mc in (1024, 7):
                ref = orc.balance(g, k, cap, part, bnd, gain, target, pw, move_cap=mc)
                dv = [torch.from_numpy(a.copy()).cuda() for a in (part, bnd, gain, target)]
                dpw = torch.from_numpy(pw.astype(np.int32)).cuda()
                rounds, moves = handle.balance(to_dev(g), k, cap, mc, dv[0], dv[1], dv[2], dv[3], dpw)
                assert (rounds, moves) == (ref["rounds"], ref["moves"]), (name, k, mc)
                assert np.array_equal(_np(dv[0]), ref["part"]), (name, k, mc)
                assert np.array_equal(_np(dv[1]), ref["boundary"]), (name, k, mc)
                assert np.array_equal(_np(dpw).astype(np.int64), ref["pw"]), (name, k, mc)


def test_partition_device_init_matches_oracle(handle, orc, gen, cases):
    """Default mode: device initial partition, balance rounds, strict cap."""
    for name, g in cases:
        for k in (2, 8, 64):
            part, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
            ref, info = orc.partition(g, k, init=_gggp(orc, gen), enforce_balance=True)
            assert np.array_equal(part, ref), (name, k)
            assert cut == info["cut"] == orc.cut(g, part), (name, k)
            assert st["level_n"] == info["level_n"] and st["level_m"] == info["level_m"], (name, k)
            assert st["uf_rounds"] == info["uf_launches"], (name, k)
            assert st["refine_rounds"] == info["refine_rounds"], (name, k)
            assert st["refine_moves"] == info["refine_moves"], (name, k)
            assert st["balance_rounds"] == info["balance_rounds"], (name, k)
            assert st["balance_moves"] == info["balance_moves"], (name, k)
            assert st["init_cut"] == info["init_cut"], (name, k)


def test_partition_reference_mode_matches_oracle(handle, orc, gen, pkg, cases):
    """The reference's own rules (MAX_PARTITION_WGT with +1, no balance rounds)."""
    for name, g in cases:
        for k in (8, 64):
            o = pkg.default_options(enforce_balance=0)
            part, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, o)
            ref, info = orc.partition(g, k, init=_gggp(orc, gen))
            assert np.array_equal(part, ref), (name, k)
            assert cut == info["cut"], (name, k)
            assert st["refine_rounds"] == info["refine_rounds"], (name, k)


@pytest.mark.skipif("not __import__('oracle').has_metis()")
def test_partition_metis_recursive_init_matches_oracle(handle, orc, gen, cases, pkg):
    """METIS's recursive bisection (metis.h:185) on the coarsest graph through
    the initial-partition callback, in both modes."""
    def init(x, a, w, vw, kk):
        return orc.metis_recursive(gen.Csr(x, a, w, vw), kk)[0]
    # Delaunay and grid cases: on the skewed circuit case in reference mode the
    # coarsest graph has vertices heavier than a bisection target, and METIS's
    # recursive bisection reports "Cannot bisect a graph with 0 vertices" and
    # leaves the part vector unspecified
    for name, g in cases[:3]:
        if g.m and g.adjwgt.min() <= 0:
            continue   # METIS requires positive edge weights
        for k in (8, 64):
            for enforce in (0, 1):
                o = pkg.default_options(enforce_balance=enforce)
                part, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, o, init=init)
                ref, info = orc.partition(g, k, init=init, enforce_balance=bool(enforce))
                assert np.array_equal(part, ref), (name, k, enforce)
                assert cut == info["cut"], (name, k, enforce)


@pytest.mark.skipif("not __import__('oracle').has_metis()")
def test_partition_metis_init_matches_oracle(handle, orc, gen, cases, pkg):
    """The reference's own configuration: METIS on the coarsest graph."""
    def metis_init(x, a, w, vw, kk):
        return orc.metis_kway(gen.Csr(x, a, w, vw), kk)[0]
    for name, g in cases:
        if g.m and g.adjwgt.min() <= 0:
            continue   # METIS requires positive edge weights (it crashes on zero weights)
        for k in (8, 64):
            o = pkg.default_options(enforce_balance=0)
            part, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, o, init=metis_init)
            ref, info = orc.partition(g, k)
            assert np.array_equal(part, ref), (name, k)
            assert cut == info["cut"], (name, k)


@pytest.mark.skipif("not __import__('os').path.exists(__import__('oracle').N11_PATH)")
def test_n11_fixture(handle, orc, gen, pkg):
    x, a, w, vw = pkg.read_metis(orc.N11_PATH)
    g = gen.Csr(x, a, w, vw)
    for k in (8, 64):
        part, cut, st = handle.partition(x, a, w, vw, k)
        ref, info = orc.partition(g, k, init=_gggp(orc, gen), enforce_balance=True)
        assert np.array_equal(part, ref)
        assert cut == info["cut"]
        assert orc.part_weights(g, part, k).max() * k <= 1.03 * g.n


def test_device_resident_partition_is_deterministic(handle, orc, gen):
    import torch
    g = weighted(gen, gen.delaunay(1 << 17, 3), seed=2)
    dg = to_dev(g)
    out = []
    for _ in range(2):
        p = torch.empty(g.n, dtype=torch.int32, device="cuda:0")
        cut, st = handle.partition_device(*dg, 64, p)
        out.append((_np(p), cut))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]
    assert out[0][1] == orc.cut(g, out[0][0])
    pw = orc.part_weights(g, out[0][0], 64)
    assert pw.sum() == g.vwgt.sum()
    assert pw.max() * 64 <= 1.03 * g.vwgt.sum()
    ref, info = orc.partition(g, 64, init=_gggp(orc, gen), enforce_balance=True)
    assert np.array_equal(out[0][0], ref)


def test_invalid_input_is_rejected(handle, pkg, gen):
    g = gen.delaunay(500, 1)
    bad = g.adjncy.copy()
    bad[3] = g.n + 5
    with pytest.raises(pkg.GkwError) as e:
        handle.partition(g.xadj, bad, g.adjwgt, g.vwgt, 4)
    assert e.value.status == pkg.GKW_E_INVALID
    selfloop = g.adjncy.copy()
    selfloop[g.xadj[10]] = 10
    with pytest.raises(pkg.GkwError):
        handle.partition(g.xadj, selfloop, g.adjwgt, g.vwgt, 4)
    with pytest.raises(pkg.GkwError):
        handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, 0)
    xb = g.xadj.copy()
    xb[5] = xb[6] + 1
    with pytest.raises(pkg.GkwError):
        handle.partition(xb, g.adjncy, g.adjwgt, g.vwgt, 4)
    # the handle is still usable afterwards
    part, cut, _ = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, 4)
    assert part.max() < 4


def test_empty_and_tiny_graphs(handle, pkg, gen, orc):
    # no vertices
    part, cut, st = handle.partition(np.zeros(1, np.int32), np.zeros(0, np.int32), None, None, 4)
    assert part.shape == (0,) and cut == 0
    # no edges
    n = 50
    part, cut, st = handle.partition(np.zeros(n + 1, np.int32), np.zeros(0, np.int32), None, None, 4)
    assert cut == 0 and part.min() >= 0 and part.max() < 4
    # k = 1
    g = gen.delaunay(300, 2)
    part, cut, _ = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, 1)
    assert cut == 0 and np.all(part == 0)


def test_autotune_keeps_results(pkg, gen):
    """The autotuner picks launch shapes by timing; results never depend on
    them: the same part vector and cut before tuning, after it, and under
    hand-set extreme shapes."""
    import torch
    from conftest import to_dev
    h = pkg.Handle(0)
    g = gen.circuit(60000, seed=3, levels=60, hub_max=2000)
    dg = to_dev(g)
    outs = []
    for shapes in (None, "tune", dict(match_lanes=(32, 2, 4, 2), level_verts_per_cta=64, level_min_ctas=1),
                   dict(match_lanes=(8, 32, 16, 4), level_verts_per_cta=4096, level_min_ctas=64)):
        if shapes == "tune":
            t = h.autotune(*dg, 32)
            assert all(x in (2, 4, 8, 16, 32) for x in t["match_lanes"])
        elif shapes is not None:
            h.set_tuning(**shapes)
            assert h.tuning()["level_verts_per_cta"] == shapes["level_verts_per_cta"]
        p = torch.empty(g.n, dtype=torch.int32, device="cuda:0")
        cut, _ = h.partition_device(*dg, 32, p)
        outs.append((p.cpu().numpy(), cut))
    for part, cut in outs[1:]:
        assert np.array_equal(part, outs[0][0]) and cut == outs[0][1]
    with pytest.raises(pkg.GkwError):
        h.set_tuning(match_lanes=(3, 8, 16, 32))
    h.close()


def test_graph_replay_matches_plain_launches(pkg, gen, orc):
    """Repeated partitions replay each coarsening level's and the initial
    partition's launch sequence from a captured CUDA graph (second sight:
    capture; later: replay).  Every result equals a handle that never
    captures (GKW_GRAPHS=0) and the oracle, also after the input's contents
    change in place (same buffers and sizes, other weights)."""
    import os
    import torch
    from conftest import to_dev
    g = weighted(gen, gen.delaunay(60000, 17), seed=3)
    os.environ["GKW_GRAPHS"] = "0"
    try:
        plain = pkg.Handle(0)
    finally:
        del os.environ["GKW_GRAPHS"]
    h = pkg.Handle(0)
    dg = to_dev(g)
    k = 24
    for step in range(6):
        if step == 3:   # new edge weights in the same device buffers
            src = np.repeat(np.arange(g.n), np.diff(g.xadj)).astype(np.int64)
            lo, hi = np.minimum(src, g.adjncy), np.maximum(src, g.adjncy)
            w = 1 + (lo * 1000003 + hi * 7919) % 8   # symmetric by construction
            dg[2].copy_(torch.from_numpy(w.astype(np.int32)))
        p1 = torch.empty(g.n, dtype=torch.int32, device="cuda:0")
        p2 = torch.empty(g.n, dtype=torch.int32, device="cuda:0")
        c1, s1 = h.partition_device(*dg, k, p1)
        c2, s2 = plain.partition_device(*dg, k, p2)
        assert np.array_equal(p1.cpu().numpy(), p2.cpu().numpy()) and c1 == c2, step
        assert s1["level_n"] == s2["level_n"] and s1["refine_rounds"] == s2["refine_rounds"], step
        if step in (2, 5):
            cur = gen.Csr(g.xadj, g.adjncy, dg[2].cpu().numpy(), g.vwgt)
            ref, info = orc.partition(cur, k, init=lambda x, a, ww, vw, kk: orc.init_partition(gen.Csr(x, a, ww, vw), kk),
                                      enforce_balance=True)
            assert np.array_equal(p1.cpu().numpy(), ref) and c1 == info["cut"], step
    h.close()
    plain.close()


def test_fused_coarsening_matches_per_phase(pkg, gen, cases):
    """A coarsening level runs either as one fused launch (grid barriers
    between the phases) or as the per-phase kernels; every level, the part
    vector and the cut are the same for every launch shape of the fused one:
    one CTA, a thread-block cluster, a wide cooperative grid."""
    from graphs import weighted
    graphs = list(cases) + [("circuit_60k_hubs", gen.circuit(60000, seed=3, levels=60, hub_max=2000)),
                            ("delaunay_60k_w", weighted(gen, gen.delaunay(60000, 17), seed=3))]
    per_phase = pkg.Handle(0)
    per_phase.set_tuning(coarsen_fused_max_n=0)
    fused = pkg.Handle(0)
    for name, g in graphs:
        for k in (8, 64):
            p0, c0, s0 = per_phase.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
            for vpc in (1 << 30, 4096, 64):   # one CTA; few CTAs (a cluster); wide
                fused.set_tuning(coarsen_fused_max_n=1 << 30, coarsen_verts_per_cta=vpc)
                p1, c1, s1 = fused.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
                assert np.array_equal(p1, p0) and c1 == c0, (name, k, vpc)
                assert s1["level_n"] == s0["level_n"] and s1["level_m"] == s0["level_m"], (name, k, vpc)
                assert s1["refine_rounds"] == s0["refine_rounds"], (name, k, vpc)
    per_phase.close()
    fused.close()
