"""GPU against the oracle at the full sizes of the configurations the
benchmark is quoted on (seeded synthetic stand-ins, see generators.py):

* 2D Delaunay of 2^20 points, k = 64 (the headline);
* 27-point grid 100 x 100 x 96, k = 64;
* road-like graph of 12M points, k = 256;
* circuit-like graph of 4M vertices, k = 256.

Each is compared bit for bit -- part vector, cut, every level's size and
every level's refinement and balance rounds -- in the default mode (device
initial partition; the oracle runs its restatement) and in the reference's
configuration (reference mode, METIS on the coarsest graph), except the
circuit-like graph in reference mode, whose coarsest graph METIS cannot
partition (it stops with "Cannot bisect a graph with 0 vertices", as the
reference would).  The 2% quality bar is checked at the headline size over
ten seeds, and the device initial partition is compared with METIS on the
identical coarsest graph.  The graphs are generated in parallel by spawned
processes."""
import concurrent.futures as cf
import multiprocessing as mp

import numpy as np
import pytest

from graphs import build_graph

pytestmark = pytest.mark.gpu

SPECS = {
    "delaunay_2e20": (("delaunay", 1 << 20, 1), 64),
    "grid27_100x100x96": (("grid27", 100, 100, 96), 64),
    "circuit_4M": (("circuit", 4_000_000, 1), 256),
    "road_12M": (("road", 12_000_000, 1), 256),
}
SEEDS = list(range(2, 11))   # seed 1 is the headline graph above


@pytest.fixture(scope="module")
def pending():
    ex = cf.ProcessPoolExecutor(max_workers=6, mp_context=mp.get_context("spawn"))
    futs = {name: ex.submit(build_graph, spec) for name, (spec, _) in SPECS.items()}
    futs.update({f"delaunay_2e20_s{s}": ex.submit(build_graph, ("delaunay", 1 << 20, s)) for s in SEEDS})
    yield futs
    ex.shutdown(wait=False, cancel_futures=True)


def _metis(orc, gen):
    return lambda x, a, w, vw, kk: orc.metis_kway(gen.Csr(x, a, w, vw), kk)[0]


def _gggp(orc, gen):
    return lambda x, a, w, vw, kk: orc.init_partition(gen.Csr(x, a, w, vw), kk)


def _same_run(st, part, cut, ref, info, what):
    nl = info["n_levels"]
    assert st["n_levels"] == nl, what
    assert list(st["level_n"][:nl]) == info["level_n"], what
    assert list(st["level_m"][:nl]) == info["level_m"], what
    assert list(st["refine_rounds"][:nl - 1]) == info["refine_rounds"], what
    assert list(st["balance_rounds"][:nl]) == info["balance_rounds"], what
    assert cut == info["cut"], what
    assert np.array_equal(part, ref), what


def _run_both(handle, pkg, orc, gen, g, k, name, reference_mode=True):
    part, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
    ref, info = orc.partition(g, k, init=_gggp(orc, gen), enforce_balance=True)
    _same_run(st, part, cut, ref, info, (name, "default mode"))
    W = int(g.vwgt.astype(np.int64).sum())
    assert np.bincount(part, weights=g.vwgt, minlength=k).max() <= 1.03 * W / k, name
    if reference_mode:
        o = pkg.default_options(enforce_balance=0)
        rpart, rcut, rst = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, opts=o, init=_metis(orc, gen))
        rref, rinfo = orc.partition(g, k, enforce_balance=False)
        _same_run(rst, rpart, rcut, rref, rinfo, (name, "reference mode"))
    return cut


@pytest.mark.parametrize("name", ["delaunay_2e20", "grid27_100x100x96", "road_12M", "circuit_4M"])
def test_configuration_matches_oracle(handle, pkg, orc, gen, pending, name):
    g = pending[name].result()
    k = SPECS[name][1]
    if name == "grid27_100x100x96":
        assert g.n_edges == 12218972
    _run_both(handle, pkg, orc, gen, g, k, name, reference_mode=(name != "circuit_4M"))


def test_delaunay_2e20_ten_seeds_within_2pct(handle, pkg, orc, gen, pending):
    """Default-mode cut against the reference configuration's cut (reference
    mode, METIS on the coarsest graph), both on the GPU, seeds 1-10: mean
    ratio <= 1.02 and balance <= 1.03 on every seed.  The GPU equals the
    oracle in both modes (test above), so the ratios are the oracle's too."""
    ratios = []
    k = 64
    o = pkg.default_options(enforce_balance=0)
    for name in ["delaunay_2e20"] + [f"delaunay_2e20_s{s}" for s in SEEDS]:
        g = pending[name].result()
        part, cut, _ = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
        _, rcut, _ = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, opts=o, init=_metis(orc, gen))
        W = int(g.vwgt.astype(np.int64).sum())
        assert np.bincount(part, weights=g.vwgt, minlength=k).max() <= 1.03 * W / k, name
        ratios.append(cut / rcut)
    print("default/reference cut ratios over 10 seeds:", [round(r, 4) for r in ratios])
    assert np.mean(ratios) <= 1.02, ratios


@pytest.mark.parametrize("name", ["delaunay_2e20", "grid27_100x100x96", "circuit_4M"])
def test_device_init_against_metis_on_the_same_coarsest_graph(handle, pkg, orc, gen, pending, name):
    """The device initial partition (GGGP recursive bisection) against host
    METIS on the identical coarsest graph (the one the default mode's device
    initial partition receives): cut within 10% of METIS's."""
    import torch
    from conftest import to_dev
    g = pending[name].result()
    k = SPECS[name][1]
    seen = {}

    def capture(x, a, w, vw, kk):
        seen["g"] = gen.Csr(x, a, w, vw)
        return orc.metis_kway(seen["g"], kk)[0]

    handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, init=capture)
    cg = seen["g"]
    dev = handle.init_partition(to_dev(cg), k).cpu().numpy()
    assert np.array_equal(dev, orc.init_partition(cg, k)), name
    dcut, mcut = orc.cut(cg, dev), orc.metis_kway(cg, k)[1]
    print(f"{name}: coarsest n={cg.n}; device initial partition cut {dcut}, METIS {mcut}")
    assert dcut <= 1.10 * mcut, (name, dcut, mcut)
