"""Seeded test graphs covering the shapes and edge cases of the partitioner."""
from __future__ import annotations

import numpy as np


def path_graph(gen, n: int):
    src = np.arange(n - 1)
    return gen.from_edges(n, src, src + 1)


def star_graph(gen, n: int):
    leaves = np.arange(1, n)
    return gen.from_edges(n, np.zeros(n - 1, dtype=np.int64), leaves)


def weighted(gen, g, seed: int, wmax: int = 8, vmax: int = 4):
    """Same topology, random symmetric edge weights U{1..wmax}, vertex weights U{1..vmax}."""
    rng = np.random.default_rng(seed)
    n = g.n
    src = np.repeat(np.arange(n), np.diff(g.xadj))
    keep = src < g.adjncy
    s, d = src[keep], g.adjncy[keep]
    w = rng.integers(1, wmax + 1, s.shape[0])
    vw = rng.integers(1, vmax + 1, n).astype(np.int32)
    return gen.from_edges(n, s, d, w, vw)


def with_isolated_and_zero(gen, seed: int):
    """A Delaunay graph plus isolated vertices, with some zero edge weights."""
    rng = np.random.default_rng(seed)
    base = gen.delaunay(3000, seed)
    n = base.n + 200
    src = np.repeat(np.arange(base.n), np.diff(base.xadj))
    keep = src < base.adjncy
    s, d = src[keep], base.adjncy[keep]
    w = rng.integers(0, 3, s.shape[0])   # zero weights included
    return gen.from_edges(n, s, d, w)


def two_components(gen, seed: int):
    a = gen.delaunay(2500, seed)
    b = gen.delaunay(1500, seed + 1)
    sa = np.repeat(np.arange(a.n), np.diff(a.xadj))
    sb = np.repeat(np.arange(b.n), np.diff(b.xadj)) + a.n
    return gen.from_edges(a.n + b.n, np.concatenate([sa, sb]), np.concatenate([a.adjncy, b.adjncy + a.n]))


def with_hub(gen, seed: int, n: int = 20000, fan: int = 10000):
    """A Delaunay graph whose vertex n/2 is also joined to `fan` random others:
    one row of about 10k entries among rows of about 6 (the skew of the
    circuit-like graphs' fan-out hubs)."""
    rng = np.random.default_rng(seed)
    base = gen.delaunay(n, seed)
    src = np.repeat(np.arange(base.n), np.diff(base.xadj))
    keep = src < base.adjncy
    s, d = src[keep], base.adjncy[keep]
    hub = n // 2
    others = rng.choice(np.setdiff1d(np.arange(n), [hub]), fan, replace=False)
    s = np.concatenate([s, np.full(fan, hub)])
    d = np.concatenate([d, others])
    w = rng.integers(1, 4, s.shape[0])
    return gen.from_edges(n, s, d, w)


def small_cases(gen):
    """(name, graph) pairs for per-phase parity; each runs in well under a second."""
    cases = [
        ("delaunay_2k", gen.delaunay(2048, 11)),
        ("delaunay_20k", gen.delaunay(20000, 5)),
        ("grid27_12x11x10", gen.grid27(12, 11, 10)),
        ("circuit_30k", gen.circuit(30000, seed=2, levels=60, hub_max=3000)),
        ("delaunay_w", weighted(gen, gen.delaunay(8000, 9), seed=4)),
        ("isolated_zero_w", with_isolated_and_zero(gen, 3)),
        ("two_components", two_components(gen, 21)),
        ("path_1500", path_graph(gen, 1500)),
        ("star_6000", star_graph(gen, 6000)),
        ("delaunay_hub10k", with_hub(gen, 13)),
    ]
    return cases


def build_graph(spec):
    """Generator call by spec, for a process pool: ("delaunay", n, seed),
    ("grid27", nx, ny, nz), ("circuit", n, seed) or ("road", n, seed)."""
    import os
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import __graft_entry__ as ge
    gen = ge.load_generators()
    kind, *args = spec
    if kind == "delaunay":
        return gen.delaunay(args[0], seed=args[1])
    if kind == "grid27":
        return gen.grid27(*args)
    if kind == "circuit":
        return gen.circuit(args[0], seed=args[1])
    if kind == "road":
        return gen.road(args[0], seed=args[1])
    raise ValueError(spec)
