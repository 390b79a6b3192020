"""Seeded synthetic graph generators for the partitioner's workloads.

Every generator returns a ``Csr`` (int32 numpy arrays, 0-based ids, rows sorted
ascending, symmetric, no self loops).  The shapes follow the workloads the
partitioner is measured on:

* ``delaunay(n, seed)``   2D Delaunay triangulation of ``n`` points uniform in the
  unit square (unit weights).  ``n = 2048`` has the shape of the DIMACS
  ``delaunay_n11`` graph the reference ships as its only fixture; ``n = 2**20``
  is the mid-size k=64 workload.
* ``grid27(nx, ny, nz)``  structured 3D grid with 26-neighbour (27-point stencil)
  adjacency, unit weights; 100x100x96 gives 960,000 vertices and 12,218,972
  undirected edges.
* ``road(n, seed)``       Euclidean MST of a Delaunay triangulation plus the
  shortest 8% of the remaining Delaunay edges (road-network-like, avg degree ~2.2).
* ``circuit(n, seed)``    levelised DAG-like timing graph: Poisson(2.5) fan-in from
  the previous 5 levels inside a 90%-local index window, 0.1% of vertices with
  power-law fan-out up to 10k; symmetrised, edge weights U{1..8}, vertex weights
  U{1..4} (the first drawn weight of a duplicated edge wins).

The real DIMACS / SuiteSparse graphs are not available offline; these seeded
stand-ins reproduce their sizes, degree distributions and weight ranges.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Csr:
    xadj: np.ndarray      # int32[n+1]
    adjncy: np.ndarray    # int32[m], 0-based
    adjwgt: np.ndarray    # int32[m]
    vwgt: np.ndarray      # int32[n]

    @property
    def n(self) -> int:
        return int(self.xadj.shape[0] - 1)

    @property
    def m(self) -> int:
        """Directed CSR entries (2 x undirected edges)."""
        return int(self.adjncy.shape[0])

    @property
    def n_edges(self) -> int:
        return self.m // 2


def from_edges(n: int, src: np.ndarray, dst: np.ndarray, wgt: np.ndarray | None = None,
               vwgt: np.ndarray | None = None) -> Csr:
    """Build a symmetric CSR from an undirected edge list.

    Self loops are dropped.  Duplicated undirected edges keep the weight of their
    first occurrence in the input order.
    """
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if wgt is None:
        wgt = np.ones(src.shape[0], dtype=np.int64)
    wgt = np.asarray(wgt, dtype=np.int64)
    keep = src != dst
    src, dst, wgt = src[keep], dst[keep], wgt[keep]
    lo = np.minimum(src, dst)
    hi = np.maximum(src, dst)
    key = lo * n + hi
    # first occurrence wins: np.unique returns the index of the first occurrence
    ukey, first = np.unique(key, return_index=True)
    w = wgt[first]
    lo = ukey // n
    hi = ukey % n
    s = np.concatenate([lo, hi])
    d = np.concatenate([hi, lo])
    ww = np.concatenate([w, w])
    order = np.lexsort((d, s))
    s, d, ww = s[order], d[order], ww[order]
    xadj = np.zeros(n + 1, dtype=np.int64)
    np.add.at(xadj, s + 1, 1)
    xadj = np.cumsum(xadj)
    if vwgt is None:
        vwgt = np.ones(n, dtype=np.int32)
    return Csr(xadj.astype(np.int32), d.astype(np.int32), ww.astype(np.int32),
               np.asarray(vwgt, dtype=np.int32))


def delaunay(n: int, seed: int = 1) -> Csr:
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    tri = Delaunay(pts).simplices.astype(np.int64)
    a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
    src = np.concatenate([a, b, a])
    dst = np.concatenate([b, c, c])
    return from_edges(n, src, dst)


def grid27(nx: int, ny: int, nz: int) -> Csr:
    n = nx * ny * nz
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = x.ravel(); y = y.ravel(); z = z.ravel()
    vid = x + nx * (y + ny * z)
    srcs, dsts = [], []
    # forward half of the 26 offsets; from_edges symmetrises
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) <= (0, 0, 0):
                    continue
                xx, yy, zz = x + dx, y + dy, z + dz
                ok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny) & (zz >= 0) & (zz < nz)
                srcs.append(vid[ok])
                dsts.append((xx + nx * (yy + ny * zz))[ok])
    return from_edges(n, np.concatenate(srcs), np.concatenate(dsts))


def road(n: int, seed: int = 1, extra_frac: float = 0.08) -> Csr:
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import minimum_spanning_tree
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2))
    tri = Delaunay(pts).simplices.astype(np.int64)
    a = np.concatenate([tri[:, 0], tri[:, 1], tri[:, 0]])
    b = np.concatenate([tri[:, 1], tri[:, 2], tri[:, 2]])
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo * n + hi)
    lo, hi = key // n, key % n
    length = np.hypot(*(pts[lo] - pts[hi]).T)
    g = coo_matrix((length, (lo, hi)), shape=(n, n)).tocsr()
    mst = minimum_spanning_tree(g).tocoo()
    in_mst = np.zeros(key.shape[0], dtype=bool)
    mkey = np.minimum(mst.row, mst.col).astype(np.int64) * n + np.maximum(mst.row, mst.col)
    in_mst[np.searchsorted(key, mkey)] = True
    rest = np.flatnonzero(~in_mst)
    n_extra = int(round(extra_frac * rest.shape[0]))
    extra = rest[np.argsort(length[rest], kind="stable")[:n_extra]]
    sel = np.concatenate([np.flatnonzero(in_mst), extra])
    return from_edges(n, lo[sel], hi[sel])


def circuit(n: int, seed: int = 1, levels: int = 200, fanin_mean: float = 2.5,
            window_levels: int = 5, local_frac: float = 0.9, hub_frac: float = 0.001,
            hub_max: int = 10000) -> Csr:
    rng = np.random.default_rng(seed)
    per = max(1, n // levels)
    lvl = np.minimum(np.arange(n) // per, levels - 1)
    lvl_start = np.searchsorted(lvl, np.arange(levels))
    lvl_start = np.append(lvl_start, n)
    deg = rng.poisson(fanin_mean, n)
    deg[lvl == 0] = 0
    src_v = np.repeat(np.arange(n), deg)
    m0 = src_v.shape[0]
    lv = lvl[src_v]
    back = rng.integers(1, window_levels + 1, m0)
    pl = np.maximum(lv - back, 0)
    lo = lvl_start[pl]
    hi = lvl_start[np.minimum(lv, levels)]   # exclusive: strictly earlier levels
    hi = np.maximum(hi, lo + 1)
    span = hi - lo
    # 90% local: pick within a window around the vertex's relative position
    rel = (src_v - lvl_start[lv]) / np.maximum(1, lvl_start[np.minimum(lv + 1, levels)] - lvl_start[lv])
    centre = lo + (rel * span).astype(np.int64)
    width = np.maximum(1, span // 20)
    local = rng.random(m0) < local_frac
    off = rng.integers(-width, width + 1)
    pick_local = np.clip(centre + off, lo, hi - 1)
    pick_any = lo + (rng.random(m0) * span).astype(np.int64)
    dst_v = np.where(local, pick_local, pick_any)
    # hubs: power-law fan-out up to hub_max into later levels
    n_hub = max(1, int(round(hub_frac * n)))
    hubs = rng.choice(n, n_hub, replace=False)
    fo = np.minimum(hub_max, (rng.pareto(1.2, n_hub) * 20 + 10).astype(np.int64))
    hs = np.repeat(hubs, fo)
    hd = rng.integers(0, n, hs.shape[0])
    src = np.concatenate([src_v, hs])
    dst = np.concatenate([dst_v, hd])
    w = rng.integers(1, 9, src.shape[0])
    vw = rng.integers(1, 5, n).astype(np.int32)
    return from_edges(n, src, dst, w, vw)


def check_csr(g: Csr) -> None:
    """Raise ValueError if ``g`` is not a symmetric, self-loop-free, sorted CSR."""
    n = g.n
    if g.xadj[0] != 0 or np.any(np.diff(g.xadj) < 0) or g.xadj[-1] != g.m:
        raise ValueError("bad xadj")
    if g.m and (g.adjncy.min() < 0 or g.adjncy.max() >= n):
        raise ValueError("neighbour id out of range")
    src = np.repeat(np.arange(n), np.diff(g.xadj))
    if np.any(src == g.adjncy):
        raise ValueError("self loop")
    fwd = src.astype(np.int64) * n + g.adjncy
    rev = g.adjncy.astype(np.int64) * n + src
    fo = np.argsort(fwd)
    ro = np.argsort(rev)
    if not np.array_equal(fwd[fo], rev[ro]) or not np.array_equal(g.adjwgt[fo], g.adjwgt[ro]):
        raise ValueError("not symmetric")


def write_metis(g: Csr, path: str) -> None:
    """Write ``g`` as a METIS .graph file: header ``n |E|`` (unit weights) or
    ``n |E| 011`` (vertex and edge weights), then one line per vertex with its
    1-based neighbours (preceded by the vertex weight and followed each by its
    edge weight in the weighted form)."""
    weighted = bool(np.any(g.adjwgt != 1) or np.any(g.vwgt != 1))
    deg = np.diff(g.xadj)
    with open(path, "w") as f:
        f.write(f"{g.n} {g.n_edges}" + (" 011" if weighted else "") + "\n")
        adj1 = (g.adjncy.astype(np.int64) + 1).astype(str)
        if weighted:
            wstr = g.adjwgt.astype(str)
        lines = []
        for v in range(g.n):
            a, b = int(g.xadj[v]), int(g.xadj[v + 1])
            if weighted:
                toks = [str(int(g.vwgt[v]))]
                for e in range(a, b):
                    toks.append(adj1[e])
                    toks.append(wstr[e])
                lines.append(" ".join(toks))
            else:
                lines.append(" ".join(adj1[a:b]) if deg[v] else "")
            if len(lines) >= 65536:
                f.write("\n".join(lines) + "\n")
                lines = []
        if lines:
            f.write("\n".join(lines) + "\n")


def _main(argv) -> int:
    """``generators.py <delaunay|grid27|road|circuit> <args...> <out.graph>``:
    delaunay N SEED | grid27 NX NY NZ | road N SEED | circuit N SEED."""
    if len(argv) < 3:
        print(_main.__doc__)
        return 2
    kind, out = argv[0], argv[-1]
    a = [int(x) for x in argv[1:-1]]
    g = {"delaunay": lambda: delaunay(a[0], a[1]), "grid27": lambda: grid27(a[0], a[1], a[2]),
         "road": lambda: road(a[0], a[1]), "circuit": lambda: circuit(a[0], a[1])}[kind]()
    write_metis(g, out)
    print(f"{out}: n={g.n} edges={g.n_edges}")
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(_main(sys.argv[1:]))
