"""Batched and served forms: every graph partitions exactly as it does alone.

The alone result is the host entry point gkw_partition on a plain handle; the
batched result comes from one gkw_partition_batch call over the concatenated
CSR (as one disjoint union, or one job per graph on the slots), the served
result from requests submitted by several host threads while others run.
Part vectors and cuts must be identical (integer work: exact)."""
import threading
import time

import numpy as np
import pytest

from graphs import path_graph, star_graph, two_components, weighted, with_isolated_and_zero

pytestmark = pytest.mark.gpu


def mixed_graphs(gen, seed=0):
    rng = np.random.default_rng(seed)
    gs = [
        gen.delaunay(2048, 11), gen.delaunay(20000, 5), gen.grid27(12, 11, 10),
        gen.circuit(30000, seed=2, levels=60, hub_max=3000), weighted(gen, gen.delaunay(8000, 9), seed=4),
        with_isolated_and_zero(gen, 3), two_components(gen, 21), path_graph(gen, 1500), star_graph(gen, 6000),
        gen.from_edges(1, np.zeros(0, np.int64), np.zeros(0, np.int64)),       # one vertex
        gen.from_edges(0, np.zeros(0, np.int64), np.zeros(0, np.int64)),       # empty
    ]
    for i in range(13):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(40000))))
        kind = i % 3
        if kind == 0:
            gs.append(gen.delaunay(n, 100 + i))
        elif kind == 1:
            a = max(2, int(round(n ** (1 / 3))))
            gs.append(gen.grid27(a, a, max(2, n // (a * a))))
        else:
            gs.append(gen.circuit(n, seed=200 + i, levels=40, hub_max=500))
    ks = [int(rng.choice([2, 3, 4, 8, 16, 32, 64])) for _ in gs]
    ks[9] = 1
    return gs, ks


def alone(pkg, gs, ks, opts=None):
    h = pkg.Handle(0)
    out = []
    for g, k in zip(gs, ks):
        part, cut, _ = h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, opts)
        out.append((part.copy(), cut))
    h.close()
    return out


def shuffled_rows(g, seed):
    """The same graph with every adjacency row in a random order."""
    rng = np.random.default_rng(seed)
    a = g.adjncy.copy()
    w = g.adjwgt.copy()
    for v in range(g.n):
        lo, hi = int(g.xadj[v]), int(g.xadj[v + 1])
        p = rng.permutation(hi - lo) + lo
        a[lo:hi] = a[p]
        w[lo:hi] = w[p]
    return type(g)(g.xadj.copy(), a, w, g.vwgt.copy())


def check_batch(pkg, srv, gs, ks, opts=None):
    ref = alone(pkg, gs, ks, opts)
    x, a, w, vw, gp = pkg.concat_graphs(gs)
    part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, ks, opts=opts)
    assert list(sts) == [0] * len(gs)
    for i, (p_ref, c_ref) in enumerate(ref):
        assert np.array_equal(part[gp[i]:gp[i + 1]], p_ref), i
        assert cuts[i] == c_ref, i


def test_union_batch_matches_alone(pkg, gen):
    """One pipeline over the disjoint union: small graphs that stop coarsening
    at once (rows in random order), graphs that stop at different depths (each
    union level holds only the graphs still present), k = 1, empty and
    one-vertex graphs, in both modes and with other balance-skip settings."""
    gs, ks = mixed_graphs(gen)
    for i in (0, 5, 6, 8):
        gs[i] = shuffled_rows(gs[i], 40 + i)
    srv = pkg.Server(0, slots=2)
    check_batch(pkg, srv, gs, ks)
    check_batch(pkg, srv, gs, ks, pkg.default_options(enforce_balance=0))
    check_batch(pkg, srv, gs, ks, pkg.default_options(balance_skip_levels=0, coarse_vertex_frac=0.0))
    check_batch(pkg, srv, gs[:12], ks[:12], pkg.default_options(balance_skip_levels=2, eps=0.05))
    st = srv.stats()
    assert st["completed"] == 3 * len(gs) + 12 and st["failed"] == 0
    assert st["peak_running"] == 0      # no slot job ran: every batch went through the union
    srv.close()


def test_union_batch_keeps_duplicate_edges(pkg, gen):
    # a small graph that stops coarsening at its input level, with a duplicated
    # edge in two rows, beside a graph that coarsens: the small graph is
    # partitioned on its own rows as given
    g = gen.delaunay(600, 7)
    u = int(g.adjncy[g.xadj[0]])   # edge 0-u listed twice in both rows
    rows = [list(zip(g.adjncy[g.xadj[v]:g.xadj[v + 1]], g.adjwgt[g.xadj[v]:g.xadj[v + 1]])) for v in range(g.n)]
    rows[0].append((u, 1))
    rows[u].append((0, 1))
    x = np.zeros(g.n + 1, np.int32)
    x[1:] = np.cumsum([len(r) for r in rows])
    a = np.array([e for r in rows for e, _ in r], np.int32)
    w = np.array([c for r in rows for _, c in r], np.int32)
    gd = type(g)(x, a, w, g.vwgt.copy())
    gs = [gen.delaunay(30000, 3), gd]
    ks = [8, 4]
    srv = pkg.Server(0, slots=2)
    check_batch(pkg, srv, gs, ks)
    srv.close()


def test_batch_matches_alone(pkg, gen):
    gs, ks = mixed_graphs(gen)
    ref = alone(pkg, gs, ks)
    x, a, w, vw, gp = pkg.concat_graphs(gs)
    srv = pkg.Server(0, slots=6, batch_union=0)
    part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, ks)
    assert list(sts) == [0] * len(gs)
    for i, (p_ref, c_ref) in enumerate(ref):
        assert np.array_equal(part[gp[i]:gp[i + 1]], p_ref), i
        assert cuts[i] == c_ref, i
    # the same batch again on the warm server, reference mode with per-graph eps
    eps = [0.03 if i % 2 else 0.05 for i in range(len(gs))]
    o = pkg.default_options(enforce_balance=0)
    part2, cuts2, _ = srv.partition_batch(x, a, w, vw, gp, ks, eps=eps, opts=o)
    h = pkg.Handle(0)
    for i, (g, k) in enumerate(zip(gs, ks)):
        oi = pkg.default_options(enforce_balance=0, eps=eps[i])
        p_ref, c_ref, _ = h.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k, oi)
        assert np.array_equal(part2[gp[i]:gp[i + 1]], p_ref), i
        assert cuts2[i] == c_ref, i
    h.close()
    st = srv.stats()
    assert st["completed"] == 2 * len(gs) and st["failed"] == 0
    assert st["peak_running"] >= 2      # jobs overlapped on the device
    srv.close()


def test_served_matches_alone_under_load(pkg, gen):
    gs, ks = mixed_graphs(gen, seed=1)
    ref = alone(pkg, gs, ks)
    srv = pkg.Server(0, slots=4)
    tickets = {}
    lock = threading.Lock()
    errors = []

    def client(idx):
        rng = np.random.default_rng(idx)
        try:
            for i in range(idx, len(gs), 3):
                g = gs[i]
                t = srv.submit(g.xadj, g.adjncy, g.adjwgt, g.vwgt, ks[i])
                with lock:
                    tickets[i] = t
                time.sleep(float(rng.uniform(0, 0.004)))
        except Exception as e:   # surfaced below
            errors.append(e)

    th = [threading.Thread(target=client, args=(c,)) for c in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for i, t in tickets.items():
        res = srv.poll(t, gs[i].n, wait_ms=-1)
        assert res is not None
        part, cut, info = res
        assert np.array_equal(part, ref[i][0]), i
        assert cut == ref[i][1], i
        assert info["latency_ms"] >= info["run_ms"] >= 0.0
        assert info["predicted_bytes"] > 0
    st = srv.stats(reset=True)
    assert st["completed"] == len(gs) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["graphs_per_s"] > 0
    assert srv.stats()["completed"] == 0
    srv.close()


def test_served_requests_drained_as_unions(pkg, gen):
    """Small requests queued faster than they run are drained into union runs;
    each result is still the graph's lone result.  A malformed request among
    them fails alone."""
    rng = np.random.default_rng(5)
    gs, ks = [], []
    for i in range(48):
        n = int(rng.integers(500, 6000))
        gs.append(gen.delaunay(n, 300 + i) if i % 2 else gen.grid27(8, 8, max(2, n // 64)))
        ks.append(int(rng.choice([2, 4, 8, 16])))
    ref = alone(pkg, gs, ks)
    bad = gen.delaunay(700, 9)
    bad_a = bad.adjncy.copy()
    bad_a[3] = bad.n + 50                    # neighbour id outside the graph
    srv = pkg.Server(0, slots=2)
    tickets = [srv.submit(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k) for g, k in zip(gs[:24], ks[:24])]
    t_bad = srv.submit(bad.xadj, bad_a, bad.adjwgt, bad.vwgt, 4)
    tickets += [srv.submit(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k) for g, k in zip(gs[24:], ks[24:])]
    sizes = []
    for i, t in enumerate(tickets):
        part, cut, info = srv.poll(t, gs[i].n, wait_ms=-1)
        assert np.array_equal(part, ref[i][0]), i
        assert cut == ref[i][1], i
        assert info["n_levels"] >= 1
        sizes.append(info["batch_graphs"])
    with pytest.raises(pkg.GkwError):
        srv.poll(t_bad, bad.n, wait_ms=-1)
    assert max(sizes) > 1                    # some requests ran together
    st = srv.stats()
    assert st["completed"] == len(gs) and st["failed"] == 1
    srv.close()


def test_server_budget_serialises_jobs(pkg, gen):
    gs, ks = mixed_graphs(gen, seed=2)
    gs, ks = gs[:8], ks[:8]
    ref = alone(pkg, gs, ks)
    srv = pkg.Server(0, slots=4, pool_bytes=1, batch_union=0)   # nothing fits beside a running job
    x, a, w, vw, gp = pkg.concat_graphs(gs)
    part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, ks)
    for i, (p_ref, c_ref) in enumerate(ref):
        assert np.array_equal(part[gp[i]:gp[i + 1]], p_ref), i
        assert cuts[i] == c_ref
    assert srv.stats()["peak_running"] == 1
    srv.close()


def test_wide_jobs_take_turns(pkg, gen):
    # every job in wide mode: the grid-barrier kernels of different slots are
    # chained on the device instead of running side by side
    gs, ks = mixed_graphs(gen, seed=3)
    gs, ks = gs[:10], ks[:10]
    ref = alone(pkg, gs, ks)
    srv = pkg.Server(0, slots=4, narrow_max_n=0, batch_union=0)
    x, a, w, vw, gp = pkg.concat_graphs(gs)
    part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, ks)
    for i, (p_ref, c_ref) in enumerate(ref):
        assert np.array_equal(part[gp[i]:gp[i + 1]], p_ref), i
        assert cuts[i] == c_ref
    srv.close()


def test_batch_reports_bad_graphs(pkg, gen):
    g0, g1, g2 = gen.delaunay(1200, 1), gen.delaunay(1300, 2), gen.delaunay(1400, 3)
    x, a, w, vw, gp = pkg.concat_graphs([g0, g1, g2])
    # rewire one edge of graph 0 into graph 1 (both directions): 0 and 1 now
    # name vertices outside their own range
    u = 0
    e = int(x[u])
    v = int(a[e])
    a = a.copy()
    a[e] = gp[1] + 5
    back = int(np.nonzero(a[x[v]:x[v + 1]] == u)[0][0]) + int(x[v])
    a[back] = gp[1] + 6
    srv = pkg.Server(0, slots=2)
    with pytest.raises(pkg.GkwError):
        srv.partition_batch(x, a, w, vw, gp, [4, 4, 4])
    part, cuts, sts = srv.partition_batch(x, a, w, vw, gp, [4, 4, 4], raise_on_error=False)
    assert sts[0] == pkg.GKW_E_INVALID and sts[2] == 0
    h = pkg.Handle(0)
    p_ref, c_ref, _ = h.partition(g2.xadj, g2.adjncy, g2.adjwgt, g2.vwgt, 4)
    h.close()
    assert np.array_equal(part[gp[2]:gp[3]], p_ref) and cuts[2] == c_ref
    with pytest.raises(pkg.GkwError):
        srv.poll(12345, 10)   # unknown ticket
    srv.close()
