"""The C-ABI library (CPU only): loads, exports every declared symbol, parses
METIS files, writes partitions; the CLI's argument handling."""
import os
import subprocess

import numpy as np
import pytest

import oracle


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    syms = pkg.exported_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_version_and_defaults(pkg):
    assert pkg.lib().gkw_version().startswith(b"gkway-b200")
    o = pkg.default_options()
    assert (o.eps, o.group_cap, o.threshold_factor, o.move_cap) == (0.03, 6, 20, 1024)
    assert o.init_method == pkg.INIT_DEVICE


def test_max_part_weight_matches_oracle(pkg):
    for W, k in [(2048, 8), (1048576, 64), (960000, 64), (10000000, 256), (17, 3)]:
        assert pkg.max_part_weight(W, k) == oracle.max_part_weight(W, k)


def write_graph(path, header, lines):
    with open(path, "w") as f:
        f.write(header + "\n")
        for ln in lines:
            f.write(ln + "\n")


def test_reader_formats(pkg, tmp_path):
    # triangle 1-2-3 plus pendant 4 on 3
    p = str(tmp_path / "a.graph")
    write_graph(p, "% comment\n4 4", ["2 3", "1 3", "1 2 4", "3"])
    x, a, w, vw = pkg.read_metis(p)
    assert list(x) == [0, 2, 4, 7, 8] and list(a) == [1, 2, 0, 2, 0, 1, 3, 2]
    assert np.all(w == 1) and np.all(vw == 1)
    # fmt 1: edge weights
    write_graph(p, "4 4 1", ["2 5 3 1", "1 5 3 2", "1 1 2 2 4 7", "3 7"])
    x, a, w, vw = pkg.read_metis(p)
    assert list(w) == [5, 1, 5, 2, 1, 2, 7, 7]
    # fmt 10: vertex weights
    write_graph(p, "4 4 10", ["3 2 3", "1 1 3", "2 1 2 4", "9 3"])
    x, a, w, vw = pkg.read_metis(p)
    assert list(vw) == [3, 1, 2, 9] and list(a) == [1, 2, 0, 2, 0, 1, 3, 2]
    # fmt 011: both
    write_graph(p, "4 4 011", ["3 2 5 3 1", "1 1 5 3 2", "2 1 1 2 2 4 7", "9 3 7"])
    x, a, w, vw = pkg.read_metis(p)
    assert list(vw) == [3, 1, 2, 9] and list(w) == [5, 1, 5, 2, 1, 2, 7, 7]
    # the reference's reading of "11": neighbour/weight pairs, no vertex weights
    write_graph(p, "4 4 11", ["2 5 3 1", "1 5 3 2", "1 1 2 2 4 7", "3 7"])
    x, a, w, vw = pkg.read_metis(p, reference_quirks=True)
    assert list(w) == [5, 1, 5, 2, 1, 2, 7, 7] and np.all(vw == 1)


def test_reader_errors(pkg, tmp_path):
    p = str(tmp_path / "b.graph")
    write_graph(p, "3 2", ["2", "1 3", "9"])        # id out of range
    with pytest.raises(pkg.GkwError):
        pkg.read_metis(p)
    write_graph(p, "3 5", ["2", "1 3", "2"])        # edge count mismatch
    with pytest.raises(pkg.GkwError):
        pkg.read_metis(p)
    write_graph(p, "3 2 0 2", ["2", "1 3", "2"])    # ncon 2
    with pytest.raises(pkg.GkwError):
        pkg.read_metis(p)
    with pytest.raises(pkg.GkwError):
        pkg.read_metis(str(tmp_path / "missing.graph"))


@pytest.mark.skipif(not os.path.exists(oracle.N11_PATH), reason="reference fixture not available")
def test_reader_matches_checker_on_n11(pkg):
    x, a, w, vw = pkg.read_metis(oracle.N11_PATH)
    g = oracle.read_metis_graph(oracle.N11_PATH)
    assert np.array_equal(x, g.xadj) and np.array_equal(a, g.adjncy)
    assert np.array_equal(w, g.adjwgt) and np.array_equal(vw, g.vwgt)


def test_write_partition(pkg, tmp_path):
    p = str(tmp_path / "o.out")
    pkg.write_partition(p, np.array([3, 0, 1, 2], np.int32))
    assert open(p).read() == "3\n0\n1\n2\n"


def test_cli_usage_and_missing_file(pkg, tmp_path):
    cli = pkg.CLI_PATH
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([cli, str(tmp_path / "nope.graph"), "4", "out"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 1 and "cannot open" in r.stderr


def test_generators(gen):
    g = gen.grid27(4, 3, 5)
    gen.check_csr(g)
    # 27-point stencil: undirected edges = sum over the 13 forward offsets of prod(n_i - |d_i|)
    def count(nx, ny, nz):
        tot = 0
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if (dz, dy, dx) <= (0, 0, 0):
                        continue
                    tot += (nx - abs(dx)) * (ny - abs(dy)) * (nz - abs(dz))
        return tot
    assert g.n_edges == count(4, 3, 5)
    assert count(100, 100, 96) == 12218972
    d = gen.delaunay(2048, 1)
    gen.check_csr(d)
    assert 6000 < d.n_edges < 6200
    c = gen.circuit(20000, seed=3, levels=50, hub_max=2000)
    gen.check_csr(c)
    assert c.adjwgt.min() >= 1 and c.adjwgt.max() <= 8 and c.vwgt.min() >= 1 and c.vwgt.max() <= 4


@pytest.mark.parametrize("kind", ["unit", "weighted"])
def test_write_metis_round_trip(pkg, gen, tmp_path, kind):
    g = gen.delaunay(3000, 5) if kind == "unit" else gen.circuit(5000, 3)
    p = str(tmp_path / "g.graph")
    gen.write_metis(g, p)
    x, a, w, vw = pkg.read_metis(p)
    assert np.array_equal(x, g.xadj) and np.array_equal(a, g.adjncy)
    assert np.array_equal(w, g.adjwgt) and np.array_equal(vw, g.vwgt)


def test_reader_large_files_parallel(pkg, gen, tmp_path):
    """Files above 8 MB are parsed by several threads; the result and the
    errors are those of the sequential reading (small files)."""
    from graphs import weighted
    g = weighted(gen, gen.delaunay(250000, 3), seed=5)
    p = str(tmp_path / "big.graph")
    gen.write_metis(g, p)
    import os
    assert os.path.getsize(p) > (8 << 20)
    x, a, w, vw = pkg.read_metis(p)
    assert np.array_equal(x, g.xadj) and np.array_equal(a, g.adjncy)
    assert np.array_equal(w, g.adjwgt) and np.array_equal(vw, g.vwgt)
    # comment lines between vertex lines, and lines after the n-th vertex
    # (never read) that would not parse
    lines = open(p).read().split("\n")
    body = lines[1:1 + g.n]
    out = [lines[0]]
    for i, ln in enumerate(body):
        if i % 5000 == 0:
            out.append("% a comment line")
        out.append(ln)
    out.append("not a vertex line")
    q = str(tmp_path / "big2.graph")
    open(q, "w").write("\n".join(out) + "\n")
    x2, a2, w2, vw2 = pkg.read_metis(q)
    assert np.array_equal(x2, g.xadj) and np.array_equal(a2, g.adjncy) and np.array_equal(w2, g.adjwgt)
    assert np.array_equal(vw2, g.vwgt)
    # a bad token late in the file is reported
    out[-2] = out[-2] + " x"
    open(q, "w").write("\n".join(out) + "\n")
    with pytest.raises(pkg.GkwError, match="bad token"):
        pkg.read_metis(q)


def test_server_config_defaults(pkg):
    """The documented defaults of gkw_server_config (no device needed)."""
    c = pkg.server_config()
    assert c.slots == 2 and c.pool_bytes == 64 << 30 and c.slot_keep_bytes == 4 << 30
    assert c.narrow_max_n == 262144 and c.batch_union == 1
    assert c.batch_max_n == 1 << 22 and c.batch_graph_max_n == 262144
    assert all(r == 0 for r in c.reserved)
    c2 = pkg.server_config(slots=5, batch_union=0)
    assert c2.slots == 5 and c2.batch_union == 0 and c2.batch_max_n == 1 << 22


def test_server_argument_errors_without_device(pkg):
    """Argument checks of the server entry points answer before any device
    work (so they hold on a machine without a GPU too)."""
    with pytest.raises(pkg.GkwError):
        pkg.Server(0, slots=0)
    with pytest.raises(pkg.GkwError):
        pkg.Server(0, batch_max_n=-1)
    with pytest.raises(pkg.GkwError):
        pkg.Server(0, narrow_max_n=-5)


def test_predicted_footprint(pkg):
    """The server's admission measure (no device needed): at least the input
    CSR and part vector, and never smaller for a larger graph or more parts."""
    f = pkg.predict_footprint
    for n, m, k in ((1000, 6000, 8), (1 << 20, 6291384, 64), (12_000_000, 26_000_000, 256)):
        assert f(n, m, k) >= 4 * (n + 1) + 8 * m + 8 * n
        assert f(2 * n, m, k) > f(n, m, k)
        assert f(n, 2 * m, k) > f(n, m, k)
        assert f(n, m, 4 * k) >= f(n, m, k)
    assert f(0, 0, 1) > 0   # empty graphs still hold the fixed per-job state


def test_concat_graphs_layout(pkg, gen):
    gs = [gen.delaunay(300, 1), gen.from_edges(0, np.zeros(0, np.int64), np.zeros(0, np.int64)),
          gen.grid27(3, 3, 3)]
    x, a, w, vw, gp = pkg.concat_graphs(gs)
    assert list(gp) == [0, gs[0].n, gs[0].n, gs[0].n + gs[2].n]
    assert x[-1] == a.shape[0] == sum(g.m for g in gs)
    for i, g in enumerate(gs):
        v0, v1 = gp[i], gp[i + 1]
        assert np.array_equal(x[v0:v1 + 1] - x[v0], g.xadj)
        assert np.array_equal(a[x[v0]:x[v1]] - v0, g.adjncy)
        assert np.array_equal(w[x[v0]:x[v1]], g.adjwgt) and np.array_equal(vw[v0:v1], g.vwgt)


def test_write_partition_many_ids(pkg, tmp_path):
    rng = np.random.default_rng(0)
    part = np.concatenate([rng.integers(0, 40000, 50000), [0, 2 ** 31 - 1, -7]]).astype(np.int32)
    p = str(tmp_path / "many.out")
    pkg.write_partition(p, part)
    assert open(p).read() == "".join(f"{v}\n" for v in part.tolist())
    pkg.write_partition(p, np.zeros(0, np.int32))
    assert open(p).read() == ""
