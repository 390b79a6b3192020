"""METIS .graph reading and part-id writing on the device: the same CSR (or
the same error) as the host reader on every format case of the host reader's
tests, the reference's "11" reading, comment lines, CRLF line ends, missing
trailing lines, lines after the n-th vertex line that would not parse, a
bad token far into a large file; and the device-written part file equal to
the host writer's."""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def write_graph(path, header, lines, end="\n"):
    with open(path, "w", newline="") as f:
        f.write(header + end + end.join(lines) + end)


def _same(handle, pkg, path, quirks=False):
    host = pkg.read_metis(path, reference_quirks=quirks)
    dev = handle.read_metis_device(path, reference_quirks=quirks)
    for a, b in zip(host, dev):
        assert np.array_equal(a, b.cpu().numpy()), path


def _both_fail(handle, pkg, path, match=None):
    with pytest.raises(pkg.GkwError, match=match):
        pkg.read_metis(path)
    with pytest.raises(pkg.GkwError, match=match):
        handle.read_metis_device(path)


def test_device_reader_formats(handle, pkg, tmp_path):
    p = str(tmp_path / "a.graph")
    cases = [
        ("% comment\n4 4", ["2 3", "1 3", "1 2 4", "3"], False),
        ("4 4 1", ["2 5 3 1", "1 5 3 2", "1 1 2 2 4 7", "3 7"], False),
        ("4 4 10", ["3 2 3", "1 1 3", "2 1 2 4", "9 3"], False),
        ("4 4 011", ["3 2 5 3 1", "1 1 5 3 2", "2 1 1 2 2 4 7", "9 3 7"], False),
        ("4 4 11", ["2 5 3 1", "1 5 3 2", "1 1 2 2 4 7", "3 7"], True),
        ("4 4 100", ["1 2 3", "1 1 3", "2 1 2 4", "7 3"], False),
        ("5 4", ["2 3", "%  a comment", "1 3", "", "  1\t2  4 ", "3"], False),   # blank and comment lines
        ("6 4", ["2 3", "1 3", "1 2 4", "3"], False),                             # missing trailing lines
        ("4 4", ["2 3", "1 3", "1 2 4", "3", "not a vertex line"], False),        # never read
    ]
    for header, lines, quirks in cases:
        write_graph(p, header, lines)
        _same(handle, pkg, p, quirks)
        write_graph(p, header, lines, end="\r\n")
        _same(handle, pkg, p, quirks)


def test_device_reader_errors(handle, pkg, tmp_path):
    p = str(tmp_path / "b.graph")
    write_graph(p, "3 2", ["2", "1 3", "9"])
    _both_fail(handle, pkg, p, "out of range")
    write_graph(p, "3 5", ["2", "1 3", "2"])
    _both_fail(handle, pkg, p, "header says")
    write_graph(p, "3 2 0 2", ["2", "1 3", "2"])
    _both_fail(handle, pkg, p, "ncon")
    write_graph(p, "3 2", ["2", "1 x3", "2"])
    _both_fail(handle, pkg, p, "bad token")
    write_graph(p, "3 2 1", ["2 1", "1 1 3", "2 1"])
    _both_fail(handle, pkg, p, "missing edge weight")
    write_graph(p, "3 2", ["2 -", "1 3", "2"])
    _both_fail(handle, pkg, p, "bad token")
    write_graph(p, "3 2", ["9 x", "1 3", "2"])      # the first error in the line is the range error
    _both_fail(handle, pkg, p, "out of range")
    write_graph(p, "3 2", ["x 9", "1 3", "2"])      # ... and here the bad token
    _both_fail(handle, pkg, p, "bad token")
    with pytest.raises(pkg.GkwError):
        handle.read_metis_device(str(tmp_path / "missing.graph"))


@pytest.mark.skipif(not os.path.exists(oracle.N11_PATH), reason="reference fixture not available")
def test_device_reader_n11(handle, pkg):
    _same(handle, pkg, oracle.N11_PATH)


def test_device_reader_large_file(handle, pkg, gen, tmp_path):
    from graphs import weighted
    g = weighted(gen, gen.delaunay(250000, 3), seed=5)
    p = str(tmp_path / "big.graph")
    gen.write_metis(g, p)
    x, a, w, vw = (t.cpu().numpy() for t in handle.read_metis_device(p))
    assert np.array_equal(x, g.xadj) and np.array_equal(a, g.adjncy)
    assert np.array_equal(w, g.adjwgt) and np.array_equal(vw, g.vwgt)
    lines = open(p).read().split("\n")
    out = [lines[0]] + lines[1:1 + g.n]
    out[-3] = out[-3] + " x"
    q = str(tmp_path / "big2.graph")
    open(q, "w").write("\n".join(out) + "\n")
    _both_fail(handle, pkg, q, "bad token")


def test_device_writer(handle, pkg, tmp_path):
    import torch
    rng = np.random.default_rng(4)
    part = np.concatenate([rng.integers(0, 40000, 50000), [0, 2 ** 31 - 1, 9, 10, 99, 100]]).astype(np.int32)
    a, b = str(tmp_path / "h.out"), str(tmp_path / "d.out")
    pkg.write_partition(a, part)
    handle.write_partition_device(b, torch.from_numpy(part).cuda())
    assert open(a, "rb").read() == open(b, "rb").read()
