"""The drop-in surfaces on a device: the g-kway CLI's success path and the
C++ classes (gk::GraphPartitioner and the free graph_partitioner()).

The CLI must write <cwd>/<out>.out with one part id per line in vertex order,
print the four timer lines and "***** h_cutsize <cut>" as the reference does
(gkway/graph_partitioner.hpp:338-353, graph.hpp:227-240), and give exactly the
part vector of gkw_partition on the same graph and k."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dac_g-kway_b200")
CLI = os.path.join(LIBDIR, "bin", "g-kway")
TIMERS = ("Total time: ", "Coarsen time: ", "Init partition time: ", "Refinement time: ")


def _graph_file(gen, tmp_path, which):
    if which == "n11":
        if not os.path.exists(oracle.N11_PATH):
            pytest.skip("the reference fixture is not available")
        return oracle.N11_PATH, oracle.read_metis_graph(oracle.N11_PATH)
    g = gen.delaunay(1 << 16, seed=3)
    path = str(tmp_path / "d16.graph")
    gen.write_metis(g, path)
    return path, g


@pytest.mark.parametrize("which,k", [("n11", 8), ("d16", 64)])
def test_cli_success_path(handle, gen, tmp_path, which, k):
    path, g = _graph_file(gen, tmp_path, which)
    r = subprocess.run([CLI, path, str(k), "result"], capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    for t in TIMERS:
        assert re.search(re.escape(t) + r"[0-9.e+-]+s", r.stdout), (t, r.stdout)
    m = re.search(r"\*\*\*\*\* h_cutsize (\d+)", r.stdout)
    assert m, r.stdout
    lines = (tmp_path / "result.out").read_text().split("\n")
    assert lines[-1] == "" and len(lines) == g.n + 1
    part = np.array([int(x) for x in lines[:-1]], np.int32)
    want, cut, _ = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
    assert np.array_equal(part, want)
    assert int(m.group(1)) == cut == oracle.cut(g, part)


PROGRAM = r'''
#include <cstdio>
#include <vector>
#include "gkway.hpp"

int main(int argc, char** argv) {
  gk::Graph g(argv[1]);
  const int k = std::atoi(argv[2]);
  gk::GraphPartitioner gp;
  const std::vector<int> part = gp.partition(g, k);
  gk::PartitionResult r = gp.partition_with_stats(g, k);
  if (r.part != part) { std::printf("partition and partition_with_stats differ\n"); return 3; }
  std::vector<gk::PartitionResult> multi = gp.partition_multi_k(g, {k, 2 * k});
  if (multi.size() != 2 || multi[0].part != part || multi[0].cut != r.cut) {
    std::printf("partition_multi_k differs\n");
    return 4;
  }
  FILE* f = std::fopen("cls.txt", "w");
  for (int p : part) std::fprintf(f, "%d\n", p);
  std::fclose(f);
  std::printf("cut=%lld levels=%d\n", (long long)r.cut, r.stats.n_levels);
  graph_partitioner(argv[1], "free", k);   // the reference's free function
  return 0;
}
'''


def test_cpp_graph_partitioner_on_device(handle, gen, tmp_path):
    path, g = _graph_file(gen, tmp_path, "d16")
    src = tmp_path / "app.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "app"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + LIBDIR, "-lgkway", "-Wl,-rpath," + LIBDIR, "-L/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath,/usr/local/cuda/lib64"], check=True, capture_output=True)
    k = 32
    r = subprocess.run([str(exe), path, str(k)], capture_output=True, text=True, cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    want, cut, st = handle.partition(g.xadj, g.adjncy, g.adjwgt, g.vwgt, k)
    cls = np.loadtxt(tmp_path / "cls.txt", dtype=np.int32)
    free = np.loadtxt(tmp_path / "free.out", dtype=np.int32)
    assert np.array_equal(cls, want) and np.array_equal(free, want)
    assert f"cut={cut} levels={st['n_levels']}" in r.stdout
    assert f"***** h_cutsize {cut}" in r.stdout
