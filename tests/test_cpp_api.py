"""The C++ drop-in surface (include/gkway.hpp) compiles into a user program and
its host-only parts run without a device: gk::Graph parsing and getters,
dump_result, and use_metis_init for both METIS entry points."""
import os
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dac_g-kway_b200")

PROGRAM = r'''
#include <cstdio>
#include <vector>
#include "gkway.hpp"

int main(int argc, char** argv) {
  gk::Graph g(argv[1]);
  std::printf("n=%d m=%lld\n", (int)g.csr().n, (long long)g.csr().nnz);
  std::vector<int> part(g.csr().n, 0);
  for (int v = 0; v < (int)part.size(); ++v) part[v] = v % 4;
  g.dump_result(part, "cpp_api");
  gkw_options o;
  gkw_default_options(&o);
  const bool kway = gk::use_metis_init(&o, argv[2]);
  const bool rec = gk::use_metis_init(&o, argv[2], /*recursive=*/true);
  std::printf("kway=%d recursive=%d callback=%d\n", (int)kway, (int)rec, (int)(o.init_method == GKW_INIT_CALLBACK));
  return 0;
}
'''


@pytest.mark.skipif(not (os.path.exists(oracle.N11_PATH) and os.path.exists(oracle.METIS_PATH)),
                    reason="fixture or METIS not available")
def test_cpp_api_host_parts(pkg, tmp_path):
    src = tmp_path / "app.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "app"
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L" + LIBDIR, "-lgkway", "-Wl,-rpath," + LIBDIR, "-L/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath,/usr/local/cuda/lib64"], check=True, capture_output=True)
    r = subprocess.run([str(exe), oracle.N11_PATH, oracle.METIS_PATH], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert "n=2048 m=12254" in r.stdout
    assert "kway=1 recursive=1 callback=1" in r.stdout
    lines = (tmp_path / "cpp_api.out").read_text().split()
    assert len(lines) == 2048 and lines[:5] == ["0", "1", "2", "3", "0"]
