"""bench.py's roofline arithmetic on synthetic per-level statistics: the
algorithmic bytes of each phase (4-byte words, every compulsory array once),
the achieved GB/s of the level kernel, and its fraction of the peak."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _stats(levels, ms_level, entries, ms_coarsen=1.0, ms_refine=2.0):
    return {"n_levels": len(levels), "level_n": [n for n, _ in levels], "level_m": [m for _, m in levels],
            "ms_level": ms_level, "round_entries": entries, "ms_coarsen": ms_coarsen, "ms_refine": ms_refine}


def test_match_bytes_of_the_million_vertex_level():
    # the heavy-edge match of level 0 of the 2^20 Delaunay graph: 4(n+1) + 8m + 4n
    n, m = 1048576, 6291384
    st = _stats([(n, m), (239829, 1400000)], [0.3, 0.2], [0, 0])
    match = 4 * (n + 1) + 8 * m + 4 * n
    assert abs(match / 1e6 - 58.7) < 0.05
    nc, mc = 239829, 1400000
    want = match + (12 * n + 4 * nc) + (4 * (n + 1) + 8 * m + 8 * n + 4 * (nc + 1) + 8 * mc)
    assert bench.coarsen_bytes(st) == want


def test_level_kernel_bytes_and_roofline(monkeypatch):
    levels = [(1000, 6000), (300, 2000), (90, 500)]
    ms = [0.5, 0.25, -1.0]          # the coarsest level had no launch
    entries = [40000, 10000, 0]
    st = _stats(levels, ms, entries, ms_coarsen=0.4, ms_refine=0.75)
    got = bench.level_kernel_launches(st)
    assert [i for i, _, _ in got] == [0, 1]

    def level_bytes(i):
        n, m = levels[i]
        b = 4 * (n + 1) + 8 * m + 4 * n + 8 * n + 8 * entries[i]
        if i + 1 < len(levels):
            b += 4 * n + 4 * levels[i + 1][0]
        return b

    assert [b for _, b, _ in got] == [level_bytes(0), level_bytes(1)]
    monkeypatch.setattr(bench, "load_peak_gbs", lambda: (1000.0, "test peak"))
    roof, phases = bench.roofline_report([st, st])
    tot_b = 2 * (level_bytes(0) + level_bytes(1))
    tot_s = 2 * (0.5 + 0.25) / 1e3
    assert roof["achieved"] == pytest.approx(tot_b / tot_s / 1e9)
    assert roof["frac"] == pytest.approx(roof["achieved"] / 1000.0)
    assert roof["launches"] == 4
    assert roof["algorithmic_bytes_per_launch"] == pytest.approx(tot_b / 4)
    assert phases["coarsen"]["bytes_per_step"] == pytest.approx(bench.coarsen_bytes(st))
    assert phases["uncoarsen"]["frac"] == pytest.approx(
        (level_bytes(0) + level_bytes(1)) / (0.75 / 1e3) / 1e9 / 1000.0)
