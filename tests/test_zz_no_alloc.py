"""gkw_cut_noalloc: the cut entry point for callers that may not allocate
device memory (its accumulators live in a fixed array inside the library).
Checked against gkw_cut on the same inputs and against the oracle's cut and
part weights, on two calls in a row -- the second call finds the array holding
the first call's values and must clear them -- on the default stream and on a
caller's stream, up to the largest k the fixed array holds (8190, whose last
part weight lands in the array's last word).  Integer results: exact equality.
This file is collected last so that a run that stops at its first failure has
run every other test before it."""
import numpy as np
import pytest

from conftest import to_dev
from graphs import weighted

pytestmark = pytest.mark.gpu


def test_cut_noalloc_matches_cut(pkg, gen, orc):
    import torch
    torch.cuda.set_device(0)
    h = pkg.Handle(0)
    side = torch.cuda.Stream()
    cases = [
        (weighted(gen, gen.delaunay(30000, 4), seed=7), 64),
        (gen.grid27(20, 18, 16), 5000),   # k above the shared-memory staging of the kernel
        (gen.delaunay(3000, 9), 3),
        (gen.grid27(24, 22, 20), 8190),   # the largest k: the array's last word is a part weight
    ]
    rng = np.random.default_rng(1)
    for g, k in cases:
        dg = to_dev(g)
        for call in range(2):
            part_np = rng.integers(0, k, g.n).astype(np.int32)
            part = torch.from_numpy(part_np).cuda()
            ref_cut, ref_pw = h.cut(dg, part, k)
            cut, pw = pkg.cut_noalloc(dg, part, k)
            assert cut == ref_cut == orc.cut(g, part_np), (g.n, k, call)
            assert np.array_equal(pw, ref_pw), (g.n, k, call)
            assert np.array_equal(pw, orc.part_weights(g, part_np, k)), (g.n, k, call)
            # the same call on a caller's stream, ordered after the uploads above
            side.wait_stream(torch.cuda.current_stream())
            cut_s, pw_s = pkg.cut_noalloc(dg, part, k, stream=side.cuda_stream)
            side.synchronize()
            assert cut_s == cut and np.array_equal(pw_s, pw), (g.n, k, call)
    h.close()


def test_cut_noalloc_rejects_bad_input(pkg, gen):
    import torch
    g = gen.delaunay(500, 2)
    dg = to_dev(g)
    part = torch.zeros(g.n, dtype=torch.int32, device="cuda:0")
    with pytest.raises(pkg.GkwError):
        pkg.cut_noalloc(dg, part, 9000)   # above the fixed capacity
    with pytest.raises(pkg.GkwError):
        pkg.cut_noalloc(dg, part, 0)      # no parts
    part[3] = 7
    with pytest.raises(pkg.GkwError):
        pkg.cut_noalloc(dg, part, 4)      # part id out of range
    part[3] = 0
    cut, pw = pkg.cut_noalloc(dg, part, 4)
    assert cut == 0 and pw[0] == g.n
