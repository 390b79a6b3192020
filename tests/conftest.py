import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__ as ge  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    return ge.load_package()


@pytest.fixture(scope="session")
def gen():
    return ge.load_generators()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def handle(pkg):
    h = pkg.Handle(0)
    yield h
    h.close()


def to_dev(g):
    import torch
    dev = torch.device("cuda:0")
    return tuple(torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev)
                 for a in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
