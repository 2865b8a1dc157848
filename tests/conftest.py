import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "brain-match_b200", "python"))
sys.path.insert(0, HERE)

GOLDEN = os.path.join(HERE, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name))
    return {k: z[k] for k in z.files}


def golden_graphs(g):
    A = (g["a_src"], g["a_dst"], g["a_w"])
    B = (g["b_src"], g["b_dst"], g["b_w"])
    return int(g["n"]), A, B


@pytest.fixture(scope="session")
def golden_small():
    return load_golden("golden_small.npz")


@pytest.fixture(scope="session")
def golden_cfg1():
    return load_golden("golden_cfg1.npz")


@pytest.fixture(scope="session")
def golden_selfloop():
    return load_golden("golden_selfloop.npz")


@pytest.fixture(scope="session")
def golden_selfloop_ref():
    return load_golden("golden_selfloop_ref.npz")


@pytest.fixture(scope="session")
def golden_simfilter():
    return load_golden("golden_simfilter.npz")


def make_engine(n, A, B, pi):
    """An engine holding graphs A, B (edge-array triples) and mapping pi."""
    import bmb200 as bm
    eng = bm.Engine(0)
    eng.set_graphs(bm.Graph(n, *A), bm.Graph(n, *B))
    eng.set_mapping(pi)
    return eng
