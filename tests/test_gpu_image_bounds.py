"""The per-vertex image list bounds (the bounds of B's lists at pi x, which
the row kernel's first-hop staging reads instead of pi x) are kept by every
kernel that moves images: single swaps, k-set permutations and subset
re-assignment.  After each kind of move the row kernel's whole rows must
equal the oracle's rows at the device's current mapping, bit for bit."""
import numpy as np
import pytest

from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    yield n, A, B, e, Oracle(n, A, B)
    e.close()


def _rows(n, seed, k=12):
    return np.random.default_rng(seed).choice(np.arange(1, n + 1), k, replace=False).astype(np.int32)


def _check(e, orc, n, seed):
    rows = _rows(n, seed)
    np.testing.assert_array_equal(e.delta_rows(rows), orc.rows(e.get_mapping(), rows))


def test_rows_after_swaps(setup):
    n, A, B, e, orc = setup
    rng = np.random.default_rng(7)
    for it in range(6):
        a, b = (int(x) for x in rng.choice(np.arange(1, n + 1), 2, replace=False))
        d = int(e.delta_rows(np.array([a], np.int32))[0, b])  # keeps the tracked score exact
        e.apply_swaps(np.array([[a, b]], np.int32), np.array([d], np.int64))
        _check(e, orc, n, 100 + it)


def test_rows_after_set_permutations(setup):
    n, A, B, e, orc = setup
    rng = np.random.default_rng(8)
    for it in range(4):
        sets = rng.choice(np.arange(1, n + 1), 3, replace=False).astype(np.int32)
        best, perm = e.kset_eval(3, sets)
        e.apply_sets(3, sets, perm.reshape(-1), best)
        _check(e, orc, n, 200 + it)


def test_rows_after_subset_assignment(setup):
    n, A, B, e, orc = setup
    e.search_hungarian(k=64, seed=3, iterations=2)
    _check(e, orc, n, 300)
