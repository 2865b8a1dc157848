"""Greedy-similarity initial matching on the device equals the host
restatement of src/greedy-match.c (same features, same order, same ties)."""
import time

import numpy as np
import pytest

import bmb200 as bm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config,kw", [(1, {}), (1, {"n": 300, "m_target": 3000, "seed": 5}), (3, {"n": 2500, "m_target": 60000, "seed": 9})])
def test_device_greedy_equals_host(config, kw):
    A, B, truth, init = bm.gen_pair(config, **kw)
    with bm.Engine(0) as e:
        got = e.greedy_match(A, B)
    np.testing.assert_array_equal(got, bm.greedy_match(A, B))
    assert bm.check_bijection(got) == 0


def test_device_greedy_duplicates_and_self_loops():
    # duplicate edges count in degrees and reach, like the reference's lists
    rng = np.random.default_rng(2)
    n = 150
    src = rng.integers(1, n + 1, 1200).astype(np.int32)
    dst = rng.integers(1, n + 1, 1200).astype(np.int32)
    src = np.concatenate([src, src[:100], np.arange(1, 11, dtype=np.int32)])
    dst = np.concatenate([dst, dst[:100], np.arange(1, 11, dtype=np.int32)])
    w = np.ones_like(src)
    A = bm.Graph(n, src, dst, w)
    perm = rng.permutation(n) + 1
    B = bm.Graph(n, perm[src - 1].astype(np.int32), perm[dst - 1].astype(np.int32), w)
    with bm.Engine(0) as e:
        got = e.greedy_match(A, B)
        np.testing.assert_array_equal(got, bm.greedy_match(A, B))
        with pytest.raises(bm.BMError):
            e.greedy_match(bm.Graph(n, np.array([0], np.int32), np.array([1], np.int32), np.array([1], np.int32)), B)


def test_device_greedy_full_scale():
    A, B, truth, init = bm.gen_pair(2, init_mode=0)
    t = time.perf_counter()
    host = bm.greedy_match(A, B)
    th = time.perf_counter() - t
    with bm.Engine(0) as e:
        e.greedy_match(A, B)  # first call pays module load and allocations
        t = time.perf_counter()
        got = e.greedy_match(A, B)
        td = time.perf_counter() - t
    np.testing.assert_array_equal(got, host)
    print(f"greedy matching n={A.n}: host {th:.3f} s, device {td:.3f} s")


@pytest.mark.parametrize("idx", range(3))
def test_device_greedy_equals_reference_fixture(idx):
    """The device matching equals the reference greedy-match binary's output
    (tests/golden/golden_greedy.npz, made by oracle/_ref/greedy-match)."""
    from test_ref_greedy import fixture_pair, greedy_cases
    A, B, pi_ref = fixture_pair(greedy_cases()[idx])
    with bm.Engine(0) as e:
        got = e.greedy_match(A, B)
    np.testing.assert_array_equal(got, pi_ref)
