"""The greedy-similarity initial matching pinned to the reference's own
greedy-match (src/greedy-match.c:450-530, compiled unmodified into
oracle/_ref/greedy-match by oracle/Makefile).

The fixture tests/golden/golden_greedy.npz holds the reference binary's
matchings of three generated pairs (its run takes minutes on the largest);
the host restatement bm_greedy_match must equal them, and, where the binary
is present, equal a live run on a small pair too.  The device version is
checked against the same fixture in tests/test_gpu_greedy.py."""
import os
import subprocess

import numpy as np
import pytest

import bmb200 as bm
from conftest import load_golden, REPO

GREEDY_BIN = os.path.join(REPO, "oracle", "_ref", "greedy-match")


def edge_digest(g):
    h = (g.src.astype(np.uint64) * np.uint64(1000003) + g.dst.astype(np.uint64)) * np.uint64(65599) \
        + g.w.astype(np.uint64)
    return np.uint64(np.bitwise_xor.reduce(h * np.uint64(0x9E3779B97F4A7C15)))


def greedy_cases():
    g = load_golden("golden_greedy.npz")
    out = []
    i = 0
    while f"case{i}" in g:
        config, seed, n, m = (int(x) for x in g[f"case{i}"])
        out.append((config, seed, n, m, g[f"digest{i}"], g[f"pi{i}"]))
        i += 1
    return out


def fixture_pair(case):
    config, seed, n, m, digest, pi = case
    A, B, truth, init = bm.gen_pair(config, n=n, m_target=m, seed=seed)
    assert edge_digest(A) == digest[0] and edge_digest(B) == digest[1], "the generator changed: remake the fixture"
    return A, B, pi


@pytest.mark.parametrize("idx", range(3))
def test_host_greedy_equals_reference_fixture(idx):
    A, B, pi_ref = fixture_pair(greedy_cases()[idx])
    assert (pi_ref[1:] > 0).all()
    np.testing.assert_array_equal(bm.greedy_match(A, B), pi_ref)


@pytest.mark.skipif(not os.path.exists(GREEDY_BIN), reason="oracle/_ref/greedy-match not built")
def test_host_greedy_equals_live_reference(tmp_path):
    A, B, truth, init = bm.gen_pair(1, n=600, m_target=9000, seed=31)
    ga, gb, out = (str(tmp_path / f) for f in ("g1.csv", "g2.csv", "match.csv"))
    bm.write_graph_csv(ga, A)
    bm.write_graph_csv(gb, B)
    subprocess.run([GREEDY_BIN, ga, gb, out], check=True, stdout=subprocess.DEVNULL)
    ref = np.loadtxt(out, delimiter=",", skiprows=1, dtype=np.int64).reshape(-1, 2)
    assert len(ref) == A.n  # every vertex has an edge: the reference's node list is 1..n
    pi_ref = np.zeros(A.n + 1, np.int32)
    pi_ref[ref[:, 0]] = ref[:, 1]
    np.testing.assert_array_equal(bm.greedy_match(A, B), pi_ref)
