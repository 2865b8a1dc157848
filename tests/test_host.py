"""Host library (libbmhost): CSV formats, generator, orderings, greedy
matching and host score.  CPU only."""
import os

import numpy as np
import pytest

import bmb200 as bm
from oracle_bind import Oracle


def test_generator_deterministic_and_clean():
    A1, B1, t1, i1 = bm.gen_pair(1, n=400, m_target=5000, seed=3)
    A2, B2, t2, i2 = bm.gen_pair(1, n=400, m_target=5000, seed=3)
    for x, y in ((A1.src, A2.src), (A1.dst, A2.dst), (A1.w, A2.w), (B1.src, B2.src), (B1.w, B2.w), (t1, t2), (i1, i2)):
        np.testing.assert_array_equal(x, y)
    A3, _, _, _ = bm.gen_pair(1, n=400, m_target=5000, seed=4)
    assert not (A3.src.shape == A1.src.shape and np.array_equal(A3.src, A1.src) and np.array_equal(A3.dst, A1.dst))
    for G in (A1, B1):
        assert G.m > 0
        assert np.all(G.src != G.dst)
        assert np.all((G.w >= 1) & (G.w <= 32767))
        keys = G.src.astype(np.int64) * (G.n + 1) + G.dst
        assert np.unique(keys).shape[0] == G.m
        assert G.src.min() >= 1 and G.dst.max() <= G.n
    assert abs(A1.m - 5000) < 500
    assert bm.check_bijection(t1) == 0 and bm.check_bijection(i1) == 0
    # about 30% of the vertices reshuffled
    assert 0.15 < np.mean(i1[1:] != t1[1:]) < 0.35


def test_generator_fullscale_shape():
    A, B, truth, init = bm.gen_pair(2, n=3000, m_target=200000, seed=9, init_mode=0)
    deg = np.bincount(A.src, minlength=A.n + 1) + np.bincount(A.dst, minlength=A.n + 1)
    assert deg.max() > 8 * deg[1:].mean()  # heavy tail
    assert np.mean(A.w <= 5) > 0.7 and A.w.max() <= 3000
    # B is A relabelled with noise: most edges survive under the truth
    akeys = set((truth[A.src].astype(np.int64) * (A.n + 1) + truth[A.dst]).tolist())
    bkeys = set((B.src.astype(np.int64) * (B.n + 1) + B.dst).tolist())
    assert len(akeys & bkeys) > 0.9 * A.m


def test_graph_csv_roundtrip(tmp_path):
    A, _, _, _ = bm.gen_pair(1, n=200, m_target=1500, seed=5)
    p = str(tmp_path / "g.csv")
    bm.write_graph_csv(p, A)
    G, bad = bm.read_graph_csv(p)
    assert bad == 0 and G.n == A.src.max().clip(min=A.dst.max()) or G.n == max(A.src.max(), A.dst.max())
    np.testing.assert_array_equal(G.src, A.src)
    np.testing.assert_array_equal(G.dst, A.dst)
    np.testing.assert_array_equal(G.w, A.w)


def test_graph_csv_malformed_lines(tmp_path):
    p = tmp_path / "g.csv"
    p.write_text("from,to,weight\n1,2,3\nbad line\n 4, 5,6\n7,8\n\n9,10,-2\n")
    G, bad = bm.read_graph_csv(str(p))
    assert G.m == 3 and bad == 3
    np.testing.assert_array_equal(G.src, [1, 4, 9])
    np.testing.assert_array_equal(G.w, [3, 6, -2])


def test_mapping_formats(tmp_path):
    p1 = tmp_path / "m1.csv"
    p1.write_text("Male Node ID,Female Node ID\nm3,f1\nm1,f2\nm2,f3\n")
    p2 = tmp_path / "m2_12345.csv"
    p2.write_text("a,b\n3,1\n1,2\n2,3\n")
    for p in (p1, p2):
        pi, cnt, mx = bm.read_mapping(str(p), 3)
        np.testing.assert_array_equal(pi, [0, 2, 3, 1])
        assert cnt == 3 and mx == 3
    out = str(tmp_path / "out.csv")
    bm.write_mapping(out, np.array([0, 2, 0, 1], np.int32))
    assert open(out).read() == "Male Node ID,Female Node ID\nm1,f2\nm3,f1\n"


def test_ordering_roundtrip(tmp_path):
    A, _, _, _ = bm.gen_pair(1, n=100, m_target=800, seed=2)
    o = bm.ordering_by_weighted_degree(A)
    assert sorted(o[1:].tolist()) == list(range(1, 101))
    p = str(tmp_path / "o.csv")
    bm.write_ordering(p, o)
    np.testing.assert_array_equal(bm.read_ordering(p, 100), o)
    rows = bm.rows_from_ordering(o)
    assert o[rows[0]] == 1 and o[rows[-1]] == 100


def test_greedy_match_is_bijection_and_beats_random():
    A, B, truth, _ = bm.gen_pair(1, n=300, m_target=3000, seed=8)
    pi = bm.greedy_match(A, B)
    assert bm.check_bijection(pi) == 0
    rng = np.random.default_rng(0)
    rnd = np.concatenate([[0], rng.permutation(300) + 1]).astype(np.int32)
    assert bm.host_score(A, B, pi) > bm.host_score(A, B, rnd)


def test_host_score_matches_oracle():
    A, B, truth, init = bm.gen_pair(1, n=300, m_target=3000, seed=6)
    orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    assert bm.host_score(A, B, init) == orc.score(init)
    assert bm.host_score(A, B, truth) == orc.score(truth)


def test_bijection_check():
    assert bm.check_bijection(np.array([0, 1, 2, 3], np.int32)) == 0
    assert bm.check_bijection(np.array([0, 1, 1, 3], np.int32)) == 2
    assert bm.check_bijection(np.array([0, 1, 2, 4], np.int32)) == 3


def test_first_appearance_and_node_metrics():
    """The graph-alignment variant's vertex list (add_node order) and its
    calculate_node_metrics, against a direct computation."""
    src = np.array([5, 2, 5, 7, 2, 9], np.int32)
    dst = np.array([2, 7, 9, 5, 5, 9], np.int32)
    w = np.array([3, 1, 4, 1, 5, 9], np.int32)
    g = bm.Graph(10, src, dst, w)
    np.testing.assert_array_equal(bm.first_appearance(g), [5, 2, 7, 9])
    rank = np.arange(11, dtype=np.int32) * 10
    m = bm.node_metrics(g, rank)
    for v in range(11):
        outd, ind = int((src == v).sum()), int((dst == v).sum())
        tot = int(w[src == v].sum() + w[dst == v].sum())
        listed = v in (5, 2, 7, 9)
        exp = [ind, outd, tot / ind if ind else 0.0, tot / outd if outd else 0.0, rank[v]] if listed else [0] * 5
        np.testing.assert_array_equal(m[v], np.array(exp, np.float64))
