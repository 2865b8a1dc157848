"""Parity of the device kernels with the reference: scores, pair deltas, whole
rows and row reductions, bit-exact (int64) against the golden fixtures made by
the reference's own functions and against the oracle."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng_small(golden_small):
    n, A, B = golden_graphs(golden_small)
    e = make_engine(n, A, B, golden_small["pi_init"])
    yield e
    e.close()


@pytest.fixture(scope="module")
def eng_cfg1(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    yield e
    e.close()


def reduce_rows(full, rows, col_lo=None):
    """first_pos / best / npos of full delta rows, in the kernel's convention."""
    out = []
    n = full.shape[1] - 1
    for r, u in enumerate(rows):
        lo = 1 if col_lo is None else col_lo[r]
        v = np.arange(n + 1)
        ok = (v >= lo) & (v != u) & (v >= 1)
        d = full[r]
        pos = np.nonzero(ok & (d > 0))[0]
        cand = np.nonzero(ok)[0]
        first = int(pos[0]) if pos.size else 0
        if cand.size:
            bd = d[cand].max()
            best = int(cand[np.nonzero(d[cand] == bd)[0][0]])
        else:
            bd, best = 0, 0
        out.append((u, first, best, int(pos.size), int(d[first]) if first else 0, int(bd)))
    return out


@pytest.mark.parametrize("case", ["golden_small", "golden_cfg1"])
def test_score_matches_reference(case, request):
    g = request.getfixturevalue(case)
    e = request.getfixturevalue("eng_small" if case == "golden_small" else "eng_cfg1")
    assert e.score() == int(g["score_init"])
    assert e.tracked_score() == int(g["score_init"])
    assert int(e.overlap().sum()) == 2 * int(g["score_init"])  # no self-loops: each edge at both ends


@pytest.mark.parametrize("case", ["golden_small", "golden_cfg1"])
def test_pair_deltas_match_reference(case, request):
    g = request.getfixturevalue(case)
    e = request.getfixturevalue("eng_small" if case == "golden_small" else "eng_cfg1")
    np.testing.assert_array_equal(e.delta_pairs(g["pairs"]), g["pair_deltas"])


@pytest.mark.parametrize("case", ["golden_small", "golden_cfg1"])
def test_row_deltas_match_reference(case, request):
    g = request.getfixturevalue(case)
    e = request.getfixturevalue("eng_small" if case == "golden_small" else "eng_cfg1")
    np.testing.assert_array_equal(e.delta_rows(g["rows"]), g["row_deltas"])


def test_all_rows_small_vs_oracle(golden_small, eng_small):
    n, A, B = golden_graphs(golden_small)
    orc = Oracle(n, A, B)
    rows = np.arange(1, n + 1, dtype=np.int32)
    np.testing.assert_array_equal(eng_small.delta_rows(rows), orc.rows(golden_small["pi_init"], rows))


def test_rows_best_matches_full_rows(golden_cfg1, eng_cfg1):
    rng = np.random.default_rng(1)
    rows = rng.choice(np.arange(1, 2001), 96, replace=False).astype(np.int32)
    full = eng_cfg1.delta_rows(rows)
    col = rng.integers(1, 2001, rows.shape[0]).astype(np.int32)
    for cl in (None, col):
        res = eng_cfg1.rows_best(rows, cl)
        exp = reduce_rows(full, rows, cl)
        got = [tuple(int(x) for x in r) for r in res]
        assert got == exp


@pytest.mark.parametrize("ctas,threads", [(1, 256), (1, 512), (2, 512), (3, 512), (4, 256), (5, 256), (7, 512),
                                          (8, 512)])
def test_row_tiling_variants_agree(golden_cfg1, eng_cfg1, ctas, threads):
    rows = np.arange(1, 2001, 37, dtype=np.int32)
    exp = Oracle(*golden_graphs(golden_cfg1)).rows(golden_cfg1["pi_init"], rows)
    eng_cfg1.set_row_tiling(ctas, threads)
    try:
        np.testing.assert_array_equal(eng_cfg1.delta_rows(rows), exp)
        masked = exp[:, 1:].copy()
        masked[np.arange(rows.shape[0]), rows - 1] = np.iinfo(np.int64).min
        np.testing.assert_array_equal(eng_cfg1.rows_best(rows)["best_delta"], masked.max(axis=1))
    finally:
        eng_cfg1.set_row_tiling(0, 512)


def test_apply_updates_state(golden_small):
    n, A, B = golden_graphs(golden_small)
    pi = golden_small["pi_init"].copy()
    orc = Oracle(n, A, B)
    e = make_engine(n, A, B, pi)
    rng = np.random.default_rng(3)
    for _ in range(25):
        u, v = rng.choice(np.arange(1, n + 1), 2, replace=False)
        d = int(e.delta_pairs(np.array([u, v], np.int32))[0])
        assert d == orc.delta(pi, u, v)
        e.apply_swaps(np.array([u, v], np.int32), np.array([d], np.int64))
        pi[u], pi[v] = pi[v], pi[u]
        np.testing.assert_array_equal(e.get_mapping(), pi)
        assert e.tracked_score() == orc.score(pi)
    ov_inc = e.overlap()
    assert e.score() == orc.score(pi)  # recomputes the overlap from scratch
    np.testing.assert_array_equal(e.overlap(), ov_inc)
    rows = rng.choice(np.arange(1, n + 1), 8, replace=False).astype(np.int32)
    np.testing.assert_array_equal(e.delta_rows(rows), orc.rows(pi, rows))
    e.close()


def test_batch_apply_independent_swaps(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"].copy()
    e = make_engine(n, A, B, pi)
    orc = Oracle(n, A, B)
    # build an independent set of swaps greedily on the host
    nb = [set() for _ in range(n + 1)]
    for s, d in zip(A[0], A[1]):
        nb[s].add(d)
        nb[d].add(s)
    rng = np.random.default_rng(4)
    blocked, pairs = set(), []
    for _ in range(400):
        u, v = (int(x) for x in rng.choice(np.arange(1, n + 1), 2, replace=False))
        if u in blocked or v in blocked:
            continue
        pairs.append((u, v))
        blocked |= {u, v} | nb[u] | nb[v]
    pairs = np.array(pairs, np.int32)
    d = e.delta_pairs(pairs)
    e.apply_swaps(pairs, d)
    for u, v in pairs:
        pi[u], pi[v] = pi[v], pi[u]
    np.testing.assert_array_equal(e.get_mapping(), pi)
    assert e.tracked_score() == orc.score(pi) == int(golden_cfg1["score_init"]) + int(d.sum())
    e.close()


def test_batch_apply_rejects_dependent_swaps(golden_small):
    n, A, B = golden_graphs(golden_small)
    e = make_engine(n, A, B, golden_small["pi_init"])
    u, v = int(A[0][0]), int(A[1][0])  # an A edge u -> v
    w = next(x for x in range(1, n + 1) if x not in (u, v))
    z = next(x for x in range(1, n + 1) if x not in (u, v, w))
    with pytest.raises(bm.BMError) as ei:
        e.apply_swaps(np.array([u, w, v, z], np.int32))
    assert ei.value.status == bm.BM_INVALID_ARG
    np.testing.assert_array_equal(e.get_mapping(), golden_small["pi_init"])
    e.close()


def test_selfloops_duplicates_exact(golden_selfloop):
    g = golden_selfloop
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    for pi, s, (u, v), s2 in zip(g["pis"], g["scores"], g["swaps"], g["swapped_scores"]):
        e = make_engine(n, A, B, pi)
        assert e.score() == s
        assert int(e.delta_pairs(np.array([u, v], np.int32))[0]) == s2 - s
        rows = np.arange(1, n + 1, dtype=np.int32)
        full = e.delta_rows(rows)
        exp = np.array([[0 if (v2 == 0 or v2 == r) else orc.exact_delta(pi, r, v2) for v2 in range(n + 1)]
                        for r in rows])
        np.testing.assert_array_equal(full, exp)
        allp = np.array([(r, c) for r in rows for c in range(1, n + 1)], np.int32)
        np.testing.assert_array_equal(e.delta_pairs(allp).reshape(n, n), full[:, 1:])
        e.close()


def test_tiny_and_empty_graphs():
    for n, A, B in [
        (2, ([1], [2], [5]), ([2], [1], [3])),
        (3, ([1, 2, 3], [2, 3, 1], [1, 2, 3]), ([1, 2], [2, 3], [3, 3])),
        (5, ([], [], []), ([], [], [])),
    ]:
        A = tuple(np.array(x, np.int32) for x in A)
        B = tuple(np.array(x, np.int32) for x in B)
        orc = Oracle(n, A, B)
        pi = np.arange(n + 1, dtype=np.int32)
        pi[1:] = pi[1:][::-1]
        e = make_engine(n, A, B, pi)
        assert e.score() == orc.score(pi)
        rows = np.arange(1, n + 1, dtype=np.int32)
        np.testing.assert_array_equal(e.delta_rows(rows), orc.rows(pi, rows))
        e.close()


def test_invalid_arguments(golden_small):
    n, A, B = golden_graphs(golden_small)
    e = bm.Engine(0)
    with pytest.raises(bm.BMError):
        e.set_mapping(golden_small["pi_init"])  # graphs not set
    e.set_graphs(bm.Graph(n, *A), bm.Graph(n, *B))
    bad = golden_small["pi_init"].copy()
    bad[2] = bad[1]
    for pi in (bad, np.zeros(n + 1, np.int32)):
        with pytest.raises(bm.BMError) as ei:
            e.set_mapping(pi)
        assert ei.value.status == bm.BM_INVALID_ARG
    with pytest.raises(bm.BMError):
        e.set_graph(bm.SIDE_A, bm.Graph(n, [1], [n + 1], [1]))
    with pytest.raises(bm.BMError):
        e.set_graph(bm.SIDE_A, bm.Graph(n, [1], [2], [40000]))
    with pytest.raises(bm.BMError):
        e.set_graph(bm.SIDE_B, bm.Graph(n, [1], [2], [-1]))
    with pytest.raises(bm.BMError):
        e.set_graph(bm.SIDE_B, bm.Graph(n + 1, [1], [2], [1]))  # n differs from A
    e.set_mapping(golden_small["pi_init"])
    with pytest.raises(bm.BMError):
        e.delta_pairs(np.array([1, n + 1], np.int32))
    with pytest.raises(bm.BMError):
        e.delta_rows(np.array([0], np.int32))
    with pytest.raises(bm.BMError):
        e.set_row_tiling(9, 0)
    assert e.score() == int(golden_small["score_init"])  # context still usable
    e.close()


def test_fullscale_properties():
    """At the full-scale size (n = 18,524, ~3M edges): rows agree with pairs,
    delta(u,v) = delta(v,u), a sample agrees with the oracle, the tracked
    score with the host score, and the overlap sums to twice the score."""
    A, B, truth, init = bm.gen_pair(2, init_mode=0, seed=2)
    n = A.n
    e = bm.Engine(0)
    e.set_graphs(A, B)
    e.set_mapping(init)
    s = e.score()
    assert s == bm.host_score(A, B, init)
    assert int(e.overlap().sum()) == 2 * s
    rng = np.random.default_rng(7)
    rows = rng.choice(np.arange(1, n + 1), 40, replace=False).astype(np.int32)
    full = e.delta_rows(rows)
    cols = rng.integers(1, n + 1, size=(rows.shape[0], 64))
    pairs = np.stack([np.repeat(rows, 64), cols.reshape(-1)], axis=1).astype(np.int32)
    d = e.delta_pairs(pairs)
    exp = full[np.repeat(np.arange(rows.shape[0]), 64), cols.reshape(-1)]
    exp[pairs[:, 0] == pairs[:, 1]] = 0
    np.testing.assert_array_equal(d, exp)
    # symmetry through the whole-row path
    sym = e.delta_rows(cols[:4, 0].astype(np.int32))
    np.testing.assert_array_equal(sym[np.arange(4), rows[:4]], full[np.arange(4), cols[:4, 0]])
    orc = Oracle(n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    np.testing.assert_array_equal(d[:300], orc.pairs(init, pairs[:300]))
    res = e.rows_best(rows)
    masked = full[:, 1:].copy()
    masked[np.arange(rows.shape[0]), rows - 1] = np.iinfo(np.int64).min
    np.testing.assert_array_equal(res["best_delta"], masked.max(axis=1))
    e.close()
