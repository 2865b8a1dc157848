"""Parity at the bench's full scale, against the reference's own functions.

The full-scale pair (n = 18,524, ~3M directed edges per graph, greedy
initial matching, ordering-driven rows) is the workload the bench times; here
every schedule that runs on it is pinned to the reference
(oracle/_ref/libref.so, src/graph-alignment-optimized-parallel.c compiled
unmodified) or to the oracle's exact restatements, within a test's budget:

* the parity sweep: the first accepts of the reference's serial loop
  (optimize_mapping, src/graph-alignment-optimized.c:513-580, with its
  re-score after every accept), same final mapping, score and accept count;
* whole rows: eight rows of the timed batches against the reference's
  calculate_swap_delta under its OpenMP m2 sweep, every partner;
* k-sets: 2-path 3-sets with all six permutations and random 8-sets with the
  best permutation and a sample of the rest, against the oracle's local
  re-scoring;
* an annealing chain at the size of the batched-chain workload (n = 17,000,
  E = 80 n, 10^5 steps) replayed bit for bit by the oracle, for one and for
  eight speculative candidates per iteration.
"""
import numpy as np
import pytest

import bmb200 as bm
from oracle_bind import Oracle, Reference, ref_available

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref/libref.so not built")


@pytest.fixture(scope="module")
def full():
    A, B, truth, init = bm.gen_pair(2)
    rows = bm.rows_from_ordering(bm.ordering_by_weighted_degree(A))
    eng = bm.Engine(0)
    eng.set_graphs(A, B)
    eng.set_mapping(init)
    yield A, B, init, rows, eng
    eng.close()


@pytest.fixture(scope="module")
def reference(full):
    A, B, init, rows, eng = full
    ref = Reference(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    yield ref
    ref.close()


@needs_ref
def test_fullscale_score_equals_reference(full, reference):
    A, B, init, rows, eng = full
    assert eng.score() == reference.score(init)


@needs_ref
def test_fullscale_rows_equal_reference(full, reference):
    """Eight whole rows (18,523 partners each) of the bench's batches: the
    first row of evenly spaced batches over the ordering pass."""
    A, B, init, rows, eng = full
    n = A.n
    pick = rows[[(k * n) // 8 for k in range(8)]].astype(np.int32)
    got = eng.delta_rows(pick)
    exp = reference.rows(init, pick)
    np.testing.assert_array_equal(got, exp)
    best = eng.rows_best(pick)
    for r in range(len(pick)):
        d = exp[r].copy()
        d[0] = np.iinfo(np.int64).min
        d[pick[r]] = np.iinfo(np.int64).min
        assert best["best_delta"][r] == d.max()
        assert best["best"][r] == int(np.argmax(d))
        assert best["npos"][r] == int((exp[r] > 0).sum())


@needs_ref
@pytest.mark.parametrize("accepts", [60])
def test_fullscale_parity_sweep_equals_reference_loop(full, reference, accepts):
    """The serial first-improvement loop from the greedy matching in ordering
    order, bounded to its first accepts: the reference (with its full
    re-score after every accept) and the engine's speculative rows agree on
    the mapping, the score and the accept count."""
    A, B, init, rows, eng = full
    pi_r, s_r, log_r, _, _ = reference.serial(init, rows=rows, max_accepts=accepts, verify=True)
    eng.set_mapping(init)
    prog, st = eng.sweep_parity(rows=rows, max_accepts=accepts)
    assert prog.accepts == len(log_r) == accepts
    np.testing.assert_array_equal(eng.get_mapping(), pi_r)
    assert prog.score == s_r == eng.score()
    eng.set_mapping(init)


def path_triples(A, n, count, rng):
    """3-sets along 2-paths u - x - y (either edge direction), distinct."""
    order = np.argsort(A.src, kind="stable")
    src, dst = A.src[order], A.dst[order]
    ptr = np.searchsorted(src, np.arange(0, n + 2))
    out = []
    while len(out) < count:
        e = int(rng.integers(0, len(src)))
        u, x = int(src[e]), int(dst[e])
        deg = ptr[x + 1] - ptr[x]
        if deg == 0:
            continue
        y = int(dst[ptr[x] + int(rng.integers(deg))])
        if len({u, x, y}) == 3:
            out.append((u, x, y))
    return np.array(out, np.int32)


def test_fullscale_3sets_equal_oracle(full):
    A, B, init, rows, eng = full
    n = A.n
    orc = Oracle(n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    rng = np.random.default_rng(44)
    sets = path_triples(A, n, 300, rng)
    best, perm, alld = eng.kset_eval(3, sets, all_deltas=True)
    import itertools
    perms = [list(p) for p in itertools.permutations(range(3))]
    for s in range(len(sets)):
        exp = np.array([orc.perm_delta(init, sets[s], p) for p in perms], np.int64)
        np.testing.assert_array_equal(alld[s], exp)
        assert best[s] == exp.max()
        assert list(perm[s]) == perms[int(np.argmax(exp))]


def test_fullscale_8sets_equal_oracle(full):
    """Random 8-subsets: the best permutation's delta, and 64 sampled
    permutations of each set (of all 40,320), against the oracle."""
    A, B, init, rows, eng = full
    n = A.n
    orc = Oracle(n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    rng = np.random.default_rng(45)
    sets = np.stack([rng.choice(n, 8, replace=False) + 1 for _ in range(120)]).astype(np.int32)
    best, perm, alld = eng.kset_eval(8, sets, all_deltas=True)
    import itertools
    lex = list(itertools.permutations(range(8)))
    for s in range(len(sets)):
        assert best[s] == alld[s].max()
        assert orc.perm_delta(init, sets[s], perm[s]) == best[s]
        assert tuple(perm[s]) == lex[int(np.argmax(alld[s]))]
        for j in rng.choice(len(lex), 64, replace=False):
            assert alld[s][j] == orc.perm_delta(init, sets[s], list(lex[j]))


@pytest.mark.parametrize("candidates", [1, 8])
def test_chain_at_batched_chain_size_replays_on_cpu(candidates):
    A, B, truth, init = bm.gen_pair(3, n=17000, m_target=80 * 17000, seed=301)
    eng = bm.Engine(0)
    batch = bm.Batch(eng)
    try:
        batch.add_pair(A, B)
        steps = 100_000
        pis, scores, acc, st = batch.sa_run([0], [1234], [init], steps, t0=5.0, t_end=0.01,
                                            candidates=candidates, chunk=25_000)
        orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
        pi_o, s_o, a_o = orc.sa(init, 1234, steps, 5.0, 0.01)
        np.testing.assert_array_equal(pis[0], pi_o)
        assert scores[0] == s_o == orc.score(pis[0])
        assert acc[0] == a_o
    finally:
        batch.close()
        eng.close()
