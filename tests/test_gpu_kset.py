"""k-vertex permutation moves (3-vertex moves and permutation sets): every
permutation's exact delta equals the oracle's local re-scoring, the best one
is the first maximum in lexicographic order, independent sets apply with an
exact tracked score, and the search keeps its score verified."""
import itertools
import math

import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


def lex_perms(k):
    return [list(p) for p in itertools.permutations(range(k))]


def path_triples(A, n, count, rng):
    nb = [[] for _ in range(n + 1)]
    for s, d in zip(A[0], A[1]):
        nb[s].append(int(d))
        nb[d].append(int(s))
    out = []
    while len(out) < count:
        u = int(rng.integers(1, n + 1))
        if not nb[u]:
            continue
        x = nb[u][int(rng.integers(len(nb[u])))]
        y = nb[x][int(rng.integers(len(nb[x])))]
        if len({u, x, y}) == 3:
            out.append((u, x, y))
    return np.array(out, np.int32)


@pytest.mark.parametrize("k", [2, 3, 4, 5])
def test_all_permutation_deltas_match_oracle(golden_small, k):
    n, A, B = golden_graphs(golden_small)
    pi = golden_small["pi_init"]
    e = make_engine(n, A, B, pi)
    orc = Oracle(n, A, B)
    rng = np.random.default_rng(k)
    sets = [rng.choice(np.arange(1, n + 1), k, replace=False) for _ in range(6)]
    if k == 3:
        sets += list(path_triples(A, n, 10, rng))  # sets with internal edges
    sets = np.array(sets, np.int32)
    best, perm, alld = e.kset_eval(k, sets, all_deltas=True)
    perms = lex_perms(k)
    for s in range(sets.shape[0]):
        exp = np.array([orc.perm_delta(pi, sets[s], p) for p in perms], np.int64)
        np.testing.assert_array_equal(alld[s], exp)
        bi = int(np.argmax(exp))
        assert best[s] == exp[bi]
        assert list(perm[s]) == perms[bi]
    if k == 2:
        np.testing.assert_array_equal(alld[:, 1], e.delta_pairs(sets))
    e.close()


def test_eight_sets_full_enumeration(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi)
    orc = Oracle(n, A, B)
    rng = np.random.default_rng(8)
    sets = np.array([rng.choice(np.arange(1, n + 1), 8, replace=False) for _ in range(2)], np.int32)
    # a set with edges inside: a vertex and seven of its neighbours
    nb = sorted(set(A[1][A[0] == A[0][0]].tolist()))[:7]
    if len(nb) == 7:
        sets = np.vstack([sets, np.array([A[0][0]] + nb, np.int32)])
    best, perm, alld = e.kset_eval(8, sets, all_deltas=True)
    perms = lex_perms(8)
    for s in range(sets.shape[0]):
        idx = np.random.default_rng(s).choice(len(perms), 2000, replace=False)
        for i in idx:
            assert alld[s, i] == orc.perm_delta(pi, sets[s], perms[i])
        assert best[s] == alld[s].max()
        assert list(perm[s]) == perms[int(np.argmax(alld[s]))]
        assert orc.perm_delta(pi, sets[s], perm[s]) == best[s]
    e.close()


@pytest.mark.parametrize("k", [4, 5, 6, 7, 8])
def test_best_permutation_without_full_output(golden_cfg1, k):
    """Sets without internal entries take the grouped enumeration when no
    per-permutation output is asked for; best delta and permutation (lowest
    lexicographic index on ties) equal the full enumeration's and the oracle's."""
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi)
    orc = Oracle(n, A, B)
    rng = np.random.default_rng(40 + k)
    sets = np.array([rng.choice(np.arange(1, n + 1), k, replace=False) for _ in range(24)], np.int32)
    best_f, perm_f, alld = e.kset_eval(k, sets, all_deltas=True)
    best, perm = e.kset_eval(k, sets)
    np.testing.assert_array_equal(best, best_f)
    np.testing.assert_array_equal(perm, perm_f)
    perms = lex_perms(k)
    for s in range(sets.shape[0]):
        assert best[s] == alld[s].max()
        assert list(perm[s]) == perms[int(np.argmax(alld[s]))]
        assert orc.perm_delta(pi, sets[s], perm[s]) == best[s]
    e.close()


def test_selfloop_sets_exact(golden_selfloop):
    g = golden_selfloop
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    rng = np.random.default_rng(5)
    for pi in g["pis"][:3]:
        e = make_engine(n, A, B, pi)
        sets = np.array([rng.choice(np.arange(1, n + 1), 4, replace=False) for _ in range(5)], np.int32)
        _, _, alld = e.kset_eval(4, sets, all_deltas=True)
        for s in range(5):
            for j, p in enumerate(lex_perms(4)):
                q = pi.copy()
                q[sets[s]] = pi[sets[s][p]]
                assert alld[s, j] == orc.score(q) - orc.score(pi)
        e.close()


def test_apply_independent_sets(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"].copy()
    e = make_engine(n, A, B, pi)
    orc = Oracle(n, A, B)
    nbr = [set() for _ in range(n + 1)]
    for s, d in zip(A[0], A[1]):
        nbr[s].add(int(d))
        nbr[d].add(int(s))
    rng = np.random.default_rng(9)
    blocked, chosen = set(), []
    while len(chosen) < 40:
        s = [int(x) for x in rng.choice(np.arange(1, n + 1), 4, replace=False)]
        if any(v in blocked for v in s):
            continue
        chosen.append(s)
        for v in s:
            blocked |= {v} | nbr[v]
    sets = np.array(chosen, np.int32)
    best, perm = e.kset_eval(4, sets)
    e.apply_sets(4, sets, perm, best)
    for s in range(sets.shape[0]):
        pi[sets[s]] = golden_cfg1["pi_init"][sets[s][perm[s]]]
    np.testing.assert_array_equal(e.get_mapping(), pi)
    assert e.tracked_score() == e.score() == orc.score(pi) == int(golden_cfg1["score_init"]) + int(best.sum())
    rows = np.array([1, 500, 1999], np.int32)
    np.testing.assert_array_equal(e.delta_rows(rows), orc.rows(pi, rows))
    with pytest.raises(bm.BMError):
        e.apply_sets(4, np.concatenate([sets[0], sets[0]]), np.concatenate([perm[0], perm[0]]))
    e.close()


@pytest.mark.parametrize("k,mode", [(8, 0), (3, 1), (4, 0)])
def test_kset_search_keeps_exact_score(golden_cfg1, k, mode):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    prog, st = e.search_ksets(k, 512, mode=mode, seed=7, max_launches=6)
    assert prog.launches == 6 and prog.evaluated == 6 * 512 * math.factorial(k)
    assert prog.score == e.score() >= int(golden_cfg1["score_init"])
    assert prog.accepts > 0
    assert bm.check_bijection(e.get_mapping()) == 0
    e.close()
