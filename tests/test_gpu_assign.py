"""Independent-subset re-assignment: the device auction against scipy's
optimal assignment, and the subset re-assignment's exact delta against the
oracle's one-sided gains solved on the host."""
import numpy as np
import pytest
from scipy.optimize import linear_sum_assignment

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k,lo,hi,seed", [(1, -5, 5, 1), (2, -5, 5, 2), (7, 0, 3, 3), (64, -1000, 1000, 4),
                                          (300, -3, 3, 5), (1000, -50000, 50000, 6)])
def test_auction_is_optimal(k, lo, hi, seed):
    rng = np.random.default_rng(seed)
    a = rng.integers(lo, hi + 1, (k, k)).astype(np.int32)
    with bm.Engine(0) as e:
        assign, total = e.lap_solve(a)
    assert sorted(assign.tolist()) == list(range(k))
    r, c = linear_sum_assignment(a, maximize=True)
    assert total == int(a[r, c].sum()) == int(a[np.arange(k), assign].sum())


def _independent_subset(n, A, k, seed):
    rng = np.random.default_rng(seed)
    adj = [set() for _ in range(n + 1)]
    for s, d in zip(A[0].tolist(), A[1].tolist()):
        adj[s].add(d)
        adj[d].add(s)
    taken, blocked = [], set()
    for v in rng.permutation(np.arange(1, n + 1)).tolist():
        if v in blocked:
            continue
        taken.append(v)
        blocked |= adj[v] | {v}
        if len(taken) == k:
            break
    return np.array(taken, np.int32), adj


def test_subset_assign_exact_and_optimal(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"].copy()
    orc = Oracle(n, A, B)
    subset, adj = _independent_subset(n, A, 24, 7)
    k = len(subset)
    base = orc.score(pi)
    # one-sided gains from the oracle's score of the (non-bijective) moved mapping
    c = np.zeros((k, k), np.int64)
    for i in range(k):
        for j in range(k):
            if i != j:
                m = pi.copy()
                m[subset[i]] = pi[subset[j]]
                c[i, j] = orc.score(m) - base
    r, col = linear_sum_assignment(c, maximize=True)
    best = int(c[r, col].sum())
    e = make_engine(n, A, B, pi)
    delta, changed = e.subset_assign(subset)
    assert delta == best >= 0
    assert e.tracked_score() == e.score() == base + delta == orc.score(e.get_mapping())
    assert bm.check_bijection(e.get_mapping()) == 0
    # members adjacent in A are refused
    s0 = int(A[0][0]), int(A[1][0])
    with pytest.raises(bm.BMError):
        e.subset_assign(np.array(s0, np.int32))
    e.close()


def test_search_hungarian_improves_exactly(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    s0 = e.score()
    prog, st = e.search_hungarian(k=512, seed=3, iterations=6)
    assert st == bm.BM_OK
    assert e.tracked_score() == e.score() == prog.score > s0
    assert bm.check_bijection(e.get_mapping()) == 0
    e.close()
