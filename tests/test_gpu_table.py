"""The exact delta table (score-lookup engine): every entry against the
oracle, the device top-K against a host sort, refresh after swaps against a
fresh table, and the table search to an exact local optimum."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


def test_table_equals_oracle(golden_small):
    n, A, B = golden_graphs(golden_small)
    pi = golden_small["pi_init"]
    e = make_engine(n, A, B, pi)
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    tab = e.table_download(d_tab, ld)
    rows = np.arange(1, n + 1, dtype=np.int32)
    exp = Oracle(n, A, B).rows(pi, rows)  # (n, n+1), v = 0..n
    np.testing.assert_array_equal(tab[1:, : n + 1], exp)
    assert np.all(tab[0] == 0) and np.all(np.diag(tab[:, : n + 1]) == 0)
    np.testing.assert_array_equal(tab[:, : n + 1], tab[:, : n + 1].T)
    e.dev_free(d_tab)
    e.close()


def _host_topk(tab, n, k):
    iu, iv = np.triu_indices(n + 1, 1)
    keep = iu >= 1
    iu, iv = iu[keep], iv[keep]
    d = tab[iu, iv].astype(np.int64)
    order = np.lexsort((iv, iu, -d))[:k]
    return np.stack([iu[order], iv[order]], 1).astype(np.int32), d[order]


@pytest.mark.parametrize("k", [1, 37, 1000, 4096])
def test_topk_matches_host_sort(golden_small, k):
    n, A, B = golden_graphs(golden_small)
    e = make_engine(n, A, B, golden_small["pi_init"])
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    tab = e.table_download(d_tab, ld)
    pairs, deltas = e.table_topk(d_tab, ld, k)
    hp, hd = _host_topk(tab, n, k)
    np.testing.assert_array_equal(deltas, hd)
    np.testing.assert_array_equal(pairs, hp)
    with pytest.raises(bm.BMError):
        e.table_topk(d_tab, ld, 4097)
    e.dev_free(d_tab)
    e.close()


def test_topk_ties_in_pair_order():
    # a graph pair where most deltas are equal: ties must come in (u, v) order
    n = 120
    A = (np.array([1, 2, 3], np.int32), np.array([2, 3, 1], np.int32), np.array([5, 5, 5], np.int32))
    B = (np.array([1, 2], np.int32), np.array([2, 3], np.int32), np.array([5, 5], np.int32))
    e = make_engine(n, A, B, np.arange(n + 1, dtype=np.int32))
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    tab = e.table_download(d_tab, ld)
    for k in (5, 300, 4096):
        pairs, deltas = e.table_topk(d_tab, ld, k)
        hp, hd = _host_topk(tab, n, k)
        np.testing.assert_array_equal(pairs, hp)
        np.testing.assert_array_equal(deltas, hd)
    e.dev_free(d_tab)
    e.close()


def test_refresh_after_swaps_equals_fresh_table(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    pairs, deltas = e.table_topk(d_tab, ld, 1)
    a, b = int(pairs[0, 0]), int(pairs[0, 1])
    e.apply_swaps(np.array([[a, b]], np.int32), deltas[:1])
    nb = set([a, b])
    for x in (a, b):
        nb |= set(A[1][A[0] == x].tolist()) | set(A[0][A[1] == x].tolist())
    e.table_refresh_dev(d_tab, ld, sorted(nb))
    got = e.table_download(d_tab, ld)
    d2, ld2 = e.table_alloc()
    e.delta_table_dev(d2, ld2)
    np.testing.assert_array_equal(got[:, : n + 1], e.table_download(d2, ld2)[:, : n + 1])
    e.dev_free(d_tab)
    e.dev_free(d2)
    e.close()


def test_table_search_reaches_exact_local_optimum(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    prog, st = e.search_table(d_tab, ld, k=512)
    assert st == bm.BM_OK and prog.converged == 1
    assert e.tracked_score() == e.score() == prog.score > int(golden_cfg1["score_init"])
    res = e.rows_best(np.arange(1, n + 1, dtype=np.int32))
    assert np.all(res["best_delta"] <= 0)
    # the table stayed exact through the refreshes
    d2, ld2 = e.table_alloc()
    e.delta_table_dev(d2, ld2)
    np.testing.assert_array_equal(e.table_download(d_tab, ld)[:, : n + 1], e.table_download(d2, ld2)[:, : n + 1])
    e.dev_free(d_tab)
    e.dev_free(d2)
    e.close()
