"""Tiered row launches: a launch of few rows runs its heaviest rows (ranked on
the device by the work estimate) in twice-wider clusters on a second stream.
Every output (full delta rows, row reductions with and without column bounds,
the device-rows entry point, reference-delta semantics) must equal the
single-launch path and the oracle bit for bit, at batch sizes on both sides
of every tier threshold, with repeated and duplicated rows."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu

# batch sizes: 1 and 20 (8-CTA clusters, no wider tier), 40, 57 and 70
# (4-CTA clusters, 8-CTA tiers while the resident clusters allow), 100 and 140
# (2-CTA clusters with 4-CTA tiers)
SIZES = (1, 20, 40, 57, 70, 100, 140)


@pytest.fixture(scope="module")
def cfg1(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    e.set_row_split(-1)
    yield n, A, B, e
    e.close()


def _rows(n, A, k, seed):
    """k rows mixing the heaviest vertices of A with light ones, shuffled,
    with one duplicate when k > 2."""
    deg = np.bincount(A[0], minlength=n + 1) + np.bincount(A[1], minlength=n + 1)
    order = np.argsort(-deg[1:], kind="stable") + 1
    rng = np.random.default_rng(seed)
    heavy = order[: max(1, k // 4)]
    light = rng.choice(order[k:], k - heavy.shape[0], replace=False)
    rows = np.concatenate([heavy, light]).astype(np.int32)
    rng.shuffle(rows)
    if k > 2:
        rows[-1] = rows[0]
    return rows


def _tier_rows(e, k):
    """Rows in the wider tier for a launch of k rows, by the library's rule:
    the cluster size c is the largest power of two up to 8 with k c <= SMs;
    below 8, H = min(k, resident c clusters - k - 1, resident 2c clusters)."""
    import ctypes as C
    v = C.c_int32()
    e.L.bm_rows_max_active_clusters(e.h, 1, 512, C.byref(v))
    sms = v.value // 2  # two CTAs per SM
    c = 1
    while c < 8 and k * c <= sms:
        c *= 2
    if c >= 8:
        return 0
    e.L.bm_rows_max_active_clusters(e.h, c, 512, C.byref(v))
    m1 = v.value
    e.L.bm_rows_max_active_clusters(e.h, 2 * c, 512, C.byref(v))
    m2 = v.value
    return max(0, min(k, m1 - k - 1, m2))


def _dev_best(e, rows):
    d_rows = e.dev_alloc(rows.nbytes)
    d_out = e.dev_alloc(bm.ROW_DTYPE.itemsize * rows.shape[0])
    try:
        e.h2d(d_rows, rows)
        c0 = e.launch_count()
        e.rows_best_dev(d_rows, None, rows.shape[0], d_out)
        launches = e.launch_count() - c0
        out = np.zeros(rows.shape[0], bm.ROW_DTYPE)
        e.d2h(out, d_out)
        e.sync()
    finally:
        e.dev_free(d_rows)
        e.dev_free(d_out)
    return out, launches


@pytest.mark.parametrize("k", SIZES)
def test_tiers_equal_single_launch_and_oracle(golden_cfg1, cfg1, k):
    n, A, B, e = cfg1
    rows = _rows(n, A, k, seed=k)
    col = np.random.default_rng(k).integers(1, n + 1, k).astype(np.int32)
    e.set_row_tiers(-1)
    try:
        base_full, base_best, base_col = e.delta_rows(rows), e.rows_best(rows), e.rows_best(rows, col)
        base_dev, l_off = _dev_best(e, rows)
        assert l_off == 1
        np.testing.assert_array_equal(base_dev, base_best)
        exp = Oracle(n, A, B).rows(golden_cfg1["pi_init"], rows[:8])
        np.testing.assert_array_equal(base_full[:8], exp)
        for tiers in (0, 3, 1000):
            e.set_row_tiers(tiers)
            np.testing.assert_array_equal(e.delta_rows(rows), base_full)
            np.testing.assert_array_equal(e.rows_best(rows), base_best)
            np.testing.assert_array_equal(e.rows_best(rows, col), base_col)
            got, launches = _dev_best(e, rows)
            np.testing.assert_array_equal(got, base_best)
            assert launches == (2 if _tier_rows(e, k) > 0 else 1), (k, tiers)
    finally:
        e.set_row_tiers(0)


def test_tiers_repeated_launches(cfg1):
    n, A, B, e = cfg1
    sets = [_rows(n, A, k, seed=100 + k) for k in (57, 40, 100, 57, 3)]
    e.set_row_tiers(-1)
    exp = [e.rows_best(r) for r in sets]
    e.set_row_tiers(0)
    for _ in range(3):
        for r, x in zip(sets, exp):
            np.testing.assert_array_equal(e.rows_best(r), x)
            np.testing.assert_array_equal(_dev_best(e, r)[0], x)


def test_tiers_reference_semantics(golden_selfloop_ref):
    """Reference-delta semantics (the REFCPU instantiation) through tiers."""
    g = golden_selfloop_ref
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    e.set_semantics("ref-cpu")
    e.set_row_split(-1)
    try:
        rows = np.resize(np.asarray(g["rows"], np.int32), 57)
        exp = np.resize(g["row_deltas"], (57, g["row_deltas"].shape[1]))
        for tiers in (-1, 0, 2):
            e.set_row_tiers(tiers)
            np.testing.assert_array_equal(e.delta_rows(rows), exp)
    finally:
        e.close()


def test_tiers_fullscale_rows_agree():
    """Full-scale pair, two 57-row batches of the weighted-degree ordering (the
    heaviest rows and a middle batch): tiered and single launches agree on
    full rows and reductions."""
    A, B, truth, init = bm.gen_pair(2, seed=2)
    order = bm.ordering_by_weighted_degree(A)
    allrows = bm.rows_from_ordering(order)
    e = bm.Engine(0)
    e.set_graphs(A, B)
    e.set_mapping(init)
    try:
        for lo in (0, A.n // 2):
            rows = np.ascontiguousarray(allrows[lo:lo + 57]).astype(np.int32)
            e.set_row_tiers(-1)
            full0, best0 = e.delta_rows(rows), e.rows_best(rows)
            dev0, _ = _dev_best(e, rows)
            np.testing.assert_array_equal(dev0, best0)
            e.set_row_tiers(0)
            np.testing.assert_array_equal(e.rows_best(rows), best0)
            dev1, launches = _dev_best(e, rows)
            assert launches == 2
            np.testing.assert_array_equal(dev1, best0)
            np.testing.assert_array_equal(e.delta_rows(rows), full0)
    finally:
        e.close()


def test_tier_setting_validation(cfg1):
    n, A, B, e = cfg1
    assert e.row_tiers() == 0
    with pytest.raises(bm.BMError):
        e.set_row_tiers(-2)
    e.set_row_tiers(5)
    assert e.row_tiers() == 5
    e.set_row_tiers(0)


def test_host_rows_graph_replays(cfg1):
    """bm_rows_best without column bounds runs as a captured CUDA graph per row
    count: replays with new rows, a new row count, changed settings and a
    changed mapping all give the device-rows path's results, and each replay
    counts its kernels."""
    n, A, B, e = cfg1
    e.set_row_tiers(0)
    for k, seed in ((57, 1), (57, 2), (57, 3), (40, 4), (57, 5), (100, 6), (100, 7)):
        rows = _rows(n, A, k, seed=200 + seed)
        c0 = e.launch_count()
        got = e.rows_best(rows)
        launches = e.launch_count() - c0
        exp, dev_launches = _dev_best(e, rows)
        np.testing.assert_array_equal(got, exp)
        assert launches == dev_launches
    rows = _rows(n, A, 57, seed=300)
    for tiers in (-1, 2, 0):
        e.set_row_tiers(tiers)
        np.testing.assert_array_equal(e.rows_best(rows), _dev_best(e, rows)[0])
        np.testing.assert_array_equal(e.rows_best(rows), _dev_best(e, rows)[0])
    # a changed mapping: the graph reads the current one
    pi0 = e.get_mapping()
    best = e.rows_best(rows)
    i = int(np.argmax(best["best_delta"]))
    assert best["best_delta"][i] > 0
    e.apply_swaps(np.array([[best["row"][i], best["best"][i]]], np.int32), np.array([best["best_delta"][i]], np.int64))
    try:
        got = e.rows_best(rows)
        np.testing.assert_array_equal(got, _dev_best(e, rows)[0])
        assert not np.array_equal(got, best)
    finally:
        e.set_mapping(pi0)
    np.testing.assert_array_equal(e.rows_best(rows), best)
