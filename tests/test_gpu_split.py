"""Split rows: a row launch with fewer rows than cluster slots spreads heavy
rows over several clusters that meet in global memory.  Every output (full
delta rows, row reductions with and without column bounds, delta-table rows)
must equal the one-cluster-per-row path and the oracle bit for bit, for every
slot count and cluster size, over repeated launches (the arrival counters
reset themselves)."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg1(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    yield n, A, B, e
    e.close()


def _skewed_rows(n, A, k, seed):
    """k rows: the heaviest vertices of A mixed with light ones, shuffled."""
    deg = np.bincount(A[0], minlength=n + 1) + np.bincount(A[1], minlength=n + 1)
    order = np.argsort(-deg[1:], kind="stable") + 1
    rng = np.random.default_rng(seed)
    heavy = order[: max(1, k // 4)]
    light = rng.choice(order[k:], k - heavy.shape[0], replace=False)
    rows = np.concatenate([heavy, light]).astype(np.int32)
    rng.shuffle(rows)
    return rows


def _outputs(e, rows, col):
    return e.delta_rows(rows), e.rows_best(rows), e.rows_best(rows, col)


@pytest.mark.parametrize("ctas", [1, 2, 4])
def test_split_equals_unsplit_and_oracle(golden_cfg1, cfg1, ctas):
    n, A, B, e = cfg1
    rows = _skewed_rows(n, A, 12, seed=ctas)
    col = np.random.default_rng(5).integers(1, n + 1, rows.shape[0]).astype(np.int32)
    exp_full = Oracle(n, A, B).rows(golden_cfg1["pi_init"], rows)
    e.set_row_tiling(ctas, 512)
    try:
        e.set_row_split(-1)
        base = _outputs(e, rows, col)
        np.testing.assert_array_equal(base[0], exp_full)
        for slots in (13, 24, 48, 100, 296):
            e.set_row_split(slots)
            got = _outputs(e, rows, col)
            np.testing.assert_array_equal(got[0], exp_full)
            np.testing.assert_array_equal(got[1], base[1])
            np.testing.assert_array_equal(got[2], base[2])
    finally:
        e.set_row_split(0)
        e.set_row_tiling(0, 512)


def test_split_repeated_launches_reset_counters(cfg1):
    n, A, B, e = cfg1
    e.set_row_split(-1)
    sets = [_skewed_rows(n, A, k, seed=k) for k in (3, 9, 1, 17, 9, 40)]
    exp = [e.rows_best(r) for r in sets]
    e.set_row_split(0)
    try:
        for _ in range(3):
            for r, x in zip(sets, exp):
                np.testing.assert_array_equal(e.rows_best(r), x)
    finally:
        e.set_row_split(0)


def test_split_table_search(golden_cfg1):
    """The delta-table search refreshes the rows around each applied swap
    through the split path; its swaps, score and table match the unsplit run."""
    n, A, B = golden_graphs(golden_cfg1)
    out = []
    for slots in (-1, 296):
        e = make_engine(n, A, B, golden_cfg1["pi_init"])
        e.set_row_split(slots)
        d_tab, ld = e.table_alloc()
        try:
            e.delta_table_dev(d_tab, ld)
            prog, st = e.search_table(d_tab, ld, k=64, max_accepts=6, max_rounds=4)
            out.append((e.get_mapping(), e.score(), e.table_download(d_tab, ld), prog.accepts))
        finally:
            e.dev_free(d_tab)
            e.close()
    (pa, sa, ta, na), (pb, sb, tb, nb) = out
    assert na == nb and na > 0
    np.testing.assert_array_equal(pa, pb)
    assert sa == sb
    np.testing.assert_array_equal(ta, tb)


def test_split_setting_validation(cfg1):
    n, A, B, e = cfg1
    assert e.row_split() == 0
    with pytest.raises(bm.BMError):
        e.set_row_split(-2)
    e.set_row_split(7)
    assert e.row_split() == 7
    e.set_row_split(0)


def test_split_fullscale_rows_agree():
    """Full-scale pair, the 57 heaviest rows of the weighted-degree ordering
    (hub rows of up to 19 item chunks): split and unsplit launches agree on
    full rows and reductions."""
    A, B, truth, init = bm.gen_pair(2, seed=2)
    order = bm.ordering_by_weighted_degree(A)
    rows = np.ascontiguousarray(bm.rows_from_ordering(order)[:57]).astype(np.int32)
    e = bm.Engine(0)
    e.set_graphs(A, B)
    e.set_mapping(init)
    try:
        e.set_row_split(-1)
        full0, best0 = e.delta_rows(rows[:8]), e.rows_best(rows)
        for slots in (0, 114):
            e.set_row_split(slots)
            np.testing.assert_array_equal(e.delta_rows(rows[:8]), full0)
            np.testing.assert_array_equal(e.rows_best(rows), best0)
    finally:
        e.close()
