"""Reference-delta semantics (bm_set_semantics).  On a pair with self-loops
the engine returns the reference's own calculate_swap_delta values
(src/graph-alignment-optimized.c:321-408) for pairs, whole rows and the delta
table, and its parity sweep makes the reference serial loop's accepts; the
reported score is the re-computed one, as in the reference loop
(:571-576).  Exact semantics stays the score difference."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


def _engine(g, mode):
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    e.set_semantics(mode)
    return e


def test_semantics_setting(golden_selfloop_ref):
    e = _engine(golden_selfloop_ref, "exact")
    assert e.semantics() == "exact"
    e.set_semantics("ref-cpu")
    assert e.semantics() == "ref-cpu"
    with pytest.raises(ValueError):
        e.set_semantics("approx")
    assert e.L.bm_set_semantics(e.h, 7) == bm.BM_INVALID_ARG
    assert e.semantics() == "ref-cpu"
    e.close()


def test_pairs_equal_reference_deltas(golden_selfloop_ref):
    g = golden_selfloop_ref
    n, A, B = golden_graphs(g)
    e = _engine(g, "ref-cpu")
    np.testing.assert_array_equal(e.delta_pairs(g["pairs"]), g["pair_deltas"])
    e.set_semantics("exact")
    orc = Oracle(n, A, B)
    exact = np.array([orc.exact_delta(g["pi_init"], u, v) if u != v else 0 for u, v in g["pairs"]])
    np.testing.assert_array_equal(e.delta_pairs(g["pairs"]), exact)
    e.close()


@pytest.mark.parametrize("ctas,threads", [(0, 512), (1, 256), (3, 512), (8, 512)])
def test_rows_equal_reference_deltas(golden_selfloop_ref, ctas, threads):
    g = golden_selfloop_ref
    rows = g["rows"]
    e = _engine(g, "ref-cpu")
    e.set_row_tiling(ctas, threads)
    np.testing.assert_array_equal(e.delta_rows(rows), g["row_deltas"])
    masked = g["row_deltas"][:, 1:].copy()
    masked[np.arange(rows.shape[0]), rows - 1] = np.iinfo(np.int64).min
    np.testing.assert_array_equal(e.rows_best(rows)["best_delta"], masked.max(axis=1))
    e.close()


def test_split_rows_equal_reference_deltas(golden_selfloop_ref):
    g = golden_selfloop_ref
    e = _engine(g, "ref-cpu")
    e.set_row_split(32)
    np.testing.assert_array_equal(e.delta_rows(g["rows"]), g["row_deltas"])
    e.close()


def test_table_equals_reference_rows(golden_selfloop_ref):
    g = golden_selfloop_ref
    n, A, B = golden_graphs(g)
    e = _engine(g, "ref-cpu")
    d_tab, ld = e.table_alloc()
    e.delta_table_dev(d_tab, ld)
    tab = e.table_download(d_tab, ld)
    exp = Oracle(n, A, B).rows(g["pi_init"], np.arange(1, n + 1, dtype=np.int32))  # calculate_swap_delta, restated
    np.testing.assert_array_equal(tab[1:, : n + 1], exp)
    e.dev_free(d_tab)
    e.close()


def test_parity_sweep_makes_reference_accepts(golden_selfloop_ref):
    g = golden_selfloop_ref
    e = _engine(g, "ref-cpu")
    prog, st = e.sweep_parity(max_sweeps=int(g["serial_max_sweeps"]))
    assert st == bm.BM_OK
    assert prog.accepts == int(g["serial_accepts"])
    assert (prog.sweeps, prog.converged) == (int(g["serial_sweeps"]), int(g["serial_converged"]))
    np.testing.assert_array_equal(e.get_mapping(), g["serial_pi"])
    assert prog.score == e.score() == int(g["serial_score"])
    e.close()
    e = _engine(g, "ref-cpu")
    prog, _ = e.sweep_parity(max_accepts=100)
    np.testing.assert_array_equal(e.get_mapping(), g["serial100_pi"])
    assert prog.score == int(g["serial100_score"])
    e.close()


def test_batched_search_and_perturb_keep_the_true_score(golden_selfloop_ref):
    g = golden_selfloop_ref
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    e = _engine(g, "ref-cpu")
    prog, st = e.search_batched(max_sweeps=3)
    assert st in (bm.BM_OK, bm.BM_TIMEOUT)
    assert prog.score == e.score() == orc.score(e.get_mapping())
    s0 = e.tracked_score()
    _, total = e.perturb(5, seed=3)
    assert e.tracked_score() == s0 + total == orc.score(e.get_mapping())
    e.close()


def test_loop_free_pair_is_unchanged(golden_small):
    g = golden_small
    e = _engine(g, "ref-cpu")
    np.testing.assert_array_equal(e.delta_pairs(g["pairs"]), g["pair_deltas"])
    np.testing.assert_array_equal(e.delta_rows(g["rows"]), g["row_deltas"])
    e.close()
