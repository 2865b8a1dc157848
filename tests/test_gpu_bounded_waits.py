"""Device-side waits that run out end their call with BM_TIMEOUT and leave the
context usable.

The tensor-core MLP scorer waits on an mbarrier for each MMA completion, and
the auction of the subset assignment runs under a clock bound.  bm_set_wait_limit
lowers both bounds to one SM cycle, so every such wait gives up on its first
check (no GPU fault is involved: the scorer then sets its error flag, waits
with the default bound for the MMAs it issued, frees its tensor memory and
returns).  Each test asserts the BM_TIMEOUT status and its message, that the
error flag is cleared (the next check reports nothing), and that the next call
on the same context, with the default bounds back, gives the same results as
before."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine

pytestmark = pytest.mark.gpu


def test_mlp_mma_wait_runs_out_and_context_recovers(golden_small):
    n, A, B = golden_graphs(golden_small)
    eng = make_engine(n, A, B, golden_small["pi_init"])
    try:
        m = bm.Mlp(eng, seed=1)
        rows = np.array([3, 77, 200], np.int32)
        good = m.score_rows(rows)
        assert eng.L.bm_set_wait_limit(eng.h, 1) == bm.BM_OK
        with pytest.raises(bm.BMError) as ex:
            m.score_rows(rows)
        assert ex.value.status == bm.BM_TIMEOUT
        assert b"MMA completion wait ran out" in eng.L.bm_ctx_last_error(eng.h)
        assert eng.L.bm_set_wait_limit(eng.h, 0) == bm.BM_OK
        m.status()  # the flag was cleared when it was reported
        np.testing.assert_array_equal(m.score_rows(rows), good)
        assert eng.score() == int(golden_small["score_init"])
        np.testing.assert_array_equal(eng.delta_rows(rows), eng.delta_rows(rows))
    finally:
        eng.close()


def test_auction_bound_runs_out_and_context_recovers():
    rng = np.random.default_rng(3)
    k = 300
    benefit = rng.integers(-1000, 1000, size=(k, k)).astype(np.int32)
    with bm.Engine(0) as eng:
        assign, total = eng.lap_solve(benefit)
        assert eng.L.bm_set_wait_limit(eng.h, 1) == bm.BM_OK
        with pytest.raises(bm.BMError) as ex:
            eng.lap_solve(benefit)
        assert ex.value.status == bm.BM_TIMEOUT
        assert b"auction did not finish within its bound" in eng.L.bm_ctx_last_error(eng.h)
        assert eng.L.bm_set_wait_limit(eng.h, 0) == bm.BM_OK
        a2, t2 = eng.lap_solve(benefit)
        assert t2 == total
        np.testing.assert_array_equal(np.sort(a2), np.arange(k))


def test_wait_limit_rejects_negative():
    with bm.Engine(0) as eng:
        assert eng.L.bm_set_wait_limit(eng.h, -5) == bm.BM_INVALID_ARG


def test_training_mma_wait_runs_out_and_context_recovers(golden_small):
    """The tensor-core training kernel's MMA-completion waits, run out the
    same way: BM_TIMEOUT, then the same gradient as before."""
    n, A, B = golden_graphs(golden_small)
    eng = make_engine(n, A, B, golden_small["pi_init"])
    try:
        m = bm.Mlp(eng, seed=2)
        rng = np.random.default_rng(9)
        pairs = rng.integers(1, n + 1, (400, 2)).astype(np.int32)
        pairs = pairs[pairs[:, 0] != pairs[:, 1]][:300]
        x = m.pair_features(pairs)
        y = rng.normal(0.0, 0.5, x.shape[0]).astype(np.float32)
        g0, l0 = m.gradients(x, y)
        assert eng.L.bm_set_wait_limit(eng.h, 1) == bm.BM_OK
        with pytest.raises(bm.BMError) as ex:
            m.gradients(x, y)
        assert ex.value.status == bm.BM_TIMEOUT
        assert eng.L.bm_set_wait_limit(eng.h, 0) == bm.BM_OK
        g1, l1 = m.gradients(x, y)
        # the same up to the order of the CTAs' atomic additions
        assert np.linalg.norm(g1 - g0) <= 1e-5 * np.linalg.norm(g0)
        assert abs(l1 - l0) <= 1e-6 * max(1.0, abs(l0))
    finally:
        eng.close()
