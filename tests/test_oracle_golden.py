"""The oracle (oracle/bm_oracle.c) pinned against the golden fixtures made by
the reference's own functions, and against the compiled reference itself when
it is present.  CPU only."""
import numpy as np
import pytest

from conftest import golden_graphs
from oracle_bind import Oracle, Reference, ref_available


@pytest.mark.parametrize("case", ["golden_small", "golden_cfg1"])
def test_oracle_score_and_deltas(case, request):
    g = request.getfixturevalue(case)
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    assert orc.score(g["pi_init"]) == int(g["score_init"])
    assert orc.score(g["pi_truth"]) == int(g["score_truth"])
    np.testing.assert_array_equal(orc.pairs(g["pi_init"], g["pairs"]), g["pair_deltas"])
    np.testing.assert_array_equal(orc.rows(g["pi_init"], g["rows"]), g["row_deltas"])


def test_oracle_serial_converges_like_reference(golden_small):
    g = golden_small
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    pi, score, log, sweeps, conv = orc.serial(g["pi_init"])
    assert conv == int(g["serial_converged"]) == 1
    assert sweeps == int(g["serial_sweeps"])
    assert score == int(g["serial_score"])
    np.testing.assert_array_equal(pi, g["serial_pi"])
    np.testing.assert_array_equal(log, g["serial_log"])
    assert orc.score(pi) == score


def test_oracle_serial_first_sweep_cfg1(golden_cfg1):
    g = golden_cfg1
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    pi, score, log, sweeps, conv = orc.serial(g["pi_init"], max_sweeps=1)
    assert len(log) == int(g["serial_accepts"])
    np.testing.assert_array_equal(log[: len(g["serial_log"])], g["serial_log"])
    np.testing.assert_array_equal(pi, g["serial_pi"])
    assert score == int(g["serial_score"])
    pi100, s100, _, _, _ = orc.serial(g["pi_init"], max_accepts=100)
    np.testing.assert_array_equal(pi100, g["serial100_pi"])
    assert s100 == int(g["serial100_score"])


def test_oracle_selfloop_scores(golden_selfloop):
    g = golden_selfloop
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    for pi, s, (u, v), s2, rd in zip(g["pis"], g["scores"], g["swaps"], g["swapped_scores"], g["ref_deltas"]):
        assert orc.score(pi) == s
        assert orc.exact_delta(pi, u, v) == s2 - s
        assert orc.delta(pi, u, v) == rd  # the reference's own (inexact here) delta, restated


def test_oracle_selfloop_reference_deltas(golden_selfloop_ref):
    """On a pair with self-loops (no duplicates) the restated
    calculate_swap_delta equals the reference's own deltas, pairs, whole rows
    and the accept sequence of the serial loop, although those deltas are not
    score differences there."""
    g = golden_selfloop_ref
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    assert orc.score(g["pi_init"]) == int(g["score_init"])
    deltas = orc.pairs(g["pi_init"], g["pairs"])
    np.testing.assert_array_equal(deltas, g["pair_deltas"])
    exact = np.array([orc.exact_delta(g["pi_init"], u, v) if u != v else 0 for u, v in g["pairs"]])
    assert (exact != deltas).sum() > 100  # the fixture exercises the self-loop rule
    np.testing.assert_array_equal(orc.rows(g["pi_init"], g["rows"]), g["row_deltas"])
    pi, _, log, sweeps, conv = orc.serial(g["pi_init"], max_sweeps=int(g["serial_max_sweeps"]))
    np.testing.assert_array_equal(log, g["serial_log"])
    np.testing.assert_array_equal(pi, g["serial_pi"])
    assert (sweeps, conv) == (int(g["serial_sweeps"]), int(g["serial_converged"]))
    assert orc.score(pi) == int(g["serial_score"])  # the reference re-scores every accept
    pi100, _, _, _, _ = orc.serial(g["pi_init"], max_accepts=100)
    np.testing.assert_array_equal(pi100, g["serial100_pi"])
    assert orc.score(pi100) == int(g["serial100_score"])


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_oracle_matches_live_reference():
    import bmb200 as bm
    for seed in (21, 22):
        Ag, Bg, truth, init = bm.gen_pair(1, n=500, m_target=6000, seed=seed)
        A, B = (Ag.src, Ag.dst, Ag.w), (Bg.src, Bg.dst, Bg.w)
        orc, ref = Oracle(Ag.n, A, B), Reference(Ag.n, A, B)
        rng = np.random.default_rng(seed)
        pairs = rng.integers(1, Ag.n + 1, size=(4000, 2)).astype(np.int32)
        np.testing.assert_array_equal(orc.pairs(init, pairs), ref.pairs(init, pairs))
        assert orc.score(truth) == ref.score(truth)
        p1, s1, l1, _, _ = orc.serial(init, max_sweeps=1)
        p2, s2, l2, _, _ = ref.serial(init, max_sweeps=1)
        np.testing.assert_array_equal(p1, p2)
        np.testing.assert_array_equal(l1, l2)
        assert s1 == s2
        ref.close()


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("seed", [31, 32, 33])
def test_oracle_matches_live_reference_with_loops_and_duplicates(seed):
    """Random pairs with self-loops (at most one per A vertex), duplicate edges
    and zero weights: the restated calculate_swap_delta, whole rows and one
    serial sweep equal the reference's own, quirks included."""
    n, m = 200, 2500
    rng = np.random.default_rng(seed)

    def graph(one_loop_per_vertex):
        s = rng.integers(1, n + 1, m).astype(np.int32)
        d = rng.integers(1, n + 1, m).astype(np.int32)
        lv = rng.choice(np.arange(1, n + 1), 40, replace=False).astype(np.int32)
        dup = rng.integers(0, m, 300)
        s, d = np.concatenate([s, lv, s[dup]]), np.concatenate([d, lv, d[dup]])
        w = rng.integers(0, 9, s.shape[0]).astype(np.int32)
        if one_loop_per_vertex:
            seen, keep = set(), []
            for i in range(s.shape[0]):
                if s[i] == d[i]:
                    if s[i] in seen:
                        continue
                    seen.add(int(s[i]))
                keep.append(i)
            s, d, w = s[keep], d[keep], w[keep]
        return s, d, w

    A, B = graph(True), graph(False)
    orc, ref = Oracle(n, A, B), Reference(n, A, B)
    pi = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
    assert orc.score(pi) == ref.score(pi)
    pairs = rng.integers(1, n + 1, size=(3000, 2)).astype(np.int32)
    np.testing.assert_array_equal(orc.pairs(pi, pairs), ref.pairs(pi, pairs))
    rows = np.array([1, 77, 200], np.int32)
    np.testing.assert_array_equal(orc.rows(pi, rows), ref.rows(pi, rows))
    p1, s1, l1, _, _ = orc.serial(pi, max_sweeps=1)
    p2, s2, l2, _, _ = ref.serial(pi, max_sweeps=1)
    np.testing.assert_array_equal(l1, l2)
    np.testing.assert_array_equal(p1, p2)
    assert s1 == s2
    ref.close()
