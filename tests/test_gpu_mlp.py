"""Learned partner proposals: the feature table, the MLP's forward and
backward kernels against the oracle's FP64 replica, the tensor-core row
scorer, top-K selection, training, and the search that uses the model."""
import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import mlp_oracle

pytestmark = pytest.mark.gpu


def _bf16(a):
    """Round float32 to BF16 (nearest even), as float32."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _b_lookup(n, B):
    keys = B[0].astype(np.int64) * (n + 1) + B[1].astype(np.int64)
    order = np.argsort(keys, kind="stable")
    return keys[order], B[2][order]


def _b_weight(tab, n, g, h):
    keys, w = tab
    q = g.astype(np.int64) * (n + 1) + h.astype(np.int64)
    i = np.clip(np.searchsorted(keys, q), 0, len(keys) - 1)
    return np.where(keys[i] == q, w[i], 0)


def test_feature_table_matches_host(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi)
    m = bm.Mlp(e, seed=1)
    t = m.features()
    assert t.shape == (n + 1, 12)
    assert np.all(t[0] == 0)
    src, dst, w = (a.astype(np.int64) for a in A)
    dout = np.bincount(src, minlength=n + 1)
    din = np.bincount(dst, minlength=n + 1)
    wout = np.bincount(src, weights=w, minlength=n + 1)
    win = np.bincount(dst, weights=w, minlength=n + 1)
    s = e.overlap().astype(np.float64)
    bt = _b_lookup(n, B)
    absent = _b_weight(bt, n, pi[src], pi[dst]) == 0
    miss = np.bincount(src, weights=absent, minlength=n + 1) + np.bincount(dst, weights=absent, minlength=n + 1)
    bout = np.bincount(B[0], minlength=n + 1)
    bin_ = np.bincount(B[1], minlength=n + 1)
    exp = np.zeros((n + 1, 12), np.float32)
    exp[:, 0] = np.log1p(dout)
    exp[:, 1] = np.log1p(din)
    exp[:, 2] = np.log1p(wout)
    exp[:, 3] = np.log1p(win)
    exp[:, 4] = np.log1p(s)
    exp[:, 5] = np.log1p(np.maximum(wout + win - s, 0))
    exp[:, 6] = np.log1p(miss)
    exp[:, 8] = np.log1p(bout[pi])
    exp[:, 9] = np.log1p(bin_[pi])
    exp[0] = 0
    np.testing.assert_allclose(t, exp, rtol=3e-6, atol=1e-6)
    e.close()


def test_pair_features_definition(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi)
    m = bm.Mlp(e, seed=1)
    t = m.features()
    rng = np.random.default_rng(3)
    pairs = rng.integers(1, n + 1, (3000, 2)).astype(np.int32)
    # include pairs joined by B edges in both directions
    inv = np.argsort(pi[1:]) + 1
    pairs[:200, 0] = inv[B[0][:200] - 1]
    pairs[:200, 1] = inv[B[1][:200] - 1]
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    x = m.pair_features(pairs)
    a, b = t[pairs[:, 0]], t[pairs[:, 1]]
    bt = _b_lookup(n, B)
    fu, fv = pi[pairs[:, 0]], pi[pairs[:, 1]]
    exp = np.zeros((len(pairs), 24), np.float32)
    exp[:, 0:7] = a[:, 0:7]
    exp[:, 7] = a[:, 8] + a[:, 9]
    exp[:, 8:15] = b[:, 0:7]
    exp[:, 15] = b[:, 8] + b[:, 9]
    exp[:, 16] = np.abs(a[:, 0] - b[:, 8])
    exp[:, 17] = np.abs(a[:, 1] - b[:, 9])
    exp[:, 18] = np.abs(b[:, 0] - a[:, 8])
    exp[:, 19] = np.abs(b[:, 1] - a[:, 9])
    exp[:, 20] = _b_weight(bt, n, fu, fv) > 0
    exp[:, 21] = _b_weight(bt, n, fv, fu) > 0
    exp[:, 22] = np.abs(a[:, 4] - b[:, 4])
    exp[:, 23] = a[:, 5] + b[:, 5]
    np.testing.assert_array_equal(x, _bf16(exp))
    assert x[:200, 20].min() == 1.0
    e.close()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("backend,npairs", [(0, 512), (0, 1000), (1, 512)])
def test_gradients_match_fp64_oracle(golden_cfg1, backend, npairs):
    """Gradients of the tensor-core training kernel (backend 0; its backward
    signals dh2, dh1 are BF16 MMA operands, and the oracle rounds them too)
    and of the SIMT kernel (backend 1) against the FP64 replica; 1,000 records
    leave the last 128-record tile partly filled."""
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=11)
    m.set_backend(backend)
    rng = np.random.default_rng(5)
    pairs = rng.integers(1, n + 1, (npairs + 100, 2)).astype(np.int32)
    pairs = pairs[pairs[:, 0] != pairs[:, 1]][:npairs]
    x = m.pair_features(pairs)
    y = rng.normal(0.0, 0.5, x.shape[0]).astype(np.float32)
    w = m.params()
    g, loss = m.gradients(x, y)
    out_o, g_o, loss_o = mlp_oracle(w, x, y, rounding=2 if backend == 0 else True)
    # forward of the same features (SIMT kernel) against the replica
    out = m.score_features(x)
    assert np.max(np.abs(out - out_o)) <= 2e-3 * (1 + np.max(np.abs(out_o)))
    assert abs(loss - loss_o) <= 1e-3 * loss_o
    # gradient, whole and per parameter block; tolerance covers BF16 rounding
    # of a hidden activation that flips between FP32 and FP64 sums
    assert _rel(g, g_o) < 2e-3
    for lo, hi in [(0, 3072), (3072, 3200), (3200, 19584), (19584, 19712), (19712, 19840)]:
        assert _rel(g[lo:hi], g_o[lo:hi]) < 1e-2, (lo, hi)
    assert abs(g[19840] - g_o[19840]) <= 1e-4 * max(1.0, abs(g_o[19840]))
    e.close()


@pytest.mark.parametrize("backend", [0, 1])
def test_row_scores_match_fp64_oracle(golden_cfg1, backend):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=2)
    m.set_backend(backend)
    rows = np.array([1, 17, 999, 1500, 2000, 640, 3, 1234, 77], np.int32)
    sc = m.score_rows(rows)
    assert sc.shape == (len(rows), n)
    for r, u in enumerate(rows):
        assert sc[r, u - 1] == -np.inf
    v = np.arange(1, n + 1, dtype=np.int32)
    pairs = np.stack([np.repeat(rows, n), np.tile(v, len(rows))], 1).astype(np.int32)
    keep = pairs[:, 0] != pairs[:, 1]
    x = m.pair_features(pairs[keep])
    o = mlp_oracle(m.params(), x, rounding=True)[0]
    got = sc.reshape(-1)[keep].astype(np.float64)
    err = np.abs(got - o) / (1.0 + np.abs(o))
    assert np.quantile(err, 0.99) < 2e-3, np.quantile(err, 0.99)
    assert err.max() < 3e-2, err.max()
    e.close()


def test_row_scores_several_rows_per_cta(golden_cfg1):
    """More rows than SMs: the scorer's CTAs take several rows each (the
    feature groups rebuild their candidate bitmaps at every row change, the
    output groups switch rows mid-pipeline).  Rows that are a CTA's second or
    third are checked against the FP64 oracle, all rows against the SIMT
    scorer, and a repeated row gives identical scores wherever it lands."""
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=5)
    rng = np.random.default_rng(11)
    R = 333  # 2 or 3 rows per CTA on a 148-SM B200 (one CTA per SM)
    rows = rng.integers(1, n + 1, R).astype(np.int32)
    rows[-1] = rows[0]
    m.set_backend(0)
    sc = m.score_rows(rows)
    m.set_backend(1)
    ref = m.score_rows(rows)
    m.set_backend(0)
    np.testing.assert_array_equal(sc[-1], sc[0])
    for r, u in enumerate(rows):
        assert sc[r, u - 1] == -np.inf
    fin = np.isfinite(ref)
    err = np.abs(sc[fin] - ref[fin]) / (1.0 + np.abs(ref[fin]))
    assert np.quantile(err, 0.99) < 2e-3, np.quantile(err, 0.99)
    pick = np.array([R - 40, R - 20, R - 2], np.int64)
    v = np.arange(1, n + 1, dtype=np.int32)
    pairs = np.stack([np.repeat(rows[pick], n), np.tile(v, len(pick))], 1).astype(np.int32)
    keep = pairs[:, 0] != pairs[:, 1]
    o = mlp_oracle(m.params(), m.pair_features(pairs[keep]), rounding=True)[0]
    got = sc[pick].reshape(-1)[keep].astype(np.float64)
    err = np.abs(got - o) / (1.0 + np.abs(o))
    assert np.quantile(err, 0.99) < 2e-3, np.quantile(err, 0.99)
    assert err.max() < 3e-2, err.max()
    e.close()


@pytest.mark.parametrize("backend", [0, 1])
def test_candidate_scores_equal_row_scores(golden_cfg1, backend):
    """bm_mlp_score_candidates on listed partners gives the row scorer's scores
    at those partners, bit for bit, on both backends; partners outside 1..n
    or equal to the row's vertex are rejected."""
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=3)
    m.set_backend(backend)
    rows = np.array([1, 17, 999, 1500, 2000, 640, 3], np.int32)
    rng = np.random.default_rng(4)
    cands = np.stack([rng.choice(np.setdiff1d(np.arange(1, n + 1), [u]), 300, replace=False) for u in rows])
    cands = cands.astype(np.int32)
    got = m.score_candidates(rows, cands)
    full = m.score_rows(rows)
    np.testing.assert_array_equal(got, full[np.arange(len(rows))[:, None], cands - 1])
    bad = cands.copy()
    bad[2, 5] = rows[2]
    with pytest.raises(bm.BMError):
        m.score_candidates(rows, bad)
    bad[2, 5] = n + 1
    with pytest.raises(bm.BMError):
        m.score_candidates(rows, bad)
    e.close()


def test_sampled_learned_search_beats_uniform(golden_cfg1):
    """The learned search over sampled partners (the model scores 256 distinct
    random partners per row and proposes its top 8) reaches the score of eight
    uniform passes of 64 random partners per row, from the same start and
    seed, with at most a quarter of the uniform search's exact checks (the
    cost that dominates both); on this pair it takes about an eighth."""
    n, A, B = golden_graphs(golden_cfg1)
    pi0 = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi0)
    m = bm.Mlp(e, seed=1)
    _, pu, su = m.search(None, topk=64, uniform=True, exact_fallback=False, max_sweeps=8, seed=7)
    e.close()
    assert pu.score > int(golden_cfg1["score_init"])
    e = make_engine(n, A, B, pi0)
    m = bm.Mlp(e, seed=1)
    m.reserve_records(1_000_000)
    m.collect_rows(np.arange(1, n + 1, dtype=np.int32), per_row=128, seed=3)
    m.fit(400, batch=4096, lr=2e-3)
    _, pl, sl = m.search(None, topk=8, sample=256, exact_fallback=False, target_score=int(pu.score), max_sweeps=40,
                         seed=7)
    assert pl.score >= pu.score, (pl.score, pu.score)
    assert sl.proposals * 4 <= su.proposals, (sl.proposals, su.proposals)
    assert e.score() == pl.score
    e.close()


def test_simt_rows_equal_simt_pairs(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=4)
    m.set_backend(1)
    rows = np.array([5, 6], np.int32)
    sc = m.score_rows(rows)
    v = np.arange(1, n + 1, dtype=np.int32)
    pairs = np.stack([np.repeat(rows, n), np.tile(v, 2)], 1).astype(np.int32)
    sp = m.score_pairs(pairs)
    np.testing.assert_array_equal(sc.reshape(-1), sp)
    e.close()


def test_topk_order_and_ties(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    e = make_engine(n, A, B, golden_cfg1["pi_init"])
    m = bm.Mlp(e, seed=9)
    rows = np.array([1, 2, 1000, 1999, 2000, 444], np.int32)
    for backend in (0, 1):
        m.set_backend(backend)
        sc = m.score_rows(rows)
        for K in (1, 7, 64):
            pv, ps = m.rows_topk(rows, K)
            for r in range(len(rows)):
                order = np.lexsort((np.arange(1, n + 1), -sc[r].astype(np.float64)))[:K] + 1
                np.testing.assert_array_equal(pv[r], order)
                np.testing.assert_array_equal(ps[r], sc[r, order - 1])
    # many equal scores: a constant model ties every partner; ids ascend
    w = np.zeros(m.nparams, np.float32)
    w[-1] = 0.5
    m.set_params(w)
    pv, ps = m.rows_topk(np.array([3], np.int32), 64)
    np.testing.assert_array_equal(pv[0], [1, 2] + list(range(4, 66)))
    assert np.all(ps == 0.5)
    with pytest.raises(bm.BMError):
        m.rows_topk(rows, 65)
    with pytest.raises(bm.BMError):
        m.score_pairs(np.array([[0, 3]], np.int32))
    e.close()


def test_training_lowers_loss_and_lifts_hit_rate(golden_cfg1):
    n, A, B = golden_graphs(golden_cfg1)
    pi0 = golden_cfg1["pi_init"]
    e = make_engine(n, A, B, pi0)
    m = bm.Mlp(e, seed=1)
    rows = np.arange(1, n + 1, dtype=np.int32)
    nrec = m.collect_rows(rows[:800], per_row=64, seed=3)
    assert nrec == 800 * 64
    first = m.fit(1, batch=4096, lr=2e-3, seed=1)
    last = m.fit(300, batch=4096, lr=2e-3, seed=1)
    assert last < 0.7 * first, (first, last)
    # one pass of proposals from the same mapping: model top-8 against 8
    # uniform partners, both judged by the exact delta
    e_u = make_engine(n, A, B, pi0)
    m_u = bm.Mlp(e_u, seed=1)
    _, pl, sl = m.search(rows, topk=8, max_sweeps=1, exact_fallback=False)
    _, pu, su = m_u.search(rows, topk=8, max_sweeps=1, exact_fallback=False, uniform=True, seed=5)
    hit_l = sl.hits / sl.proposals
    hit_u = su.hits / su.proposals
    assert sl.proposals == su.proposals == n * 8
    assert hit_l > 2.0 * hit_u, (hit_l, hit_u)
    assert pl.score > int(golden_cfg1["score_init"])
    for eng in (e, e_u):
        assert bm.check_bijection(eng.get_mapping()) == 0
        assert eng.tracked_score() == eng.score()
    e.close()
    e_u.close()


def test_learned_search_converges_to_exact_local_optimum(golden_small):
    n, A, B = golden_graphs(golden_small)
    e = make_engine(n, A, B, golden_small["pi_init"])
    m = bm.Mlp(e, seed=1)
    st, prog, stats = m.search(topk=16, train_every=1, train_batch=512, lr=1e-3, seed=2)
    assert st == bm.BM_OK and prog.converged == 1
    assert stats.exact_passes >= 1 and stats.train_steps > 0
    assert e.tracked_score() == e.score() == prog.score
    res = e.rows_best(np.arange(1, n + 1, dtype=np.int32))
    assert np.all(res["best_delta"] <= 0)
    e.close()
