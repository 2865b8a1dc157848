"""Batched annealing chains on the device replay bit for bit on the CPU: the
same Philox proposals, the same exact deltas, the same acceptance decisions,
hence the same final mapping, score and accept count, for every number of
speculative candidates per iteration."""
import numpy as np
import pytest

import bmb200 as bm
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pairs():
    out = []
    for seed, n, m in ((31, 300, 3000), (32, 450, 6000), (33, 200, 1500)):
        A, B, truth, init = bm.gen_pair(1, n=n, m_target=m, seed=seed)
        out.append((A, B, init))
    return out


@pytest.mark.parametrize("candidates,threads", [(1, 0), (4, 0), (16, 0), (1, 256), (4, 256), (16, 256)])
def test_chains_replay_on_cpu(pairs, candidates, threads):
    eng = bm.Engine(0)
    batch = bm.Batch(eng)
    for A, B, _ in pairs:
        batch.add_pair(A, B)
    chain_pair = [0, 1, 2, 0, 1]
    keys = [11, 12, 13, 14, 15]
    inits = [pairs[p][2] for p in chain_pair]
    steps = 6000
    pis, scores, acc, st = batch.sa_run(chain_pair, keys, inits, steps, t0=5.0, t_end=0.01,
                                        candidates=candidates, chunk=1000, threads=threads)
    assert st.candidates == candidates and st.launches == 6
    assert st.ctas_per_chain == 2  # 5 chains fill at most half the SMs: a pair of CTAs per chain
    assert st.threads_per_cta == (threads or 512)
    for c, p in enumerate(chain_pair):
        A, B, init = pairs[p]
        orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
        pi_o, s_o, a_o = orc.sa(init, keys[c], steps, 5.0, 0.01)
        np.testing.assert_array_equal(pis[c], pi_o)
        assert scores[c] == s_o == orc.score(pis[c])
        assert acc[c] == a_o
    batch.close()
    eng.close()


def test_uneven_batch_autotuned(tmp_path, monkeypatch):
    """Sixteen pairs of uneven size, four chains each (the batched-chain
    workload at reduced n): every chain ends on a consistent score, and the
    autotuned run equals a fixed-candidate run."""
    monkeypatch.setenv("BM_TUNE_CACHE", str(tmp_path / "tune.txt"))
    eng = bm.Engine(0)
    batch = bm.Batch(eng)
    rng = np.random.default_rng(3)
    data = []
    for i in range(16):
        n = int(rng.integers(200, 2001))
        A, B, truth, init = bm.gen_pair(3, n=n, m_target=20 * n, seed=100 + i)
        batch.add_pair(A, B)
        data.append((A, B, init))
    chain_pair = [i // 4 for i in range(64)]
    keys = list(range(1000, 1064))
    inits = [data[p][2] for p in chain_pair]
    steps = 3000
    p1, s1, a1, st1 = batch.sa_run(chain_pair, keys, inits, steps, candidates=0, chunk=1500)
    p2, s2, a2, st2 = batch.sa_run(chain_pair, keys, inits, steps, candidates=2, chunk=700)
    assert 1 <= st1.candidates <= 32
    np.testing.assert_array_equal(s1, s2)
    np.testing.assert_array_equal(a1, a2)
    for c in range(64):
        np.testing.assert_array_equal(p1[c], p2[c])
        A, B, _ = data[chain_pair[c]]
        assert bm.check_bijection(p1[c]) == 0
        assert s1[c] == bm.host_score(A, B, p1[c])
    assert (tmp_path / "tune.txt").exists()
    batch.close()
    eng.close()


def test_chains_one_cta_each_replay_on_cpu():
    """More chains than half the SMs: one CTA per chain (the other kernel
    instantiation); chains still replay bit for bit."""
    eng = bm.Engine(0)
    batch = bm.Batch(eng)
    pairs = []
    for seed, n, m in ((51, 160, 1200), (52, 220, 2000)):
        A, B, truth, init = bm.gen_pair(1, n=n, m_target=m, seed=seed)
        batch.add_pair(A, B)
        pairs.append((A, B, init))
    nch = 80
    chain_pair = [c % 2 for c in range(nch)]
    keys = [700 + c for c in range(nch)]
    inits = [pairs[p][2] for p in chain_pair]
    steps = 3000
    pis, scores, acc, st = batch.sa_run(chain_pair, keys, inits, steps, t0=5.0, t_end=0.01, candidates=4, chunk=1000)
    assert st.ctas_per_chain == 1
    for c in (0, 1, 41, 79):
        A, B, init = pairs[chain_pair[c]]
        orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
        pi_o, s_o, a_o = orc.sa(init, keys[c], steps, 5.0, 0.01)
        np.testing.assert_array_equal(pis[c], pi_o)
        assert scores[c] == s_o and acc[c] == a_o
    batch.close()
    eng.close()
