"""The oracle's FP64 MLP replica: its backward formulas against central
differences (rounding off, where the loss is smooth), and the rounding rules
it applies with rounding on."""
import numpy as np

from oracle_bind import mlp_oracle

N_PARAMS = 24 * 128 + 128 + 128 * 128 + 128 + 128 + 1
OFF = {"W1": 0, "b1": 3072, "W2": 3200, "b2": 19584, "w3": 19712, "b3": 19840}


def _params(seed):
    rng = np.random.default_rng(seed)
    w = np.zeros(N_PARAMS, np.float32)
    w[:3072] = rng.uniform(-0.4, 0.4, 3072)
    w[3072:3200] = rng.uniform(-0.1, 0.1, 128)
    w[3200:19584] = rng.uniform(-0.15, 0.15, 16384)
    w[19584:19712] = rng.uniform(-0.1, 0.1, 128)
    w[19712:19840] = rng.uniform(-0.2, 0.2, 128)
    w[19840] = 0.05
    return w


def test_oracle_gradient_matches_central_differences():
    rng = np.random.default_rng(7)
    w = _params(3)
    x = rng.uniform(0, 3, (40, 24)).astype(np.float32)
    y = rng.normal(0, 0.5, 40).astype(np.float32)
    _, g, loss = mlp_oracle(w, x, y, rounding=False)
    assert loss > 0
    picks = [OFF["W1"] + 5, OFF["W1"] + 24 * 64 + 3, OFF["b1"] + 7, OFF["W2"] + 128 * 10 + 99, OFF["W2"] + 777,
             OFF["b2"] + 31, OFF["w3"] + 12, OFF["w3"] + 100, OFF["b3"]]
    for i in picks:
        h = 1e-2
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        hp = float(wp[i]) - float(w[i])
        hm = float(w[i]) - float(wm[i])
        lp = mlp_oracle(wp, x, y, rounding=False)[2]
        lm = mlp_oracle(wm, x, y, rounding=False)[2]
        fd = (lp - lm) / (hp + hm)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g[i])) + 1e-6, (i, fd, g[i])


def test_oracle_rounding_rules():
    w = _params(5)
    x = np.random.default_rng(1).uniform(0, 3, (16, 24)).astype(np.float32)
    o_r = mlp_oracle(w, x, rounding=True)[0]
    o_e = mlp_oracle(w, x, rounding=False)[0]
    # BF16 operands change the output a little, never by much
    assert np.max(np.abs(o_r - o_e)) < 0.05 * (1 + np.max(np.abs(o_e)))
    # inputs already on the BF16 grid give the same first layer either way
    xb = (x.view(np.uint32) & 0xFFFF0000).view(np.float32)
    wb = w.copy()
    wb[:3072] = (w[:3072].view(np.uint32) & 0xFFFF0000).view(np.float32)
    assert np.all(np.isfinite(mlp_oracle(wb, xb, rounding=True)[0]))
