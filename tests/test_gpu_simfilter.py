"""The similarity-filtered pass of the reference's graph-alignment variant
(src/graph-alignment.c:489-595) on the device (bm_sweep_similarity): equal to
the variant itself (the golden fixture its own pass wrote) and to the oracle's
restatement (orc_sim_sweep, pinned to the variant compiled live) on
generated pairs, one with self-loops in the reference-delta mode."""
import sys

import numpy as np
import pytest

import bmb200 as bm
from conftest import GOLDEN, golden_graphs
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu

sys.path.insert(0, GOLDEN)


def device_pass(n, A, B, init, rank_m, rank_f, refcpu=False):
    Ag, Bg = bm.Graph(n, *A), bm.Graph(n, *B)
    nodes = bm.first_appearance(Ag)
    ma, mb = bm.node_metrics(Ag, rank_m), bm.node_metrics(Bg, rank_f)
    with bm.Engine(0) as e:
        e.set_graphs(Ag, Bg)
        e.set_mapping(init)
        if refcpu:
            e.L.bm_set_semantics(e.h, 1)
        prog, st = e.sweep_similarity(nodes, ma, mb)
        assert st == bm.BM_OK and prog.sweeps == 1
        return e.get_mapping(), int(prog.score), int(prog.accepts), e.score()


def test_pass_equals_reference_fixture(golden_simfilter):
    g = golden_simfilter
    n, A, B = golden_graphs(g)
    pi, score, acc, check = device_pass(n, A, B, g["pi_init"], g["rank_m"], g["rank_f"])
    np.testing.assert_array_equal(pi, g["pass_pi"])
    assert score == check == int(g["pass_score"]) and acc > 0


@pytest.mark.parametrize("seed,loops", [(14, 0), (15, 0), (16, 60)])
def test_pass_equals_oracle(seed, loops):
    from make_golden import simfilter_inputs
    n, A, B, init, rank_m, rank_f = simfilter_inputs(seed, loops=loops)
    pi, score, acc, check = device_pass(n, A, B, init, rank_m, rank_f, refcpu=loops > 0)
    orc = Oracle(n, A, B)
    pi_o, acc_o = orc.sim_sweep(init, rank_m, rank_f)
    np.testing.assert_array_equal(pi, pi_o)
    assert acc == acc_o and check == orc.score(pi_o)


def test_pass_resumes_after_a_budget_of_accepts(golden_simfilter):
    """Stopping after every few accepts and resuming gives the same pass."""
    g = golden_simfilter
    n, A, B = golden_graphs(g)
    Ag, Bg = bm.Graph(n, *A), bm.Graph(n, *B)
    nodes = bm.first_appearance(Ag)
    ma, mb = bm.node_metrics(Ag, g["rank_m"]), bm.node_metrics(Bg, g["rank_f"])
    with bm.Engine(0) as e:
        e.set_graphs(Ag, Bg)
        e.set_mapping(g["pi_init"])
        prog = bm.Progress()
        for _ in range(10000):
            prog, st = e.sweep_similarity(nodes, ma, mb, max_accepts=7, prog=prog)
            if prog.sweeps == 1:
                break
        np.testing.assert_array_equal(e.get_mapping(), g["pass_pi"])
