"""The similarity-filtered single pass of the reference's graph-alignment
variant (src/graph-alignment.c:489-595), restated in the oracle
(orc_sim_sweep): against the golden fixture made by the variant itself, and
against the live variant (oracle/_ref/libref_ga.so) where it was built.
CPU only."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden_graphs
from oracle_bind import Oracle, ref_ga_available

sys.path.insert(0, GOLDEN)


def test_oracle_pass_equals_reference_fixture(golden_simfilter):
    g = golden_simfilter
    n, A, B = golden_graphs(g)
    orc = Oracle(n, A, B)
    pi, accepts = orc.sim_sweep(g["pi_init"], g["rank_m"], g["rank_f"])
    np.testing.assert_array_equal(pi, g["pass_pi"])
    assert accepts > 0 and orc.score(pi) == int(g["pass_score"])


@pytest.mark.skipif(not ref_ga_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("seed,loops", [(14, 0), (15, 0), (16, 60)])
def test_oracle_pass_equals_live_reference(seed, loops):
    from make_golden import ref_simfilter_pass, simfilter_inputs
    n, A, B, init, rank_m, rank_f = simfilter_inputs(seed, loops=loops)
    pi_ref, score_ref = ref_simfilter_pass(A, B, init, rank_m, rank_f)
    orc = Oracle(n, A, B)
    pi, _ = orc.sim_sweep(init, rank_m, rank_f)
    np.testing.assert_array_equal(pi, pi_ref)
    assert orc.score(pi) == score_ref
    assert not np.array_equal(pi, init)
