"""Schedules on the device: the parity sweep reproduces the reference's serial
first-improvement loop exactly; the batched search keeps an exact score; the
bm-align CLI runs end to end."""
import os
import subprocess

import numpy as np
import pytest

import bmb200 as bm
from conftest import golden_graphs, make_engine
from oracle_bind import Oracle

pytestmark = pytest.mark.gpu


def test_parity_sweep_converges_like_reference(golden_small):
    g = golden_small
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    prog, st = e.sweep_parity()
    assert st == bm.BM_OK and prog.converged == 1
    assert prog.accepts == int(g["serial_accepts"])
    assert prog.sweeps == int(g["serial_sweeps"])
    np.testing.assert_array_equal(e.get_mapping(), g["serial_pi"])
    assert prog.score == e.score() == int(g["serial_score"])
    e.close()


def test_parity_first_sweep_cfg1(golden_cfg1):
    g = golden_cfg1
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    prog, st = e.sweep_parity(max_sweeps=1)
    assert prog.accepts == int(g["serial_accepts"])
    np.testing.assert_array_equal(e.get_mapping(), g["serial_pi"])
    assert prog.score == int(g["serial_score"])
    e.close()


def test_parity_max_accepts_and_resume(golden_cfg1):
    g = golden_cfg1
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    prog, _ = e.sweep_parity(max_accepts=37)
    assert prog.accepts == 37
    prog, _ = e.sweep_parity(max_accepts=63, prog=prog)
    assert prog.accepts == 100
    np.testing.assert_array_equal(e.get_mapping(), g["serial100_pi"])
    assert e.tracked_score() == int(g["serial100_score"])
    e.close()


def test_parity_custom_row_order(golden_small):
    g = golden_small
    n, A, B = golden_graphs(g)
    rows = np.random.default_rng(9).permutation(np.arange(1, n + 1)).astype(np.int32)
    orc = Oracle(n, A, B)
    pi_o, s_o, log_o, _, _ = orc.serial(g["pi_init"], rows=rows, max_sweeps=1)
    e = make_engine(n, A, B, g["pi_init"])
    prog, _ = e.sweep_parity(rows=rows, max_sweeps=1)
    assert prog.accepts == len(log_o)
    np.testing.assert_array_equal(e.get_mapping(), pi_o)
    assert prog.score == s_o
    e.close()


@pytest.mark.parametrize("case", ["golden_small", "golden_cfg1"])
def test_batched_search_reaches_local_optimum(case, request):
    g = request.getfixturevalue(case)
    n, A, B = golden_graphs(g)
    e = make_engine(n, A, B, g["pi_init"])
    prog, st = e.search_batched(max_sweeps=200)
    assert prog.converged == 1
    pi = e.get_mapping()
    assert bm.check_bijection(pi) == 0
    orc = Oracle(n, A, B)
    assert prog.score == e.score() == orc.score(pi)
    assert prog.score > int(g["score_init"])
    res = e.rows_best(np.arange(1, n + 1, dtype=np.int32))
    assert res["best_delta"].max() <= 0  # no improving pairwise swap left
    e.close()


def test_cli_parity_end_to_end(golden_small, tmp_path):
    g = golden_small
    n, A, B = golden_graphs(g)
    gm, gf = str(tmp_path / "gm.csv"), str(tmp_path / "gf.csv")
    bm.write_graph_csv(gm, bm.Graph(n, *A))
    bm.write_graph_csv(gf, bm.Graph(n, *B))
    om, of = str(tmp_path / "om.csv"), str(tmp_path / "of.csv")
    bm.write_ordering(om, bm.ordering_by_weighted_degree(bm.Graph(n, *A)))
    bm.write_ordering(of, bm.ordering_by_weighted_degree(bm.Graph(n, *B)))
    inp, out = str(tmp_path / "in_5047.csv"), str(tmp_path / "out.csv")
    bm.write_mapping(inp, g["pi_init"])
    r = subprocess.run([os.path.join(bm.BIN_DIR, "bm-align"), gm, gf, om, of, inp, out], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "[INFO] Expected score from filename: 5047" in r.stdout
    assert "[INFO] Initial alignment score: 5,047" in r.stdout
    assert "Final score: 7,724" in r.stdout
    pi, cnt, _ = bm.read_mapping(out, n)
    np.testing.assert_array_equal(pi, g["serial_pi"])
