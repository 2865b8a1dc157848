"""bm-align / bm-gen command-line contract on the CPU side (usage and load
errors exit 1, like graph-alignment-optimized's main)."""
import os
import subprocess

import bmb200 as bm


def run(args, **kw):
    return subprocess.run(args, capture_output=True, text=True, timeout=120, **kw)


def test_usage_exits_1():
    r = run([os.path.join(bm.BIN_DIR, "bm-align"), "a", "b"])
    assert r.returncode == 1
    assert "Usage:" in r.stderr


def test_missing_graph_exits_1(tmp_path):
    r = run([os.path.join(bm.BIN_DIR, "bm-align")] + [str(tmp_path / f"x{i}.csv") for i in range(6)])
    assert r.returncode == 1
    assert "Failed to load male graph" in r.stderr


def test_unknown_option_exits_1(tmp_path):
    r = run([os.path.join(bm.BIN_DIR, "bm-align")] + [str(tmp_path / f"x{i}.csv") for i in range(6)] + ["--bogus", "1"])
    assert r.returncode == 1


def test_bad_semantics_exits_1(tmp_path):
    r = run([os.path.join(bm.BIN_DIR, "bm-align")] + [str(tmp_path / f"x{i}.csv") for i in range(6)] +
            ["--semantics", "approx"])
    assert r.returncode == 1
    assert "--semantics must be exact or ref-cpu" in r.stderr


def test_bm_gen_writes_reference_formats(tmp_path):
    r = run([os.path.join(bm.BIN_DIR, "bm-gen"), "1", "5", str(tmp_path), "--n", "150", "--m", "1200"])
    assert r.returncode == 0, r.stderr
    g, bad = bm.read_graph_csv(str(tmp_path / "gm.csv"))
    assert bad == 0 and g.m > 1000
    pi, cnt, mx = bm.read_mapping(str(tmp_path / "init_mapping.csv"), 150)
    assert cnt == 150 and bm.check_bijection(pi) == 0
    assert open(tmp_path / "gm_order.csv").readline().strip() == "Node ID,Order"
    A, B, truth, init = bm.gen_pair(1, n=150, m_target=1200, seed=5)
    assert f"score(init)={bm.host_score(A, B, init)}" in r.stdout
