"""bm-score and bm-verify against the reference's own score-matching and
verify-mapping, compiled from the reference sources into oracle/_ref (the
comparison is skipped where those binaries were not built)."""
import os
import subprocess

import numpy as np
import pytest

import bmb200 as bm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref")
ref_tools = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "verify-mapping")),
                               reason="reference checkers not built (no reference sources here)")


def run(args):
    return subprocess.run(args, capture_output=True, text=True, timeout=300)


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("chk")
    A, B, truth, init = bm.gen_pair(1, n=400, m_target=5000, seed=21)
    bm.write_graph_csv(str(d / "gm.csv"), A)
    bm.write_graph_csv(str(d / "gf.csv"), B)
    bm.write_mapping(str(d / "init.csv"), init)
    moved = init.copy()
    rng = np.random.default_rng(1)
    for a, b in rng.integers(1, 401, (30, 2)):
        moved[a], moved[b] = moved[b], moved[a]
    bm.write_mapping(str(d / "moved.csv"), moved)
    with open(d / "dup.csv", "w") as f:  # female 7 given to two males, male 9 given two females
        f.write("Male Node ID,Female Node ID\n")
        for i in range(1, 401):
            f.write(f"m{i},f{init[i]}\n")
        f.write("m3,f7\nm9,f11\n")
    return d, A, B, init, moved


def test_usage():
    assert run([os.path.join(bm.BIN_DIR, "bm-verify")]).returncode == 1
    assert run([os.path.join(bm.BIN_DIR, "bm-score"), "x"]).returncode == 1


def test_score_host_matches_library(files):
    d, A, B, init, moved = files
    r = run([os.path.join(bm.BIN_DIR, "bm-score"), str(d / "gm.csv"), str(d / "gf.csv"), str(d / "moved.csv"),
             "--host"])
    assert r.returncode == 0, r.stdout + r.stderr
    assert int(r.stdout.strip().splitlines()[-1]) == bm.host_score(A, B, moved)


def _after(text, marker):
    lines = text.splitlines()
    return lines[lines.index(marker):]


@ref_tools
def test_verify_matches_reference(files):
    d, *_ = files
    for a, b in (("init.csv", "moved.csv"), ("init.csv", "dup.csv"), ("moved.csv", "init.csv")):
        ours = run([os.path.join(bm.BIN_DIR, "bm-verify"), str(d / a), str(d / b)])
        ref = run([os.path.join(REF, "verify-mapping"), str(d / a), str(d / b)])
        assert ours.returncode == ref.returncode == 0
        # from the verification on, the reports are identical
        assert _after(ours.stdout, "Verifying initial mapping...") == _after(ref.stdout, "Verifying initial mapping...")
    assert "Test mapping is invalid" in run([os.path.join(bm.BIN_DIR, "bm-verify"), str(d / "init.csv"),
                                             str(d / "dup.csv")]).stdout


@ref_tools
def test_score_matches_reference(files):
    d, *_ = files
    for m in ("init.csv", "moved.csv"):
        ours = run([os.path.join(bm.BIN_DIR, "bm-score"), str(d / "gm.csv"), str(d / "gf.csv"), str(d / m), "--host"])
        ref = run([os.path.join(REF, "score-matching"), str(d / "gm.csv"), str(d / "gf.csv"), str(d / m)])
        assert ours.returncode == ref.returncode == 0, ref.stdout[-500:]
        # the reference prints the score as its only bare integer line, between timestamp lines
        ref_score = [ln for ln in ref.stdout.splitlines() if ln.strip().lstrip("-").isdigit()]
        assert ref_score and ours.stdout.strip().splitlines()[-1] == ref_score[-1].strip()


@pytest.mark.gpu
def test_score_gpu_path(files):
    d, A, B, init, moved = files
    r = run([os.path.join(bm.BIN_DIR, "bm-score"), str(d / "gm.csv"), str(d / "gf.csv"), str(d / "moved.csv")])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Score computed on the GPU" in r.stdout
    assert int(r.stdout.strip().splitlines()[-1]) == bm.host_score(A, B, moved)
