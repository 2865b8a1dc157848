"""The end-to-end baseline script (oracle/ref_e2e.py) on a short run: the
unmodified reference search binary loads the full-scale synthetic pair in the
reference's CSV formats and computes the same initial score as the host
scorer.  CPU only; skipped where the reference binary was not built."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

REF_BIN = os.path.join(REPO, "oracle", "_ref", "graph-alignment-optimized-parallel")


@pytest.mark.skipif(not os.path.exists(REF_BIN), reason="oracle/_ref not built (reference sources absent)")
def test_reference_binary_scores_like_the_host():
    work = os.path.join(REPO, "oracle", "_ref", "e2e_test")  # beside the binary, out of version control
    r = subprocess.run([sys.executable, os.path.join(REPO, "oracle", "ref_e2e.py"), "--seconds", "15",
                        "--threads", "2", "--workdir", work],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["initial_score_reference"] == out["initial_score_host"] > 0
    for t, rows, score in out["saves"]:
        assert rows % 25 == 24 and score >= out["initial_score_host"]
