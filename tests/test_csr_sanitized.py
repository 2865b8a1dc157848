"""The host-side builder of the device graph layout (bm_csr.hpp), compiled
with AddressSanitizer and UndefinedBehaviorSanitizer and checked on random
graphs with duplicates, self-loops and zero weights.  CPU only."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def test_csr_builder_under_sanitizers(tmp_path):
    exe = str(tmp_path / "csr_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-o", exe, os.path.join(HERE, "csr_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "csr_check ok" in r.stdout
