"""End-to-end CPU baseline: the unmodified reference search binary on the
full-scale synthetic pair, score versus time.

TEST INFRASTRUCTURE ONLY: a baseline measurement of the reference, never the
product.  The binary is oracle/_ref/graph-alignment-optimized-parallel, which
oracle/Makefile compiles unmodified from
src/graph-alignment-optimized-parallel.c where the reference sources are
present.  Its loop never ends (while(true), :514), so it runs for a fixed wall
time and is then stopped.

Progress is read two ways.  (1) The mapping the reference saves every 25
outer rows (save_intermediate_mapping at :538-541, written before row 25k is
processed, so it holds rows 1..25k-1): each new file is scored on the host
(bm_host_score, equal to the reference's calculate_alignment_score) and
stamped with its time of appearance.  (2) Its own progress lines every 100
outer rows (:521-535: rows processed, "Current score", rows per second).

The pair and the initial matching are those of the bench's workload
(bm-gen config 2, seed 2: n = 18,524, ~3M edges per graph, greedy-similarity
initial matching), written in the reference's CSV formats.

    python oracle/ref_e2e.py [--seconds 600] [--threads 0] [--workdir DIR]

The CSV files and the reference's output mapping go to DIR (default
oracle/_ref/e2e, beside the binary) and are deleted at the end unless --keep
is given.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import signal
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "brain-match_b200", "python"))

import bmb200 as bm  # noqa: E402

REF_BIN = os.path.join(HERE, "_ref", "graph-alignment-optimized-parallel")
GEN_BIN = os.path.join(REPO, "brain-match_b200", "bin", "bm-gen")
NUM = r"([0-9][0-9,]*)"


def num(s: str) -> int:
    return int(s.replace(",", ""))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class Lines(threading.Thread):
    """Reads the reference's stdout; keeps the parsed progress lines."""

    def __init__(self, stream, t0):
        super().__init__(daemon=True)
        self.stream, self.t0 = stream, t0
        self.initial = None
        self.t_opt = None
        self.progress = []  # [s since start, rows processed, score, improvements, rows/s]
        self._row = {}

    def run(self):
        for line in self.stream:
            now = round(time.perf_counter() - self.t0, 3)
            m = re.search(r"Starting optimization with initial score: " + NUM, line)
            if m:
                self.initial, self.t_opt = num(m.group(1)), now
            for key, pat in (("rows", r"Processed: " + NUM + "/"), ("score", r"Current score: " + NUM),
                             ("impr", r"Improvements found: " + NUM)):
                m = re.search(pat, line)
                if m:
                    self._row[key] = num(m.group(1))
            m = re.search(r"Processing speed: ([0-9.]+) nodes/sec", line)
            if m:
                r = self._row
                self.progress.append([now, r.get("rows"), r.get("score"), r.get("impr"), float(m.group(1))])
                self._row = {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=600.0)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--workdir", default=None)
    ap.add_argument("--keep", action="store_true", help="keep the generated CSV files")
    args = ap.parse_args()
    if not os.path.exists(REF_BIN):
        raise SystemExit(f"{REF_BIN} missing: run make -C oracle where the reference sources exist")
    work = args.workdir or os.path.join(HERE, "_ref", "e2e")
    os.makedirs(work, exist_ok=True)
    subprocess.run([GEN_BIN, "2", "2", work], check=True, capture_output=True)
    A = bm.read_graph_csv(os.path.join(work, "gm.csv"))[0]
    B = bm.read_graph_csv(os.path.join(work, "gf.csv"))[0]
    n = max(A.n, B.n)
    A.n = B.n = n
    init = bm.read_mapping(os.path.join(work, "init_mapping.csv"), n)[0]
    init_score = bm.host_score(A, B, init)
    out_path = os.path.join(work, "ref_out_mapping.csv")
    if os.path.exists(out_path):
        os.remove(out_path)

    env = dict(os.environ)
    threads = args.threads or os.cpu_count()
    env["OMP_NUM_THREADS"] = str(threads)
    # line-buffered stdout; timeout only as the last bound should this script die
    cmd = ["timeout", "-k", "30", str(int(args.seconds + 300)), "stdbuf", "-oL", REF_BIN,
           os.path.join(work, "gm.csv"), os.path.join(work, "gf.csv"), os.path.join(work, "gm_order.csv"),
           os.path.join(work, "gf_order.csv"), os.path.join(work, "init_mapping.csv"), out_path]
    t0 = time.perf_counter()
    wall0 = time.time()
    proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, env=env,
                            start_new_session=True)
    lines = Lines(proc.stdout, t0)
    lines.start()
    saves = []  # [s since start, rows done, score]
    last_mtime = None
    try:
        while time.perf_counter() - t0 < args.seconds and proc.poll() is None:
            time.sleep(0.5)
            try:
                st = os.stat(out_path)
            except FileNotFoundError:
                continue
            if st.st_mtime_ns == last_mtime:
                continue
            time.sleep(1.0)  # let the writer finish the file
            try:
                if os.stat(out_path).st_mtime_ns != st.st_mtime_ns:
                    continue
                pi = bm.read_mapping(out_path, n)[0]
            except (OSError, RuntimeError):
                continue
            last_mtime = st.st_mtime_ns
            saves.append([round(st.st_mtime - wall0, 1), 25 * (len(saves) + 1) - 1, bm.host_score(A, B, pi)])
    finally:
        if proc.poll() is None:
            os.killpg(proc.pid, signal.SIGTERM)
            try:
                proc.wait(timeout=30)
            except subprocess.TimeoutExpired:
                os.killpg(proc.pid, signal.SIGKILL)
                proc.wait()
    lines.join(timeout=5)
    if not args.keep:
        for name in ("gm.csv", "gf.csv", "gm_order.csv", "gf_order.csv", "init_mapping.csv", "truth_mapping.csv",
                     "ref_out_mapping.csv"):
            path = os.path.join(work, name)
            if os.path.exists(path):
                os.remove(path)
    print(json.dumps({
        "binary": "graph-alignment-optimized-parallel (unmodified reference)",
        "workload": "bm-gen config 2 seed 2 (n = 18,524, ~3M edges per graph, greedy initial matching)",
        "threads": threads, "cpu": cpu_model(), "seconds": args.seconds,
        "initial_score_reference": lines.initial, "initial_score_host": init_score,
        "s_to_optimisation_start": lines.t_opt,
        "saves_columns": ["s since start", "rows done", "score (host re-score of the saved mapping)"],
        "saves": saves,
        "progress_columns": ["s since start", "rows processed", "score", "improvements", "rows/s"],
        "progress": lines.progress}), flush=True)


if __name__ == "__main__":
    sys.exit(main())
