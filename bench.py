"""Benchmark: exact swap-deltas/s on the full-scale synthetic pair.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: seeded synthetic graph pair, n = 18,524 vertices per side, ~3M
directed edges per graph (joint in/out power law, heavy-tailed int weights,
5% edge noise), greedy-similarity initial matching.  Rows are visited in
ordering-rank order (weighted degree); one step evaluates one batch of 57 rows
x all 18,523 partners = 1,055,811 >= 2^20 exact int64 swap deltas with the
whole-row kernel and reduces each row (first improving partner, best partner,
count).  L2 is flushed before every step (the graphs and the hash fit in L2).

value  = deltas of all ranks / max over ranks of the summed kernel times
         (CUDA events on the engine's stream, inputs resident in HBM)
e2e    = the same through the public C ABI bm_rows_best with host buffers
         (rows in, row results out), wall clock per call
--impl reference times the reference's own calculate_swap_delta under its
OpenMP m2 sweep (oracle/_ref, compiled from the reference sources; the
restated oracle if that library is absent) on the same row batches.  Its
process loads no library of this engine: a child process writes the workload
(generator and greedy matching) to a temporary file, read back with numpy.
Under torchrun every rank takes disjoint row batches (weak scaling); only a
barrier and a max of the timings cross ranks (gloo), there is no data-path
collective.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "brain-match_b200", "python"))

import bmb200 as bm  # noqa: E402

WORKLOAD = ("full-scale synthetic pair: n=18,524 per side, ~3M directed edges per graph, joint in/out power law "
            "(mean ~160), weights 80% in 1..5 with a tail to 3,000, 5% edge noise, greedy-similarity initial "
            "matching; ordering-driven rows, 57 rows x 18,523 partners (>= 2^20 candidates) per step")


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        return ws, rank, local, dist
    return 1, 0, 0, None


def dist_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def make_workload():
    A, B, truth, init = bm.gen_pair(2)
    order = bm.ordering_by_weighted_degree(A)
    rows = bm.rows_from_ordering(order)
    return A, B, truth, init, rows


WORKLOAD_KEYS = ("a_src", "a_dst", "a_w", "b_src", "b_dst", "b_w", "init", "rows")


def write_workload(path):
    """The workload as plain arrays (the reference arm's input)."""
    A, B, truth, init, rows = make_workload()
    np.savez(path, n=np.int64(A.n), a_src=A.src, a_dst=A.dst, a_w=A.w, b_src=B.src, b_dst=B.dst, b_w=B.w, init=init,
             rows=rows)


def read_workload_isolated():
    """The workload made by a child process and read back with numpy, so the
    calling process loads no library of this engine."""
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "workload.npz")
        subprocess.run([sys.executable, os.path.abspath(__file__), "--write-workload", path], check=True,
                       env=dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0"))
        z = np.load(path)
        return int(z["n"]), {k: np.ascontiguousarray(z[k]) for k in WORKLOAD_KEYS}


def algorithmic_bytes_per_row(A: bm.Graph, B: bm.Graph, pi: np.ndarray) -> np.ndarray:
    """Bytes the whole-row algorithm must read for each row u (1-indexed array):
    4 B per second-hop list entry, 16 B per first-hop item (entry, pointer
    pair, image), 16 B of hash probes per A neighbour, 4 B x n of S(v) in the
    finalise pass."""
    n = A.n
    pinv = np.zeros(n + 1, np.int64)
    pinv[pi[1:]] = np.arange(1, n + 1)
    dAo = np.bincount(A.src, minlength=n + 1)
    dAi = np.bincount(A.dst, minlength=n + 1)
    dBo = np.bincount(B.src, minlength=n + 1)
    dBi = np.bincount(B.dst, minlength=n + 1)
    t = np.zeros(n + 1, np.int64)
    np.add.at(t, A.src, dBi[pi[A.dst]])
    np.add.at(t, A.dst, dBo[pi[A.src]])
    np.add.at(t, pinv[B.src], dAi[pinv[B.dst]])
    np.add.at(t, pinv[B.dst], dAo[pinv[B.src]])
    first = dAo + dAi + dBo[pi] + dBi[pi]
    return 4 * t + 16 * first + 16 * (dAo + dAi) + 4 * n


class ClockSampler:
    """SM clock and clock-event reasons of the engine's GPU, polled through NVML
    every ~2 ms in a background thread while the timed region runs (read-only
    queries; no GPU setting is changed)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, pci_bus_id: str):
        import threading
        self.samples, self.reasons, self.max_mhz = [], 0, 0.0
        self.stop_ev = threading.Event()
        self.thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(pci_bus_id.encode())
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                self.reasons |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
            except Exception:
                pass
            self.stop_ev.wait(0.002)

    def stop(self) -> dict | None:
        if self.thread is None:
            return None
        self.stop_ev.set()
        self.thread.join()
        if not self.samples:
            return None
        names = sorted(k for k, bit in self.REASONS.items() if self.reasons & bit)
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples), "source": "NVML, 2 ms polling during the warm-up and timed steps"}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def pinned_array(nbytes: int, dtype, count: int):
    p = C.c_void_p()
    st = bm.cuda_lib().bm_host_alloc_pinned(nbytes, C.byref(p))
    if st != bm.BM_OK:
        raise bm.BMError(st, "bm_host_alloc_pinned")
    buf = (C.c_char * nbytes).from_address(p.value)
    return np.frombuffer(buf, dtype=dtype, count=count), p.value


def cpu_baseline(A, B, init, rows, starts, budget_s=12.0):
    """The reference's calculate_swap_delta under its OpenMP m2 sweep, on a
    bounded sample of the same rows (the first row of each timed batch, as
    many as fit the budget); all host threads."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from oracle_bind import Oracle, Reference, ref_available
    threads = os.cpu_count() or 1
    Ae, Be = (A.src, A.dst, A.w), (B.src, B.dst, B.w)
    if ref_available():
        impl, kind = Reference(A.n, Ae, Be), "reference"
    else:
        impl, kind = Oracle(A.n, Ae, Be), "port"
    done, t_total = 0, 0.0
    for st in starts:
        t0 = time.perf_counter()
        impl.rows(init, rows[st:st + 1], threads)
        t_total += time.perf_counter() - t0
        done += 1
        if t_total >= budget_s:
            break
    if kind == "reference":
        impl.close()
    val = done * (A.n - 1) / t_total
    return {"value": val, "unit": "deltas/s", "cores": threads, "kind": kind,
            "sample": f"{done} rows x {A.n - 1} partners, the first row of each timed batch ({t_total:.1f} s)"}


def step_starts(n: int, steps: int, offset: float = 0.0):
    """Start positions (in the ordering) of the timed batches: evenly spaced over
    one full pass, so the K measured batches are a stratified sample of it."""
    return [int(((s + offset) * n) // steps) % n for s in range(steps)]


def bench_config(n, mA, mB, R, ws):
    """The `config` of a bench line; both arms print the same one."""
    return {"workload": WORKLOAD, "n": n, "edges_A": mA, "edges_B": mB, "rows_per_step": R,
            "candidates_per_step": R * (n - 1), "l2": "flushed before every step",
            "parallelism": f"row batches sharded over {ws} rank(s), no data-path collective"}


def run_reference(args, ws, rank, dist):
    """The reference's calculate_swap_delta under its OpenMP m2 sweep on the
    bench's own row batches (all partners of each row), all host threads.
    Rank 0 alone runs it.  A step is the same batch as in the engine's arm
    when K such steps fit --ref-budget seconds, else the first rows of it."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from oracle_bind import Oracle, Reference, ref_available
    n, w = read_workload_isolated()
    init, rows = w["init"], w["rows"]
    R = args.rows_per_step
    threads = os.cpu_count() or 1
    Ae, Be = (w["a_src"], w["a_dst"], w["a_w"]), (w["b_src"], w["b_dst"], w["b_w"])
    if ref_available():
        impl, kind = Reference(n, Ae, Be), "reference"
    else:
        impl, kind = Oracle(n, Ae, Be), "port"
    # warm-up: one row at each of W evenly spaced positions; their mean time
    # estimates a row, and the whole batch is timed per step if K steps fit
    # the budget, else fewer rows of it
    t0 = time.perf_counter()
    wstarts = step_starts(n, args.warmup, 0.5)
    for st in wstarts:
        impl.rows(init, rows[st:st + 1], threads)
    est = (time.perf_counter() - t0) / max(1, len(wstarts))
    rps = max(1, min(R, int(args.ref_budget / max(1e-9, est * args.steps))))
    total = 0.0
    starts = step_starts(n, args.steps)
    for st in starts:
        idx = (st + np.arange(rps)) % n
        t0 = time.perf_counter()
        impl.rows(init, np.ascontiguousarray(rows[idx]), threads)
        total += time.perf_counter() - t0
    if kind == "reference":
        impl.close()
    v = args.steps * rps * (n - 1) / total
    sample = (f"the engine arm's batches: {rps} rows x {n - 1} partners per step" if rps == R else
              f"the first {rps} of the {R} rows of each of the engine arm's batches x {n - 1} partners per step")
    base = {"value": v, "unit": "deltas/s", "cores": threads, "kind": kind, "sample": sample}
    cfg = bench_config(n, int(w["a_src"].shape[0]), int(w["b_src"].shape[0]), R, 1)
    if rps != R:
        cfg["reference_rows_per_step"] = rps
    out = {"impl": "reference", "metric": "exact swap-deltas/s", "value": v, "unit": "deltas/s", "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
           "config": cfg, "cpu_baseline": base,
           "e2e": {"value": v, "unit": "deltas/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args, ws, rank, local, dist):
    A, B, truth, init, rows = make_workload()
    n = A.n
    R = args.rows_per_step
    eng = bm.Engine(local)
    eng.set_graphs(A, B)
    eng.set_mapping(init)
    score0 = eng.score()
    bytes_row = algorithmic_bytes_per_row(A, B, init)

    starts = step_starts(n, args.warmup, 0.5) + step_starts(n, args.steps)
    nsteps = args.warmup + args.steps

    def batch(step):
        idx = (starts[step] + rank * R + np.arange(R)) % n
        return np.ascontiguousarray(rows[idx])

    # every batch's rows staged on the device before timing
    all_rows = np.concatenate([batch(s) for s in range(nsteps)]).astype(np.int32)
    d_rows = eng.dev_alloc(all_rows.nbytes)
    eng.h2d(d_rows, all_rows)
    d_res = eng.dev_alloc(bm.ROW_DTYPE.itemsize * R)
    ev = [(eng.event(), eng.event()) for _ in range(nsteps)]

    def device_step(step):
        eng.l2_flush()
        eng.record(ev[step][0])
        eng.rows_best_dev(d_rows + 4 * R * step, None, R, d_res)
        eng.record(ev[step][1])

    # clocks are sampled from the warm-up on: the timed region alone lasts a
    # few milliseconds, shorter than a few NVML polls
    clocks = ClockSampler(eng.pci_bus_id())
    for s in range(args.warmup):
        device_step(s)
    eng.sync()
    barrier(dist)
    t_wall = time.perf_counter()
    launches_a = eng.launch_count()
    for s in range(args.warmup, nsteps):
        device_step(s)
    eng.sync()
    wall = time.perf_counter() - t_wall
    launches_b = eng.launch_count()
    clk = clocks.stop()
    barrier(dist)
    step_ms = [eng.elapsed_ms(*ev[s]) for s in range(args.warmup, nsteps)]
    total_ms = float(sum(step_ms))
    total_bytes = int(sum(int(bytes_row[batch(s)].sum()) for s in range(args.warmup, nsteps)))

    deltas_step = R * (n - 1)
    max_ms = dist_max(dist, total_ms)
    all_deltas = dist_sum(dist, float(deltas_step * args.steps))
    value = all_deltas / (max_ms / 1000.0)

    # e2e through the C ABI with host buffers (pinned): rows in, row results out
    h_rows, p_rows = pinned_array(4 * R, np.int32, R)
    h_res, p_res = pinned_array(bm.ROW_DTYPE.itemsize * R, bm.ROW_DTYPE, R)
    L = bm.cuda_lib()
    e2e_s = 0.0
    for s in range(args.warmup + args.steps):
        h_rows[:] = batch(s)
        eng.l2_flush()
        eng.sync()
        t0 = time.perf_counter()
        st = L.bm_rows_best(eng.h, p_rows, None, R, p_res)
        dt = time.perf_counter() - t0
        if st != bm.BM_OK:
            raise bm.BMError(st, "bm_rows_best")
        if s >= args.warmup:
            e2e_s += dt
    e2e_s = dist_max(dist, e2e_s)
    e2e_val = all_deltas / e2e_s

    peak, peak_kind = measured_peaks()
    achieved = total_bytes / (total_ms / 1000.0) / 1e9
    traffic, traffic_rec = recorded_traffic(args.steps, args.warmup, R)
    l2 = l2_peak(eng)
    out = {"metric": "exact swap-deltas/s", "value": value, "unit": "deltas/s", "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int64", "data": "synthetic",
           "config": bench_config(n, A.m, B.m, R, ws),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak,
                        "traffic": traffic, "peak_source": peak_kind,
                        "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of the row launches, "
                                           f"summed per step (a step's rows may run as two launches), mean of "
                                           f"{traffic_rec['steps']} timed steps of this command, kernel "
                                           f"source digest {traffic_rec['kernel_digest']}") if traffic_rec else
                                          "no ncu record of this kernel source and command",
                        "l2_peak": l2, "l2_frac": (achieved / l2) if l2 else None,
                        "l2_peak_source": "measured in this run: 16-byte ld.cg reads of a 64 MiB L2-resident buffer, "
                                          "20 passes, CUDA events",
                        "kernel": "rows_kernel (whole-row 2-hop scatter, fused row reduction)",
                        "bytes_per_step": total_bytes / args.steps},
           "e2e": {"value": e2e_val, "unit": "deltas/s", "h2d_bytes_per_step": 4 * R,
                   "d2h_bytes_per_step": bm.ROW_DTYPE.itemsize * R},
           "gpu_launches": int(launches_b - launches_a), "timed_wall_s": wall, "score_init": score0}
    if clk:
        out["clocks"] = clk
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(A, B, init, rows, starts[args.warmup:], budget_s=args.ref_seconds)
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        out["reference_gpu"] = reference_gpu(A, B, init, batch(args.warmup))
        rg = out["reference_gpu"]
        if "deltas_per_s" in rg:
            # the engine's row kernel on that same batch, from the timed steps
            rg["engine_deltas_per_s_same_batch"] = deltas_step / (step_ms[0] / 1e3)
    converged_pi = None
    if rank == 0 and ws == 1 and args.search_seconds > 0:
        out["search"] = plain_search(eng, rows, args.search_seconds)
        if out["search"]["converged"]:
            converged_pi = eng.get_mapping()
    eng.close()
    if rank == 0 and ws == 1 and args.learned_seconds > 0 and out.get("search", {}).get("converged"):
        out["learned_vs_plain"] = learned_compare(local, A, B, init, rows, out["search"], args.learned_seconds)
    if rank == 0 and ws == 1 and args.learned_seconds > 0:
        out["learned_vs_uniform"] = learned_vs_uniform(local, A, B, init, rows)
    if rank == 0 and ws == 1 and not args.no_extras:
        out["initial_matching"] = initial_matching(local, A, B, init)
        out["higher_order"] = higher_order(local, A, B, init, not args.no_reference_gpu)
        out["delta_table"] = delta_table(local, A, B, init, out.get("search", {}))
        out["subset_assignment"] = [subset_assignment(local, A, B, init, "initial matching")]
        if converged_pi is not None:
            out["subset_assignment"].append(subset_assignment(local, A, B, converged_pi,
                                                              "plain search's local optimum"))
        out["sa_chains"] = sa_chains(local, args.sa_steps)
    if rank == 0:
        print(json.dumps(out), flush=True)


TRAFFIC_RECORD = os.path.join(REPO, "profiles", "rows_kernel_traffic.json")
ROWS_KERNEL_SOURCES = ("brain-match_b200/csrc/bm_rows.cu",)


def rows_kernel_digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for rel in ROWS_KERNEL_SOURCES:
        with open(os.path.join(REPO, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def recorded_traffic(steps: int, warmup: int, rows_per_step: int):
    """DRAM bytes (read + write) of the row kernel per step (the step's
    launches summed) from an ncu capture of this bench's own launches (the
    record names the capture and the digest of the kernel's sources it was
    taken on); None unless the record is of the current kernel source and of
    this run's steps, warm-up and batch size."""
    try:
        with open(TRAFFIC_RECORD) as f:
            rec = json.load(f)
        if (rec["kernel_digest"] == rows_kernel_digest() and rec["steps"] == steps and rec["warmup"] == warmup
                and rec["rows_per_step"] == rows_per_step):
            return float(rec["dram_bytes_per_step"]), rec
    except (OSError, ValueError, KeyError):
        pass
    return None, None


def l2_peak(eng):
    """Measured L2 read bandwidth of this GPU (GB/s), 64 MiB read 20 times."""
    g = C.c_double()
    st = bm.cuda_lib().bm_probe_l2_bandwidth(eng.h, 64 << 20, 20, C.byref(g))
    return g.value if st == bm.BM_OK else None


def reference_gpu(A, B, init, rows_batch):
    """The reference's own GPU swap-delta kernel (calculateSwapDeltasKernelQuick,
    src/graph-re-alignment-gpu.cu:139-248, compiled for sm_100a into
    oracle/_ref/librefgpu.so) on one of the timed batches: the rows as its
    changed vertices, every partner, dense int16 matrices as its driver builds
    them; CUDA events around three launches after one warm-up."""
    path = os.path.join(REPO, "oracle", "_ref", "librefgpu.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/librefgpu.so not built"}
    L = C.CDLL(path)
    vp = C.c_void_p
    L.refgpu_quick.restype = C.c_int
    L.refgpu_quick.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, C.c_longlong, vp, vp, vp, vp, vp, C.c_int, C.c_int,
                               C.POINTER(C.c_float), vp, vp]
    L.refgpu_total_pairs.restype = C.c_longlong
    L.refgpu_total_pairs.argtypes = [C.c_int, C.c_int]
    r = np.ascontiguousarray(rows_batch, np.int32)
    ms = C.c_float()
    st = L.refgpu_quick(A.n, A.m, A.src.ctypes.data, A.dst.ctypes.data, A.w.ctypes.data, B.m, B.src.ctypes.data,
                        B.dst.ctypes.data, B.w.ctypes.data, init.ctypes.data, r.ctypes.data, len(r), 3, C.byref(ms),
                        None, None)
    if st != 0:
        return {"unavailable": f"reference kernel returned CUDA error {st}"}
    pairs = int(L.refgpu_total_pairs(A.n, len(r)))
    return {"kernel": "calculateSwapDeltasKernelQuick", "rows": len(r), "pairs_per_launch": pairs,
            "ms_per_launch": ms.value, "deltas_per_s": pairs / (ms.value / 1e3),
            "timing": "CUDA events, 3 launches after one warm-up, inputs resident"}


def reference_gpu3(A, B, init, rows, batch=4096):
    """The reference's own 3-vertex GPU kernel (calculateThreeNodeSwapKernel,
    src/graph-re-alignment-gpu-3-swap.cu:43-305, oracle/_ref/librefgpu3.so) on
    the first `batch` triplets of its enumeration around six rows: triplets/s,
    each with five permutations over dense int16 matrices."""
    path = os.path.join(REPO, "oracle", "_ref", "librefgpu3.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/librefgpu3.so not built"}
    L = C.CDLL(path)
    vp = C.c_void_p
    L.refgpu3_triplets.restype = C.c_int
    L.refgpu3_triplets.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, C.c_longlong, vp, vp, vp, vp, vp, C.c_int,
                                   C.c_int, C.c_int, C.POINTER(C.c_float), vp, vp]
    changed = np.ascontiguousarray(rows[A.n // 4:A.n // 4 + 6], np.int32)
    ms = C.c_float()
    st = L.refgpu3_triplets(A.n, A.m, A.src.ctypes.data, A.dst.ctypes.data, A.w.ctypes.data, B.m, B.src.ctypes.data,
                            B.dst.ctypes.data, B.w.ctypes.data, init.ctypes.data, changed.ctypes.data, 6, batch, 1,
                            C.byref(ms), None, None)
    if st != 0:
        return {"unavailable": f"reference kernel returned CUDA error {st}"}
    return {"kernel": "calculateThreeNodeSwapKernel", "triplets": batch, "ms_per_launch": ms.value,
            "sets_per_s": batch / (ms.value / 1e3), "permutations_per_set": 5,
            "timing": "CUDA events, one launch after one warm-up, inputs resident"}


MLP_FLOP_PER_PAIR = 2 * (24 * 128 + 128 * 128 + 128)
# forward, then dW2 = H1^T dH2, dH1 = dH2 W2^T, dW1 = X^T dH1, dw3 and dh2
MLP_TRAIN_FLOP_PER_RECORD = MLP_FLOP_PER_PAIR + 2 * 128 * 128 + 2 * 128 * 128 + 2 * 24 * 128 + 3 * 128


def bf16_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def scorer_throughput(device, A, B, init, rows):
    """The MLP row scorer on 1,184 rows (8 per SM pair of CTAs), inputs
    resident: tensor-core and SIMT kernels, CUDA events, and the tensor-core
    kernel against the measured BF16 peak."""
    n = A.n
    out = {}
    e = bm.Engine(device)
    e.set_graphs(A, B)
    e.set_mapping(init)
    m = bm.Mlp(e, seed=1)
    R = min(n, 1184)
    d_rows = e.dev_alloc(4 * R)
    e.h2d(d_rows, np.ascontiguousarray(rows[:R]))
    d_sc = e.dev_alloc(4 * R * n)
    a, b = e.event(), e.event()
    for backend, reps, name in ((0, 5, "tcgen05"), (1, 1, "simt")):
        m.set_backend(backend)
        m.score_rows_dev(d_rows, R, d_sc)
        e.sync()
        e.record(a)
        for _ in range(reps):
            m.score_rows_dev(d_rows, R, d_sc)
        e.record(b)
        e.sync()
        m.status()
        ms = e.elapsed_ms(a, b) / reps
        pairs = R * (n - 1)
        out[f"scorer_{name}"] = {"pairs_per_s": pairs / (ms / 1e3),
                                 "tflops": pairs * MLP_FLOP_PER_PAIR / (ms / 1e3) / 1e12, "ms_per_launch": ms,
                                 "rows_per_launch": R}
    # training: minibatch steps (gather, gradient, AdamW) of 8,192 records
    m.reserve_records(1 << 18)
    m.collect_rows(rows[:1024], per_row=128, seed=3)
    for backend, steps, name in ((0, 200, "tcgen05"), (1, 20, "simt")):
        m.set_backend(backend)
        m.fit(2, batch=8192, lr=1e-3)
        e.sync()
        e.record(a)
        m.fit(steps, batch=8192, lr=1e-3)
        e.record(b)
        e.sync()
        ms = e.elapsed_ms(a, b) / steps
        out[f"training_{name}"] = {"records_per_s": 8192 / (ms / 1e3), "ms_per_step": ms,
                                   "tflops": 8192 * MLP_TRAIN_FLOP_PER_RECORD / (ms / 1e3) / 1e12,
                                   "batch": 8192, "steps": steps,
                                   "timing": "CUDA events around whole steps: gather, gradient, AdamW"}
    m.set_backend(0)
    peak, kind = bf16_peak()
    tc = out["scorer_tcgen05"]["tflops"]
    out["roofline_scorer"] = {"bound": "tensor", "achieved": tc, "peak": peak, "unit": "TFLOP/s", "frac": tc / peak,
                              "peak_source": kind, "kernel": "mlp_rows_tc_kernel",
                              "flop_per_pair": MLP_FLOP_PER_PAIR}
    e.dev_free(d_rows)
    e.dev_free(d_sc)
    e.close()
    return out


def learned_compare(device, A, B, init, rows, plain, seconds):
    """Learned vs plain proposals from the same initial matching: time to the
    plain search's converged score (record harvest, training and inference
    included), hit rates of one proposal pass, and the tensor-core scorer's
    throughput against the measured BF16 peak."""
    n = A.n

    def engine():
        e = bm.Engine(device)
        e.set_graphs(A, B)
        e.set_mapping(init)
        return e

    out = {"plain_seconds": plain["seconds"], "plain_score": plain["score"]}
    out.update(scorer_throughput(device, A, B, init, rows))

    def one_pass(mm, uniform):
        _, p, s = mm.search(rows, topk=64, max_sweeps=1, exact_fallback=False, uniform=uniform, seed=7)
        return {"hit_rate": s.hits / max(1, s.proposals), "proposals": int(s.proposals), "accepts": int(p.accepts),
                "score": int(p.score)}

    e = engine()
    out["pass_uniform"] = one_pass(bm.Mlp(e, seed=1), True)
    e.close()
    # learned: harvest + training + search, all inside the clock
    e = engine()
    t0 = time.perf_counter()
    m = bm.Mlp(e, seed=1)
    m.reserve_records(5_000_000)
    nrec = m.collect_rows(rows, per_row=256, seed=3)
    l0 = m.fit(1, batch=8192, lr=2e-3)
    l1 = m.fit(1500, batch=8192, lr=2e-3)
    e.sync()
    t_train = time.perf_counter() - t0
    w = m.params()
    st, p, s = m.search(rows, topk=64, exact_fallback=True, fallback_accepts=n // 100, train_every=4,
                        train_batch=4096, lr=5e-4, target_score=plain["score"], time_budget=seconds)
    t_total = time.perf_counter() - t0
    out["learned"] = {"seconds_to_plain_score": t_total if p.score >= plain["score"] else None,
                      "seconds": t_total, "score": int(p.score), "records": int(nrec), "harvest_train_s": t_train,
                      "loss_first": l0, "loss_last": l1, "t_propose": s.t_propose, "t_exact": s.t_exact,
                      "t_train_online": s.t_train, "hit_rate": s.hits / max(1, s.proposals),
                      "exact_passes": int(s.exact_passes), "timed_out": st == bm.BM_TIMEOUT}
    e.close()
    e = engine()
    m = bm.Mlp(e, seed=1)
    m.set_params(w)
    out["pass_trained"] = one_pass(m, False)
    e.close()
    e = engine()
    out["pass_untrained"] = one_pass(bm.Mlp(e, seed=1), False)
    e.close()
    return out


def learned_vs_uniform(device, A, B, init, rows, uniform_seconds=8.0):
    """Proposal searches with exact checks from the greedy matching: uniform
    random partners (64 per row, 4,736 rows per batch: the fastest of the
    uniform settings measured) for uniform_seconds, then the model's top 32 of
    1,024 sampled partners per row (2,368 rows per batch, feature table
    refreshed every 4 batches) until it reaches the uniform search's score,
    with record harvest and training inside its clock.  Same seed and start."""
    def engine():
        e = bm.Engine(device)
        e.set_graphs(A, B)
        e.set_mapping(init)
        return e

    e = engine()
    m = bm.Mlp(e, seed=1)
    t0 = time.perf_counter()
    _, p, s = m.search(rows, topk=64, uniform=True, exact_fallback=False, time_budget=uniform_seconds, seed=7,
                       rows_per_batch=4736)
    t_u = time.perf_counter() - t0
    out = {"uniform": {"seconds": t_u, "score": int(p.score), "proposals": int(s.proposals), "sweeps": int(p.sweeps),
                       "hit_rate": s.hits / max(1, s.proposals), "topk": 64, "rows_per_batch": 4736}}
    e.close()
    e = engine()
    t0 = time.perf_counter()
    m = bm.Mlp(e, seed=1)
    m.reserve_records(5_000_000)
    nrec = m.collect_rows(rows, per_row=256, seed=3)
    m.fit(1500, batch=8192, lr=2e-3)
    e.sync()
    t_train = time.perf_counter() - t0
    st, p2, s2 = m.search(rows, topk=32, sample=1024, exact_fallback=False, target_score=out["uniform"]["score"],
                          time_budget=2 * uniform_seconds, seed=7, rows_per_batch=2368, refresh_batches=4)
    t_l = time.perf_counter() - t0
    reached = p2.score >= out["uniform"]["score"]
    out["learned"] = {"seconds": t_l, "reached": bool(reached), "score": int(p2.score), "harvest_train_s": t_train,
                      "records": int(nrec), "proposals": int(s2.proposals), "sweeps": int(p2.sweeps),
                      "hit_rate": s2.hits / max(1, s2.proposals), "t_propose": s2.t_propose, "t_exact": s2.t_exact,
                      "topk": 32, "sample": 1024, "rows_per_batch": 2368}
    out["time_ratio"] = (t_l / t_u) if reached else None
    e.close()
    return out


def higher_order(device, A, B, init, reference_kernels=True):
    """Exact k-set permutation deltas on the full-scale pair: 4,096 random
    8-subsets (8! = 40,320 permutations each) and 65,536 3-vertex sets along
    2-paths u -> x -> y (all 6 permutations), best permutation per set."""
    n = A.n
    e = bm.Engine(device)
    e.set_graphs(A, B)
    e.set_mapping(init)
    rng = np.random.default_rng(4)
    sets8 = np.stack([rng.choice(n, 8, replace=False) + 1 for _ in range(4096)]).astype(np.int32)
    order = np.argsort(A.src, kind="stable")
    src, dst = A.src[order], A.dst[order]
    ptr = np.searchsorted(src, np.arange(0, n + 2))  # out-list of v: [ptr[v], ptr[v+1])
    e_idx = rng.integers(0, len(src), 4 * 65536)
    u, x = src[e_idx], dst[e_idx]
    deg = ptr[x + 1] - ptr[x]
    ok = deg > 0
    pick = ptr[x] + (rng.random(len(x)) * np.maximum(deg, 1)).astype(np.int64)
    y = np.where(ok, dst[np.minimum(pick, len(dst) - 1)], 0)
    good = ok & (y != u) & (y != x) & (u != x)
    sets3 = np.stack([u[good], x[good], y[good]], 1)[:65536].astype(np.int32)
    out = {}
    for k, sets, nperm in ((8, sets8, 40320), (3, sets3, 6)):
        e.kset_eval(k, sets[:64])
        t0 = time.perf_counter()
        best, _ = e.kset_eval(k, sets)
        dt = time.perf_counter() - t0
        out[f"k{k}"] = {"sets": int(len(sets)), "sets_per_s": len(sets) / dt,
                        "permutation_deltas_per_s": len(sets) * nperm / dt, "improving_sets": int((best > 0).sum()),
                        "seconds": dt, "timing": "host call, transfers included"}
    # device time of the 3-sets alone, for the reference kernel beside it
    d_sets = e.dev_alloc(sets3.nbytes)
    e.h2d(d_sets, sets3)
    d_best = e.dev_alloc(8 * len(sets3))
    d_perm = e.dev_alloc(4 * 3 * len(sets3))
    d_status = e.dev_alloc(4)
    e.h2d(d_status, np.zeros(1, np.int32))
    a, b = e.event(), e.event()
    e.kset_eval_dev(3, d_sets, len(sets3), d_best, d_perm, d_status)
    e.record(a)
    e.kset_eval_dev(3, d_sets, len(sets3), d_best, d_perm, d_status)
    e.record(b)
    e.sync()
    ms = e.elapsed_ms(a, b)
    out["k3"]["device_sets_per_s"] = len(sets3) / (ms / 1e3)
    e.close()
    if reference_kernels:
        order = bm.rows_from_ordering(bm.ordering_by_weighted_degree(A))
        out["k3_reference_gpu"] = reference_gpu3(A, B, init, order)
    return out


def sa_chains(device, steps, candidates=0):
    """Batched annealing chains: 16 pairs with n uniform in 2,000..20,000 and
    80 n edges, 4 chains per pair, T 5 -> 0.01 geometric."""
    rng = np.random.default_rng(3)
    e = bm.Engine(device)
    batch = bm.Batch(e)
    inits, ns = [], []
    t_gen = time.perf_counter()
    for i in range(16):
        n = int(rng.integers(2000, 20001))
        A, B, truth, init = bm.gen_pair(3, n=n, m_target=80 * n, seed=300 + i)
        batch.add_pair(A, B)
        inits.append(init)
        ns.append(n)
    t_gen = time.perf_counter() - t_gen
    chain_pair = np.repeat(np.arange(16), 4).astype(np.int32)
    keys = 1000 + np.arange(64)
    init_pis = [inits[p] for p in chain_pair]
    batch.sa_run(chain_pair, keys, init_pis, 2000, candidates=candidates)  # autotune and warm-up
    t0 = time.perf_counter()
    pis, scores, acc, st = batch.sa_run(chain_pair, keys, init_pis, steps, t0=5.0, t_end=0.01, candidates=candidates)
    dt = time.perf_counter() - t0
    out = {"chains": 64, "pairs": 16, "n_range": [min(ns), max(ns)], "steps_per_chain": steps,
           "proposals_per_s": 64 * steps / dt, "seconds": dt, "candidates_per_iteration": int(st.candidates),
           "ctas_per_chain": int(st.ctas_per_chain), "threads_per_cta": int(st.threads_per_cta),
           "launches": int(st.launches), "accepts_mean": float(np.mean(acc)), "generation_s": t_gen,
           "timing": "host call: graph replay, transfers and final scores included"}
    batch.close()
    e.close()
    return out


def initial_matching(device, A, B, init):
    """Greedy-similarity initial matching of the full-scale pair: the host
    library (all host cores) and the device version, which must agree."""
    t = time.perf_counter()
    host = bm.greedy_match(A, B)
    th = time.perf_counter() - t
    with bm.Engine(device) as e:
        e.greedy_match(A, B)
        t = time.perf_counter()
        dev = e.greedy_match(A, B)
        td = time.perf_counter() - t
    return {"host_seconds": th, "device_seconds": td, "equal": bool(np.array_equal(host, dev)),
            "equals_workload_init": bool(np.array_equal(dev, init)), "host_cores": os.cpu_count()}


def delta_table(device, A, B, init, plain):
    """The exact delta table of the full-scale pair (every pair, int32), its
    top-1,024, and the table search from the initial matching to its local
    optimum, against the plain search's score."""
    n = A.n
    with bm.Engine(device) as e:
        e.set_graphs(A, B)
        e.set_mapping(init)
        d_tab, ld = e.table_alloc()
        a, b = e.event(), e.event()
        e.delta_table_dev(d_tab, ld)  # warm-up
        e.sync()
        e.record(a)
        e.delta_table_dev(d_tab, ld)
        e.record(b)
        e.sync()
        t_build = e.elapsed_ms(a, b) / 1e3
        e.table_topk(d_tab, ld, 1024)  # warm-up (scratch allocated on first use)
        t = time.perf_counter()
        e.table_topk(d_tab, ld, 1024)
        t_topk = time.perf_counter() - t
        prog, st = e.search_table(d_tab, ld, k=1024, time_budget=60.0)
        out = {"table_bytes": 4 * (n + 1) * ld, "build_seconds": t_build,
               "build_deltas_per_s": n * (n - 1) / t_build, "topk1024_seconds": t_topk,
               "search_seconds": prog.seconds, "search_score": int(prog.score), "search_accepts": int(prog.accepts),
               "search_rounds": int(prog.sweeps), "converged": int(prog.converged),
               "plain_score": plain.get("score"), "plain_seconds": plain.get("seconds")}
        e.dev_free(d_tab)
    return out


def subset_assignment(device, A, B, start_pi, label):
    """Independent-subset re-assignment (random A-independent subsets of up
    to 4,096 members, optimal assignment of their images) from a given
    mapping: time per iteration and the score it adds."""
    with bm.Engine(device) as e:
        e.set_graphs(A, B)
        e.set_mapping(start_pi)
        s0 = e.score()
        prog, st = e.search_hungarian(k=4096, seed=5, iterations=10)
        return {"start": label, "start_score": int(s0), "score": int(prog.score), "gain": int(prog.score - s0),
                "iterations": int(prog.launches), "members_per_iteration": int(prog.rows_done // max(1, prog.launches)),
                "moved": int(prog.accepts), "seconds": prog.seconds,
                "seconds_per_iteration": prog.seconds / max(1, prog.launches)}


def plain_search(eng, rows, seconds):
    """Time-to-score of the plain batched search from the same initial matching."""
    traj = []
    prog = bm.Progress()
    t0 = time.perf_counter()
    traj.append([0.0, eng.tracked_score()])
    while time.perf_counter() - t0 < seconds:
        prog, st = eng.search_batched(rows=rows, time_budget=min(1.0, seconds), prog=prog)
        traj.append([round(time.perf_counter() - t0, 3), int(prog.score)])
        if prog.converged:
            break
    return {"seconds": round(time.perf_counter() - t0, 3), "accepts": int(prog.accepts),
            "evaluated": int(prog.evaluated), "trajectory": traj, "converged": int(prog.converged),
            "score": int(prog.score)}


def run_section(args):
    """One side section of the bench on the full-scale workload, alone."""
    if args.only == "sa_chains":
        out = sa_chains(0, args.sa_steps, args.sa_candidates)
    else:
        A, B, truth, init, rows = make_workload()
        if args.only == "initial_matching":
            out = initial_matching(0, A, B, init)
        elif args.only == "higher_order":
            out = higher_order(0, A, B, init)
        elif args.only == "delta_table":
            out = delta_table(0, A, B, init, {})
        elif args.only == "mlp_scorer":
            out = scorer_throughput(0, A, B, init, rows)
        elif args.only == "learned_vs_uniform":
            out = learned_vs_uniform(0, A, B, init, rows)
        else:
            out = subset_assignment(0, A, B, init, "initial matching")
    print(json.dumps({"section": args.only, "result": out}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows-per-step", type=int, default=57)
    ap.add_argument("--ref-seconds", type=float, default=12.0, help="budget of the engine arm's cpu_baseline sample")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="budget of the reference arm's timed steps (seconds); larger K get fewer rows per step")
    ap.add_argument("--write-workload", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU kernels on the same batches")
    ap.add_argument("--search-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned-seconds", type=float, default=90.0)
    ap.add_argument("--no-extras", action="store_true", help="skip the k-set and annealing-chain sections")
    ap.add_argument("--sa-steps", type=int, default=1_000_000)
    ap.add_argument("--sa-candidates", type=int, default=0, help="starting proposals per iteration (0: autotuned)")
    ap.add_argument("--only", default=None,
                    choices=["initial_matching", "higher_order", "delta_table", "subset_assignment", "sa_chains",
                             "mlp_scorer", "learned_vs_uniform"],
                    help="run one side section alone and print its result (a profiling target, not a bench line)")
    args = ap.parse_args()
    if args.write_workload:
        write_workload(args.write_workload)
        return
    if args.only:
        run_section(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local, dist = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank, dist)
        else:
            run_ours(args, ws, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
