"""The sharded search through the C ABI on the GPU.

Two ranks (processes) share the one GPU of this machine over the TCP
transport: their kernels never wait on each other (the exchange is on the
host), and they must end with the same mapping as a single-process replay of
the protocol (each rank's rows evaluated under the same mapping, candidates
concatenated in rank order, bm_select_independent, bm_apply_swaps).  The NCCL
transport runs as a world of one (one GPU here): its collectives must give the
same search as the TCP transport."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

import bmb200 as bm

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PY = os.path.join(os.path.dirname(HERE), "brain-match_b200", "python")
RPR = 24  # rows per rank and round


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _pair():
    A, B, truth, init = bm.gen_pair(1, n=1200, m_target=24000, seed=21)
    rows = bm.rows_from_ordering(bm.ordering_by_weighted_degree(A))
    return A, B, init, rows


def _rank_worker(rank, world, port, q):
    sys.path.insert(0, PY)
    import bmb200 as bm
    A, B, init, rows = _pair()
    eng = bm.Engine(0)
    eng.set_graphs(A, B)
    eng.set_mapping(init)
    comm = bm.Comm(bm.BM_COMM_TCP, rank, world, f"127.0.0.1:{port}", timeout=120.0, eng=eng)
    try:
        prog, st = comm.search_sharded(rows=rows, rows_per_rank=RPR)
        q.put((rank, eng.get_mapping().tolist(), int(prog.score), int(prog.accepts), int(prog.converged),
               int(eng.score())))
    finally:
        comm.close()
        eng.close()


def _replay(world, rpr=RPR):
    """The protocol of bm_search_sharded in one process, through the engine."""
    A, B, init, rows = _pair()
    eng = bm.Engine(0)
    eng.set_graphs(A, B)
    eng.set_mapping(init)
    n = A.n
    per_round = world * rpr
    rounds_per_pass = -(-n // per_round)
    rnd = 0
    pass_acc = 0
    while True:
        idx = (rnd * per_round + np.arange(per_round)) % n
        pairs, deltas = [], []
        for r in range(world):
            res = eng.rows_best(rows[idx[r::world]])
            for x in res:
                if x["best_delta"] > 0:
                    pairs.append((x["row"], x["best"]))
                    deltas.append(x["best_delta"])
        p = np.array(pairs, np.int32).reshape(-1, 2)
        d = np.array(deltas, np.int64)
        chosen = eng.select_independent(p, d)
        if len(chosen):
            eng.apply_swaps(p[chosen], d[chosen])
            pass_acc += len(chosen)
        rnd += 1
        if rnd % rounds_per_pass == 0:
            if pass_acc == 0:
                break
            pass_acc = 0
    out = eng.get_mapping().tolist(), eng.score()
    eng.close()
    return out


def test_two_ranks_share_a_gpu_over_tcp():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=600)
        out[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    pi0, s0, a0, c0, e0 = out[0]
    pi1, s1, a1, c1, e1 = out[1]
    assert pi0 == pi1 and s0 == s1 == e0 == e1 and a0 == a1 and c0 == c1 == 1
    pi_r, s_r = _replay(2)
    assert pi0 == pi_r and s0 == s_r


def test_nccl_world_of_one_equals_tcp():
    A, B, init, rows = _pair()
    res = {}
    for kind in (bm.BM_COMM_TCP, bm.BM_COMM_NCCL):
        eng = bm.Engine(0)
        eng.set_graphs(A, B)
        eng.set_mapping(init)
        comm = bm.Comm(kind, 0, 1, None, timeout=120.0, eng=eng)
        try:
            prog, st = comm.search_sharded(rows=rows, rows_per_rank=2 * RPR)
            assert prog.converged == 1
            assert comm.allreduce_sum(41) == 41
            gp, gd = comm.allgather_swaps(np.array([[5, 9], [7, 2]], np.int32), np.array([3, -4], np.int64), cap=8)
            assert gp.tolist() == [[5, 9], [7, 2]] and gd.tolist() == [3, -4]
            pi = eng.get_mapping()
            best, br, q = comm.island_best(int(prog.score), pi)
            assert best == prog.score and br == 0 and q.tolist() == pi.tolist()
            res[kind] = (pi.tolist(), int(prog.score), int(prog.accepts))
        finally:
            comm.close()
            eng.close()
    assert res[bm.BM_COMM_TCP] == res[bm.BM_COMM_NCCL]
    pi_r, s_r = _replay(1, 2 * RPR)
    assert res[bm.BM_COMM_NCCL][0] == pi_r and res[bm.BM_COMM_NCCL][1] == s_r


def test_cli_two_ranks(tmp_path):
    """bm-align --ranks 2: two processes of the drop-in CLI on the one GPU over
    TCP; rank 0 writes the mapping, which equals the engine-level two-rank
    search with the same rows per rank and row order."""
    import subprocess
    A, B, init, rows = _pair()
    n = A.n
    gm, gf = str(tmp_path / "gm.csv"), str(tmp_path / "gf.csv")
    bm.write_graph_csv(gm, A)
    bm.write_graph_csv(gf, B)
    om, of = str(tmp_path / "om.csv"), str(tmp_path / "of.csv")
    bm.write_ordering(om, bm.ordering_by_weighted_degree(A))
    bm.write_ordering(of, bm.ordering_by_weighted_degree(B))
    inp = str(tmp_path / "in.csv")
    bm.write_mapping(inp, init)
    port = _free_port()
    procs = []
    for r in range(2):
        out = str(tmp_path / f"out{r}.csv")
        cmd = [os.path.join(bm.BIN_DIR, "bm-align"), gm, gf, om, of, inp, out, "--mode", "search", "--schedule",
               "ordering", "--rows-per-batch", str(RPR), "--ranks", "2", "--rank", str(r), "--addr",
               f"127.0.0.1:{port}", "--comm", "tcp", "--comm-timeout", "120"]
        procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=600) for p in procs]
    assert all(p.returncode == 0 for p in procs), [o[1] for o in outs]
    assert "Converged: yes" in outs[0][0] and "Rank 0 of 2" in outs[0][0]
    assert outs[1][0] == ""  # rank 1 prints no progress lines
    assert not os.path.exists(str(tmp_path / "out1.csv"))
    pi, cnt, _ = bm.read_mapping(str(tmp_path / "out0.csv"), n)
    pi_r, s_r = _replay(2)
    assert pi.tolist() == pi_r
