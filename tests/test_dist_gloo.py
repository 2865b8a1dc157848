"""The multi-rank path on the CPU: world-size-2 gloo process groups run the
sharded row search protocol (each rank its rows, candidates all-gathered,
the same deterministic selection everywhere, so the mappings stay identical)
and the island synchronisation.  Row evaluation uses the oracle here, in place
of each rank's GPU; the exchange and the selection are the product's
(bm_dist.py, bm_select_independent_host)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _select(A, pairs, deltas):
    import bmb200 as bm
    L = bm.host_lib()
    L.bm_select_independent_host.restype = C.c_int
    L.bm_select_independent_host.argtypes = [C.POINTER(bm.Edges), C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                             C.POINTER(C.c_int32)]
    e = A.edges_struct()
    p = np.ascontiguousarray(pairs.reshape(-1).astype(np.int32))
    d = np.ascontiguousarray(deltas.astype(np.int64))
    chosen = np.zeros(max(1, d.shape[0]), np.int32)
    nc = C.c_int32()
    assert L.bm_select_independent_host(C.byref(e), p.ctypes.data, d.ctypes.data, d.shape[0], chosen.ctypes.data,
                                        C.byref(nc)) == 0
    return chosen[: nc.value]


def _sharded_round(orc, A, pi, rows):
    full = orc.rows(pi, rows) if rows.shape[0] else np.zeros((0, A.n + 1), np.int64)
    pairs, deltas = [], []
    for i, u in enumerate(rows):
        d = full[i].copy()
        d[0] = np.iinfo(np.int64).min
        d[u] = np.iinfo(np.int64).min
        v = int(np.argmax(d))
        if d[v] > 0:
            pairs.append((u, v))
            deltas.append(d[v])
    return np.array(pairs, np.int32).reshape(-1, 2), np.array(deltas, np.int64)


def _worker(rank, world, port, results):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "brain-match_b200", "python"))
    sys.path.insert(0, HERE)
    import torch.distributed as dist

    import bm_dist
    import bmb200 as bm
    from oracle_bind import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        A, B, truth, init = bm.gen_pair(1, n=300, m_target=3000, seed=11)
        orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
        order = np.arange(1, A.n + 1, dtype=np.int32)
        pi = init.copy()
        score = orc.score(pi)
        hist = []
        for rnd in range(12):
            rows = bm_dist.round_rows(order, rnd, 16, rank, world)
            pairs, deltas = _sharded_round(orc, A, pi, rows)
            gp, gd = bm_dist.gather_candidates(pairs, deltas)
            for i in _select(A, gp, gd):
                u, v = gp[i]
                pi[u], pi[v] = pi[v], pi[u]
                score += int(gd[i])
            hist.append((score, int(pi.astype(np.int64).dot(np.arange(pi.shape[0])) % (1 << 61))))
        assert score == orc.score(pi)
        # island synchronisation: ranks diverge, then adopt the best
        rng = np.random.default_rng(rank)
        q = pi.copy()
        for _ in range(3 + rank):
            a, b = rng.choice(np.arange(1, A.n + 1), 2, replace=False)
            q[a], q[b] = q[b], q[a]
        best, best_rank, qb = bm_dist.island_best(orc.score(q), q)
        results[rank] = (hist, pi.tolist(), best, best_rank, qb.tolist(), orc.score(q))
    finally:
        dist.destroy_process_group()


def test_sharded_search_and_island_sync_two_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    results = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    h0, pi0, b0, br0, q0, s0 = results[0]
    h1, pi1, b1, br1, q1, s1 = results[1]
    assert h0 == h1 and pi0 == pi1  # identical trajectories on both ranks
    assert h0[-1][0] > h0[0][0] or h0[0][0] > 0
    assert b0 == b1 == max(s0, s1) and br0 == br1 and q0 == q1

    # the same protocol in one process (both ranks' rows, rank-order gather) gives the same result
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "brain-match_b200", "python"))
    import bm_dist
    import bmb200 as bm
    from oracle_bind import Oracle
    A, B, truth, init = bm.gen_pair(1, n=300, m_target=3000, seed=11)
    orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    order = np.arange(1, A.n + 1, dtype=np.int32)
    pi = init.copy()
    for rnd in range(12):
        parts = [_sharded_round(orc, A, pi, bm_dist.round_rows(order, rnd, 16, r, 2)) for r in range(2)]
        gp = np.concatenate([p[0] for p in parts]).reshape(-1, 2)
        gd = np.concatenate([p[1] for p in parts])
        for i in _select(A, gp, gd):
            u, v = gp[i]
            pi[u], pi[v] = pi[v], pi[u]
    assert pi.tolist() == pi0
