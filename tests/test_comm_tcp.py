"""The multi-rank path on the CPU, over the library's own TCP transport (no
MPI, no PyTorch): world-size-2 process pairs run the sharded row-search
protocol (each rank its rows, candidates all-gathered in rank order, the same
deterministic selection everywhere, so the mappings stay identical) and the
island synchronisation, and a rank that leaves makes the other's next
collective end with BM_TIMEOUT instead of waiting for ever.  Row evaluation
uses the oracle here in place of each rank's GPU; the exchange and the
selection are the product's (bm_comm_*, bm_select_independent_host)."""
import ctypes as C
import multiprocessing as mp
import os
import socket
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PY = os.path.join(os.path.dirname(HERE), "brain-match_b200", "python")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def round_rows(order, rnd, rows_per_rank, rank, world):
    """Rows of round `rnd` owned by `rank`, as bm_search_sharded deals them:
    world * rows_per_rank consecutive rows of `order` (cyclically), every
    world-th from the rank's own position."""
    n = order.shape[0]
    idx = (rnd * world * rows_per_rank + np.arange(world * rows_per_rank)) % n
    return np.ascontiguousarray(order[idx[rank::world]])


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


def _protocol_worker(rank, world, port, q):
    sys.path.insert(0, PY)
    sys.path.insert(0, HERE)
    import bmb200 as bm
    from oracle_bind import Oracle
    comm = bm.Comm(bm.BM_COMM_TCP, rank, world, f"127.0.0.1:{port}", timeout=60.0)
    try:
        A, B, truth, init = bm.gen_pair(1, n=300, m_target=3000, seed=11)
        orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
        order = np.arange(1, A.n + 1, dtype=np.int32)
        pi = init.copy()
        score = orc.score(pi)
        hist = []
        for rnd in range(12):
            rows = round_rows(order, rnd, 16, rank, world)
            pairs, deltas = _sharded_round(orc, A, pi, rows)
            gp, gd = comm.allgather_swaps(pairs, deltas, cap=world * 16)
            for i in _select(A, gp, gd):
                u, v = gp[i]
                pi[u], pi[v] = pi[v], pi[u]
                score += int(gd[i])
            hist.append((score, int(pi.astype(np.int64).dot(np.arange(pi.shape[0])) % (1 << 61))))
        assert score == orc.score(pi)
        total = comm.allreduce_sum(rank + 1)
        comm.barrier()
        # island synchronisation: ranks diverge, then adopt the best
        rng = np.random.default_rng(rank)
        qpi = pi.copy()
        for _ in range(3 + rank):
            a, b = rng.choice(np.arange(1, A.n + 1), 2, replace=False)
            qpi[a], qpi[b] = qpi[b], qpi[a]
        own = orc.score(qpi)
        best, best_rank, qb = comm.island_best(own, qpi)
        q.put((rank, hist, pi.tolist(), total, best, best_rank, qb.tolist(), own))
    finally:
        comm.close()


def test_sharded_protocol_and_island_sync_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_protocol_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=240)
        out[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    h0, pi0, t0, b0, br0, q0, s0 = out[0]
    h1, pi1, t1, b1, br1, q1, s1 = out[1]
    assert h0 == h1 and pi0 == pi1  # identical trajectories on both ranks
    assert h0[-1][0] > h0[0][0] or h0[0][0] > 0
    assert t0 == t1 == 3
    assert b0 == b1 == max(s0, s1) and br0 == br1 == (0 if s0 >= s1 else 1) and q0 == q1

    # the same protocol in one process (both ranks' rows, rank-order gather) gives the same result
    sys.path.insert(0, PY)
    import bmb200 as bm
    from oracle_bind import Oracle
    A, B, truth, init = bm.gen_pair(1, n=300, m_target=3000, seed=11)
    orc = Oracle(A.n, (A.src, A.dst, A.w), (B.src, B.dst, B.w))
    order = np.arange(1, A.n + 1, dtype=np.int32)
    pi = init.copy()
    for rnd in range(12):
        parts = [_sharded_round(orc, A, pi, round_rows(order, rnd, 16, r, 2)) for r in range(2)]
        gp = np.concatenate([p[0] for p in parts]).reshape(-1, 2)
        gd = np.concatenate([p[1] for p in parts])
        for i in _select(A, gp, gd):
            u, v = gp[i]
            pi[u], pi[v] = pi[v], pi[u]
    assert pi.tolist() == pi0


def _leaving_worker(rank, world, port, q):
    sys.path.insert(0, PY)
    import bmb200 as bm
    comm = bm.Comm(bm.BM_COMM_TCP, rank, world, f"127.0.0.1:{port}", timeout=2.0)
    comm.barrier()
    if rank == 1:
        comm.close()  # leaves between steps, before the next collective
        q.put((rank, "left", 0.0))
        return
    t = time.perf_counter()
    try:
        comm.allgather_swaps(np.zeros((0, 2), np.int32), np.zeros(0, np.int64), cap=8)
        q.put((rank, "no error", time.perf_counter() - t))
    except bm.BMError as e:
        q.put((rank, (e.status, str(e)), time.perf_counter() - t))
    comm.close()


def test_rank_that_leaves_ends_the_others_collective():
    import bmb200 as bm
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r = q.get(timeout=120)
        out[r[0]] = r[1:]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    res, dt = out[0]
    assert res != "no error"
    assert res[0] == bm.BM_TIMEOUT and "rank 1" in res[1]
    assert dt < 30


def test_comm_rejects_bad_arguments():
    sys.path.insert(0, PY)
    import bmb200 as bm
    L = bm.cuda_lib()
    h = C.c_void_p()
    assert L.bm_comm_create(0, 2, 2, b"127.0.0.1:1", 1.0, None, C.byref(h)) == bm.BM_INVALID_ARG  # rank >= world
    assert L.bm_comm_create(1, 0, 1, None, 1.0, None, C.byref(h)) == bm.BM_INVALID_ARG  # NCCL needs a context
    assert L.bm_comm_create(0, 1, 2, b"no-port", 1.0, None, C.byref(h)) == bm.BM_INVALID_ARG
    c = bm.Comm(bm.BM_COMM_TCP, 0, 1)  # a world of one needs no address
    assert c.allreduce_sum(7) == 7
    gp, gd = c.allgather_swaps(np.array([[3, 4]], np.int32), np.array([5], np.int64), cap=4)
    assert gp.tolist() == [[3, 4]] and gd.tolist() == [5]
    c.close()
