"""Coordination of a search sharded over ranks (one process per GPU), with
torch.distributed as plumbing only.

Sharded row search (the multi-GPU plan of the reference's MPI drivers,
src/graph-re-alignment-mpi-omp.c:76-123, restated for one replicated mapping):
every rank evaluates its share of a round's rows on its own GPU, keeps each
row's best improving partner, the candidates are all-gathered in rank order,
and every rank runs the same deterministic independent-subset selection on the
same list, so all ranks apply the same swaps and the mapping stays replicated
without broadcasting it.

Island synchronisation (the reference's sync_best_solutions,
src/graph-re-alignment-mpi-omp.c:76-123: gather scores, pick the best rank,
send its mapping): one all-reduce of a packed (score, rank) key picks the best
rank (lowest rank on ties) and one broadcast sends its mapping to every rank.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def round_rows(order: np.ndarray, rnd: int, rows_per_rank: int, rank: int, world: int) -> np.ndarray:
    """Rows of round `rnd` owned by `rank`: the round takes world*rows_per_rank
    consecutive rows of `order` (cyclically) and deals them round-robin."""
    n = order.shape[0]
    start = (rnd * world * rows_per_rank) % n
    idx = (start + np.arange(world * rows_per_rank)) % n
    return np.ascontiguousarray(order[idx[rank::world]])


def gather_candidates(pairs: np.ndarray, deltas: np.ndarray):
    """All-gather variable-length candidate lists in rank order: returns the
    concatenated (pairs (k,2) int32, deltas (k,) int64)."""
    world = dist.get_world_size()
    cnt = torch.tensor([pairs.shape[0]], dtype=torch.int64)
    counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(counts, cnt)
    counts = [int(c.item()) for c in counts]
    mx = max(max(counts), 1)
    buf = torch.zeros((mx, 4), dtype=torch.int64)
    if pairs.shape[0]:
        buf[: pairs.shape[0], 0] = torch.from_numpy(pairs[:, 0].astype(np.int64))
        buf[: pairs.shape[0], 1] = torch.from_numpy(pairs[:, 1].astype(np.int64))
        buf[: pairs.shape[0], 2] = torch.from_numpy(deltas.astype(np.int64))
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    allp, alld = [], []
    for r in range(world):
        b = bufs[r][: counts[r]].numpy()
        allp.append(b[:, :2].astype(np.int32))
        alld.append(b[:, 2].astype(np.int64))
    return np.concatenate(allp).reshape(-1, 2), np.concatenate(alld)


def island_best(score: int, pi: np.ndarray):
    """Every rank adopts the mapping of the rank with the best score."""
    rank, world = dist.get_rank(), dist.get_world_size()
    key = torch.tensor([(int(score) << 16) | (0xFFFF - rank)], dtype=torch.int64)
    dist.all_reduce(key, op=dist.ReduceOp.MAX)
    best_rank = 0xFFFF - int(key.item() & 0xFFFF)
    best_score = int(key.item() >> 16)
    t = torch.from_numpy(np.ascontiguousarray(pi.astype(np.int32)))
    dist.broadcast(t, src=best_rank)
    return best_score, best_rank, t.numpy().copy()
