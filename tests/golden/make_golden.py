"""Generate the golden fixtures of tests/golden/ from the reference's own
functions (calculate_alignment_score, calculate_swap_delta and the loop order
of optimize_mapping), compiled from the reference sources into
oracle/_ref/libref.so by oracle/Makefile.

Run in a checkout where the reference sources are present:
    make -C oracle && python tests/golden/make_golden.py

Each fixture holds the graph pair itself (so it does not depend on the
generator staying unchanged), the mappings, and the reference's outputs.
golden_greedy.npz is the exception: its pairs are too large to store, so it
holds their generator parameters and edge checksums beside the matchings the
reference's greedy-match binary (oracle/_ref/greedy-match) wrote for them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "brain-match_b200", "python"))
sys.path.insert(0, os.path.join(REPO, "tests"))

import bmb200 as bm  # noqa: E402
from oracle_bind import Reference, ref_available  # noqa: E402


def edges(g):
    return g.src, g.dst, g.w


def make_pair_case(name, config, seed, n, m, npairs, nrows, max_sweeps, log_cap, verify):
    A, B, truth, init = bm.gen_pair(config, n=n, m_target=m, seed=seed)
    ref = Reference(A.n, edges(A), edges(B))
    rng = np.random.default_rng(seed)
    pairs = rng.integers(1, A.n + 1, size=(npairs, 2)).astype(np.int32)
    rows = rng.choice(np.arange(1, A.n + 1), size=nrows, replace=False).astype(np.int32)
    out = {
        "n": np.int64(A.n),
        "a_src": A.src, "a_dst": A.dst, "a_w": A.w,
        "b_src": B.src, "b_dst": B.dst, "b_w": B.w,
        "pi_init": init, "pi_truth": truth,
        "score_init": np.int64(ref.score(init)), "score_truth": np.int64(ref.score(truth)),
        "pairs": pairs, "pair_deltas": ref.pairs(init, pairs),
        "rows": rows, "row_deltas": ref.rows(init, rows),
    }
    pi_f, score_f, log, sweeps, conv = ref.serial(init, max_sweeps=max_sweeps, verify=verify)
    out.update({
        "serial_max_sweeps": np.int64(max_sweeps),
        "serial_pi": pi_f, "serial_score": np.int64(score_f), "serial_accepts": np.int64(len(log)),
        "serial_log": log[:log_cap], "serial_sweeps": np.int64(sweeps), "serial_converged": np.int64(conv),
    })
    # the first 100 accepts only, to pin the early order exactly
    pi_k, score_k, log_k, _, _ = ref.serial(init, max_accepts=100, verify=verify)
    out.update({"serial100_pi": pi_k, "serial100_score": np.int64(score_k)})
    ref.close()
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, {k: (v if np.ndim(v) == 0 else np.shape(v)) for k, v in out.items() if k in
                 ("n", "score_init", "score_truth", "serial_score", "serial_accepts", "serial_sweeps",
                  "serial_converged")})


def make_selfloop_case(name, seed=17, n=40, m=400):
    """A pair with self-loops, duplicate edges and zero weights.  The score is
    well defined there; calculate_swap_delta is not exact (it counts a self-loop
    twice against the old image), so the fixture records scores of mapping
    pairs (pi, pi after one swap) and the reference's delta for comparison."""
    rng = np.random.default_rng(seed)
    s = rng.integers(1, n + 1, m).astype(np.int32)
    d = rng.integers(1, n + 1, m).astype(np.int32)
    w = rng.integers(0, 9, m).astype(np.int32)
    seen, keep = set(), []
    for i in range(m):  # at most one self-loop per A vertex
        if s[i] == d[i]:
            if s[i] in seen:
                continue
            seen.add(int(s[i]))
        keep.append(i)
    A = (s[keep], d[keep], w[keep])
    B = (rng.integers(1, n + 1, m).astype(np.int32), rng.integers(1, n + 1, m).astype(np.int32),
         rng.integers(0, 9, m).astype(np.int32))
    ref = Reference(n, A, B)
    pis, scores, swaps, swapped_scores, ref_deltas = [], [], [], [], []
    for _ in range(8):
        pi = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
        pis.append(pi)
        scores.append(ref.score(pi))
        u, v = rng.choice(np.arange(1, n + 1), 2, replace=False)
        swaps.append((u, v))
        q = pi.copy()
        q[u], q[v] = q[v], q[u]
        swapped_scores.append(ref.score(q))
        ref_deltas.append(int(ref.pairs(pi, np.array([u, v], np.int32))[0]))
    ref.close()
    np.savez_compressed(os.path.join(HERE, name), n=np.int64(n), a_src=A[0], a_dst=A[1], a_w=A[2], b_src=B[0],
                        b_dst=B[1], b_w=B[2], pis=np.array(pis), scores=np.array(scores, np.int64),
                        swaps=np.array(swaps, np.int32), swapped_scores=np.array(swapped_scores, np.int64),
                        ref_deltas=np.array(ref_deltas, np.int64))
    print(name, "scores", scores[:3])


def make_selfloop_ref_case(name, seed=23, n=300, m=3000, loops=75):
    """A pair with self-loops on a quarter of the vertices of each graph, no
    duplicate edges and weights 1..8: the inputs where calculate_swap_delta
    differs from the score difference (a self-loop of a swapped vertex counted
    once as an out-edge and once as an in-edge, both against the old image).
    Records the reference's pair deltas, whole-row deltas and its serial loop
    with the re-score of every accept (optimize_mapping :571-576), so that the
    engine's reference-delta mode can be pinned to the reference itself."""
    rng = np.random.default_rng(seed)

    def graph():
        s = rng.integers(1, n + 1, m).astype(np.int32)
        d = rng.integers(1, n + 1, m).astype(np.int32)
        lv = rng.choice(np.arange(1, n + 1), loops, replace=False).astype(np.int32)
        s, d = np.concatenate([s, lv]), np.concatenate([d, lv])
        _, first = np.unique(s.astype(np.int64) * (n + 1) + d, return_index=True)
        keep = np.sort(first)
        return s[keep], d[keep], rng.integers(1, 9, keep.shape[0]).astype(np.int32)

    A, B = graph(), graph()
    ref = Reference(n, A, B)
    init = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
    pairs = rng.integers(1, n + 1, size=(2000, 2)).astype(np.int32)
    rows = rng.choice(np.arange(1, n + 1), size=4, replace=False).astype(np.int32)
    out = {
        "n": np.int64(n), "a_src": A[0], "a_dst": A[1], "a_w": A[2], "b_src": B[0], "b_dst": B[1], "b_w": B[2],
        "pi_init": init, "score_init": np.int64(ref.score(init)),
        "pairs": pairs, "pair_deltas": ref.pairs(init, pairs), "rows": rows, "row_deltas": ref.rows(init, rows),
    }
    # bounded: with these deltas a swap and its reverse can both look
    # improving, so the loop need not converge
    pi_f, score_f, log, sweeps, conv = ref.serial(init, max_sweeps=8, verify=True)
    out.update({"serial_max_sweeps": np.int64(8), "serial_pi": pi_f, "serial_score": np.int64(score_f), "serial_accepts": np.int64(len(log)),
                "serial_log": log, "serial_sweeps": np.int64(sweeps), "serial_converged": np.int64(conv)})
    pi_k, score_k, _, _, _ = ref.serial(init, max_accepts=100, verify=True)
    out.update({"serial100_pi": pi_k, "serial100_score": np.int64(score_k)})
    ref.close()
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, {k: (v if np.ndim(v) == 0 else np.shape(v)) for k, v in out.items() if k in
                 ("n", "score_init", "serial_score", "serial_accepts", "serial_sweeps", "serial_converged")})


def simfilter_inputs(seed, n=300, m=3000, loops=0):
    """A pair for the similarity-filtered variant: the generator's pair (or,
    with loops > 0, a random pair with that many self-loops per graph and no
    duplicate edges), the largest id present in both graphs (the variant sizes
    its arrays by each graph's largest id), and orderings by weighted degree."""
    if loops:
        rng = np.random.default_rng(seed)

        def graph():
            s_ = rng.integers(1, n + 1, m).astype(np.int32)
            d_ = rng.integers(1, n + 1, m).astype(np.int32)
            lv = rng.choice(np.arange(1, n + 1), loops, replace=False).astype(np.int32)
            s_, d_ = np.concatenate([s_, lv]), np.concatenate([d_, lv])
            _, first = np.unique(s_.astype(np.int64) * (n + 1) + d_, return_index=True)
            keep = np.sort(first)
            return [s_[keep], d_[keep], rng.integers(1, 9, keep.shape[0]).astype(np.int32)]

        A, B = graph(), graph()
        init = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
    else:
        Ag, Bg, _, init = bm.gen_pair(1, n=n, m_target=m, seed=seed)
        A, B = [Ag.src, Ag.dst, Ag.w], [Bg.src, Bg.dst, Bg.w]
    for G in (A, B):
        if max(int(G[0].max()), int(G[1].max())) < n:
            G[0] = np.append(G[0], n).astype(np.int32)
            G[1] = np.append(G[1], 1).astype(np.int32)
            G[2] = np.append(G[2], 1).astype(np.int32)
    rank_m = bm.ordering_by_weighted_degree(bm.Graph(n, *A))
    rank_f = bm.ordering_by_weighted_degree(bm.Graph(n, *B))
    return n, tuple(A), tuple(B), init, rank_m, rank_f


def ref_simfilter_pass(A, B, init, rank_m, rank_f):
    """One pass of the reference variant (its orderings read from CSV files
    written beside the reference libraries)."""
    from oracle_bind import ReferenceGA
    tmp = os.path.join(REPO, "oracle", "_ref", "ga_tmp")
    os.makedirs(tmp, exist_ok=True)
    pm, pf = os.path.join(tmp, "order_m.csv"), os.path.join(tmp, "order_f.csv")
    bm.write_ordering(pm, rank_m)
    bm.write_ordering(pf, rank_f)
    ref = ReferenceGA(A, B)
    try:
        pi = ref.sweep(init, pm, pf, os.path.join(tmp, "out_mapping.csv"))
        return pi, ref.score(pi)
    finally:
        ref.close()


def make_simfilter_case(name, seed=13):
    """The similarity-filtered single pass of src/graph-alignment.c on a
    300-vertex pair: its final mapping and score."""
    n, A, B, init, rank_m, rank_f = simfilter_inputs(seed)
    pi, score = ref_simfilter_pass(A, B, init, rank_m, rank_f)
    np.savez_compressed(os.path.join(HERE, name), n=np.int64(n), a_src=A[0], a_dst=A[1], a_w=A[2], b_src=B[0],
                        b_dst=B[1], b_w=B[2], pi_init=init, rank_m=rank_m, rank_f=rank_f, pass_pi=pi,
                        pass_score=np.int64(score))
    print(name, "moved", int((pi != init).sum()), "score", score)


CASES = {
    "golden_small.npz": lambda: make_pair_case("golden_small.npz", 1, 11, 300, 3000, 3000, 6, max_sweeps=-1,
                                               log_cap=1 << 16, verify=True),
    "golden_cfg1.npz": lambda: make_pair_case("golden_cfg1.npz", 1, 1, 2000, 40000, 5000, 4, max_sweeps=1,
                                              log_cap=3000, verify=False),
    "golden_selfloop.npz": lambda: make_selfloop_case("golden_selfloop.npz"),
    "golden_selfloop_ref.npz": lambda: make_selfloop_ref_case("golden_selfloop_ref.npz"),
    "golden_simfilter.npz": lambda: make_simfilter_case("golden_simfilter.npz"),
    "golden_greedy.npz": lambda: make_greedy_case("golden_greedy.npz"),
}


GREEDY_REF = os.path.join(REPO, "oracle", "_ref", "greedy-match")
# (config, seed, n, edges): generated pairs on which the reference's
# greedy-match runs in seconds to minutes (its loader and 2-hop counts are
# quadratic); every vertex has an edge, so its node list is 1..n
GREEDY_CASES = ((1, 7, 3000, 60000), (3, 9, 2500, 200000), (2, 5, 4000, 640000))


def edge_digest(g):
    """A checksum of an edge list, so a test notices a changed generator."""
    h = (g.src.astype(np.uint64) * np.uint64(1000003) + g.dst.astype(np.uint64)) * np.uint64(65599) \
        + g.w.astype(np.uint64)
    return np.uint64(np.bitwise_xor.reduce(h * np.uint64(0x9E3779B97F4A7C15)))


def run_ref_greedy(A, B, workdir):
    """The reference's greedy-match binary on A and B written as its CSV input;
    returns its matching as a 1-indexed array."""
    import subprocess
    os.makedirs(workdir, exist_ok=True)
    ga, gb, out = (os.path.join(workdir, f) for f in ("g1.csv", "g2.csv", "match.csv"))
    bm.write_graph_csv(ga, A)
    bm.write_graph_csv(gb, B)
    subprocess.run([GREEDY_REF, ga, gb, out], check=True, stdout=subprocess.DEVNULL)
    ref = np.loadtxt(out, delimiter=",", skiprows=1, dtype=np.int64).reshape(-1, 2)
    pi = np.zeros(A.n + 1, np.int32)
    pi[ref[:, 0]] = ref[:, 1]
    return pi


def make_greedy_case(name):
    import tempfile
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for i, (config, seed, n, m) in enumerate(GREEDY_CASES):
            A, B, truth, init = bm.gen_pair(config, n=n, m_target=m, seed=seed)
            out[f"case{i}"] = np.array([config, seed, n, m], np.int64)
            out[f"digest{i}"] = np.array([edge_digest(A), edge_digest(B)], np.uint64)
            out[f"pi{i}"] = run_ref_greedy(A, B, os.path.join(tmp, str(i)))
            print(name, i, config, seed, n, m, "matched", int((out[f"pi{i}"][1:] > 0).sum()))
    np.savez_compressed(os.path.join(HERE, name), **out)


def main():
    """Make every fixture, or only those named on the command line."""
    if not ref_available():
        raise SystemExit("oracle/_ref/libref.so missing: run make -C oracle where the reference sources exist")
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()


if __name__ == "__main__":
    main()
