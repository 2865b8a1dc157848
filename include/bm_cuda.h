/*
 * bm_cuda.h — C ABI of the B200 swap-search engine (libbmcuda.so).
 *
 * Plain C types only: pointers, sizes and status codes.  Every entry point
 * returns a bm_status; the library never calls exit().  One context owns one
 * device and one CUDA stream; a context is not re-entrant, different contexts
 * may be driven from different host threads.
 *
 * Problem: two weighted directed graphs A ("male", gm) and B ("female", gf)
 * on vertex ids 1..n, and a bijection pi: A-vertex -> B-vertex stored 1-indexed
 * in an int32 array of length n+1 (slot 0 unused), exactly like the `mapping`
 * array of the reference tools.  The objective is the edge-overlap score
 *     score(pi) = sum over A edges (x->y, w) of min(w, w_B(pi x, pi y))
 * (w_B = 0 for absent edges), computed in int64.
 *
 * Semantics ("exact"): a swap delta is score(pi after swapping pi(u),pi(v))
 * minus score(pi), with score as in calculate_alignment_score
 * (src/graph-alignment-optimized.c:292-307): every A edge-list entry counts
 * (duplicate A edges count once per entry), B is a matrix (the last duplicate
 * weight wins, src/graph-alignment-optimized.c:185).  Self-loops are scored
 * exactly; on graphs without self-loops this equals calculate_swap_delta
 * (src/graph-alignment-optimized.c:321-408) for every pair.  The optional
 * reference-delta mode (bm_set_semantics) reproduces calculate_swap_delta
 * itself on graphs with self-loops.
 *
 * Limits: n <= 131071, 0 <= w <= 32767 (the reference stores B weights as
 * int16), fewer than 2^31 edges per graph, at most one self-loop per A vertex.
 * Inputs outside these limits are rejected with BM_INVALID_ARG.
 */
#ifndef BM_CUDA_H
#define BM_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bm_status {
    BM_OK = 0,
    BM_INVALID_ARG = 1,   /* bad size, id, weight, non-bijective mapping, missing graph */
    BM_OOM = 2,           /* device or host allocation failed */
    BM_CUDA_ERROR = 3,    /* a CUDA runtime call or kernel launch failed */
    BM_TIMEOUT = 4,       /* a time or iteration budget ran out before completion */
    BM_PARITY_FAIL = 5,   /* a self-check (score re-verification) disagreed */
    BM_UNSUPPORTED = 6,   /* the request exceeds what the chosen kernel supports */
    BM_NO_DEVICE = 7      /* no CUDA device, or the requested ordinal does not exist */
} bm_status;

typedef struct bm_ctx bm_ctx;

#define BM_SIDE_A 0   /* "male" graph gm: the graph whose edges are scored */
#define BM_SIDE_B 1   /* "female" graph gf: the graph looked up at mapped ends */

/* ---------------------------------------------------------------- lifecycle */

/* Create a context on `device` (ordinal).  Replaces the implicit global state
 * of the reference tools (main in src/graph-alignment-optimized.c:682-738,
 * cudaSetDevice in src/graph-re-alignment-gpu.cu:1304). */
bm_status bm_ctx_create(int device, bm_ctx** out);
void bm_ctx_destroy(bm_ctx* ctx);
const char* bm_status_str(bm_status s);
/* Last error message recorded on this context ("" if none). */
const char* bm_ctx_last_error(const bm_ctx* ctx);
/* The context's cudaStream_t, as an opaque pointer. */
void* bm_ctx_stream(bm_ctx* ctx);
bm_status bm_sync(bm_ctx* ctx);

/* ------------------------------------------------------------------- graphs */

/* Upload one graph from an edge list (ids 1..n).  The library copies; the
 * caller keeps ownership of the host arrays.  Replaces load_graph_from_csv +
 * add_edge (src/graph-alignment-optimized.c:183-204, 635-679): A keeps every
 * list entry, B keeps the last weight of a duplicated edge.  Both graphs must
 * share the same n.  Setting a graph invalidates the mapping. */
bm_status bm_set_graph(bm_ctx* ctx, int side, int32_t n, int64_t m,
                       const int32_t* src, const int32_t* dst, const int32_t* w);

/* Graph statistics after upload: n, non-self entries, max in+out degree. */
bm_status bm_graph_info(bm_ctx* ctx, int side, int32_t* n, int64_t* m_nonself,
                        int32_t* max_degree, int64_t* max_weighted_degree);

/* ------------------------------------------------------------------ mapping */

/* Set pi (host, n+1 entries, 1-indexed, slot 0 ignored).  pi must be a
 * bijection of 1..n (the check of verify_mapping, src/verify-mapping.c:199-232).
 * Recomputes the per-vertex overlap and the score on the device. */
bm_status bm_set_mapping(bm_ctx* ctx, const int32_t* pi);
/* Copy the current pi back to the host (n+1 entries, slot 0 = 0). */
bm_status bm_get_mapping(bm_ctx* ctx, int32_t* pi);

/* ------------------------------------------------------------------- scoring */

/* Full score of the current pi, recomputed from scratch on the device.
 * Replaces calculate_alignment_score (src/graph-alignment-optimized.c:292-307)
 * and score-matching's calculate_score_sparse (src/score-matching.c:558-597). */
bm_status bm_score(bm_ctx* ctx, int64_t* score);
/* Score tracked incrementally by the engine (sum of applied deltas).  In the
 * reference-delta mode (bm_set_semantics) the deltas need not be score
 * differences, so between a schedule's end-of-call re-score and the next
 * one it may differ from bm_score. */
bm_status bm_tracked_score(bm_ctx* ctx, int64_t* score);
/* Per-vertex overlap S(v) = sum of min(w, w_B) over non-self A entries incident
 * to v (each edge counts at both ends), host array of n+1 int32. */
bm_status bm_get_overlap(bm_ctx* ctx, int32_t* ov);

/* ------------------------------------------------------------ swap deltas */

/* Exact deltas for k arbitrary pairs (u_i, v_i) = (pairs[2i], pairs[2i+1]).
 * Host buffers.  Replaces calculate_swap_delta
 * (src/graph-alignment-optimized.c:321-408) and the reference GPU kernels
 * calculateSwapDeltasKernel(Quick) (src/graph-re-alignment-gpu.cu:46-248).
 * u == v gives 0. */
bm_status bm_delta_pairs(bm_ctx* ctx, const int32_t* pairs, int64_t k, int64_t* deltas);
/* Same, device pointers, asynchronous on the context stream. */
bm_status bm_delta_pairs_dev(bm_ctx* ctx, const int32_t* d_pairs, int64_t k, int64_t* d_deltas);

/* Exact deltas of whole rows: for each row u = rows[r], delta(u, v) for
 * v = 0..n is written to deltas[r*(n+1) + v] (v == 0 and v == u give 0).
 * Host buffers.  This is the m2 sweep of one m1 row of optimize_mapping
 * (src/graph-alignment-optimized.c:542-579) evaluated at once. */
bm_status bm_delta_rows(bm_ctx* ctx, const int32_t* rows, int32_t nrows, int64_t* deltas);
bm_status bm_delta_rows_dev(bm_ctx* ctx, const int32_t* d_rows, int32_t nrows, int64_t* d_deltas);

/* Per-row reduction of whole-row deltas, without materialising them. */
typedef struct bm_row_result {
    int32_t row;         /* u */
    int32_t first_pos;   /* smallest v >= col_lo, v != u, with delta > 0; 0 if none */
    int32_t best;        /* v with the largest delta (smallest v on ties), v >= col_lo, v != u */
    int32_t npos;        /* number of v >= col_lo with delta > 0 */
    int64_t first_delta; /* delta(u, first_pos), 0 if none */
    int64_t best_delta;  /* delta(u, best) */
} bm_row_result;

/* col_lo may be NULL (all columns); otherwise col_lo[r] is the first column
 * considered for row r.  Host buffers.  Without col_lo (and up to 4,096 rows,
 * no split plan) the call replays a CUDA graph whose kernels write the
 * results into pinned memory and returns as soon as every row's result has
 * arrived; the graph's last steps finish in the context's stream order
 * before any later work of the context. */
bm_status bm_rows_best(bm_ctx* ctx, const int32_t* rows, const int32_t* col_lo,
                       int32_t nrows, bm_row_result* out);
bm_status bm_rows_best_dev(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo,
                           int32_t nrows, bm_row_result* d_out);

/* --------------------------------------------------------------- moves */

/* Apply k swaps pi(a_i) <-> pi(b_i) that must be pairwise independent (no shared
 * vertex and no A edge between the endpoint sets of two swaps; k == 1 is always
 * independent), updating pi, the per-vertex overlap and the tracked score by
 * the given deltas.  Host buffers.  Replaces the swap of optimize_mapping
 * (src/graph-alignment-optimized.c:556-566). */
bm_status bm_apply_swaps(bm_ctx* ctx, const int32_t* pairs, const int64_t* deltas, int32_t k);

/* ------------------------------------------------------------- schedules */

typedef struct bm_progress {
    int64_t rows_done;       /* rows (m1 values) completed */
    int64_t evaluated;       /* exact deltas evaluated (full rows count n-1) */
    int64_t accepts;         /* swaps applied */
    int64_t score;           /* tracked score at return */
    int64_t launches;        /* kernel batches launched */
    int32_t next_row_pos;    /* position in row_order to resume from */
    int32_t next_col;        /* column to resume from in that row */
    int32_t sweeps;          /* completed passes over row_order */
    int32_t converged;       /* 1 if a full pass found no improving swap */
    double seconds;          /* wall time spent */
} bm_progress;

/* Serial first-improvement hill-climb, bit-exact with the loop of
 * optimize_mapping (src/graph-alignment-optimized.c:513-580): rows in
 * row_order (NULL = 1..n), columns v = 1..n ascending, accept the first
 * delta > 0 and continue from the next column under the new mapping.
 * Stops at convergence (a full pass without an accept), after max_accepts
 * accepts (<0: no limit), max_sweeps passes (<0: no limit) or time_budget_s
 * seconds (<=0: no limit; BM_TIMEOUT is returned when it ran out).  `prog`
 * may carry a resume position (next_row_pos, next_col) in; it is updated. */
bm_status bm_sweep_parity(bm_ctx* ctx, const int32_t* row_order, int32_t nrows,
                          int64_t max_accepts, int32_t max_sweeps, double time_budget_s,
                          bm_progress* prog);

/* Throughput search: batches of rows (row_order, cycled), best improving
 * partner per row, then a deterministic conflict-free subset of those swaps
 * (descending delta, ascending row) applied together.  Stops like
 * bm_sweep_parity; target_score > 0 also stops once the score reaches it. */
bm_status bm_search_batched(bm_ctx* ctx, const int32_t* row_order, int32_t nrows,
                            int32_t rows_per_batch, int64_t max_accepts, int32_t max_sweeps,
                            double time_budget_s, int64_t target_score, bm_progress* prog);

/* The single pass of optimize_mapping in the reference's graph-alignment
 * variant (src/graph-alignment.c:489-595), with its similarity filter
 * (:545-553): m1 and then m2 run over nodes[0..nnodes) (the variant's vertex
 * list, bm_first_appearance in bm_host.h); the swap is evaluated only when
 * calculate_node_similarity (:274-284, FP64, the same operations in the same
 * order) of the swapped images beats the current pair's, and a positive delta
 * is applied at once.  metrics_a, metrics_b: five doubles per vertex id
 * 0..n of each graph (bm_node_metrics).  One pass, resumable through
 * prog->next_row_pos / next_col (positions in nodes[]); stops early after
 * max_accepts (-1: none) or the time budget (BM_TIMEOUT).  The deltas follow
 * bm_set_semantics: BM_SEMANTICS_REF_CPU reproduces the variant on graphs
 * with self-loops too. */
bm_status bm_sweep_similarity(bm_ctx* ctx, const int32_t* nodes, int32_t nnodes, const double* metrics_a,
                              const double* metrics_b, int64_t max_accepts, double time_budget_s, bm_progress* prog);

/* Deterministic independent-subset selection of candidate swaps (pairs[2i],
 * pairs[2i+1]) with deltas[i]: among delta > 0, in descending delta then
 * ascending index, a swap is taken when neither endpoint lies in the closed A
 * neighbourhood of an endpoint already taken (the independence rule of
 * src/independent-hungarian/hungarianSubset.c:657-740).  Every rank of a
 * sharded search runs it on the same gathered list, so the ranks apply the
 * same swaps and keep identical mappings.  chosen gets candidate indices. */
bm_status bm_select_independent(bm_ctx* ctx, const int32_t* pairs, const int64_t* deltas, int32_t count,
                                int32_t* chosen, int32_t* nchosen);

/* Perturbation: k disjoint swaps selected[i] <-> selected[i+k] over 2k
 * distinct vertices (random_swap_k_vertices, src/graph-re-alignment-gpu.cu:
 * 763-810); mode 0 draws all 2k uniformly, mode 1 draws the first k with
 * probability proportional to 7*out-weight + 3*in-weight of A (the weighted
 * variant of src/graph-re-alignment-gpu-swap.cu:767-887), the next k
 * uniformly.  Draws come from Philox4x32-10 keyed by seed, starting at stream
 * position `counter`.  The exact deltas are applied in order; changed (2k
 * ints, optional) receives the vertices, total_delta their sum. */
bm_status bm_perturb(bm_ctx* ctx, int32_t k, int32_t mode, uint64_t seed, uint64_t counter,
                     int32_t* changed, int64_t* total_delta);
/* Batched search with perturbation restarts (the pattern of
 * src/graph-re-alignment-gpu.cu:1004-1028): converge with bm_search_batched,
 * perturb with k_perturb swaps, repeat up to max_restarts times or until the
 * budget ends; the best mapping seen is restored at the end and its score
 * returned in best_score. */
bm_status bm_search_restarts(bm_ctx* ctx, const int32_t* row_order, int32_t nrows, int32_t rows_per_batch,
                             int32_t k_perturb, int32_t mode, uint64_t seed, int32_t max_restarts,
                             double time_budget_s, bm_progress* prog, int64_t* best_score);

/* --------------------------------------------------- k-vertex permutations */

/* Exact deltas of every permutation of small vertex sets (2 <= k <= 8):
 * sets[i*k + a] is member a of set i.  For each set the best permutation
 * (largest delta, the first in lexicographic order on ties; the identity,
 * delta 0, when nothing improves) is returned as best_perm[i*k + a] = the
 * member whose image member a takes, with its delta in best_delta[i].
 * all_deltas (optional, nsets * k! entries) receives every permutation's
 * delta in lexicographic order.  k = 3 gives the 3-vertex moves of
 * calculateThreeNodeSwapKernel (src/graph-re-alignment-gpu-3-swap.cu:43-305);
 * k = 4..8 the permutation sets of src/graph-alignment-permset-parallel.c:
 * 304-363, with exact deltas for edges inside a set.  Host buffers. */
bm_status bm_kset_eval(bm_ctx* ctx, int32_t k, const int32_t* sets, int64_t nsets, int64_t* best_delta,
                       int32_t* best_perm, int64_t* all_deltas);
/* Device-pointer form; *d_status (device int32, zeroed by the caller) gets bit
 * 0 for a rejected set (bad or repeated id) and bit 1 for a set with more than
 * 256 A entries between its members (both evaluated as delta 0). */
bm_status bm_kset_eval_dev(bm_ctx* ctx, int32_t k, const int32_t* d_sets, int64_t nsets,
                           int64_t* d_best_delta, int32_t* d_best_perm, int32_t* d_status);
/* Apply permutations of pairwise independent sets (no shared vertex, no A
 * edge between two sets), as apply_permutation does for triples
 * (src/graph-re-alignment-gpu-3-swap.cu:925-956).  Host buffers. */
bm_status bm_apply_sets(bm_ctx* ctx, int32_t k, const int32_t* sets, const int32_t* perms,
                        const int64_t* deltas, int32_t nsets);
/* Search by k-vertex permutations: each launch draws sets_per_launch sets
 * (mode 0: k random distinct vertices; mode 1, k = 3 only: a path u - x - y of
 * A), evaluates all k! permutations of each, and applies a greedy independent
 * subset of the improving ones (descending delta).  Sets come from
 * Philox4x32-10 keyed by seed, so a run is reproducible. */
bm_status bm_search_ksets(bm_ctx* ctx, int32_t k, int32_t sets_per_launch, int32_t mode, uint64_t seed,
                          int64_t max_launches, double time_budget_s, bm_progress* prog);

/* ------------------------------------------------- annealing chains */

/* A batch of graph pairs of uneven size, for many independent annealing
 * chains in one persistent kernel.  Pairs are added like bm_set_graph (same
 * limits and duplicate rules); each gets an index 0, 1, ...  A batch runs on
 * its context's device and stream; destroy it before the context. */
typedef struct bm_batch bm_batch;
bm_status bm_batch_create(bm_ctx* ctx, bm_batch** out);
void bm_batch_destroy(bm_batch* b);
bm_status bm_batch_add_pair(bm_batch* b, int32_t n,
                            int64_t mA, const int32_t* srcA, const int32_t* dstA, const int32_t* wA,
                            int64_t mB, const int32_t* srcB, const int32_t* dstB, const int32_t* wB,
                            int32_t* pair_index);

typedef struct bm_sa_params {
    int64_t steps;       /* proposals per chain */
    double t0;           /* starting temperature */
    double t_end;        /* final temperature: T_i = t0 * exp(ln(t_end/t0) * i / steps) */
    int32_t candidates;  /* proposals evaluated together per iteration at the start, 1..16; 0 = autotuned
                          * (with the CTAs per chain: 1, or a pair of CTAs when the chains fill at most
                          * half the SMs; the tuner times a prefix of the run for each choice and caches
                          * the best per device, sizes and chain count).  Each chain then adapts it (up
                          * to 64) to its own acceptances: doubled after an iteration with none,
                          * 2 (j + 1) after the j-th is accepted. */
    int64_t chunk;       /* proposals per chain per kernel launch (0 = 65536) */
    int32_t threads_per_cta; /* 256 or 512 with a set candidates value; 0 = 512 there, and with
                              * candidates = 0 the tuner chooses it as well (256 or 512) */
} bm_sa_params;

typedef struct bm_sa_stats {
    int32_t candidates;      /* value used */
    int32_t ctas_per_chain;  /* 1, or 2: a pair of CTAs (a cluster) per chain */
    int64_t launches;        /* graph replays */
    double seconds;      /* wall time of the chain launches */
    int32_t threads_per_cta; /* 256 or 512 */
} bm_sa_stats;

/* Simulated annealing, the loop of simulated_annealing in
 * src/best-swap/score-lookup.c:346-408 with exact int64 deltas.  Chain c runs
 * on pair chain_pair[c]; its proposals come from Philox4x32-10 keyed by
 * chain_key[c] with the step as counter, and the acceptance test
 * u < exp(delta/T) uses the library's own exp, so every chain is
 * deterministic and independent of `candidates`.  init_pi and final_pi hold
 * the chains' mappings back to back, n_c + 1 ints each (slot 0 ignored);
 * bm_sa_layout_size gives the total.  final_score and accepts have nchains
 * entries.  Any output pointer may be NULL. */
bm_status bm_sa_run(bm_batch* b, int32_t nchains, const int32_t* chain_pair, const uint64_t* chain_key,
                    const int32_t* init_pi, const bm_sa_params* params, int32_t* final_pi,
                    int64_t* final_score, int64_t* accepts, bm_sa_stats* stats);
int64_t bm_sa_layout_size(bm_batch* b, int32_t nchains, const int32_t* chain_pair);

/* The chains of bm_sa_run, computed without allocating any device memory.
 * No counterpart in the reference.  For callers that cannot call
 * cudaMalloc/cudaFree while they run (device memory owned by their own pool
 * under a fixed budget, or a serving path that must not take cudaFree's
 * device-wide synchronisation).  The batch itself is built beforehand with
 * bm_batch_add_pair, which does allocate.  All scratch lives in one static
 * device array of 8,486,912 bytes.  bm_ctx_create looks up its device address
 * (which loads the module holding it), so the array is reserved on a device
 * when the first context on it is created and held until the process exits;
 * the entry point itself reserves nothing, on its first call too
 * (bm_alloc_count does not move).  A device reset invalidates the contexts
 * on the device; create a new one after it.  The array limits a call to 256
 * pairs, 1,024 chains and a total of 2^20 mapping entries (sum over chains
 * of n + 1); larger requests return BM_INVALID_ARG.  Calls share the array
 * and it keeps the last call's contents: calls that overlap on the GPU race
 * and must be serialised by the caller.  candidates == 0 uses 8 (no
 * autotuning: the tuner would allocate).  Arguments and outputs as
 * bm_sa_run, without stats. */
bm_status bm_sa_run_noalloc(bm_batch* b, int32_t nchains, const int32_t* chain_pair, const uint64_t* chain_key,
                            const int32_t* init_pi, const bm_sa_params* params, int32_t* final_pi,
                            int64_t* final_score, int64_t* accepts);

/* ----------------------------------------------------- multi-rank search */

/* Ranks of a sharded search, one process per GPU on a node, with no MPI and
 * no PyTorch: the replacement of the reference's MPI drivers
 * (src/graph-re-alignment-mpi-omp.c, src/graph-re-alignment-mpi-gpu.cu).
 * BM_COMM_TCP: host sockets in a star around rank 0, which listens on addr
 * ("host:port"); the others connect to it (retrying while it starts).  It
 * needs no GPU (ctx may be NULL for the exchange calls).  BM_COMM_NCCL: NCCL
 * (libnccl.so.2, loaded when asked for) over NVLink on ctx's device and
 * stream; rank 0's socket carries only the ncclUniqueId (world 1 needs no
 * address).  Every call below is collective: every rank makes the same calls
 * in the same order.  Each wait is bounded by timeout_s: a rank that leaves or
 * stops answering makes the others' calls return BM_TIMEOUT (an NCCL
 * communicator is aborted then, and later calls return BM_TIMEOUT at once).
 * bm_comm_last_error gives the message. */
typedef struct bm_comm bm_comm;
enum { BM_COMM_TCP = 0, BM_COMM_NCCL = 1 };
bm_status bm_comm_create(int32_t kind, int32_t rank, int32_t world, const char* addr, double timeout_s, bm_ctx* ctx,
                         bm_comm** out);
void bm_comm_destroy(bm_comm* comm);
const char* bm_comm_last_error(const bm_comm* comm);
bm_status bm_comm_barrier(bm_comm* comm);
/* Sum of value over the ranks (a consistency check of replicated state). */
bm_status bm_comm_allreduce_sum(bm_comm* comm, int64_t value, int64_t* total);
/* Candidate swaps of every rank, concatenated in rank order (each rank's in
 * its own order): all_pairs gets 2 ints and all_deltas one value per
 * candidate, *total their count (at most cap, else BM_INVALID_ARG). */
bm_status bm_comm_allgather_swaps(bm_comm* comm, const int32_t* pairs, const int64_t* deltas, int32_t count, int32_t cap,
                                  int32_t* all_pairs, int64_t* all_deltas, int32_t* total);
/* Island synchronisation (sync_best_solutions,
 * src/graph-re-alignment-mpi-omp.c:76-123): every rank adopts the mapping
 * pi[0..n] of the rank with the best score (the lowest rank on ties), in
 * place; best_score and best_rank (optional) receive the winner.  Scores
 * must lie in 0..2^47. */
bm_status bm_comm_island_best(bm_comm* comm, int64_t score, int32_t* pi, int32_t n, int64_t* best_score,
                              int32_t* best_rank);
/* Sharded batched search.  Round r takes world * rows_per_rank consecutive
 * rows of row_order (cyclically; NULL = 1..n; rows_per_rank 0 = 2 x SMs) and
 * each rank evaluates every world-th of them, from its rank on, on its GPU
 * (best improving partner per row, the row argmax of
 * src/re-alignment-parallel.c:598-618).  The candidates are all-gathered in
 * rank order and every rank applies bm_select_independent's choice from the
 * same list, so the replicated mapping stays identical on every rank with
 * no broadcast.  Stops after max_rounds (-1: none), when a full pass applies
 * nothing (converged), or after the round in which some rank's time budget
 * ran out (BM_TIMEOUT; every rank stops there).  Ends with a full re-score
 * and a comparison of the ranks' mappings (BM_PARITY_FAIL if they differ).
 * All ranks must pass the same row_order, rows_per_rank and max_rounds. */
bm_status bm_search_sharded(bm_ctx* ctx, bm_comm* comm, const int32_t* row_order, int32_t nrows,
                            int32_t rows_per_rank, int64_t max_rounds, double time_budget_s, bm_progress* prog);

/* ------------------------------------------------------------ delta table */

/* The table of every pair's exact delta, the score-lookup engine of
 * src/best-swap/score-lookup.c (create_score_lookup :246-293), kept exact:
 * entry (u, v) of a device int32 array at d_table[u * ld + v] for
 * 1 <= u, v <= n (0 on the diagonal and in row and column 0), ld >= n + 1.
 * The caller owns the array ((n + 1) * ld * 4 bytes: 1.37 GB at n = 18,524).
 * Deltas fit int32 (the engine rejects weighted degrees that could overflow);
 * the reference truncates them to short. */
bm_status bm_delta_table_dev(bm_ctx* ctx, int32_t* d_table, int64_t ld);
/* Recompute rows d_rows[0..nrows) and the matching columns.  After a swap of
 * a and b, the rows of a, b and their A neighbours are all that change (the
 * reference's update_lookup_and_heap, :129-244, recomputes the pairs of a and b
 * only and lets the rest go stale). */
bm_status bm_table_refresh_dev(bm_ctx* ctx, int32_t* d_table, int64_t ld, const int32_t* d_rows, int32_t nrows);
/* The k (1..4096) best pairs u < v of the table, largest delta first, then
 * smallest u, then smallest v: the order the reference's max-heap
 * (heap.c:79-164) extracts swaps in, with its ties made deterministic.
 * pairs receives 2*count ints, deltas count values; count = min(k, n(n-1)/2).
 * _dev: device outputs (count may be NULL), asynchronous. */
bm_status bm_table_topk(bm_ctx* ctx, const int32_t* d_table, int64_t ld, int32_t k, int32_t* pairs,
                        int64_t* deltas, int32_t* count);
bm_status bm_table_topk_dev(bm_ctx* ctx, const int32_t* d_table, int64_t ld, int32_t k, int32_t* d_pairs,
                            int64_t* d_deltas, int32_t* d_count);
/* Best-swap search on the table (the optimize loop of score-lookup,
 * :530-…, without its annealing phases): take the k best pairs, apply the
 * improving ones that are independent of better ones (bm_select_independent's
 * rule), refresh the changed rows, repeat until the best delta is <= 0 or a
 * budget ends.  The table must hold the current mapping's deltas
 * (bm_delta_table_dev) and stays exact; every call ends with a full re-score
 * (BM_PARITY_FAIL on a mismatch). */
bm_status bm_search_table(bm_ctx* ctx, int32_t* d_table, int64_t ld, int32_t k, int64_t max_accepts,
                          int32_t max_rounds, double time_budget_s, bm_progress* prog);

/* ------------------------------------------- independent-subset assignment */

/* Optimal linear assignment of a k x k integer benefit matrix (row-major,
 * |benefit| <= 2^30, 1 <= k <= 4096): assign[i] = the column of row i in a
 * permutation maximising the total, *total that total.  Replaces the
 * reference's Hungarian method (src/independent-hungarian/hungarian.c:144-334)
 * with the auction algorithm on the device; ties between optimal permutations
 * may be broken differently. */
bm_status bm_lap_solve(bm_ctx* ctx, const int32_t* benefit, int32_t k, int32_t* assign, int64_t* total);
/* Re-assign the images of an A-independent subset (no A edge between two of
 * its k <= 4096 members) by the best permutation of those images, as
 * src/independent-hungarian/hungarianSubset.c:657-795 does with the one-sided
 * gains of one_side_swap_delta (:414-459), self-loops included (the reference
 * skips them and re-scores).  *delta >= 0 is the exact score change, *changed
 * the number of members that moved. */
bm_status bm_subset_assign(bm_ctx* ctx, const int32_t* subset, int32_t k, int64_t* delta, int32_t* changed);
/* Repeat: draw a random A-independent subset of up to k members (Philox keyed
 * by seed), re-assign it optimally; `iterations` times (< 0: until the
 * budget).  Ends with a full re-score (BM_PARITY_FAIL on a mismatch). */
bm_status bm_search_hungarian(bm_ctx* ctx, int32_t k, uint64_t seed, int32_t iterations, double time_budget_s,
                              bm_progress* prog);

/* ------------------------------------------------------- initial matching */

/* Greedy-similarity initial matching on the device: the algorithm of
 * src/greedy-match.c (features compute_vertex_features/compute_2hop_metrics
 * :213-293; vertices sorted by descending feature sum :295-300; each A vertex
 * in turn takes the unmatched B vertex at the smallest L1 feature distance
 * :442-530), ties broken by vertex id; the same mapping as bm_greedy_match in
 * bm_host.h.  Edge lists with ids 1..n; weights are not used and duplicate
 * edges count, like the reference's adjacency lists.  pi receives n+1 ints
 * (slot 0 = 0).  The context provides the device and stream only; its graphs
 * and mapping are not touched. */
bm_status bm_greedy_match_dev(bm_ctx* ctx, int32_t n, int64_t mA, const int32_t* srcA, const int32_t* dstA,
                              int64_t mB, const int32_t* srcB, const int32_t* dstB, int32_t* pi);

/* ------------------------------------------------------ learned proposals */

/* A 24 -> 128 -> 128 -> 1 MLP that scores swap partners v of a vertex u from
 * structural features, trained on (candidate, exact delta) records.  No
 * counterpart in the reference: its only guided proposal is the
 * degree-weighted random swap of src/graph-re-alignment-gpu-swap.cu:767-887.
 * It only proposes; every accepted swap is gated by the exact int64 delta.
 * BF16 inputs, weights and activations, FP32 accumulation and FP32 master
 * weights.  Parameters are packed as W1[24][128] b1[128] W2[128][128] b2[128]
 * w3[128] b3 (W[i][j]: input i, output j), bm_mlp_num_params() floats.
 * A model is bound to the context (and the graphs) it was created on.
 * bm_mlp_create returns BM_UNSUPPORTED when the tensor-core row scorer's
 * shared memory (about 141 KB + n / 2 bytes of candidate bitmaps) exceeds the
 * device's per-block limit: n above about 180,000 vertices on a B200. */
typedef struct bm_mlp bm_mlp;

bm_status bm_mlp_create(bm_ctx* ctx, uint64_t seed, bm_mlp** out);
void bm_mlp_destroy(bm_mlp* m);
int32_t bm_mlp_num_params(void);
bm_status bm_mlp_get_params(bm_mlp* m, float* params);
bm_status bm_mlp_set_params(bm_mlp* m, const float* params);
/* Row scoring back end: 0 = tcgen05 tensor-core kernel (default), 1 = SIMT. */
bm_status bm_mlp_set_backend(bm_mlp* m, int32_t backend);

/* Recompute the per-vertex table (12 floats per vertex, row 0 zero) for the
 * current mapping; read it back ((n+1)*12 floats). */
bm_status bm_mlp_refresh_features(bm_mlp* m);
bm_status bm_mlp_get_features(bm_mlp* m, float* table);
/* The 24 features (BF16 values) of k pairs, from the current table. */
bm_status bm_mlp_pair_features(bm_mlp* m, const int32_t* pairs, int64_t k, float* feats);

/* Model scores: of k pairs (SIMT); of k explicit feature rows (k x 24, SIMT);
 * of whole rows (nrows x n floats, partner v at r*n + v-1, -inf at v == u,
 * by the selected back end). */
bm_status bm_mlp_score_pairs(bm_mlp* m, const int32_t* pairs, int64_t k, float* scores);
bm_status bm_mlp_score_features(bm_mlp* m, const float* x, int64_t k, float* scores);
bm_status bm_mlp_score_rows(bm_mlp* m, const int32_t* rows, int32_t nrows, float* scores);
/* Same on device buffers, asynchronous on the context stream (the scores are
 * produced in the model's own buffer and copied to d_scores).  A tensor-core
 * wait that ran out is reported by the next bm_mlp_status or host-side call. */
bm_status bm_mlp_score_rows_dev(bm_mlp* m, const int32_t* d_rows, int32_t nrows, float* d_scores);
/* Scores of listed partners: scores[r * S + i] for partner cands[r * S + i]
 * of row rows[r] (1..n, not the row's own vertex), on the same kernels as
 * bm_mlp_score_rows and equal to its scores at those partners. */
bm_status bm_mlp_score_candidates(bm_mlp* m, const int32_t* rows, int32_t nrows, const int32_t* cands, int32_t S,
                                  float* scores);
/* Synchronise and report (then clear) the tensor-core kernel's error flag:
 * BM_TIMEOUT if an MMA completion wait ran out, else BM_OK. */
bm_status bm_mlp_status(bm_mlp* m);
/* The K (1..64) best-scored partners of each row, best first, ties by lower
 * id; partners[r*K + j], scores optional. */
bm_status bm_mlp_rows_topk(bm_mlp* m, const int32_t* rows, int32_t nrows, int32_t K, int32_t* partners,
                           float* scores);

/* Loss mean((out - y)^2) over k feature rows and its gradient
 * (bm_mlp_num_params() floats), without updating the model. */
bm_status bm_mlp_gradients(bm_mlp* m, const float* x, const float* y, int64_t k, float* grads, float* loss);
/* One AdamW step (beta 0.9 / 0.999, eps 1e-8, decoupled weight decay) on
 * explicit features and targets. */
bm_status bm_mlp_adamw_step(bm_mlp* m, const float* x, const float* y, int64_t k, float lr, float weight_decay,
                            float* loss);

/* Training records (features under the mapping of the moment, target
 * sign(d) * log1p(|d|) / 8 of the exact delta d) kept on the device in a ring.
 * collect_rows evaluates whole rows with the exact row kernel and keeps per
 * row up to per_row/2 improving partners plus uniform random partners;
 * *nrecords = records held. */
bm_status bm_mlp_reserve_records(bm_mlp* m, int64_t capacity);
bm_status bm_mlp_collect_rows(bm_mlp* m, const int32_t* rows, int32_t nrows, int32_t per_row, uint64_t seed,
                              int64_t* nrecords);
bm_status bm_mlp_clear_records(bm_mlp* m);
/* AdamW steps on random minibatches of the held records; *loss = loss of the
 * last minibatch. */
bm_status bm_mlp_fit(bm_mlp* m, int32_t steps, int32_t batch, float lr, float weight_decay, uint64_t seed,
                     float* loss);

typedef struct bm_learned_params {
    int32_t topk;             /* partners proposed per row, 1..64 (0: 64) */
    int32_t rows_per_batch;   /* rows per launch (0: 2 x SMs) */
    int32_t refresh_batches;  /* feature table refreshed every this many batches (0: 1) */
    int32_t uniform;          /* 1: uniform random partners instead of the model (the yardstick for the hit rate) */
    int32_t exact_fallback;   /* 1: after a pass with at most fallback_accepts accepts, an exact row pass
                                 runs; a pass of it without accepts ends the search (converged) */
    int32_t fallback_accepts; /* threshold of the above (0: only passes without accepts) */
    int32_t train_every;      /* online AdamW step every this many batches (0: no online training) */
    int32_t train_batch;      /* records per online step (0: 4096) */
    float lr, weight_decay;
    uint64_t seed;
    int64_t max_accepts;      /* < 0: unlimited */
    int32_t max_sweeps;       /* < 0: unlimited */
    double time_budget_s;     /* <= 0: none */
    int64_t target_score;     /* > 0: stop once the score reaches it */
    int32_t sample;           /* 0: the model scores every partner of a row; S > 0: it scores S distinct
                                 random partners per row (Philox, fresh per batch) and proposes the top-K
                                 of those (S below K counts as K; S of n - 1 or more means every partner) */
} bm_learned_params;

typedef struct bm_learned_stats {
    int64_t proposals;        /* (u, v) proposals checked by the exact delta */
    int64_t hits;             /* of which improving (delta > 0) */
    int64_t exact_passes;
    int64_t train_steps;
    double t_propose, t_exact, t_train;  /* seconds in features + scoring + top-K, exact checks + applies, training */
} bm_learned_stats;

/* Search that proposes the top-K partners of each row (model, over all
 * partners or over a random sample of them, or uniform), checks them with the
 * exact delta, and applies the best improving proposal of each row when it is
 * independent of those already taken (descending delta).  Stats accumulate
 * into *stats. */
bm_status bm_search_learned(bm_ctx* ctx, bm_mlp* m, const int32_t* row_order, int32_t nrows,
                            const bm_learned_params* params, bm_progress* prog, bm_learned_stats* stats);

/* ------------------------------------------------------- device utilities */

/* Device memory, copies and events on the context stream, for callers that
 * keep inputs resident (benchmarks, pipelines).  No PyTorch needed. */
bm_status bm_dev_alloc(bm_ctx* ctx, int64_t bytes, void** d_ptr);
bm_status bm_dev_free(bm_ctx* ctx, void* d_ptr);
bm_status bm_memcpy_h2d(bm_ctx* ctx, void* d_dst, const void* h_src, int64_t bytes);
bm_status bm_memcpy_d2h(bm_ctx* ctx, void* h_dst, const void* d_src, int64_t bytes);
bm_status bm_host_alloc_pinned(int64_t bytes, void** h_ptr);
bm_status bm_host_free_pinned(void* h_ptr);
/* Write a device buffer larger than L2 so the next kernel starts cold. */
bm_status bm_l2_flush(bm_ctx* ctx);
bm_status bm_event_create(bm_ctx* ctx, void** ev);
bm_status bm_event_destroy(bm_ctx* ctx, void* ev);
bm_status bm_event_record(bm_ctx* ctx, void* ev);
bm_status bm_event_elapsed_ms(bm_ctx* ctx, void* ev_start, void* ev_stop, float* ms);
/* Kernel launches issued by this context since creation (all entry points). */
int64_t bm_launch_count(const bm_ctx* ctx);
/* PCI bus id of the context's device ("0000:1b:00.0"), for NVML queries. */
bm_status bm_device_pci_bus_id(bm_ctx* ctx, char* buf, int32_t len);
/* Device and pinned-host allocations and releases (cudaMalloc, cudaFree,
 * cudaMallocHost, cudaHostAlloc, cudaFreeHost) the library has made in this
 * process, over all contexts.  A diagnostic: an entry point that allocates
 * nothing leaves it unchanged. */
uint64_t bm_alloc_count(void);
/* L2 read bandwidth of the context's device in GB/s: a read kernel streams a
 * buffer of `bytes` (1 MiB .. the L2 size) through L2 `reps` times after one
 * pass that makes it resident, timed with CUDA events.  The roofline
 * denominator of kernels whose working set stays in L2; no reference
 * counterpart (a measurement utility). */
bm_status bm_probe_l2_bandwidth(bm_ctx* ctx, int64_t bytes, int32_t reps, double* gbs);
/* Bound, in SM clock cycles, of the context's device-side waits: each
 * MMA-completion wait of the tensor-core MLP scorer (default 4e9, about two
 * seconds) and the auction of bm_lap_solve / bm_subset_assign (default 2e10).
 * 0 restores the defaults.  A wait that runs out makes its call return
 * BM_TIMEOUT and leaves the context usable: the scorer sets an error flag,
 * waits (with the default bound) for the MMAs it issued, frees its tensor
 * memory and returns; the flag is cleared when it is reported.  A testing and
 * diagnosis aid; the reference has no counterpart (its kernels do not wait). */
bm_status bm_set_wait_limit(bm_ctx* ctx, int64_t cycles);
/* Free and total memory of the context's device (cudaMemGetInfo). */
bm_status bm_device_memory(bm_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes);

/* Delta semantics of pairwise swaps.  BM_SEMANTICS_EXACT (default): the
 * score difference.  BM_SEMANTICS_REF_CPU: the value calculate_swap_delta
 * (src/graph-alignment-optimized.c:321-408) returns, which differs from the
 * score difference only when a swapped A vertex x has a self-loop of weight
 * s: its out-edge loop (:327-340) and in-edge loop (:343-356) each meet the
 * self-loop and compare min(s, B(f1, f2)) or min(s, B(f2, f1)) against
 * min(s, B(f_x, f_x)) of the old image.  The mode applies to every pairwise
 * swap delta (bm_delta_pairs, bm_delta_rows, bm_rows_best, the delta table
 * and the schedules that accept swaps by them), so bm_sweep_parity makes the
 * reference loop's accepts on such graphs; the score a schedule reports is
 * re-computed at its end, as the reference re-scores after every accept
 * (:571-576), instead of being checked against the sum of the deltas.
 * Permutation sets, 3-rotations, annealing chains and one-sided gains stay
 * exact.  Duplicate A edges between the two swapped vertices still count once
 * per list entry (the reference counts the matrix's last weight once).  The
 * mode applies to deltas computed after the call: a delta table built before
 * it keeps its values until rebuilt or refreshed. */
#define BM_SEMANTICS_EXACT 0
#define BM_SEMANTICS_REF_CPU 1
bm_status bm_set_semantics(bm_ctx* ctx, int32_t mode);
bm_status bm_get_semantics(bm_ctx* ctx, int32_t* mode);

/* Tuning knobs of the row kernel: CTAs per row (1..8: a thread-block cluster
 * sharing the row through distributed shared memory) and threads per CTA
 * (256 or 512).  0 keeps the current value. */
bm_status bm_set_row_tiling(bm_ctx* ctx, int32_t ctas_per_row, int32_t threads);
bm_status bm_get_row_tiling(bm_ctx* ctx, int32_t* ctas_per_row, int32_t* threads);
/* Split rows: in a row launch whose rows the caller passed from the host
 * (bm_rows_best, bm_delta_rows and the search schedules; not the _dev entry
 * points), heavy rows (by a per-row work estimate refreshed when the mapping
 * is set and when a search starts) are spread over several thread-block
 * clusters, each taking a strided share of the row's first-hop items, whose
 * partial sums meet in global memory; results are identical either way.
 * slots: 0 = automatic (default: split rows of at least ~300k 2-hop entries
 * when the resident clusters of the launch's shape are at least 4x the rows),
 * -1 = off (one cluster per row), k > 0 = up to k slots (capped at 2 x SMs),
 * splitting every row it can.  No reference counterpart: the reference
 * evaluates one pair per thread. */
bm_status bm_set_row_split(bm_ctx* ctx, int32_t slots);
bm_status bm_get_row_split(bm_ctx* ctx, int32_t* slots);
/* Tiered row launches: a launch of few rows in c-CTA clusters that leaves
 * resident CTA slots free runs its heaviest rows (by the same work estimate,
 * ranked on the device, so the _dev entry points use it too) in 2c-CTA
 * clusters, in a second launch on the context's second stream concurrent with
 * the first; the calling stream waits for both.  Results are identical
 * either way.  heavy_rows: 0 = automatic (default: as many rows as keep both
 * launches resident together, by the device's resident-cluster counts for
 * the two cluster sizes), -1 = off, k > 0 = at most k rows.  Not used when the CTAs per row are set (bm_set_row_tiling) or a
 * split plan is active.  No reference counterpart. */
bm_status bm_set_row_tiers(bm_ctx* ctx, int32_t heavy_rows);
bm_status bm_get_row_tiers(bm_ctx* ctx, int32_t* heavy_rows);
/* How many row clusters of the given shape can be resident at once on the
 * device for the current n (cudaOccupancyMaxActiveClusters). */
bm_status bm_rows_max_active_clusters(bm_ctx* ctx, int32_t ctas_per_row, int32_t threads, int32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* BM_CUDA_H */
