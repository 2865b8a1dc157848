/*
 * bm-align — drop-in replacement for graph-alignment-optimized
 * (src/graph-alignment-optimized.c:682-738):
 *
 *   bm-align <male graph> <female graph> <male ordering> <female ordering>
 *            <in mapping> <out mapping> [options]
 *
 * Same positional arguments, CSV formats, [INFO] progress lines and exit codes
 * (0, or 1 on a usage or load error).  The search runs on the GPU through the
 * C ABI of libbmcuda.  Unlike the reference, whose loop never ends
 * (while(true), :513), the run stops when a full pass finds no improving swap
 * or when a budget runs out; the best mapping is written to <out mapping>
 * periodically and at the end.
 *
 * Options (after the six positionals):
 *   --mode parity|search   parity: the reference's serial first-improvement
 *                          order, bit-exact (default); search: batched
 *                          best-improvement with conflict-free apply
 *   --schedule natural|ordering   rows 1..n (default) or by male ordering rank
 *   --time-budget S        stop after S seconds (default: none)
 *   --max-accepts K        stop after K applied swaps
 *   --max-sweeps K         stop after K full passes
 *   --save-interval S      seconds between checkpoints (default 60)
 *   --rows-per-batch R     rows per launch in search mode (default 2 x SMs)
 *   --device D             CUDA device ordinal (default 0)
 *   --semantics exact|ref-cpu   swap deltas as score differences (default),
 *                          or as calculate_swap_delta computes them
 *                          (:321-408), which differ on graphs with
 *                          self-loops; ref-cpu with --mode parity makes the
 *                          reference loop's accepts on such graphs
 *   --ranks N --rank R     run as rank R of N processes (one per GPU) of a
 *                          sharded search (bm_search_sharded; --mode search),
 *                          in place of the reference's MPI drivers; every
 *                          rank reads the same inputs, rank 0 writes
 *                          <out mapping> and prints the progress lines
 *   --addr HOST:PORT       rank 0's address (default 127.0.0.1:29517)
 *   --comm tcp|nccl        the ranks' transport (default nccl)
 *   --comm-timeout S       bound of every exchange (default 120)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bm_cuda.h"
#include "bm_host.h"

static int g_quiet = 0; /* ranks other than 0 of a sharded run print no progress lines */
#define LOG_INFO(...) do { if (!g_quiet) { printf("[INFO] " __VA_ARGS__); printf("\n"); fflush(stdout); } } while (0)
#define LOG_ERROR(...) do { fprintf(stderr, "[ERROR] " __VA_ARGS__); fprintf(stderr, "\n"); } while (0)

static const char* commas(long long v, char* buf) {
    char tmp[32];
    snprintf(tmp, sizeof tmp, "%lld", v < 0 ? -v : v);
    int len = (int)strlen(tmp), j = 0;
    if (v < 0) buf[j++] = '-';
    for (int i = 0; i < len; i++) {
        buf[j++] = tmp[i];
        if ((len - i - 1) > 0 && (len - i - 1) % 3 == 0) buf[j++] = ',';
    }
    buf[j] = 0;
    return buf;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static int load_graph(const char* path, bm_edges* e) {
    int64_t bad = 0;
    if (bm_read_graph_csv(path, e, &bad) != 0) {
        LOG_ERROR("Failed to open file: %s", path);
        return -1;
    }
    char b1[32];
    LOG_INFO("Loading graph from %s (%s lines)", path, commas(e->m + bad, b1));
    if (bad) LOG_ERROR("Malformed lines in CSV: %lld", (long long)bad);
    LOG_INFO("Graph loaded successfully:");
    LOG_INFO("  - Edges: %s", commas(e->m, b1));
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 7) {
        LOG_ERROR("Usage: %s <male graph> <female graph> <male ordering> <female ordering> <in mapping> <out mapping> "
                  "[--mode parity|search] [--schedule natural|ordering] [--time-budget S] [--max-accepts K] "
                  "[--max-sweeps K] [--save-interval S] [--rows-per-batch R] [--device D] "
                  "[--semantics exact|ref-cpu] [--ranks N --rank R [--addr HOST:PORT] [--comm tcp|nccl] "
                  "[--comm-timeout S]]",
                  argv[0]);
        return 1;
    }
    const char* mode = "parity";
    const char* schedule = "natural";
    const char* semantics = "exact";
    double budget = 0, save_interval = 60, comm_timeout = 120;
    long long max_accepts = -1;
    int max_sweeps = -1, device = 0, rows_per_batch = 0, ranks = 1, rank = 0;
    const char* addr = "127.0.0.1:29517";
    const char* comm_kind = "nccl";
    for (int i = 7; i < argc; i++) {
        const char* a = argv[i];
        const char* v = (i + 1 < argc) ? argv[i + 1] : NULL;
        if (!v) { LOG_ERROR("option %s needs a value", a); return 1; }
        if (!strcmp(a, "--mode")) mode = v;
        else if (!strcmp(a, "--schedule")) schedule = v;
        else if (!strcmp(a, "--time-budget")) budget = atof(v);
        else if (!strcmp(a, "--max-accepts")) max_accepts = atoll(v);
        else if (!strcmp(a, "--max-sweeps")) max_sweeps = atoi(v);
        else if (!strcmp(a, "--save-interval")) save_interval = atof(v);
        else if (!strcmp(a, "--rows-per-batch")) rows_per_batch = atoi(v);
        else if (!strcmp(a, "--device")) device = atoi(v);
        else if (!strcmp(a, "--semantics")) semantics = v;
        else if (!strcmp(a, "--ranks")) ranks = atoi(v);
        else if (!strcmp(a, "--rank")) rank = atoi(v);
        else if (!strcmp(a, "--addr")) addr = v;
        else if (!strcmp(a, "--comm")) comm_kind = v;
        else if (!strcmp(a, "--comm-timeout")) comm_timeout = atof(v);
        else { LOG_ERROR("unknown option %s", a); return 1; }
        i++;
    }
    if (strcmp(mode, "parity") && strcmp(mode, "search")) { LOG_ERROR("--mode must be parity or search"); return 1; }
    if (strcmp(schedule, "natural") && strcmp(schedule, "ordering")) {
        LOG_ERROR("--schedule must be natural or ordering");
        return 1;
    }
    if (strcmp(semantics, "exact") && strcmp(semantics, "ref-cpu")) {
        LOG_ERROR("--semantics must be exact or ref-cpu");
        return 1;
    }
    if (ranks < 1 || rank < 0 || rank >= ranks) { LOG_ERROR("--rank must lie in 0..--ranks-1"); return 1; }
    if (strcmp(comm_kind, "tcp") && strcmp(comm_kind, "nccl")) { LOG_ERROR("--comm must be tcp or nccl"); return 1; }
    if (ranks > 1 && strcmp(mode, "search")) { LOG_ERROR("a multi-rank run needs --mode search"); return 1; }
    g_quiet = rank != 0;
    double t_start = now_s();
    LOG_INFO("Graph Alignment Tool v1.0");
    LOG_INFO("Starting process with:");
    LOG_INFO("  - Male graph: %s", argv[1]);
    LOG_INFO("  - Female graph: %s", argv[2]);
    LOG_INFO("  - Output mapping: %s", argv[6]);

    bm_edges gm, gf;
    if (load_graph(argv[1], &gm)) { LOG_ERROR("Failed to load male graph"); return 1; }
    if (load_graph(argv[2], &gf)) { LOG_ERROR("Failed to load female graph"); bm_edges_free(&gm); return 1; }
    int32_t map_max = 0;
    if (bm_scan_mapping_max_id(argv[5], &map_max) != 0) {
        LOG_ERROR("Failed to open file: %s", argv[5]);
        LOG_ERROR("Failed to load benchmark mapping");
        return 1;
    }
    int32_t n = gm.n;
    if (gf.n > n) n = gf.n;
    if (map_max > n) n = map_max;
    char b1[32], b2[32];
    LOG_INFO("  - Nodes: %s", commas(n, b1));
    const char* us = strrchr(argv[5], '_');
    if (us) LOG_INFO("Expected score from filename: %d", atoi(us + 1));
    LOG_INFO("Loading benchmark mapping from %s", argv[5]);
    int32_t* pi = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int64_t cnt = 0;
    if (!pi || bm_read_mapping(argv[5], n, pi, &cnt, NULL) != 0) {
        LOG_ERROR("Failed to load benchmark mapping");
        return 1;
    }
    LOG_INFO("Loaded %s mappings", commas(cnt, b1));
    int32_t bad = bm_check_bijection(n, pi);
    if (bad) {
        LOG_ERROR("mapping is not a bijection of 1..%d (first bad id %d)", n, bad);
        return 1;
    }
    gm.n = n;
    gf.n = n;
    int64_t initial_host = bm_host_score(&gm, &gf, pi);

    bm_ctx* ctx = NULL;
    bm_status st = bm_ctx_create(device, &ctx);
    if (st != BM_OK) { LOG_ERROR("bm_ctx_create(%d): %s", device, bm_status_str(st)); return 1; }
    if ((st = bm_set_graph(ctx, BM_SIDE_A, n, gm.m, gm.src, gm.dst, gm.w)) != BM_OK ||
        (st = bm_set_graph(ctx, BM_SIDE_B, n, gf.m, gf.src, gf.dst, gf.w)) != BM_OK ||
        (st = bm_set_mapping(ctx, pi)) != BM_OK ||
        (st = bm_set_semantics(ctx, strcmp(semantics, "ref-cpu") ? BM_SEMANTICS_EXACT : BM_SEMANTICS_REF_CPU)) != BM_OK) {
        LOG_ERROR("%s: %s", bm_status_str(st), bm_ctx_last_error(ctx));
        bm_ctx_destroy(ctx);
        return 1;
    }
    int64_t score = 0;
    bm_tracked_score(ctx, &score);
    if (score != initial_host) LOG_ERROR("Score mismatch - device: %lld, host: %lld", (long long)score, (long long)initial_host);
    LOG_INFO("Initial alignment score: %s", commas(score, b1));

    /* orderings are read like the reference does; the ordering schedule uses the male one */
    int32_t* order_m = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t* order_f = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    LOG_INFO("Reading ordering from %s", argv[3]);
    if (bm_read_ordering(argv[3], n, order_m) != 0) { LOG_ERROR("Error opening file: %s", argv[3]); return 1; }
    LOG_INFO("Reading ordering from %s", argv[4]);
    if (bm_read_ordering(argv[4], n, order_f) != 0) { LOG_ERROR("Error opening file: %s", argv[4]); return 1; }
    int32_t* rows = NULL;
    if (!strcmp(schedule, "ordering")) {
        rows = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        bm_rows_from_ordering(n, order_m, rows);
    }

    bm_comm* comm = NULL;
    if (ranks > 1) {
        st = bm_comm_create(strcmp(comm_kind, "tcp") ? BM_COMM_NCCL : BM_COMM_TCP, rank, ranks, addr, comm_timeout,
                            ctx, &comm);
        if (st != BM_OK) {
            LOG_ERROR("rank %d of %d: %s: %s", rank, ranks, bm_status_str(st), bm_ctx_last_error(ctx));
            bm_ctx_destroy(ctx);
            return 1;
        }
        LOG_INFO("Rank %d of %d (%s transport, rank 0 at %s)", rank, ranks, comm_kind, addr);
    }
    int64_t initial = score;
    LOG_INFO("Starting optimization with initial score: %s", commas(initial, b1));
    bm_progress prog;
    memset(&prog, 0, sizeof prog);
    double t0 = now_s(), last_save = t0;
    for (;;) {
        double left = budget > 0 ? budget - (now_s() - t0) : 0;
        if (budget > 0 && left <= 0) break;
        double chunk = save_interval > 0 ? save_interval : 60;
        if (budget > 0 && left < chunk) chunk = left;
        long long acc_left = max_accepts >= 0 ? max_accepts - prog.accepts : -1;
        if (max_accepts >= 0 && acc_left <= 0) break;
        int sw_left = max_sweeps >= 0 ? max_sweeps - prog.sweeps : -1;
        if (max_sweeps >= 0 && sw_left <= 0) break;
        int32_t sweeps_before = prog.sweeps;
        if (comm)
            st = bm_search_sharded(ctx, comm, rows, rows ? n : 0, rows_per_batch, -1, chunk, &prog);
        else if (!strcmp(mode, "parity"))
            st = bm_sweep_parity(ctx, rows, rows ? n : 0, acc_left, sw_left >= 0 ? sweeps_before + sw_left : -1,
                                 chunk, &prog);
        else
            st = bm_search_batched(ctx, rows, rows ? n : 0, rows_per_batch, acc_left,
                                   sw_left >= 0 ? sweeps_before + sw_left : -1, chunk, 0, &prog);
        if (st != BM_OK && st != BM_TIMEOUT) {
            LOG_ERROR("%s: %s", bm_status_str(st), bm_ctx_last_error(ctx));
            if (st != BM_PARITY_FAIL || comm) { bm_comm_destroy(comm); bm_ctx_destroy(ctx); return 1; }
        }
        double el = now_s() - t0;
        LOG_INFO("Optimization progress:");
        LOG_INFO("  - Processed: %s rows, %d full passes", commas(prog.rows_done, b1), prog.sweeps);
        LOG_INFO("  - Current score: %s", commas(prog.score, b1));
        LOG_INFO("  - Improvements found: %s", commas(prog.accepts, b1));
        LOG_INFO("  - Processing speed: %.1f nodes/sec, %.3g deltas/sec", el > 0 ? prog.rows_done / el : 0.0,
                 el > 0 ? prog.evaluated / el : 0.0);
        if (rank == 0 && (now_s() - last_save >= save_interval || prog.converged || st == BM_OK)) {
            bm_get_mapping(ctx, pi);
            if (bm_write_mapping(argv[6], n, pi) != 0) LOG_ERROR("Error creating file: %s", argv[6]);
            last_save = now_s();
        }
        if (prog.converged || st == BM_OK) break;
        if (comm) {
            /* the ranks' clocks differ: they stop together when any rank's budget is spent */
            int64_t stops = 0;
            const int my_stop = budget > 0 && budget - (now_s() - t0) <= 0;
            if ((st = bm_comm_allreduce_sum(comm, my_stop, &stops)) != BM_OK) {
                LOG_ERROR("%s: %s", bm_status_str(st), bm_comm_last_error(comm));
                bm_comm_destroy(comm);
                bm_ctx_destroy(ctx);
                return 1;
            }
            if (stops > 0) break;
        }
    }
    bm_comm_destroy(comm);
    bm_get_mapping(ctx, pi);
    if (rank == 0 && bm_write_mapping(argv[6], n, pi) != 0) { LOG_ERROR("Error creating file: %s", argv[6]); return 1; }
    int64_t final_dev = 0;
    bm_score(ctx, &final_dev);
    int64_t final_host = bm_host_score(&gm, &gf, pi);
    if (final_host != final_dev) LOG_ERROR("Score mismatch - device: %lld, host: %lld", (long long)final_dev, (long long)final_host);
    double t_end = now_s();
    LOG_INFO("Optimization completed:");
    LOG_INFO("  - Final score: %s", commas(final_host, b1));
    LOG_INFO("  - Total improvements: %s", commas(prog.accepts, b1));
    LOG_INFO("  - Converged: %s", prog.converged ? "yes" : "no");
    LOG_INFO("  - Time taken: %.1f minutes", (t_end - t0) / 60);
    LOG_INFO("Process completed:");
    LOG_INFO("  - Initial score: %s", commas(initial, b1));
    LOG_INFO("  - Final score: %s", commas(final_host, b2));
    LOG_INFO("  - Improvement: %.2f%%", initial ? (double)(final_host - initial) / (double)initial * 100.0 : 0.0);
    LOG_INFO("  - Total time: %.1f minutes", (t_end - t_start) / 60);
    bm_ctx_destroy(ctx);
    bm_edges_free(&gm);
    bm_edges_free(&gf);
    free(pi);
    free(order_m);
    free(order_f);
    free(rows);
    return 0;
}
