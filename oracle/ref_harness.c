/*
 * ref_harness.c — TEST INFRASTRUCTURE ONLY: a thin driver around the
 * reference's own functions, compiled from the reference's source file where
 * it lies (REF_SRC, given by oracle/Makefile) into oracle/_ref/libref.so.
 * Nothing of the reference is copied into this repository; the file is
 * included at build time with its main() renamed.
 *
 * It builds the reference's Graph structures with new_graph/add_edge and
 * exposes calculate_alignment_score, calculate_swap_delta, a bounded driver of
 * the optimize_mapping loop order (src/graph-alignment-optimized.c:513-580,
 * which itself never returns) and the OpenMP m2 sweep of
 * src/graph-alignment-optimized-parallel.c:544 without applies (the CPU
 * baseline).  The reference fixes NUM_NODES = 18524, so graphs with fewer
 * vertices are padded with isolated vertices mapped to themselves; such
 * vertices never yield a positive delta.
 */
#define main ref_main
#include REF_SRC
#undef main

#include <stdint.h>

static Graph* g_ref[2] = {NULL, NULL};
static int g_n_active = 0;

int ref_num_nodes(void) { return NUM_NODES; }

/* Build graph `which` (0 = male gm, 1 = female gf) by add_edge in input order. */
int ref_build(int which, int n_active, long long m, const int* src, const int* dst, const int* w) {
    if (which < 0 || which > 1 || n_active > NUM_NODES) return -1;
    if (g_ref[which]) { free_graph(g_ref[which]); g_ref[which] = NULL; }
    Graph* g = new_graph();
    for (long long e = 0; e < m; e++) add_edge(g, src[e], dst[e], w[e]);
    if (g->edges == NULL) { /* add_edge allocates the lists lazily */
        g->edges = calloc(MAX_NODES, sizeof(EdgeMap));
        g->reverse_edges = calloc(MAX_NODES, sizeof(EdgeMap));
    }
    g_ref[which] = g;
    g_n_active = n_active;
    return 0;
}

void ref_free(void) {
    for (int i = 0; i < 2; i++)
        if (g_ref[i]) { free_graph(g_ref[i]); g_ref[i] = NULL; }
}

/* mapping of length n_active+1 -> the reference's NUM_NODES+1 array */
static int* padded(const int* mapping) {
    int* p = malloc(sizeof(int) * (NUM_NODES + 1));
    for (int i = 0; i <= NUM_NODES; i++) p[i] = (i <= g_n_active) ? mapping[i] : i;
    p[0] = 0;
    return p;
}

int ref_score(const int* mapping) {
    int* p = padded(mapping);
    int s = calculate_alignment_score(g_ref[0], g_ref[1], p);
    free(p);
    return s;
}

void ref_pairs(const int* mapping, const int* pairs, long long k, int* out) {
    int* p = padded(mapping);
    for (long long i = 0; i < k; i++)
        out[i] = (pairs[2 * i] == pairs[2 * i + 1]) ? 0
                 : calculate_swap_delta(g_ref[0], g_ref[1], p, pairs[2 * i], pairs[2 * i + 1]);
    free(p);
}

/* Bounded driver in the order of optimize_mapping: m1 over rows, m2 = 1..n,
 * accept delta > 0 with the swap of :559-561 and, if verify, the full
 * re-score of :571-576 ("trust the verification").  Columns above n_active
 * are isolated padding and are skipped (they never improve). */
long long ref_serial(int* mapping, const int* rows, int nrows, long long max_accepts, int max_sweeps, int verify,
                     long long* score, int* log_m1, int* log_m2, int* log_delta, long long log_cap, int* sweeps_done,
                     int* converged) {
    int* p = padded(mapping);
    int cur = calculate_alignment_score(g_ref[0], g_ref[1], p);
    long long accepts = 0;
    int sweeps = 0;
    *converged = 0;
    for (;;) {
        long long pass_acc = 0;
        for (int r = 0; r < nrows; r++) {
            int m1 = rows ? rows[r] : r + 1;
            for (int m2 = 1; m2 <= g_n_active; m2++) {
                if (m1 == m2) continue;
                if (max_accepts >= 0 && accepts >= max_accepts) goto done;
                int delta = calculate_swap_delta(g_ref[0], g_ref[1], p, m1, m2);
                if (delta > 0) {
                    int f1 = p[m1], f2 = p[m2];
                    p[m1] = f2;
                    p[m2] = f1;
                    cur += delta;
                    if (verify) {
                        int v = calculate_alignment_score(g_ref[0], g_ref[1], p);
                        if (v != cur) cur = v;
                    }
                    if (accepts < log_cap) { log_m1[accepts] = m1; log_m2[accepts] = m2; log_delta[accepts] = delta; }
                    accepts++;
                    pass_acc++;
                }
            }
        }
        sweeps++;
        if (pass_acc == 0) { *converged = 1; break; }
        if (max_sweeps >= 0 && sweeps >= max_sweeps) break;
    }
done:
    for (int i = 0; i <= g_n_active; i++) mapping[i] = p[i];
    free(p);
    *score = cur;
    *sweeps_done = sweeps;
    return accepts;
}

/* The OpenMP m2 sweep (src/graph-alignment-optimized-parallel.c:544) calling
 * the reference calculate_swap_delta, deltas only: out[r*(n_active+1)+m2]. */
void ref_rows_omp(const int* mapping, const int* rows, int nrows, int* out, int threads) {
    int* p = padded(mapping);
    int n = g_n_active;
    if (threads > 0) omp_set_num_threads(threads);
    for (int r = 0; r < nrows; r++) {
        int m1 = rows[r];
        int* o = out + (long long)r * (n + 1);
        o[0] = 0;
#pragma omp parallel for schedule(dynamic)
        for (int m2 = 1; m2 <= n; m2++) o[m2] = (m2 == m1) ? 0 : calculate_swap_delta(g_ref[0], g_ref[1], p, m1, m2);
    }
    free(p);
}
