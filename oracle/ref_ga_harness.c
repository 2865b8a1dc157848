/*
 * ref_ga_harness.c — TEST INFRASTRUCTURE ONLY: a thin driver around the
 * reference's similarity-filtered variant, src/graph-alignment.c, compiled
 * from that source where it lies (REF_GA_SRC, given by oracle/Makefile) into
 * oracle/_ref/libref_ga.so.  Nothing of the reference is copied into this
 * repository; the file is included at build time with its main() renamed.
 *
 * It builds the variant's Graph structures with its own add_edge (which also
 * records the vertex order, add_node) and runs its optimize_mapping
 * (:489-595), which makes one filtered first-improvement pass and returns.
 * The orderings are read by the variant itself from the CSV paths given.
 * The caller keeps inputs inside the variant's assumptions: the largest vertex
 * id appears in both graphs and in both ordering files, so the metric and
 * ordering arrays it sizes by the largest id of each graph are never
 * indexed past their end.
 */
#define main refga_main
#include REF_GA_SRC
#undef main

static Graph* g_ga[2] = {NULL, NULL};

/* Build graph `which` (0 = male gm, 1 = female gf) by add_edge in input order. */
int refga_build(int which, long long m, const int* src, const int* dst, const int* w) {
    if (which < 0 || which > 1) return -1;
    if (g_ga[which]) { free_graph(g_ga[which]); g_ga[which] = NULL; }
    Graph* g = new_graph();
    for (long long e = 0; e < m; e++) add_edge(g, src[e], dst[e], w[e]);
    g_ga[which] = g;
    return 0;
}

void refga_free(void) {
    for (int i = 0; i < 2; i++)
        if (g_ga[i]) { free_graph(g_ga[i]); g_ga[i] = NULL; }
}

/* Largest vertex id of graph `which` (the size its arrays are given). */
int refga_max_node(int which) { return get_max_node(g_ga[which]); }

int refga_score(const int* mapping) { return calculate_alignment_score(g_ga[0], g_ga[1], (int*)mapping); }

/* One pass of optimize_mapping from `mapping` (length > the largest id of
 * gm); the result is copied into `out` (same length).  Returns 0. */
int refga_sweep(const int* mapping, int len, const char* ord_m, const char* ord_f, const char* out_path, int* out) {
    int max_node = get_max_node(g_ga[0]);
    if (len < max_node + 1) return -1;
    int* init = malloc(sizeof(int) * (size_t)len);
    memcpy(init, mapping, sizeof(int) * (size_t)len);
    int* res = optimize_mapping(g_ga[0], g_ga[1], init, ord_m, ord_f, out_path);
    memcpy(out, init, sizeof(int) * (size_t)len);
    memcpy(out, res, sizeof(int) * (size_t)(max_node + 1));
    free(res);
    free(init);
    return 0;
}
