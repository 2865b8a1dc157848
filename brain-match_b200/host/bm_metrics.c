/*
 * bm_metrics.c — inputs of the similarity-filtered pass of the reference's
 * graph-alignment variant (src/graph-alignment.c), for bm_sweep_similarity:
 *
 *   bm_first_appearance  the variant's vertex list g->nodes: every vertex in
 *                        order of first appearance, the source then the
 *                        target of each edge in file order (add_node called
 *                        from add_edge, :159-200)
 *   bm_node_metrics      calculate_node_metrics (:235-272) for the listed
 *                        vertices: in/out degree (edge counts), the weight
 *                        total of both directions, that total over the in-
 *                        and over the out-degree, and the ordering rank
 */
#include <stdlib.h>
#include <string.h>

#include "bm_host.h"

int bm_first_appearance(const bm_edges* e, int32_t* nodes, int32_t* count) {
    if (!e || !nodes || !count || e->n < 0) return -1;
    char* seen = (char*)calloc((size_t)e->n + 1, 1);
    if (!seen) return -1;
    int32_t c = 0;
    for (int64_t i = 0; i < e->m; i++) {
        const int32_t ends[2] = {e->src[i], e->dst[i]};
        for (int k = 0; k < 2; k++) {
            const int32_t v = ends[k];
            if (v < 1 || v > e->n) { free(seen); return -1; }
            if (!seen[v]) {
                seen[v] = 1;
                nodes[c++] = v;
            }
        }
    }
    free(seen);
    *count = c;
    return 0;
}

int bm_node_metrics(const bm_edges* e, const int32_t* rank, double* metrics) {
    if (!e || !metrics || e->n < 0) return -1;
    const size_t n1 = (size_t)e->n + 1;
    int64_t* indeg = (int64_t*)calloc(n1, sizeof(int64_t));
    int64_t* outdeg = (int64_t*)calloc(n1, sizeof(int64_t));
    int64_t* wsum = (int64_t*)calloc(n1, sizeof(int64_t));
    char* listed = (char*)calloc(n1, 1);
    if (!indeg || !outdeg || !wsum || !listed) {
        free(indeg); free(outdeg); free(wsum); free(listed);
        return -1;
    }
    for (int64_t i = 0; i < e->m; i++) {
        const int32_t s = e->src[i], d = e->dst[i];
        if (s < 1 || s > e->n || d < 1 || d > e->n) {
            free(indeg); free(outdeg); free(wsum); free(listed);
            return -1;
        }
        outdeg[s]++;
        indeg[d]++;
        wsum[s] += e->w[i];
        wsum[d] += e->w[i];
        listed[s] = listed[d] = 1;
    }
    memset(metrics, 0, sizeof(double) * 5 * n1);
    for (size_t v = 1; v < n1; v++) {
        if (!listed[v]) continue;
        double* m = metrics + 5 * v;
        m[0] = (double)indeg[v];
        m[1] = (double)outdeg[v];
        if (indeg[v] > 0) m[2] = (double)(int32_t)wsum[v] / (double)(int32_t)indeg[v];
        if (outdeg[v] > 0) m[3] = (double)(int32_t)wsum[v] / (double)(int32_t)outdeg[v];
        m[4] = rank ? (double)rank[v] : 0.0;
    }
    free(indeg); free(outdeg); free(wsum); free(listed);
    return 0;
}
