/*
 * bm-score — the score of a matching, as score-matching
 * (src/score-matching.c:599-700) prints it:
 *
 *   bm-score <g1.csv> <g2.csv> <matching.csv> [--host] [--device D]
 *
 * score = sum over the entries (x -> y, w) of g1 of min(w, w2(pi x, pi y)),
 * w2 the weight of that edge in g2 (the last duplicate wins) and 0 when it is
 * absent (calculate_score_sparse, :558-597).  The last line of stdout is the
 * score; exit 0, or 1 on a usage or load error.  With a mapping that is a
 * bijection of 1..n the score is computed on the GPU (bm_score), otherwise,
 * or with --host, by the host library.  A vertex missing from the matching
 * contributes nothing (the reference's calloc'd matching sends it to the
 * first vertex it registered instead).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bm_cuda.h"
#include "bm_host.h"

static int load_graph(const char* path, bm_edges* e) {
    int64_t bad = 0;
    if (bm_read_graph_csv(path, e, &bad) != 0) return -1;
    if (bad > 0) fprintf(stderr, "Warning: %lld malformed lines skipped in %s\n", (long long)bad, path);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stdout, "Usage: %s <g1.csv> <g2.csv> <matching.csv> [--host] [--device D]\n", argv[0]);
        return 1;
    }
    int host_only = 0, device = 0;
    for (int i = 4; i < argc; i++) {
        if (!strcmp(argv[i], "--host")) host_only = 1;
        else if (!strcmp(argv[i], "--device") && i + 1 < argc) device = atoi(argv[++i]);
        else {
            fprintf(stdout, "Unknown option %s\n", argv[i]);
            return 1;
        }
    }
    bm_edges A = {0}, B = {0};
    if (load_graph(argv[1], &A) != 0) {
        fprintf(stdout, "Failed to load first graph: %s\n", argv[1]);
        return 1;
    }
    if (load_graph(argv[2], &B) != 0) {
        fprintf(stdout, "Failed to load second graph: %s\n", argv[2]);
        bm_edges_free(&A);
        return 1;
    }
    int32_t mx = 0;
    if (bm_scan_mapping_max_id(argv[3], &mx) != 0) {
        fprintf(stdout, "Failed to load matching: %s\n", argv[3]);
        bm_edges_free(&A);
        bm_edges_free(&B);
        return 1;
    }
    int32_t n = A.n > B.n ? A.n : B.n;
    if (mx > n) n = mx;
    A.n = B.n = n;
    int32_t* pi = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int64_t cnt = 0;
    if (!pi || bm_read_mapping(argv[3], n, pi, &cnt, NULL) != 0) {
        fprintf(stdout, "Failed to load matching: %s\n", argv[3]);
        return 1;
    }
    printf("Processing graphs with:\n");
    printf("  Graph 1: %d vertices and %lld edges\n", n, (long long)A.m);
    printf("  Graph 2: %d vertices and %lld edges\n", n, (long long)B.m);
    printf("  Matching: %lld lines\n", (long long)cnt);
    long long score = -1;
    if (!host_only && bm_check_bijection(n, pi) == 0) {
        bm_ctx* ctx = NULL;
        int64_t s = 0;
        if (bm_ctx_create(device, &ctx) == BM_OK && bm_set_graph(ctx, BM_SIDE_A, n, A.m, A.src, A.dst, A.w) == BM_OK &&
            bm_set_graph(ctx, BM_SIDE_B, n, B.m, B.src, B.dst, B.w) == BM_OK && bm_set_mapping(ctx, pi) == BM_OK &&
            bm_score(ctx, &s) == BM_OK) {
            score = s;
            printf("Score computed on the GPU\n");
        } else if (ctx) {
            fprintf(stderr, "GPU scoring failed (%s); using the host\n", bm_ctx_last_error(ctx));
        }
        if (ctx) bm_ctx_destroy(ctx);
    }
    if (score < 0) {
        score = bm_host_score(&A, &B, pi);
        printf("Score computed on the host\n");
    }
    printf("%lld\n", score);
    free(pi);
    bm_edges_free(&A);
    bm_edges_free(&B);
    return score < 0 ? 1 : 0;
}
