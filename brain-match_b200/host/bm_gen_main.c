/*
 * bm-gen — write a seeded synthetic graph pair in the reference's CSV formats:
 *
 *   bm-gen <config 1..5> <seed> <outdir> [--n N] [--m M]
 *
 * outdir/gm.csv, gf.csv            edge lists "from,to,weight"
 * outdir/gm_order.csv, gf_order.csv "Node ID,Order" by weighted degree
 * outdir/init_mapping.csv          initial matching "m<id>,f<id>"
 * outdir/truth_mapping.csv         planted permutation
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bm_host.h"

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <config 1..5> <seed> <outdir> [--n N] [--m M]\n", argv[0]);
        return 1;
    }
    bm_gen_params p;
    if (bm_gen_defaults(atoi(argv[1]), &p) != 0) { fprintf(stderr, "unknown config %s\n", argv[1]); return 1; }
    p.seed = strtoull(argv[2], NULL, 10);
    for (int i = 4; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--n")) p.n = atoi(argv[i + 1]);
        else if (!strcmp(argv[i], "--m")) p.m_target = atoll(argv[i + 1]);
    }
    int32_t* truth = calloc((size_t)p.n + 1, sizeof(int32_t));
    int32_t* init = calloc((size_t)p.n + 1, sizeof(int32_t));
    int32_t* order = calloc((size_t)p.n + 1, sizeof(int32_t));
    bm_edges A, B;
    if (!truth || !init || !order || bm_gen_pair(&p, &A, &B, truth, init) != 0) {
        fprintf(stderr, "generation failed\n");
        return 1;
    }
    char path[4096];
    snprintf(path, sizeof path, "%s/gm.csv", argv[3]);
    if (bm_write_graph_csv(path, &A)) { fprintf(stderr, "cannot write %s\n", path); return 1; }
    snprintf(path, sizeof path, "%s/gf.csv", argv[3]);
    if (bm_write_graph_csv(path, &B)) { fprintf(stderr, "cannot write %s\n", path); return 1; }
    bm_ordering_by_weighted_degree(&A, order);
    snprintf(path, sizeof path, "%s/gm_order.csv", argv[3]);
    bm_write_ordering(path, p.n, order);
    bm_ordering_by_weighted_degree(&B, order);
    snprintf(path, sizeof path, "%s/gf_order.csv", argv[3]);
    bm_write_ordering(path, p.n, order);
    snprintf(path, sizeof path, "%s/init_mapping.csv", argv[3]);
    bm_write_mapping(path, p.n, init);
    snprintf(path, sizeof path, "%s/truth_mapping.csv", argv[3]);
    bm_write_mapping(path, p.n, truth);
    printf("n=%d mA=%lld mB=%lld score(init)=%lld score(truth)=%lld\n", p.n, (long long)A.m, (long long)B.m,
           (long long)bm_host_score(&A, &B, init), (long long)bm_host_score(&A, &B, truth));
    bm_edges_free(&A);
    bm_edges_free(&B);
    free(truth);
    free(init);
    free(order);
    return 0;
}
