/*
 * bm_greedy.c — greedy similarity initial matching and a host scorer.
 *
 * bm_greedy_match restates the algorithm of src/greedy-match.c:
 *   features  compute_vertex_features / compute_2hop_metrics  :213-293
 *   sort      qsort by total_score descending                 :296-300, :478-479
 *   greedy    nearest unmatched by L1 feature distance        :442-447, :483-510
 * The reference's qsort is not stable; here ties are broken by vertex id so the
 * result does not depend on the C library.
 */
#include "bm_host.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t n;
    int32_t* ptr;  /* n+2 */
    int32_t* adj;  /* targets */
} csr_t;

static int build_csr(const bm_edges* g, int reverse, csr_t* c) {
    int32_t n = g->n;
    c->n = n;
    c->ptr = (int32_t*)calloc((size_t)n + 2, sizeof(int32_t));
    c->adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g->m > 0 ? g->m : 1));
    if (!c->ptr || !c->adj) return -1;
    for (int64_t e = 0; e < g->m; e++) {
        int32_t s = reverse ? g->dst[e] : g->src[e];
        c->ptr[s + 1]++;
    }
    for (int32_t i = 1; i <= n + 1; i++) c->ptr[i] += c->ptr[i - 1];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    if (!fill) return -1;
    memcpy(fill, c->ptr, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t e = 0; e < g->m; e++) {
        int32_t s = reverse ? g->dst[e] : g->src[e];
        int32_t d = reverse ? g->src[e] : g->dst[e];
        c->adj[fill[s]++] = d;
    }
    free(fill);
    return 0;
}

static void free_csr(csr_t* c) { free(c->ptr); free(c->adj); }

typedef struct {
    int32_t id;
    int32_t f[4];   /* in_degree, out_degree, reachable_2hop, can_reach_2hop */
    int64_t total;
} feat_t;

static void features(const bm_edges* g, feat_t* F) {
    csr_t out, in;
    build_csr(g, 0, &out);
    build_csr(g, 1, &in);
    int32_t n = g->n;
#pragma omp parallel
    {
        int32_t* stamp = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
        int32_t tag = 0;
#pragma omp for schedule(dynamic, 64)
        for (int32_t v = 1; v <= n; v++) {
            F[v - 1].id = v;
            F[v - 1].f[0] = in.ptr[v + 1] - in.ptr[v];
            F[v - 1].f[1] = out.ptr[v + 1] - out.ptr[v];
            for (int dir = 0; dir < 2; dir++) {
                const csr_t* c = dir == 0 ? &out : &in;
                tag++;
                int32_t cnt = 0;
                for (int32_t i = c->ptr[v]; i < c->ptr[v + 1]; i++) {
                    int32_t x = c->adj[i];
                    for (int32_t j = c->ptr[x]; j < c->ptr[x + 1]; j++) {
                        int32_t y = c->adj[j];
                        if (stamp[y] != tag) { stamp[y] = tag; cnt++; }
                    }
                }
                F[v - 1].f[2 + dir] = cnt;
            }
            F[v - 1].total = (int64_t)F[v - 1].f[0] + F[v - 1].f[1] + F[v - 1].f[2] + F[v - 1].f[3];
        }
        free(stamp);
    }
    free_csr(&out);
    free_csr(&in);
}

static int cmp_feat(const void* a, const void* b) {
    const feat_t* x = (const feat_t*)a;
    const feat_t* y = (const feat_t*)b;
    if (x->total != y->total) return x->total > y->total ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

int bm_greedy_match(const bm_edges* A, const bm_edges* B, int32_t* pi) {
    int32_t n = A->n > B->n ? A->n : B->n;
    bm_edges a = *A, b = *B;
    a.n = n;
    b.n = n;
    feat_t* FA = (feat_t*)calloc((size_t)n, sizeof(feat_t));
    feat_t* FB = (feat_t*)calloc((size_t)n, sizeof(feat_t));
    unsigned char* used = (unsigned char*)calloc((size_t)n, 1);
    if (!FA || !FB || !used) return -1;
    features(&a, FA);
    features(&b, FB);
    qsort(FA, (size_t)n, sizeof(feat_t), cmp_feat);
    qsort(FB, (size_t)n, sizeof(feat_t), cmp_feat);
    memset(pi, 0, sizeof(int32_t) * ((size_t)n + 1));
    for (int32_t i = 0; i < n; i++) {
        int64_t best = LLONG_MAX;
        int32_t bj = -1;
#pragma omp parallel
        {
            int64_t lb = LLONG_MAX;
            int32_t lj = -1;
#pragma omp for schedule(static) nowait
            for (int32_t j = 0; j < n; j++) {
                if (used[j]) continue;
                int64_t d = 0;
                for (int k = 0; k < 4; k++) {
                    int64_t t = (int64_t)FA[i].f[k] - FB[j].f[k];
                    d += t < 0 ? -t : t;
                }
                if (d < lb) { lb = d; lj = j; }
            }
#pragma omp critical
            {
                if (lj >= 0 && (lb < best || (lb == best && lj < bj))) { best = lb; bj = lj; }
            }
        }
        if (bj >= 0) {
            used[bj] = 1;
            pi[FA[i].id] = FB[bj].id;
        }
    }
    free(FA);
    free(FB);
    free(used);
    return 0;
}

/* ------------------------------------------------------------ host score */

typedef struct { uint64_t* slot; uint64_t mask; } wmap;

static uint64_t mixk(uint64_t k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return k;
}

int64_t bm_host_score(const bm_edges* A, const bm_edges* B, const int32_t* pi) {
    uint64_t cap = 16;
    while (cap < (uint64_t)(B->m * 2 + 16)) cap <<= 1;
    uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    int32_t* val = (int32_t*)malloc(sizeof(int32_t) * cap);
    if (!key || !val) return -1;
    memset(key, 0xff, sizeof(uint64_t) * cap);
    for (int64_t e = 0; e < B->m; e++) {
        uint64_t k = ((uint64_t)(uint32_t)B->src[e] << 32) | (uint32_t)B->dst[e];
        uint64_t h = mixk(k) & (cap - 1);
        while (key[h] != ~0ull && key[h] != k) h = (h + 1) & (cap - 1);
        key[h] = k;
        val[h] = B->w[e]; /* last duplicate wins, like the dense matrix */
    }
    int64_t s = 0;
    for (int64_t e = 0; e < A->m; e++) {
        int32_t x = A->src[e], y = A->dst[e];
        uint64_t k = ((uint64_t)(uint32_t)pi[x] << 32) | (uint32_t)pi[y];
        uint64_t h = mixk(k) & (cap - 1);
        int32_t bw = 0;
        while (key[h] != ~0ull) {
            if (key[h] == k) { bw = val[h]; break; }
            h = (h + 1) & (cap - 1);
        }
        int32_t aw = A->w[e];
        s += aw < bw ? aw : bw;
    }
    free(key);
    free(val);
    return s;
}

/* ------------------------------------------- independent-subset selection */

typedef struct { int64_t d; int32_t i; } dsel;

static int cmp_dsel(const void* a, const void* b) {
    const dsel* x = (const dsel*)a;
    const dsel* y = (const dsel*)b;
    if (x->d != y->d) return x->d > y->d ? -1 : 1;
    return x->i < y->i ? -1 : (x->i > y->i);
}

int bm_select_independent_host(const bm_edges* A, const int32_t* pairs, const int64_t* deltas, int32_t count,
                               int32_t* chosen, int32_t* nchosen) {
    const int32_t n = A->n;
    /* undirected closed neighbourhoods as a CSR over both edge directions */
    int32_t* deg = (int32_t*)calloc((size_t)n + 2, sizeof(int32_t));
    int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(2 * A->m + 1));
    dsel* ord = (dsel*)malloc(sizeof(dsel) * (size_t)(count > 0 ? count : 1));
    uint8_t* mark = (uint8_t*)calloc((size_t)n + 1, 1);
    if (!deg || !adj || !ord || !mark) { free(deg); free(adj); free(ord); free(mark); return -1; }
    for (int64_t e = 0; e < A->m; e++) { deg[A->src[e] + 1]++; deg[A->dst[e] + 1]++; }
    for (int32_t v = 1; v <= n + 1; v++) deg[v] += deg[v - 1];
    int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    memcpy(fill, deg, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t e = 0; e < A->m; e++) {
        if (A->w[e] == 0) continue;
        adj[fill[A->src[e]]++] = A->dst[e];
        adj[fill[A->dst[e]]++] = A->src[e];
    }
    int32_t k = 0;
    for (int32_t i = 0; i < count; i++)
        if (deltas[i] > 0 && pairs[2 * i] != pairs[2 * i + 1]) { ord[k].d = deltas[i]; ord[k].i = i; k++; }
    qsort(ord, (size_t)k, sizeof(dsel), cmp_dsel);
    int32_t c = 0;
    for (int32_t t = 0; t < k; t++) {
        const int32_t i = ord[t].i, u = pairs[2 * i], v = pairs[2 * i + 1];
        if (mark[u] || mark[v]) continue;
        const int32_t ends[2] = {u, v};
        for (int q = 0; q < 2; q++) {
            const int32_t x = ends[q];
            mark[x] = 1;
            for (int32_t j = deg[x]; j < fill[x]; j++) mark[adj[j]] = 1;
        }
        chosen[c++] = i;
    }
    *nchosen = c;
    free(deg); free(adj); free(ord); free(mark); free(fill);
    return 0;
}
