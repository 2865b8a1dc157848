/*
 * bm_oracle.c — CPU restatement of the reference's swap-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the GPU kernels are
 * compared against; it is loaded by tests/, by __graft_entry__.smoke() and by
 * the CPU-baseline leg of bench.py, and by nothing else.  The engine
 * (libbmcuda) never calls it and has no CPU fallback.
 *
 * Each function follows the named reference function line by line in
 * behaviour (data layout differs: edge lists in insertion order as EdgeMap
 * keeps them, and the dense int16 matrix replaced by a hash with the same
 * last-write-wins rule):
 *   orc_score       calculate_alignment_score  src/graph-alignment-optimized.c:292-307
 *   orc_swap_delta  calculate_swap_delta       src/graph-alignment-optimized.c:321-408
 *   orc_serial      optimize_mapping loop      src/graph-alignment-optimized.c:513-580
 *                   (bounded: the reference loops forever)
 *   orc_rows_omp    the OpenMP m2 sweep        src/graph-alignment-optimized-parallel.c:544
 *                   (deltas only, no applies)
 *   orc_sim_sweep   the similarity-filtered    src/graph-alignment.c:489-595
 *                   pass of the graph-alignment variant
 *   orc_mlp         FP64 replica of the engine's learned-proposal MLP (no
 *                   reference counterpart), the checker of its gradients
 * Parity is pinned by tests/golden/ fixtures produced by the reference's own
 * functions compiled from its sources (oracle/ref_harness.c).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* The chains' RNG (Philox4x32-10) and exp are defined by the engine; the
 * replay below uses the same definitions so a chain can be checked step by
 * step.  Both are pinned separately (known-answer vectors, error bounds). */
#include "../brain-match_b200/csrc/bm_rng.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int32_t n;
    int64_t m;
    int32_t* optr;  /* n+2: out-lists in insertion order (EdgeMap edges) */
    int32_t* oto;
    int32_t* ow;
    int32_t* iptr;  /* n+2: in-lists (EdgeMap reverse_edges) */
    int32_t* ifrom;
    int32_t* iw;
    /* vertices in order of first appearance (from, then to, of each edge) */
    int32_t* nodes;
    int32_t nnodes;
    /* matrix lookups: key (s,d) -> last weight */
    uint64_t* hkey;
    int32_t* hval;
    uint64_t hmask;
} orc_graph;

static uint64_t orc_mix(uint64_t k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33;
    return k;
}

static int32_t mat(const orc_graph* g, int32_t s, int32_t d) {
    uint64_t k = ((uint64_t)(uint32_t)s << 32) | (uint32_t)d;
    uint64_t h = orc_mix(k) & g->hmask;
    while (g->hkey[h] != ~0ull) {
        if (g->hkey[h] == k) return g->hval[h];
        h = (h + 1) & g->hmask;
    }
    return 0;
}

#define MIN(a, b) ((a) < (b) ? (a) : (b))

void orc_graph_free(orc_graph* g) {
    if (!g) return;
    free(g->optr); free(g->oto); free(g->ow);
    free(g->iptr); free(g->ifrom); free(g->iw);
    free(g->hkey); free(g->hval);
    free(g->nodes);
    free(g);
}

/* add_edge (src/graph-alignment-optimized.c:183-204): the edge goes to the
 * end of from's out-list and to's in-list; the matrix keeps the last weight. */
orc_graph* orc_graph_new(int32_t n, int64_t m, const int32_t* src, const int32_t* dst, const int32_t* w) {
    orc_graph* g = (orc_graph*)calloc(1, sizeof(orc_graph));
    if (!g) return NULL;
    g->n = n;
    g->m = m;
    g->optr = (int32_t*)calloc((size_t)n + 2, sizeof(int32_t));
    g->iptr = (int32_t*)calloc((size_t)n + 2, sizeof(int32_t));
    g->oto = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    g->ow = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    g->ifrom = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    g->iw = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    uint64_t cap = 16;
    while (cap < (uint64_t)(2 * m + 16)) cap <<= 1;
    g->hkey = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    g->hval = (int32_t*)malloc(sizeof(int32_t) * cap);
    g->nodes = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    if (!g->optr || !g->iptr || !g->oto || !g->ow || !g->ifrom || !g->iw || !g->hkey || !g->hval || !g->nodes) {
        orc_graph_free(g);
        return NULL;
    }
    g->hmask = cap - 1;
    memset(g->hkey, 0xff, sizeof(uint64_t) * cap);
    for (int64_t e = 0; e < m; e++) { g->optr[src[e] + 1]++; g->iptr[dst[e] + 1]++; }
    for (int32_t i = 1; i <= n + 1; i++) { g->optr[i] += g->optr[i - 1]; g->iptr[i] += g->iptr[i - 1]; }
    int32_t* fo = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    int32_t* fi = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    memcpy(fo, g->optr, sizeof(int32_t) * ((size_t)n + 1));
    memcpy(fi, g->iptr, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t e = 0; e < m; e++) {
        int32_t s = src[e], d = dst[e];
        g->oto[fo[s]] = d; g->ow[fo[s]++] = w[e];
        g->ifrom[fi[d]] = s; g->iw[fi[d]++] = w[e];
        uint64_t k = ((uint64_t)(uint32_t)s << 32) | (uint32_t)d;
        uint64_t h = orc_mix(k) & g->hmask;
        while (g->hkey[h] != ~0ull && g->hkey[h] != k) h = (h + 1) & g->hmask;
        g->hkey[h] = k;
        g->hval[h] = (int32_t)(int16_t)w[e]; /* the matrix is short */
    }
    free(fo);
    free(fi);
    /* add_node (src/graph-alignment.c:159-174) for from, then to */
    uint8_t* seen = (uint8_t*)calloc((size_t)n + 1, 1);
    if (!seen) { orc_graph_free(g); return NULL; }
    for (int64_t e = 0; e < m; e++) {
        const int32_t v2[2] = {src[e], dst[e]};
        for (int k = 0; k < 2; k++)
            if (!seen[v2[k]]) { seen[v2[k]] = 1; g->nodes[g->nnodes++] = v2[k]; }
    }
    free(seen);
    return g;
}

/* calculate_alignment_score, src/graph-alignment-optimized.c:292-307 */
int64_t orc_score(const orc_graph* gm, const orc_graph* gf, const int32_t* mapping) {
    int64_t score = 0;
    for (int32_t s = 1; s <= gm->n; s++)
        for (int32_t j = gm->optr[s]; j < gm->optr[s + 1]; j++) {
            int32_t d = gm->oto[j];
            score += MIN(gm->ow[j], mat(gf, mapping[s], mapping[d]));
        }
    return score;
}

/* calculate_swap_delta, src/graph-alignment-optimized.c:321-408 */
int64_t orc_swap_delta(const orc_graph* gm, const orc_graph* gf, const int32_t* mapping, int32_t m1, int32_t m2) {
    int32_t f1 = mapping[m1], f2 = mapping[m2];
    int64_t delta = 0;
    for (int32_t j = gm->optr[m1]; j < gm->optr[m1 + 1]; j++) {          /* out of m1 :327-340 */
        int32_t d = gm->oto[j];
        if (d == m2) continue;
        int32_t w = gm->ow[j], df = mapping[d];
        delta += MIN(w, mat(gf, f2, df)) - MIN(w, mat(gf, f1, df));
    }
    for (int32_t j = gm->iptr[m1]; j < gm->iptr[m1 + 1]; j++) {          /* into m1 :343-356 */
        int32_t s = gm->ifrom[j];
        if (s == m2) continue;
        int32_t w = gm->iw[j], sf = mapping[s];
        delta += MIN(w, mat(gf, sf, f2)) - MIN(w, mat(gf, sf, f1));
    }
    for (int32_t j = gm->optr[m2]; j < gm->optr[m2 + 1]; j++) {          /* out of m2 :359-372 */
        int32_t d = gm->oto[j];
        if (d == m1) continue;
        int32_t w = gm->ow[j], df = mapping[d];
        delta += MIN(w, mat(gf, f1, df)) - MIN(w, mat(gf, f2, df));
    }
    for (int32_t j = gm->iptr[m2]; j < gm->iptr[m2 + 1]; j++) {          /* into m2 :375-388 */
        int32_t s = gm->ifrom[j];
        if (s == m1) continue;
        int32_t w = gm->iw[j], sf = mapping[s];
        delta += MIN(w, mat(gf, sf, f1)) - MIN(w, mat(gf, sf, f2));
    }
    int32_t a = mat(gm, m1, m2);                                          /* m1 -> m2 :392-397 */
    if (a > 0) delta += MIN(a, mat(gf, f2, f1)) - MIN(a, mat(gf, f1, f2));
    int32_t b = mat(gm, m2, m1);                                          /* m2 -> m1 :400-405 */
    if (b > 0) delta += MIN(b, mat(gf, f1, f2)) - MIN(b, mat(gf, f2, f1));
    return delta;
}

/* Exact delta by re-scoring: score(pi with m1,m2 swapped) - score(pi).  The
 * ground truth on graphs with self-loops, where calculate_swap_delta counts a
 * self-loop twice against the old image. */
int64_t orc_exact_delta(const orc_graph* gm, const orc_graph* gf, int32_t* mapping, int32_t m1, int32_t m2) {
    int64_t before = orc_score(gm, gf, mapping);
    int32_t t = mapping[m1]; mapping[m1] = mapping[m2]; mapping[m2] = t;
    int64_t after = orc_score(gm, gf, mapping);
    t = mapping[m1]; mapping[m1] = mapping[m2]; mapping[m2] = t;
    return after - before;
}

/* Bounded serial first-improvement loop of optimize_mapping
 * (src/graph-alignment-optimized.c:513-580): for m1 in rows, for m2 = 1..n,
 * m2 != m1: accept the first delta > 0 and apply it at once.  Stops after a
 * pass without accepts, after max_sweeps passes, or after max_accepts accepts.
 * Accepted moves are logged (m1, m2, delta) up to log_cap entries.
 * Returns the number of accepts; *score is updated by the deltas. */
int64_t orc_serial(const orc_graph* gm, const orc_graph* gf, int32_t* mapping, const int32_t* rows, int32_t nrows,
                   int64_t max_accepts, int32_t max_sweeps, int64_t* score, int32_t* log_m1, int32_t* log_m2,
                   int64_t* log_delta, int64_t log_cap, int32_t* sweeps_done, int32_t* converged) {
    int32_t n = gm->n;
    int64_t accepts = 0;
    int32_t sweeps = 0;
    *converged = 0;
    for (;;) {
        int64_t pass_acc = 0;
        for (int32_t r = 0; r < nrows; r++) {
            int32_t m1 = rows ? rows[r] : r + 1;
            for (int32_t m2 = 1; m2 <= n; m2++) {
                if (m1 == m2) continue;
                if (max_accepts >= 0 && accepts >= max_accepts) goto done;
                int64_t delta = orc_swap_delta(gm, gf, mapping, m1, m2);
                if (delta > 0) {
                    int32_t f1 = mapping[m1], f2 = mapping[m2];
                    mapping[m1] = f2;
                    mapping[m2] = f1;
                    *score += delta;
                    if (accepts < log_cap) {
                        log_m1[accepts] = m1;
                        log_m2[accepts] = m2;
                        log_delta[accepts] = delta;
                    }
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
    *sweeps_done = sweeps;
    return accepts;
}

/* The OpenMP m2 sweep (src/graph-alignment-optimized-parallel.c:544) without
 * applies: deltas of rows x all columns, out[r*(n+1)+m2]. */
void orc_rows_omp(const orc_graph* gm, const orc_graph* gf, const int32_t* mapping, const int32_t* rows,
                  int32_t nrows, int64_t* out, int32_t threads) {
    int32_t n = gm->n;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    for (int32_t r = 0; r < nrows; r++) {
        int32_t m1 = rows[r];
        int64_t* o = out + (size_t)r * ((size_t)n + 1);
        o[0] = 0;
#pragma omp parallel for schedule(dynamic, 64)
        for (int32_t m2 = 1; m2 <= n; m2++)
            o[m2] = (m2 == m1) ? 0 : orc_swap_delta(gm, gf, mapping, m1, m2);
    }
}

/* Deltas of arbitrary pairs. */
void orc_pairs(const orc_graph* gm, const orc_graph* gf, const int32_t* mapping, const int32_t* pairs, int64_t k,
               int64_t* out) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < k; i++) {
        int32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        out[i] = (u == v) ? 0 : orc_swap_delta(gm, gf, mapping, u, v);
    }
}

/* Per-vertex metrics of calculate_node_metrics (src/graph-alignment.c:235-272)
 * for the vertices the graph lists: degree counts, the weight total of both
 * directions, that total divided by the out- and by the in-degree, and the
 * ordering rank.  Vertices the graph does not list keep zeros. */
typedef struct {
    int32_t indeg, outdeg, wsum, rank;
    double avg_in, avg_out;
} orc_vmetrics;

static orc_vmetrics* orc_metrics(const orc_graph* g, const int32_t* rank) {
    orc_vmetrics* mt = (orc_vmetrics*)calloc((size_t)g->n + 1, sizeof(orc_vmetrics));
    if (!mt) return NULL;
    for (int32_t i = 0; i < g->nnodes; i++) {
        const int32_t v = g->nodes[i];
        orc_vmetrics* x = &mt[v];
        x->outdeg = g->optr[v + 1] - g->optr[v];
        for (int32_t j = g->optr[v]; j < g->optr[v + 1]; j++) x->wsum += g->ow[j];
        x->indeg = g->iptr[v + 1] - g->iptr[v];
        for (int32_t j = g->iptr[v]; j < g->iptr[v + 1]; j++) x->wsum += g->iw[j];
        if (x->outdeg > 0) x->avg_out = (double)x->wsum / x->outdeg;
        if (x->indeg > 0) x->avg_in = (double)x->wsum / x->indeg;
        x->rank = rank[v];
    }
    return mt;
}

/* calculate_node_similarity (src/graph-alignment.c:274-284), the same
 * operations in the same order: 0.7 x (5|d in| + 5|d out| + |d avg in| +
 * |d avg out|) + 0.3 x |d rank|, negated. */
static double orc_similarity(const orc_vmetrics* a, const orc_vmetrics* b) {
    double s = 5 * fabs((double)(a->indeg - b->indeg)) + 5 * fabs((double)(a->outdeg - b->outdeg)) +
               fabs(a->avg_in - b->avg_in) + fabs(a->avg_out - b->avg_out);
    double o = fabs((double)(a->rank - b->rank));
    s = 0.7 * s + 0.3 * o;
    return -s;
}

/* The single pass of optimize_mapping in the graph-alignment variant
 * (src/graph-alignment.c:512-578): m1 and m2 run over gm's vertices in order
 * of first appearance; a swap is evaluated only when the similarity of the
 * swapped images is higher than the current one (:545-553), and a positive
 * delta is applied at once.  rank_m, rank_f: ordering ranks per vertex (0 for
 * vertices absent from the ordering).  The variant reads B weights by list
 * scan (first duplicate); this restatement uses the last, so the two agree on
 * graphs without duplicate edges.  Returns the number of accepts. */
int64_t orc_sim_sweep(const orc_graph* gm, const orc_graph* gf, int32_t* mapping, const int32_t* rank_m,
                      const int32_t* rank_f) {
    orc_vmetrics* mm = orc_metrics(gm, rank_m);
    orc_vmetrics* mf = orc_metrics(gf, rank_f);
    int64_t accepts = -1;
    if (mm && mf) {
        accepts = 0;
        for (int32_t i = 0; i < gm->nnodes; i++) {
            const int32_t m1 = gm->nodes[i];
            for (int32_t j = 0; j < gm->nnodes; j++) {
                const int32_t m2 = gm->nodes[j];
                if (m1 == m2) continue;
                const int32_t f1 = mapping[m1], f2 = mapping[m2];
                const double cur = orc_similarity(&mm[m1], &mf[f1]) + orc_similarity(&mm[m2], &mf[f2]);
                const double swp = orc_similarity(&mm[m1], &mf[f2]) + orc_similarity(&mm[m2], &mf[f1]);
                if (swp > cur && orc_swap_delta(gm, gf, mapping, m1, m2) > 0) {
                    mapping[m1] = f2;
                    mapping[m2] = f1;
                    accepts++;
                }
            }
        }
    }
    free(mm);
    free(mf);
    return accepts;
}

/* Simulated-annealing chain of simulated_annealing
 * (src/best-swap/score-lookup.c:346-408), restated with the engine's chain
 * definition: proposal s from Philox4x32-10(key, s) (bm_sa_proposal), the
 * exact delta (calculate_swap_delta, exact on graphs without self-loops),
 * acceptance delta >= 0 or u < exp(delta / T_s) with T_s of the geometric
 * schedule, immediate apply.  log_ratio = log(t_end / t0).  Returns accepts;
 * mapping and *score are updated in place. */
int64_t orc_sa_run(const orc_graph* gm, const orc_graph* gf, int32_t* mapping, uint64_t key, int64_t steps,
                   double t0, double t_end, int64_t* score) {
    const double lr = log(t_end / t0);
    int64_t accepts = 0;
    for (int64_t s = 0; s < steps; s++) {
        bm_proposal p = bm_sa_proposal(key, (uint64_t)s, gm->n);
        int64_t d = orc_swap_delta(gm, gf, mapping, p.u, p.v);
        if (bm_sa_accept(d, p.uni, bm_sa_temperature(t0, lr, (uint64_t)s, (uint64_t)steps))) {
            int32_t t = mapping[p.u];
            mapping[p.u] = mapping[p.v];
            mapping[p.v] = t;
            *score += d;
            accepts++;
        }
    }
    return accepts;
}

/* Philox4x32-10 and exp as seen from the CPU, for known-answer and
 * error-bound tests. */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { bm_philox4x32_10(ctr, key, out); }
double orc_exp(double x) { return bm_exp(x); }

/* Delta of a permutation of a vertex set: member i takes the image of member
 * perm[i].  Follows calculate_permutation_delta
 * (src/graph-alignment-permset-parallel.c:304-339) — every A entry touching
 * the set, old contribution out, new one in — except that an entry between two
 * members is counted once (from its source's out-list), where the reference
 * counts it from both ends.  Exact, including self-loops. */
int64_t orc_perm_delta(const orc_graph* gm, const orc_graph* gf, const int32_t* mapping, const int32_t* verts,
                       int32_t k, const int32_t* perm) {
    int32_t newf[16];
    for (int32_t i = 0; i < k; i++) newf[i] = mapping[verts[perm[i]]];
    int64_t delta = 0;
    for (int32_t i = 0; i < k; i++) {
        const int32_t v = verts[i];
        for (int32_t j = gm->optr[v]; j < gm->optr[v + 1]; j++) {
            const int32_t x = gm->oto[j], w = gm->ow[j];
            int32_t xm = -1;
            for (int32_t q = 0; q < k; q++)
                if (verts[q] == x) xm = q;
            const int32_t nx = xm >= 0 ? newf[xm] : mapping[x];
            delta += MIN(w, mat(gf, newf[i], nx)) - MIN(w, mat(gf, mapping[v], mapping[x]));
        }
        for (int32_t j = gm->iptr[v]; j < gm->iptr[v + 1]; j++) {
            const int32_t x = gm->ifrom[j], w = gm->iw[j];
            int32_t xm = -1;
            for (int32_t q = 0; q < k; q++)
                if (verts[q] == x) xm = q;
            if (xm >= 0) continue; /* counted from x's out-list */
            delta += MIN(w, mat(gf, mapping[x], newf[i])) - MIN(w, mat(gf, mapping[x], mapping[v]));
        }
    }
    return delta;
}

/* ------------------------------------------------ learned-proposal model */

/* FP64 replica of the engine's 24 -> 128 -> 128 -> 1 ReLU MLP (no reference
 * counterpart).  With rounding != 0 it applies the engine's roundings: inputs,
 * W1, W2 and w3 rounded to BF16 (nearest even); each hidden pre-activation
 * (sum + bias) rounded to FP32, then ReLU, then BF16; sums in FP64.  With
 * rounding == 0 everything stays FP64 (a smooth function, for checking the
 * backward formulas by finite differences).  rounding == 2 also rounds the
 * backward signals dh2 and dh1 (pre-activation gradients of the two hidden
 * layers) to BF16, as the tensor-core training kernel does (they are its MMA
 * operands); the bias gradients then sum the rounded values.  Parameters packed as W1[24][128]
 * b1 W2[128][128] b2 w3 b3.  Writes out[k] when out != NULL and, when grads
 * != NULL, the gradient of mean((out - y)^2) and *loss. */
#define ORC_IN 24
#define ORC_H 128
static double orc_bf16(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) {
        u += 0x7FFFu + ((u >> 16) & 1u);
        u &= 0xFFFF0000u;
    }
    float r;
    memcpy(&r, &u, 4);
    return (double)r;
}

int orc_mlp(const float* w, const float* x, const float* y, int64_t k, int rounding, double* out, double* grads,
            double* loss) {
    const int o_b1 = ORC_IN * ORC_H, o_w2 = o_b1 + ORC_H, o_b2 = o_w2 + ORC_H * ORC_H, o_w3 = o_b2 + ORC_H,
              o_b3 = o_w3 + ORC_H, np = o_b3 + 1;
    double* wr = (double*)malloc(sizeof(double) * (size_t)np);
    if (!wr) return -1;
    for (int i = 0; i < np; i++) wr[i] = (double)w[i];
    if (rounding) {
        for (int i = 0; i < ORC_IN * ORC_H; i++) wr[i] = orc_bf16(w[i]);
        for (int i = 0; i < ORC_H * ORC_H; i++) wr[o_w2 + i] = orc_bf16(w[o_w2 + i]);
        for (int i = 0; i < ORC_H; i++) wr[o_w3 + i] = orc_bf16(w[o_w3 + i]);
    }
    if (grads) memset(grads, 0, sizeof(double) * (size_t)np);
    double lsum = 0.0;
    for (int64_t p = 0; p < k; p++) {
        double xb[ORC_IN], h1[ORC_H], h2[ORC_H], dh2[ORC_H];
        for (int i = 0; i < ORC_IN; i++) xb[i] = rounding ? orc_bf16(x[p * ORC_IN + i]) : (double)x[p * ORC_IN + i];
        for (int j = 0; j < ORC_H; j++) {
            double a = 0.0;
            for (int i = 0; i < ORC_IN; i++) a += xb[i] * wr[i * ORC_H + j];
            const double pre = a + wr[o_b1 + j];
            if (rounding) {
                const float pf = (float)pre;
                h1[j] = orc_bf16(pf > 0.f ? pf : 0.f);
            } else {
                h1[j] = pre > 0.0 ? pre : 0.0;
            }
        }
        for (int j = 0; j < ORC_H; j++) {
            double a = 0.0;
            for (int i = 0; i < ORC_H; i++) a += h1[i] * wr[o_w2 + i * ORC_H + j];
            const double pre = a + wr[o_b2 + j];
            if (rounding) {
                const float pf = (float)pre;
                h2[j] = orc_bf16(pf > 0.f ? pf : 0.f);
            } else {
                h2[j] = pre > 0.0 ? pre : 0.0;
            }
        }
        double o = wr[o_b3];
        for (int j = 0; j < ORC_H; j++) o += h2[j] * wr[o_w3 + j];
        if (out) out[p] = o;
        if (!grads) continue;
        const double r = o - (double)y[p];
        lsum += r * r;
        const double d = 2.0 * r / (double)k;
        grads[o_b3] += d;
        for (int j = 0; j < ORC_H; j++) {
            grads[o_w3 + j] += d * h2[j];
            dh2[j] = h2[j] > 0.0 ? d * wr[o_w3 + j] : 0.0;
            if (rounding == 2) dh2[j] = orc_bf16((float)dh2[j]);
            grads[o_b2 + j] += dh2[j];
        }
        for (int i = 0; i < ORC_H; i++) {
            for (int j = 0; j < ORC_H; j++) grads[o_w2 + i * ORC_H + j] += h1[i] * dh2[j];
            if (h1[i] > 0.0) {
                double a = 0.0;
                for (int j = 0; j < ORC_H; j++) a += wr[o_w2 + i * ORC_H + j] * dh2[j];
                if (rounding == 2) a = orc_bf16((float)a);
                grads[o_b1 + i] += a;
                for (int q = 0; q < ORC_IN; q++) grads[q * ORC_H + i] += xb[q] * a;
            }
        }
    }
    if (loss) *loss = lsum / (double)(k > 0 ? k : 1);
    free(wr);
    return 0;
}
