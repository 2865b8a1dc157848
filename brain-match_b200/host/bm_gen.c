/*
 * bm_gen.c — seeded synthetic graph pairs standing in for the VNC male and
 * female connectomes, which the reference reads from data/gm.csv and
 * data/gf.csv (absent from the reference repository).
 *
 * A is drawn from a power-law degree model; B is A relabelled by a random
 * permutation sigma (the planted truth), with a fraction of edges deleted, new
 * edges added and weights jittered.  No self-loops, no duplicate edges,
 * weights in 1..32767, so the reference's swap delta is exact on these
 * inputs.  Every random draw comes from SplitMix64 (Steele, Lea & Flood,
 * OOPSLA 2014) seeded by the caller, so a seed fixes the pair bit for bit.
 */
#include "bm_host.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

uint64_t bm_splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double urand(uint64_t* s) { return (double)(bm_splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

/* uniform integer in [0, k) */
static uint32_t urange(uint64_t* s, uint32_t k) {
    return (uint32_t)(((bm_splitmix64(s) >> 32) * (uint64_t)k) >> 32);
}

/* ------------------------------------------------------------- edge set */

typedef struct {
    uint64_t* keys;
    uint64_t mask;
    int64_t count;
} keyset;

static uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

static int keyset_init(keyset* s, int64_t expected) {
    uint64_t cap = 16;
    while (cap < (uint64_t)(expected * 2 + 16)) cap <<= 1;
    s->keys = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    if (!s->keys) return -1;
    memset(s->keys, 0xff, sizeof(uint64_t) * cap);
    s->mask = cap - 1;
    s->count = 0;
    return 0;
}

/* returns 1 if inserted, 0 if present */
static int keyset_insert(keyset* s, uint64_t key) {
    uint64_t h = mix64(key) & s->mask;
    for (;;) {
        uint64_t k = s->keys[h];
        if (k == key) return 0;
        if (k == ~0ull) { s->keys[h] = key; s->count++; return 1; }
        h = (h + 1) & s->mask;
    }
}


static void keyset_free(keyset* s) { free(s->keys); s->keys = NULL; }

static uint64_t ekey(int32_t a, int32_t b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

/* ------------------------------------------------------------- weights */

static int32_t draw_weight(const bm_gen_params* p, uint64_t* rng) {
    double u = urand(rng);
    if (u < p->tail_frac) {
        /* log-uniform heavy tail */
        double lo = p->weight_model == 0 ? 1.0 : 6.0;
        double v = lo * exp(urand(rng) * log((double)p->tail_max / lo));
        int32_t w = (int32_t)v;
        if (w < 1) w = 1;
        if (w > p->tail_max) w = p->tail_max;
        return w;
    }
    if (p->weight_model == 0) {
        double g = urand(rng);
        if (g <= 0.0) g = 1e-300;
        int32_t w = 1 + (int32_t)floor(log(g) / log(1.0 - p->geo_p));
        if (w < 1) w = 1;
        if (w > 32767) w = 32767;
        return w;
    }
    return 1 + (int32_t)urange(rng, 5);
}

/* ----------------------------------------------------------- edge buffer */

typedef struct {
    int32_t* src;
    int32_t* dst;
    int32_t* w;
    int64_t m, cap;
} ebuf;

static int ebuf_push(ebuf* b, int32_t s, int32_t d, int32_t w) {
    if (b->m == b->cap) {
        int64_t nc = b->cap ? b->cap * 2 : 1024;
        int32_t* ns = (int32_t*)realloc(b->src, sizeof(int32_t) * (size_t)nc);
        if (!ns) return -1;
        b->src = ns;
        int32_t* nd = (int32_t*)realloc(b->dst, sizeof(int32_t) * (size_t)nc);
        if (!nd) return -1;
        b->dst = nd;
        int32_t* nw = (int32_t*)realloc(b->w, sizeof(int32_t) * (size_t)nc);
        if (!nw) return -1;
        b->w = nw;
        b->cap = nc;
    }
    b->src[b->m] = s;
    b->dst[b->m] = d;
    b->w[b->m] = w;
    b->m++;
    return 0;
}

/* inverse-CDF draw from cumulative weights cum[0..n-1] (cum[n-1] = total) */
static int32_t draw_cdf(const double* cum, int32_t n, uint64_t* rng) {
    double t = urand(rng) * cum[n - 1];
    int32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (cum[mid] > t) hi = mid; else lo = mid + 1;
    }
    return lo;
}

static void shuffle_i32(int32_t* a, int32_t k, uint64_t* rng) {
    for (int32_t i = k - 1; i > 0; i--) {
        int32_t j = (int32_t)urange(rng, (uint32_t)(i + 1));
        int32_t t = a[i]; a[i] = a[j]; a[j] = t;
    }
}

int bm_gen_defaults(int config, bm_gen_params* p) {
    memset(p, 0, sizeof(*p));
    switch (config) {
    case 1:
        p->n = 2000; p->m_target = 40000; p->degree_model = 0; p->alpha = 2.1; p->max_degree = 500;
        p->weight_model = 0; p->geo_p = 0.4; p->tail_frac = 0.01; p->tail_max = 500;
        p->del_frac = 0.10; p->add_frac = 0.10; p->jitter = 1;
        p->shuffle_frac = 0.30; p->init_mode = 0; p->seed = 1;
        return 0;
    case 2: case 4: case 5:
        p->n = 18524; p->m_target = 3000000; p->degree_model = 1; p->alpha = 2.1; p->max_degree = 8000;
        p->weight_model = 1; p->geo_p = 0.4; p->tail_frac = 0.20; p->tail_max = 3000;
        p->del_frac = 0.05; p->add_frac = 0.05; p->jitter = 1;
        p->shuffle_frac = 0.30; p->init_mode = 1; p->seed = (uint64_t)config;
        return 0;
    case 3:
        p->n = 2000; p->m_target = 160000; p->degree_model = 1; p->alpha = 2.1; p->max_degree = 2000;
        p->weight_model = 1; p->geo_p = 0.4; p->tail_frac = 0.20; p->tail_max = 3000;
        p->del_frac = 0.05; p->add_frac = 0.05; p->jitter = 1;
        p->shuffle_frac = 0.30; p->init_mode = 0; p->seed = 3;
        return 0;
    default:
        return -1;
    }
}

/* Expected degrees theta_i (sum = m) of the Chung-Lu model: a power law
 * theta_r ~ (r + i0)^(-1/(alpha-1)) over ranks r, with i0 chosen so the largest
 * is max_degree, then assigned to vertices by a random permutation. */
static int chung_lu_theta(const bm_gen_params* p, double* theta, uint64_t* rng) {
    int32_t n = p->n;
    double gam = 1.0 / (p->alpha - 1.0);
    double mean = (double)p->m_target / n;
    double target = (double)p->max_degree / mean;
    if (target < 1.0) target = 1.0;
    double lo = 1e-6, hi = (double)n * 4;
    for (int it = 0; it < 200; it++) {
        double i0 = sqrt(lo * hi);
        double s = 0;
        for (int32_t r = 0; r < n; r++) s += pow(r + i0, -gam);
        double ratio = pow(i0, -gam) / (s / n);
        if (ratio > target) lo = i0; else hi = i0;
    }
    double i0 = sqrt(lo * hi);
    double s = 0;
    for (int32_t r = 0; r < n; r++) s += pow(r + i0, -gam);
    int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    if (!perm) return -1;
    for (int32_t i = 0; i < n; i++) perm[i] = i;
    shuffle_i32(perm, n, rng);
    for (int32_t r = 0; r < n; r++) theta[perm[r]] = (double)p->m_target * pow(r + i0, -gam) / s;
    free(perm);
    return 0;
}

/* Out-degrees of the model-0 graph: Pareto draws floor(xm * u^(-1/(alpha-1))),
 * at least 1 and at most max_degree, with xm bisected so the sum is m_target. */
static int pareto_outdeg(const bm_gen_params* p, int32_t* deg, uint64_t* rng) {
    int32_t n = p->n;
    double* u = (double*)malloc(sizeof(double) * (size_t)n);
    if (!u) return -1;
    double gam = 1.0 / (p->alpha - 1.0);
    int32_t cap = p->max_degree < n - 1 ? p->max_degree : n - 1;
    for (int32_t i = 0; i < n; i++) {
        double v = urand(rng);
        if (v <= 0) v = 1e-12;
        u[i] = pow(v, -gam);
    }
    double lo = 1e-3, hi = (double)cap;
    for (int it = 0; it < 100; it++) {
        double xm = 0.5 * (lo + hi);
        int64_t s = 0;
        for (int32_t i = 0; i < n; i++) {
            double d = floor(xm * u[i]);
            if (d < 1) d = 1;
            if (d > cap) d = cap;
            s += (int64_t)d;
        }
        if (s > p->m_target) hi = xm; else lo = xm;
    }
    for (int32_t i = 0; i < n; i++) {
        double d = floor(lo * u[i]);
        if (d < 1) d = 1;
        if (d > cap) d = cap;
        deg[i] = (int32_t)d;
    }
    free(u);
    return 0;
}

int bm_gen_pair(const bm_gen_params* p, bm_edges* A, bm_edges* B, int32_t* pi_true, int32_t* pi_init) {
    int32_t n = p->n;
    if (n < 2 || p->m_target < 1) return -1;
    uint64_t rng = p->seed * 0x2545F4914F6CDD1Dull + 0x1234567ull;
    memset(A, 0, sizeof(*A));
    memset(B, 0, sizeof(*B));
    ebuf ea = {0}, eb = {0};
    keyset ka, kb;
    int64_t mmax = p->m_target + (int64_t)(p->add_frac * (double)p->m_target) + 16;
    if (keyset_init(&ka, mmax) || keyset_init(&kb, mmax)) return -1;
    double* cum_src = (double*)malloc(sizeof(double) * (size_t)n);
    double* cum_dst = (double*)malloc(sizeof(double) * (size_t)n);
    if (!cum_src || !cum_dst) return -1;

    /* ---- A */
    if (p->degree_model == 0) {
        int32_t* deg = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        if (!deg || pareto_outdeg(p, deg, &rng)) return -1;
        for (int32_t x = 0; x < n; x++) {
            int32_t got = 0;
            int64_t tries = 0;
            while (got < deg[x] && tries < (int64_t)deg[x] * 50 + 100) {
                tries++;
                int32_t y = (int32_t)urange(&rng, (uint32_t)n);
                if (y == x) continue;
                if (!keyset_insert(&ka, ekey(x + 1, y + 1))) continue;
                if (ebuf_push(&ea, x + 1, y + 1, draw_weight(p, &rng))) return -1;
                got++;
            }
        }
        double c = 0;
        for (int32_t x = 0; x < n; x++) { c += deg[x]; cum_src[x] = c; cum_dst[x] = (double)(x + 1); }
        free(deg);
    } else {
        double* theta = (double*)malloc(sizeof(double) * (size_t)n);
        if (!theta || chung_lu_theta(p, theta, &rng)) return -1;
        double c = 0;
        for (int32_t x = 0; x < n; x++) { c += theta[x]; cum_src[x] = c; cum_dst[x] = c; }
        free(theta);
        int64_t tries = 0, max_tries = p->m_target * 50;
        while (ea.m < p->m_target && tries < max_tries) {
            tries++;
            int32_t x = draw_cdf(cum_src, n, &rng);
            int32_t y = draw_cdf(cum_dst, n, &rng);
            if (x == y) continue;
            if (!keyset_insert(&ka, ekey(x + 1, y + 1))) continue;
            if (ebuf_push(&ea, x + 1, y + 1, draw_weight(p, &rng))) return -1;
        }
    }

    /* ---- planted permutation sigma: A vertex x -> B vertex sigma(x) */
    int32_t* sigma = pi_true;
    sigma[0] = 0;
    for (int32_t i = 1; i <= n; i++) sigma[i] = i;
    shuffle_i32(sigma + 1, n, &rng);

    /* ---- B = sigma(A) minus deletions, jittered */
    for (int64_t e = 0; e < ea.m; e++) {
        if (urand(&rng) < p->del_frac) continue;
        int32_t w = ea.w[e];
        if (p->jitter > 0) {
            w += (int32_t)urange(&rng, (uint32_t)(2 * p->jitter + 1)) - p->jitter;
            if (w < 1) w = 1;
            if (w > 32767) w = 32767;
        }
        int32_t s = sigma[ea.src[e]], d = sigma[ea.dst[e]];
        keyset_insert(&kb, ekey(s, d));
        if (ebuf_push(&eb, s, d, w)) return -1;
    }
    /* ---- added edges, endpoints drawn like A's (through sigma) */
    int64_t add = (int64_t)(p->add_frac * (double)ea.m);
    int64_t added = 0, tries = 0;
    while (added < add && tries < add * 50 + 100) {
        tries++;
        int32_t x = draw_cdf(cum_src, n, &rng) + 1;
        int32_t y = draw_cdf(cum_dst, n, &rng) + 1;
        if (x == y) continue;
        int32_t s = sigma[x], d = sigma[y];
        if (!keyset_insert(&kb, ekey(s, d))) continue;
        if (ebuf_push(&eb, s, d, draw_weight(p, &rng))) return -1;
        added++;
    }
    keyset_free(&ka);
    keyset_free(&kb);
    free(cum_src);
    free(cum_dst);

    A->n = n; A->m = ea.m; A->src = ea.src; A->dst = ea.dst; A->w = ea.w;
    B->n = n; B->m = eb.m; B->src = eb.src; B->dst = eb.dst; B->w = eb.w;

    /* ---- initial matching */
    if (p->init_mode == 1) {
        if (bm_greedy_match(A, B, pi_init)) return -1;
    } else {
        memcpy(pi_init, sigma, sizeof(int32_t) * (size_t)(n + 1));
        int32_t k = (int32_t)llround(p->shuffle_frac * n);
        int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
        int32_t* img = (int32_t*)malloc(sizeof(int32_t) * (size_t)(k > 0 ? k : 1));
        if (!idx || !img) return -1;
        for (int32_t i = 0; i < n; i++) idx[i] = i + 1;
        /* partial Fisher-Yates: the first k entries are a uniform k-subset */
        for (int32_t i = 0; i < k; i++) {
            int32_t j = i + (int32_t)urange(&rng, (uint32_t)(n - i));
            int32_t t = idx[i]; idx[i] = idx[j]; idx[j] = t;
        }
        for (int32_t i = 0; i < k; i++) img[i] = sigma[idx[i]];
        shuffle_i32(img, k, &rng);
        for (int32_t i = 0; i < k; i++) pi_init[idx[i]] = img[i];
        free(idx);
        free(img);
    }
    pi_init[0] = 0;
    return 0;
}

/* ------------------------------------------------------------ orderings */

typedef struct { int64_t key; int32_t id; } kid;

static int cmp_kid_desc(const void* a, const void* b) {
    const kid* x = (const kid*)a;
    const kid* y = (const kid*)b;
    if (x->key != y->key) return x->key > y->key ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

static int cmp_kid_asc(const void* a, const void* b) {
    const kid* x = (const kid*)a;
    const kid* y = (const kid*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

void bm_ordering_by_weighted_degree(const bm_edges* g, int32_t* order) {
    int32_t n = g->n;
    kid* k = (kid*)calloc((size_t)n + 1, sizeof(kid));
    for (int32_t i = 0; i < n; i++) k[i].id = i + 1;
    for (int64_t e = 0; e < g->m; e++) {
        if (g->src[e] >= 1 && g->src[e] <= n) k[g->src[e] - 1].key += g->w[e];
        if (g->dst[e] >= 1 && g->dst[e] <= n) k[g->dst[e] - 1].key += g->w[e];
    }
    qsort(k, (size_t)n, sizeof(kid), cmp_kid_desc);
    order[0] = 0;
    for (int32_t r = 0; r < n; r++) order[k[r].id] = r + 1;
    free(k);
}

void bm_rows_from_ordering(int32_t n, const int32_t* order, int32_t* rows) {
    kid* k = (kid*)malloc(sizeof(kid) * (size_t)n);
    for (int32_t i = 0; i < n; i++) { k[i].id = i + 1; k[i].key = order[i + 1]; }
    qsort(k, (size_t)n, sizeof(kid), cmp_kid_asc);
    for (int32_t i = 0; i < n; i++) rows[i] = k[i].id;
    free(k);
}
