/*
 * bm_host.h — host-side C library (libbmhost.so): CSV formats of the
 * reference tools, the seeded synthetic graph-pair generator, orderings and
 * the greedy-similarity initial matching.  No CUDA here.
 */
#ifndef BM_HOST_H
#define BM_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* An edge list with ids 1..n (malloc'd arrays, freed by bm_edges_free). */
typedef struct bm_edges {
    int32_t n;
    int64_t m;
    int32_t* src;
    int32_t* dst;
    int32_t* w;
} bm_edges;

void bm_edges_free(bm_edges* e);

/* ------------------------------------------------------------- CSV formats */

/* Edge CSV: one header line, then "from,to,weight" lines
 * (load_graph_from_csv, src/graph-alignment-optimized.c:635-679).  Malformed
 * lines are counted in *malformed and skipped, like the reference.  e->n is
 * the largest id seen.  Returns 0 on success, -1 if the file cannot be read. */
int bm_read_graph_csv(const char* path, bm_edges* e, int64_t* malformed);
int bm_write_graph_csv(const char* path, const bm_edges* e);

/* Ordering CSV "Node ID,Order" (read_ordering, src/graph-alignment-optimized.c:216-239).
 * order must hold n+1 ints; ids outside 1..n are ignored. */
int bm_read_ordering(const char* path, int32_t n, int32_t* order);
int bm_write_ordering(const char* path, int32_t n, const int32_t* order);

/* Mapping CSV: header, then "m<id>,f<id>" or "<id>,<id>" lines
 * (load_benchmark_mapping, src/graph-alignment-optimized.c:428-475).
 * pi must hold n+1 ints (zeroed first); *count = lines parsed; *max_id = the
 * largest id seen on either side.  Ids above n are counted but not stored. */
int bm_read_mapping(const char* path, int32_t n, int32_t* pi, int64_t* count, int32_t* max_id);
/* Writes "Male Node ID,Female Node ID" then "m%d,f%d" for pi(i) != 0
 * (write_mapping, src/graph-alignment-optimized.c:410-425).  Atomic: the file
 * is written under a temporary name and renamed. */
int bm_write_mapping(const char* path, int32_t n, const int32_t* pi);

/* Every (male, female) id pair of a mapping file in file order (header
 * skipped, malformed lines skipped), as two malloc'd arrays the caller frees.
 * For checkers that must see duplicate assignments (verify-mapping,
 * src/verify-mapping.c:113-232). */
int bm_read_mapping_pairs(const char* path, int32_t** male, int32_t** female, int64_t* count);

/* Largest id in a mapping file without storing it (to size arrays). */
int bm_scan_mapping_max_id(const char* path, int32_t* max_id);

/* ------------------------------------------------------------ generator */

typedef struct bm_gen_params {
    int32_t n;
    int64_t m_target;       /* directed edges of A (before noise) */
    int32_t degree_model;   /* 0: out-degree power law, uniform targets; 1: joint in/out Chung-Lu */
    double alpha;           /* power-law exponent */
    int32_t max_degree;     /* cap on a vertex's expected degree */
    int32_t weight_model;   /* 0: geometric(p) + tail; 1: 80% uniform 1..5 + tail */
    double geo_p;           /* geometric parameter (weight_model 0) */
    double tail_frac;       /* fraction of heavy-tail weights */
    int32_t tail_max;       /* largest tail weight */
    double del_frac;        /* B: fraction of A's edges deleted */
    double add_frac;        /* B: fraction of new edges added (relative to m) */
    int32_t jitter;         /* B: weights jittered by a uniform integer in [-jitter, jitter], clamped >= 1 */
    double shuffle_frac;    /* initial pi: fraction of vertices reshuffled from the truth */
    int32_t init_mode;      /* 0: shuffled truth; 1: greedy similarity (bm_greedy_match) */
    uint64_t seed;
} bm_gen_params;

/* Defaults of the named workloads: 1 = n 2,000 / ~40k edges (CPU-runnable);
 * 2 = n 18,524 / ~3M edges (full scale); 3 = one pair of the batched-chain
 * workload (n and seed given by the caller); 4 and 5 = the full-scale pair.
 * Returns -1 for an unknown config. */
int bm_gen_defaults(int config, bm_gen_params* p);

/* Generate A, B, the planted truth pi_true (A vertex -> B vertex) and the
 * initial matching pi_init (both n+1 ints, 1-indexed).  No self-loops, no
 * duplicate edges, weights in 1..32767.  Deterministic in p->seed. */
int bm_gen_pair(const bm_gen_params* p, bm_edges* A, bm_edges* B,
                int32_t* pi_true, int32_t* pi_init);

/* Ordering ranks (n+1 ints, 1..n) by descending weighted degree, ties by id:
 * the "Node ID,Order" file the reference reads (read_ordering). */
void bm_ordering_by_weighted_degree(const bm_edges* g, int32_t* order);
/* Row visiting order (n ints) sorted by ascending ordering rank, ties by id. */
void bm_rows_from_ordering(int32_t n, const int32_t* order, int32_t* rows);

/* Greedy similarity matching (src/greedy-match.c:213-293, 450-530): features
 * in/out degree and distinct 2-hop reach in both directions; vertices of both
 * graphs sorted by descending feature sum (ties by id); each A vertex in turn
 * takes the unmatched B vertex at least L1 feature distance (first in sorted
 * order on ties).  pi: n+1 ints.  Uses OpenMP threads. */
int bm_greedy_match(const bm_edges* A, const bm_edges* B, int32_t* pi);

/* Host score of pi (B looked up through a hash; same semantics as the device
 * score).  Used by the CLI's final report. */
int64_t bm_host_score(const bm_edges* A, const bm_edges* B, const int32_t* pi);

/* Bijection check of pi on 1..n: 0 if valid, else the first bad id (> 0). */
int32_t bm_check_bijection(int32_t n, const int32_t* pi);

/* The deterministic selection of a sharded search (the same rule as
 * bm_select_independent in bm_cuda.h, on the host): among candidates with
 * delta > 0, in descending delta then ascending index, take a swap when
 * neither endpoint lies in the closed A neighbourhood of an endpoint already
 * taken.  chosen receives candidate indices, *nchosen their count. */
int bm_select_independent_host(const bm_edges* A, const int32_t* pairs, const int64_t* deltas, int32_t count,
                               int32_t* chosen, int32_t* nchosen);

/* Inputs of the similarity-filtered pass (bm_sweep_similarity in
 * bm_cuda.h), as the reference's graph-alignment variant builds them:
 * bm_first_appearance writes the vertices in order of first appearance in
 * the edge list, the source then the target of each edge (its g->nodes,
 * add_node from add_edge, src/graph-alignment.c:159-200; nodes needs n
 * entries); bm_node_metrics writes calculate_node_metrics (:235-272) for the
 * listed vertices, five doubles per vertex id 0..n: in-degree, out-degree,
 * the weight total of both directions over the in-degree and over the
 * out-degree, and rank[v] (the ordering rank; NULL gives 0); unlisted
 * vertices get zeros.  Both return 0, or -1 on a bad id or no memory. */
int bm_first_appearance(const bm_edges* e, int32_t* nodes, int32_t* count);
int bm_node_metrics(const bm_edges* e, const int32_t* rank, double* metrics);

/* SplitMix64 step and a uniform double in [0,1) — the generator's RNG. */
uint64_t bm_splitmix64(uint64_t* state);

#ifdef __cplusplus
}
#endif

#endif /* BM_HOST_H */
