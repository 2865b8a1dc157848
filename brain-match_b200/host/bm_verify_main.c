/*
 * bm-verify — the checks of verify-mapping (src/verify-mapping.c:301-342):
 *
 *   bm-verify <initial_mapping.csv> <test_mapping.csv>
 *
 * Loads both mapping files (header line, then "m<id>,f<id>" or "<id>,<id>"),
 * reports whether each is a valid one-to-one assignment (no female id given to
 * two males, no male id given two females: verify_mapping, :199-232) and, when
 * both are valid, lists the males whose assignment differs, the males present
 * in only one file, the summary counts and the change histogram over male id
 * deciles (analyze_differences, :235-299).  Exit 0 after the report, 1 on a
 * usage or load error, as the reference.
 *
 * Ids are accepted in 1..131071 (the engine's limit); the reference accepts
 * 1..18524 (its NUM_NODES), so on the VNC-sized data both accept the same ids.
 * The histogram's deciles are taken over 18,524 as in the reference, or over
 * the largest id seen when that is larger.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bm_host.h"

#define MAX_ID 131071
#define REF_NODES 18524  /* NUM_NODES of the reference tools */

typedef struct {
    int32_t n;            /* largest id slot allocated */
    int32_t* m2f;         /* male -> female (last line wins) */
    int32_t* f2m;         /* female -> male (last line wins) */
    unsigned char* mused;
    unsigned char* fused;
    int64_t count;        /* lines with valid ids */
} mapping_t;

static void free_mapping(mapping_t* m) {
    free(m->m2f); free(m->f2m); free(m->mused); free(m->fused);
}

static int load(const char* path, mapping_t* m) {
    int32_t *a = NULL, *b = NULL;
    int64_t cnt = 0;
    if (bm_read_mapping_pairs(path, &a, &b, &cnt) != 0) {
        fprintf(stderr, "Error opening file: %s\n", path);
        return -1;
    }
    memset(m, 0, sizeof(*m));
    m->n = MAX_ID;
    m->m2f = (int32_t*)calloc((size_t)MAX_ID + 1, sizeof(int32_t));
    m->f2m = (int32_t*)calloc((size_t)MAX_ID + 1, sizeof(int32_t));
    m->mused = (unsigned char*)calloc((size_t)MAX_ID + 1, 1);
    m->fused = (unsigned char*)calloc((size_t)MAX_ID + 1, 1);
    if (!m->m2f || !m->f2m || !m->mused || !m->fused) { free(a); free(b); free_mapping(m); return -1; }
    for (int64_t i = 0; i < cnt; i++) {
        if (a[i] <= 0 || a[i] > MAX_ID || b[i] <= 0 || b[i] > MAX_ID) {
            printf("Warning: Invalid vertex IDs on line %lld: %d,%d\n", (long long)i + 1, a[i], b[i]);
            continue;
        }
        m->m2f[a[i]] = b[i];
        m->f2m[b[i]] = a[i];
        m->mused[a[i]] = 1;
        m->fused[b[i]] = 1;
        m->count++;
    }
    free(a);
    free(b);
    printf("Successfully loaded %lld mappings from %s\n", (long long)m->count, path);
    return 0;
}

static int verify(const mapping_t* m) {
    int valid = 1;
    int32_t* cnt = (int32_t*)calloc((size_t)MAX_ID + 1, sizeof(int32_t));
    if (!cnt) return 0;
    for (int32_t i = 1; i <= MAX_ID; i++)
        if (m->mused[i] && ++cnt[m->m2f[i]] > 1) {
            printf("ERROR: Female vertex %d (f%d) is assigned to multiple male vertices\n", m->m2f[i], m->m2f[i]);
            valid = 0;
        }
    memset(cnt, 0, sizeof(int32_t) * ((size_t)MAX_ID + 1));
    for (int32_t i = 1; i <= MAX_ID; i++)
        if (m->fused[i] && ++cnt[m->f2m[i]] > 1) {
            printf("ERROR: Male vertex %d (m%d) is assigned to multiple female vertices\n", m->f2m[i], m->f2m[i]);
            valid = 0;
        }
    free(cnt);
    return valid;
}

static void differences(const mapping_t* a, const mapping_t* b) {
    printf("\nAnalyzing differences between mappings:\n");
    printf("----------------------------------------\n");
    int32_t top = 1;
    for (int32_t i = 1; i <= MAX_ID; i++)
        if (a->mused[i] || b->mused[i]) top = i;
    int64_t diff = 0, miss_init = 0, miss_test = 0;
    for (int32_t i = 1; i <= top; i++) {
        if (a->mused[i] && !b->mused[i]) {
            printf("Male vertex %d (m%d) is in initial but missing from test mapping\n", i, i);
            miss_test++;
        } else if (!a->mused[i] && b->mused[i]) {
            printf("Male vertex %d (m%d) is in test but missing from initial mapping\n", i, i);
            miss_init++;
        } else if (a->mused[i] && b->mused[i] && a->m2f[i] != b->m2f[i]) {
            printf("Difference: %d (m%d) maps to %d (f%d) in initial, %d (f%d) in test\n", i, i, a->m2f[i], a->m2f[i],
                   b->m2f[i], b->m2f[i]);
            diff++;
        }
    }
    printf("\nSummary Statistics:\n");
    printf("------------------\n");
    printf("Initial mapping count: %lld\n", (long long)a->count);
    printf("Test mapping count: %lld\n", (long long)b->count);
    printf("Number of differences: %lld\n", (long long)diff);
    printf("Vertices in initial but missing from test: %lld\n", (long long)miss_test);
    printf("Vertices in test but missing from initial: %lld\n", (long long)miss_init);
    if (a->count > 0) printf("Percentage changed: %.2f%%\n", (double)diff / (double)a->count * 100.0);
    if (diff > 0) {
        printf("\nChange Distribution:\n");
        printf("-------------------\n");
        int64_t ranges[10] = {0};
        for (int32_t i = 1; i <= top; i++)
            if (a->mused[i] && b->mused[i] && a->m2f[i] != b->m2f[i]) {
                const int32_t denom = top > REF_NODES ? top : REF_NODES;
                int r = (int)(((int64_t)i * 10) / denom);
                if (r >= 10) r = 9;
                ranges[r]++;
            }
        for (int r = 0; r < 10; r++) {
            printf("%3d-%3d%%: ", r * 10, (r + 1) * 10);
            for (int64_t j = 0; j < ranges[r] * 50 / diff; j++) putchar('*');
            printf(" (%lld)\n", (long long)ranges[r]);
        }
    }
}

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "Usage: %s <initial_mapping.csv> <test_mapping.csv>\n", argv[0]);
        return 1;
    }
    mapping_t init, test;
    printf("Loading initial mapping from %s\n", argv[1]);
    if (load(argv[1], &init) != 0) {
        fprintf(stderr, "Failed to load initial mapping\n");
        return 1;
    }
    printf("Loading test mapping from %s\n", argv[2]);
    if (load(argv[2], &test) != 0) {
        fprintf(stderr, "Failed to load test mapping\n");
        free_mapping(&init);
        return 1;
    }
    printf("\nVerifying initial mapping...\n");
    const int vi = verify(&init);
    printf("Initial mapping is %s\n", vi ? "valid" : "invalid");
    printf("\nVerifying test mapping...\n");
    const int vt = verify(&test);
    printf("Test mapping is %s\n", vt ? "valid" : "invalid");
    if (vi && vt) differences(&init, &test);
    free_mapping(&init);
    free_mapping(&test);
    return 0;
}
