/*
 * bm_io.c — the CSV formats of the reference tools, read with a single
 * buffered pass instead of fgets+sscanf per line, with the same acceptance
 * rules:
 *   edge CSV     load_graph_from_csv    src/graph-alignment-optimized.c:635-679
 *   ordering CSV read_ordering          src/graph-alignment-optimized.c:216-239
 *   mapping CSV  load_benchmark_mapping src/graph-alignment-optimized.c:428-475
 *                write_mapping          src/graph-alignment-optimized.c:410-425
 */
#define _GNU_SOURCE
#include "bm_host.h"

#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

void bm_edges_free(bm_edges* e) {
    if (!e) return;
    free(e->src);
    free(e->dst);
    free(e->w);
    e->src = e->dst = e->w = NULL;
    e->m = 0;
}

/* Whole file into memory, NUL-terminated. */
static char* slurp(const char* path, size_t* len) {
    FILE* f = fopen(path, "rb");
    if (!f) return NULL;
    if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return NULL; }
    long sz = ftell(f);
    if (sz < 0) { fclose(f); return NULL; }
    rewind(f);
    char* buf = (char*)malloc((size_t)sz + 1);
    if (!buf) { fclose(f); return NULL; }
    size_t got = fread(buf, 1, (size_t)sz, f);
    fclose(f);
    buf[got] = '\0';
    if (len) *len = got;
    return buf;
}

/* scanf-style "%d": optional leading whitespace, optional sign, >= 1 digit.
 * Returns the position after the number, or NULL. */
static const char* scan_int(const char* p, const char* end, long long* out) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) p++;
    int neg = 0;
    if (p < end && (*p == '-' || *p == '+')) { neg = (*p == '-'); p++; }
    if (p >= end || !isdigit((unsigned char)*p)) return NULL;
    long long v = 0;
    while (p < end && isdigit((unsigned char)*p)) {
        if (v < 100000000000LL) v = v * 10 + (*p - '0');
        p++;
    }
    *out = neg ? -v : v;
    return p;
}

static const char* next_line(const char* p, const char* end) {
    const char* q = memchr(p, '\n', (size_t)(end - p));
    return q ? q + 1 : end;
}

int bm_read_graph_csv(const char* path, bm_edges* e, int64_t* malformed) {
    memset(e, 0, sizeof(*e));
    if (malformed) *malformed = 0;
    size_t len = 0;
    char* buf = slurp(path, &len);
    if (!buf) return -1;
    const char* end = buf + len;
    /* count lines for capacity */
    int64_t lines = 0;
    for (const char* p = buf; p < end; p = next_line(p, end)) lines++;
    int64_t cap = lines > 0 ? lines : 1;
    e->src = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    e->dst = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    e->w = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    if (!e->src || !e->dst || !e->w) { free(buf); bm_edges_free(e); return -1; }
    const char* p = next_line(buf, end); /* skip the header line */
    int32_t maxid = 0;
    int64_t bad = 0;
    while (p < end) {
        const char* le = next_line(p, end);
        long long a, b, c;
        const char* q = scan_int(p, le, &a);
        if (q && q < le && *q == ',') q = scan_int(q + 1, le, &b); else q = NULL;
        if (q && q < le && *q == ',') q = scan_int(q + 1, le, &c); else q = NULL;
        if (q && a >= 0 && b >= 0 && a <= 0x7fffffff && b <= 0x7fffffff &&
            c >= -0x7fffffffLL && c <= 0x7fffffffLL) {
            e->src[e->m] = (int32_t)a;
            e->dst[e->m] = (int32_t)b;
            e->w[e->m] = (int32_t)c;
            if (a > maxid) maxid = (int32_t)a;
            if (b > maxid) maxid = (int32_t)b;
            e->m++;
        } else {
            bad++;
        }
        p = le;
    }
    e->n = maxid;
    if (malformed) *malformed = bad;
    free(buf);
    return 0;
}

int bm_write_graph_csv(const char* path, const bm_edges* e) {
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    static char iobuf[1 << 20];
    setvbuf(f, iobuf, _IOFBF, sizeof iobuf);
    fprintf(f, "from,to,weight\n");
    for (int64_t i = 0; i < e->m; i++) fprintf(f, "%d,%d,%d\n", e->src[i], e->dst[i], e->w[i]);
    return fclose(f) == 0 ? 0 : -1;
}

int bm_read_ordering(const char* path, int32_t n, int32_t* order) {
    size_t len = 0;
    char* buf = slurp(path, &len);
    if (!buf) return -1;
    memset(order, 0, sizeof(int32_t) * (size_t)(n + 1));
    const char* end = buf + len;
    const char* p = next_line(buf, end);
    while (p < end) {
        const char* le = next_line(p, end);
        long long a, b;
        const char* q = scan_int(p, le, &a);
        if (q && q < le && *q == ',') q = scan_int(q + 1, le, &b); else q = NULL;
        if (q && a >= 1 && a <= n) order[a] = (int32_t)b;
        p = le;
    }
    free(buf);
    return 0;
}

int bm_write_ordering(const char* path, int32_t n, const int32_t* order) {
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    fprintf(f, "Node ID,Order\n");
    for (int32_t i = 1; i <= n; i++) fprintf(f, "%d,%d\n", i, order[i]);
    return fclose(f) == 0 ? 0 : -1;
}

/* One mapping line: "%d,%d" first, else the "m<id>,f<id>" form with the
 * prefixes stripped and the rest read like atoi. */
static int parse_mapping_line(const char* p, const char* le, long long* a, long long* b) {
    const char* q = scan_int(p, le, a);
    if (q && q < le && *q == ',') {
        q = scan_int(q + 1, le, b);
        if (q) return 1;
    }
    const char* comma = memchr(p, ',', (size_t)(le - p));
    if (!comma || comma == p) return 0;
    const char* s1 = p;
    while (s1 < comma && isspace((unsigned char)*s1)) s1++;
    if (s1 < comma && *s1 == 'm') s1++;
    const char* s2 = comma + 1;
    while (s2 < le && isspace((unsigned char)*s2)) s2++;
    if (s2 >= le) return 0;
    if (*s2 == 'f') s2++;
    long long x = 0, y = 0;
    if (!scan_int(s1, comma, &x)) x = 0;
    if (!scan_int(s2, le, &y)) y = 0;
    *a = x;
    *b = y;
    return 1;
}

int bm_scan_mapping_max_id(const char* path, int32_t* max_id) {
    size_t len = 0;
    char* buf = slurp(path, &len);
    if (!buf) return -1;
    const char* end = buf + len;
    const char* p = next_line(buf, end);
    long long mx = 0;
    while (p < end) {
        const char* le = next_line(p, end);
        long long a, b;
        if (parse_mapping_line(p, le, &a, &b)) {
            if (a > mx) mx = a;
            if (b > mx) mx = b;
        }
        p = le;
    }
    free(buf);
    *max_id = (int32_t)(mx > 0x7fffffff ? 0x7fffffff : mx);
    return 0;
}

int bm_read_mapping(const char* path, int32_t n, int32_t* pi, int64_t* count, int32_t* max_id) {
    size_t len = 0;
    char* buf = slurp(path, &len);
    if (!buf) return -1;
    memset(pi, 0, sizeof(int32_t) * (size_t)(n + 1));
    const char* end = buf + len;
    const char* p = next_line(buf, end);
    int64_t cnt = 0;
    long long mx = 0;
    while (p < end) {
        const char* le = next_line(p, end);
        long long a, b;
        if (parse_mapping_line(p, le, &a, &b)) {
            cnt++;
            if (a > mx) mx = a;
            if (b > mx) mx = b;
            if (a >= 1 && a <= n && b >= 0 && b <= 0x7fffffff) pi[a] = (int32_t)b;
        }
        p = le;
    }
    free(buf);
    if (count) *count = cnt;
    if (max_id) *max_id = (int32_t)(mx > 0x7fffffff ? 0x7fffffff : mx);
    return 0;
}

int bm_read_mapping_pairs(const char* path, int32_t** a, int32_t** b, int64_t* count) {
    size_t len = 0;
    char* buf = slurp(path, &len);
    if (!buf) return -1;
    const char* end = buf + len;
    int64_t cap = 1024, cnt = 0;
    int32_t* xa = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    int32_t* xb = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
    if (!xa || !xb) { free(xa); free(xb); free(buf); return -1; }
    const char* p = next_line(buf, end);
    while (p < end) {
        const char* le = next_line(p, end);
        long long x, y;
        if (parse_mapping_line(p, le, &x, &y)) {
            if (cnt == cap) {
                cap *= 2;
                int32_t* na = (int32_t*)realloc(xa, sizeof(int32_t) * (size_t)cap);
                if (na) xa = na;
                int32_t* nb = (int32_t*)realloc(xb, sizeof(int32_t) * (size_t)cap);
                if (nb) xb = nb;
                if (!na || !nb) { free(xa); free(xb); free(buf); return -1; }
            }
            xa[cnt] = (int32_t)(x > 0x7fffffff ? 0x7fffffff : (x < -0x7fffffff ? -0x7fffffff : x));
            xb[cnt] = (int32_t)(y > 0x7fffffff ? 0x7fffffff : (y < -0x7fffffff ? -0x7fffffff : y));
            cnt++;
        }
        p = le;
    }
    free(buf);
    *a = xa;
    *b = xb;
    *count = cnt;
    return 0;
}

int bm_write_mapping(const char* path, int32_t n, const int32_t* pi) {
    size_t plen = strlen(path);
    char* tmp = (char*)malloc(plen + 32);
    if (!tmp) return -1;
    snprintf(tmp, plen + 32, "%s.tmp.%d", path, (int)getpid());
    FILE* f = fopen(tmp, "w");
    if (!f) { free(tmp); return -1; }
    fprintf(f, "Male Node ID,Female Node ID\n");
    for (int32_t i = 1; i <= n; i++)
        if (pi[i] != 0) fprintf(f, "m%d,f%d\n", i, pi[i]);
    if (fclose(f) != 0) { unlink(tmp); free(tmp); return -1; }
    int rc = rename(tmp, path);
    if (rc != 0) unlink(tmp);
    free(tmp);
    return rc == 0 ? 0 : -1;
}

int32_t bm_check_bijection(int32_t n, const int32_t* pi) {
    unsigned char* seen = (unsigned char*)calloc((size_t)n + 1, 1);
    if (!seen) return -1;
    int32_t bad = 0;
    for (int32_t i = 1; i <= n && !bad; i++) {
        int32_t f = pi[i];
        if (f < 1 || f > n || seen[f]) bad = i;
        else seen[f] = 1;
    }
    free(seen);
    return bad;
}
