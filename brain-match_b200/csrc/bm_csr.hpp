// bm_csr.hpp — host-side construction of the device graph layout (plain C++,
// no CUDA: also compiled on its own under AddressSanitizer by the CPU tests).
//
// From an edge list with ids 1..n it builds
//   optr/oent   out-lists (CSR) sorted by (src, dst)
//   iptr/ient   in-lists (CSC) sorted by (dst, src)
// with packed uint32 entries (neighbour id in bits 0..16, weight in bits
// 17..31).  Every list is padded to a multiple of 4 entries with null entries
// (0), so each list starts on a 16-byte boundary; out and in lists are padded
// separately, so the two totals differ.  Graph B additionally gets
//   otw/itw     index of the same edge in the other direction (-1 for padding)
//   htab        open-addressing table (g*(n+1)+h) -> w, load <= 1/2
// The acceptance rules follow add_edge (src/graph-alignment-optimized.c:183-204):
// A keeps every list entry, B keeps the last weight of a duplicated edge (its
// matrix store).  Zero weights never contribute to min(w, .) and are dropped.
// Self-loops are kept out of the lists, in self[].
#pragma once

#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#ifdef __CUDACC__
#define BM_HD __host__ __device__ __forceinline__
#else
#define BM_HD inline
#endif

#define BM_ID_BITS 17
#define BM_ID_MASK ((1u << BM_ID_BITS) - 1u)
#define BM_MAX_N ((int32_t)BM_ID_MASK)
#define BM_MAX_W 32767
#define BM_HASH_EMPTY 0xFFFFFFFFFFFFFFFFull

BM_HD uint32_t bm_pack(uint32_t id, uint32_t w) { return id | (w << BM_ID_BITS); }
BM_HD int32_t bm_eid(uint32_t e) { return (int32_t)(e & BM_ID_MASK); }
BM_HD int32_t bm_ew(uint32_t e) { return (int32_t)(e >> BM_ID_BITS); }

// Fibonacci hashing of a 64-bit key to `log2` bits.
BM_HD unsigned long long bm_hash_slot0(unsigned long long key, int log2) {
    return (key * 0x9E3779B97F4A7C15ull) >> (64 - log2);
}

struct HostCsr {
    int32_t n = 0;
    int64_t m_real = 0;  // non-self edges kept
    std::vector<int32_t> optr, iptr;
    std::vector<uint32_t> oent, ient;
    std::vector<int32_t> otw, itw;
    std::vector<int32_t> self;
    std::vector<unsigned long long> htab;
    int hlog2 = 0;
    int has_self = 0;
    int32_t max_deg = 0;
    int64_t max_wdeg = 0;
    int64_t m_out() const { return optr.empty() ? 0 : optr.back(); }
    int64_t m_in() const { return iptr.empty() ? 0 : iptr.back(); }
};

// Returns 0 on success, 1 for invalid input (message in err).
inline int bm_build_host_csr(bool side_b, int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                             const int32_t* w, HostCsr& G, std::string& err) {
    char buf[256];
    if (n < 1 || n > BM_MAX_N) {
        snprintf(buf, sizeof buf, "n=%d outside 1..%d", n, BM_MAX_N);
        err = buf;
        return 1;
    }
    // padding adds at most 3 slots per vertex and list; offsets are int32
    if (m < 0 || m >= (int64_t)0x7fffffff - 4 * (int64_t)BM_MAX_N) {
        snprintf(buf, sizeof buf, "edge count %lld out of range", (long long)m);
        err = buf;
        return 1;
    }
    if (m > 0 && (!src || !dst || !w)) {
        err = "null edge arrays";
        return 1;
    }
    for (int64_t e = 0; e < m; e++) {
        if (src[e] < 1 || src[e] > n || dst[e] < 1 || dst[e] > n) {
            snprintf(buf, sizeof buf, "edge %lld: id outside 1..%d", (long long)e, n);
            err = buf;
            return 1;
        }
        if (w[e] < 0 || w[e] > BM_MAX_W) {
            snprintf(buf, sizeof buf, "edge %lld: weight %d outside 0..%d", (long long)e, w[e], BM_MAX_W);
            err = buf;
            return 1;
        }
    }
    G = HostCsr();
    G.n = n;
    G.self.assign((size_t)n + 1, 0);
    std::vector<char> keep((size_t)m, 1);
    const unsigned long long np1 = (unsigned long long)n + 1;
    if (side_b) {
        int64_t cap = 1024;
        G.hlog2 = 10;
        // load <= 1/2: most lookups are for absent edges, and an unsuccessful
        // linear probe costs about (1 + 1/(1-load)^2)/2 slots, 2.5 at 1/2
        // against 8.5 at 3/4; a warp waits for its longest probe
        while (cap < 2 * (m + 1)) { cap <<= 1; G.hlog2++; }
        const unsigned long long mask = (unsigned long long)(cap - 1);
        // key -> last edge index, in a temporary table
        std::vector<unsigned long long> kk((size_t)cap, BM_HASH_EMPTY);
        std::vector<int64_t> vi((size_t)cap, -1);
        for (int64_t e = 0; e < m; e++) {
            const unsigned long long key = (unsigned long long)src[e] * np1 + (unsigned long long)dst[e];
            unsigned long long s = bm_hash_slot0(key, G.hlog2);
            while (kk[s] != BM_HASH_EMPTY && kk[s] != key) s = (s + 1) & mask;
            if (kk[s] == key) keep[(size_t)vi[s]] = 0;
            kk[s] = key;
            vi[s] = e;
        }
        G.htab.assign((size_t)cap, BM_HASH_EMPTY);
        for (int64_t e = 0; e < m; e++) {
            if (!keep[e]) continue;
            if (w[e] == 0) { keep[e] = 0; continue; }
            if (src[e] == dst[e]) { G.self[src[e]] = w[e]; G.has_self = 1; keep[e] = 0; continue; }
            const unsigned long long key = (unsigned long long)src[e] * np1 + (unsigned long long)dst[e];
            unsigned long long s = bm_hash_slot0(key, G.hlog2);
            while (G.htab[s] != BM_HASH_EMPTY) s = (s + 1) & mask;
            G.htab[s] = (key << 16) | (unsigned long long)w[e];
        }
    } else {
        for (int64_t e = 0; e < m; e++) {
            if (w[e] == 0) { keep[e] = 0; continue; }
            if (src[e] == dst[e]) {
                if (G.self[src[e]] != 0) {
                    snprintf(buf, sizeof buf, "vertex %d has more than one self-loop in graph A", src[e]);
                    err = buf;
                    return 1;
                }
                G.self[src[e]] = w[e];
                G.has_self = 1;
                keep[e] = 0;
            }
        }
    }
    std::vector<int32_t> ocnt((size_t)n + 1, 0), icnt((size_t)n + 1, 0);
    int64_t mk = 0;
    for (int64_t e = 0; e < m; e++)
        if (keep[e]) { ocnt[(size_t)src[e]]++; icnt[(size_t)dst[e]]++; mk++; }
    G.m_real = mk;
    G.optr.assign((size_t)n + 2, 0);
    G.iptr.assign((size_t)n + 2, 0);
    for (int32_t i = 0; i <= n; i++) {
        G.optr[(size_t)i + 1] = G.optr[(size_t)i] + ((ocnt[(size_t)i] + 3) & ~3);
        G.iptr[(size_t)i + 1] = G.iptr[(size_t)i] + ((icnt[(size_t)i] + 3) & ~3);
    }
    // stable counting sorts: edges by dst, and by src
    std::vector<int64_t> by_dst((size_t)mk), by_src((size_t)mk);
    {
        std::vector<int64_t> f((size_t)n + 1, 0), g((size_t)n + 1, 0);
        for (int32_t i = 1; i <= n; i++) { f[(size_t)i] = f[(size_t)i - 1] + icnt[(size_t)i - 1]; g[(size_t)i] = g[(size_t)i - 1] + ocnt[(size_t)i - 1]; }
        for (int64_t e = 0; e < m; e++) if (keep[e]) by_dst[(size_t)f[(size_t)dst[e]]++] = e;
        for (int64_t e = 0; e < m; e++) if (keep[e]) by_src[(size_t)g[(size_t)src[e]]++] = e;
    }
    G.oent.assign((size_t)G.m_out(), 0u);
    G.ient.assign((size_t)G.m_in(), 0u);
    std::vector<int32_t> opos_of((size_t)(side_b ? m : 0)), ipos_of((size_t)(side_b ? m : 0));
    {
        // out: edges in dst order placed by src (stable) -> rows sorted by dst
        std::vector<int32_t> f(G.optr.begin(), G.optr.end() - 1);
        for (int64_t k = 0; k < mk; k++) {
            const int64_t e = by_dst[(size_t)k];
            const int32_t p = f[(size_t)src[e]]++;
            G.oent[(size_t)p] = bm_pack((uint32_t)dst[e], (uint32_t)w[e]);
            if (side_b) opos_of[(size_t)e] = p;
        }
        std::vector<int32_t> g(G.iptr.begin(), G.iptr.end() - 1);
        for (int64_t k = 0; k < mk; k++) {
            const int64_t e = by_src[(size_t)k];
            const int32_t p = g[(size_t)dst[e]]++;
            G.ient[(size_t)p] = bm_pack((uint32_t)src[e], (uint32_t)w[e]);
            if (side_b) ipos_of[(size_t)e] = p;
        }
    }
    if (side_b) {
        G.otw.assign((size_t)G.m_out(), -1);
        G.itw.assign((size_t)G.m_in(), -1);
        for (int64_t e = 0; e < m; e++)
            if (keep[e]) {
                G.otw[(size_t)opos_of[(size_t)e]] = ipos_of[(size_t)e];
                G.itw[(size_t)ipos_of[(size_t)e]] = opos_of[(size_t)e];
            }
    }
    std::vector<int64_t> wd((size_t)n + 1, 0);
    for (int64_t e = 0; e < m; e++)
        if (keep[e]) { wd[(size_t)src[e]] += w[e]; wd[(size_t)dst[e]] += w[e]; }
    for (int32_t v = 1; v <= n; v++) {
        const int32_t d = ocnt[(size_t)v] + icnt[(size_t)v];
        if (d > G.max_deg) G.max_deg = d;
        if (wd[(size_t)v] + G.self[(size_t)v] > G.max_wdeg) G.max_wdeg = wd[(size_t)v] + G.self[(size_t)v];
    }
    if (!side_b && G.max_wdeg >= ((int64_t)1 << 29)) {
        snprintf(buf, sizeof buf, "weighted degree %lld of graph A is 2^29 or more", (long long)G.max_wdeg);
        err = buf;
        return 1;
    }
    return 0;
}

// Reorders the real entries of every list (the padding stays at the end) so
// that the row kernel's shared-memory scatter meets fewer bank conflicts.  A
// warp's lanes take consecutive 4-entry quads of a list, and its c-th atomic
// instruction adds at entry c of each lane's quad, at accumulator word id
// (bank id mod 32).  Position p of a list is given, where the list has one,
// an entry of bank ((p >> 2) + 8 (p & 3)) mod 32, else the next bank up that
// still has entries: entry c of 32 consecutive quads then lands in 32
// different banks when the list's banks are balanced.  Sums over the lists do
// not depend on the order; nothing may rely on these lists being sorted.
inline void bm_bank_spread_lists(const std::vector<int32_t>& ptr, std::vector<uint32_t>& ent) {
    std::vector<uint32_t> bucket[32];
    for (size_t v = 0; v + 1 < ptr.size(); v++) {
        const int32_t lo = ptr[v], hi = ptr[v + 1];
        int32_t cnt = 0;
        for (int b = 0; b < 32; b++) bucket[b].clear();
        for (int32_t j = lo; j < hi; j++) {
            const uint32_t e = ent[(size_t)j];
            if (e) { bucket[bm_eid(e) & 31].push_back(e); cnt++; }
        }
        if (cnt < 2) continue;
        size_t head[32] = {0};
        for (int32_t p = 0; p < cnt; p++) {
            int b = ((p >> 2) + 8 * (p & 3)) & 31;
            while (head[b] >= bucket[b].size()) b = (b + 1) & 31;
            ent[(size_t)lo + p] = bucket[b][head[b]++];
        }
    }
}
