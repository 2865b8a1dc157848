// CPU check of the device graph layout builder (brain-match_b200/csrc/bm_csr.hpp),
// compiled with AddressSanitizer and UndefinedBehaviorSanitizer by
// tests/test_csr_sanitized.py.  Random graphs with duplicates, self-loops and
// zero weights; every invariant the kernels rely on is checked.  Exit code 0
// means all checks passed.
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <map>
#include <random>
#include <utility>

#include "../brain-match_b200/csrc/bm_csr.hpp"

#define CHECK(c)                                                        \
    do {                                                                \
        if (!(c)) {                                                     \
            fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
            exit(1);                                                    \
        }                                                               \
    } while (0)

static int32_t hash_get(const HostCsr& G, int32_t g, int32_t h) {
    const unsigned long long key = (unsigned long long)g * (unsigned long long)(G.n + 1) + (unsigned long long)h;
    const unsigned long long mask = G.htab.size() - 1;
    unsigned long long s = bm_hash_slot0(key, G.hlog2);
    for (size_t it = 0; it < G.htab.size(); it++) {
        const unsigned long long v = G.htab[s];
        if (v == BM_HASH_EMPTY) return 0;
        if ((v >> 16) == key) return (int32_t)(v & 0xFFFF);
        s = (s + 1) & mask;
    }
    return 0;
}

static void check_bank_spread(const HostCsr& G);

static void check_graph(bool side_b, int32_t n, const std::vector<int32_t>& s, const std::vector<int32_t>& d,
                        const std::vector<int32_t>& w) {
    HostCsr G;
    std::string err;
    const int rc = bm_build_host_csr(side_b, n, (int64_t)s.size(), s.data(), d.data(), w.data(), G, err);
    // expected multiset of kept non-self entries
    std::map<std::pair<int, int>, std::vector<int>> exp;
    std::map<std::pair<int, int>, int> last;
    std::vector<int> self(n + 1, 0), nself(n + 1, 0);
    for (size_t e = 0; e < s.size(); e++) {
        if (side_b) last[{s[e], d[e]}] = w[e];
        else if (w[e] != 0) {
            if (s[e] == d[e]) { self[s[e]] = w[e]; nself[s[e]]++; }
            else exp[{s[e], d[e]}].push_back(w[e]);
        }
    }
    if (!side_b) {
        bool dup_self = false;
        for (int v = 1; v <= n; v++) dup_self |= nself[v] > 1;
        if (dup_self) { CHECK(rc == 1); return; }
    } else {
        for (auto& kv : last)
            if (kv.second != 0) {
                if (kv.first.first == kv.first.second) self[kv.first.first] = kv.second;
                else exp[kv.first].push_back(kv.second);
            }
    }
    CHECK(rc == 0);
    CHECK((int)G.optr.size() == n + 2 && (int)G.iptr.size() == n + 2);
    CHECK(G.optr[0] == 0 && G.optr[1] == 0 && G.iptr[0] == 0 && G.iptr[1] == 0);
    CHECK((int64_t)G.oent.size() == G.m_out() && (int64_t)G.ient.size() == G.m_in());
    int64_t real = 0;
    for (auto& kv : exp) real += (int64_t)kv.second.size();
    CHECK(G.m_real == real);
    std::map<std::pair<int, int>, std::vector<int>> got_o, got_i;
    for (int v = 0; v <= n; v++) {
        CHECK(G.optr[v] % 4 == 0 && G.iptr[v] % 4 == 0);
        bool pad = false;
        int prev = -1;
        for (int j = G.optr[v]; j < G.optr[v + 1]; j++) {
            const uint32_t e = G.oent[j];
            if (e == 0) { pad = true; continue; }
            CHECK(!pad);  // padding only at the end
            CHECK(bm_eid(e) >= 1 && bm_eid(e) <= n && bm_eid(e) != v);
            CHECK(bm_eid(e) >= prev);  // sorted by target
            prev = bm_eid(e);
            got_o[{v, bm_eid(e)}].push_back(bm_ew(e));
            if (side_b) {
                const int t = G.otw[j];
                CHECK(t >= 0 && t < G.m_in());
                CHECK(G.ient[t] == bm_pack((uint32_t)v, (uint32_t)bm_ew(e)));
                CHECK(G.itw[t] == j);
            }
        }
        CHECK(G.optr[v + 1] - G.optr[v] < 4 || G.oent[G.optr[v + 1] - 4] != 0);  // at most 3 pads
        pad = false;
        for (int j = G.iptr[v]; j < G.iptr[v + 1]; j++) {
            const uint32_t e = G.ient[j];
            if (e == 0) { pad = true; if (side_b) CHECK(G.itw[j] == -1); continue; }
            CHECK(!pad);
            got_i[{bm_eid(e), v}].push_back(bm_ew(e));
        }
    }
    for (auto& kv : exp) {
        std::vector<int> a = kv.second, b = got_o[kv.first], c = got_i[kv.first];
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        std::sort(c.begin(), c.end());
        CHECK(a == b && a == c);
        if (side_b) CHECK(hash_get(G, kv.first.first, kv.first.second) == kv.second[0]);
    }
    CHECK(got_o.size() == exp.size() && got_i.size() == exp.size());
    check_bank_spread(G);
    for (int v = 1; v <= n; v++) CHECK(G.self[v] == self[v]);
    if (side_b)
        for (int t = 0; t < 2000; t++) {
            const int g = 1 + rand() % n, h = 1 + rand() % n;
            auto it = last.find({g, h});
            const int want = (g == h || it == last.end()) ? 0 : it->second;
            CHECK(hash_get(G, g, h) == want);
        }
}

// bm_bank_spread_lists permutes the real entries inside each list and keeps
// the padding last; on a list with balanced banks, entry c of any 32
// consecutive quads falls in 32 different banks.
static void check_bank_spread(const HostCsr& G) {
    std::vector<uint32_t> oe = G.oent, ie = G.ient;
    bm_bank_spread_lists(G.optr, oe);
    bm_bank_spread_lists(G.iptr, ie);
    for (int pass = 0; pass < 2; pass++) {
        const std::vector<int32_t>& ptr = pass ? G.iptr : G.optr;
        const std::vector<uint32_t>& before = pass ? G.ient : G.oent;
        const std::vector<uint32_t>& after = pass ? ie : oe;
        CHECK(after.size() == before.size());
        for (size_t v = 0; v + 1 < ptr.size(); v++) {
            std::vector<uint32_t> a(before.begin() + ptr[v], before.begin() + ptr[v + 1]);
            std::vector<uint32_t> b(after.begin() + ptr[v], after.begin() + ptr[v + 1]);
            bool pad = false;
            for (uint32_t e : b) {
                if (e == 0) pad = true;
                else CHECK(!pad);
            }
            std::sort(a.begin(), a.end());
            std::sort(b.begin(), b.end());
            CHECK(a == b);
        }
    }
}

static void check_bank_spread_balanced() {
    // one list of 256 entries, eight per bank, given in id order
    std::vector<int32_t> ptr = {0, 0, 256};
    std::vector<uint32_t> ent;
    for (uint32_t i = 1; i <= 256; i++) ent.push_back(bm_pack(i, 1));
    bm_bank_spread_lists(ptr, ent);
    for (int q0 = 0; q0 + 32 <= 64; q0++)
        for (int c = 0; c < 4; c++) {
            unsigned seen = 0;
            for (int k = 0; k < 32; k++) seen |= 1u << (bm_eid(ent[(size_t)(4 * (q0 + k) + c)]) & 31);
            CHECK(seen == 0xFFFFFFFFu);
        }
}

int main() {
    check_bank_spread_balanced();
    std::mt19937 rng(12345);
    for (int trial = 0; trial < 300; trial++) {
        const int n = 1 + (int)(rng() % 60) + (trial % 10 == 0 ? 2000 : 0);
        const int m = (int)(rng() % (4 * n + 5));
        std::vector<int32_t> s(m), d(m), w(m);
        for (int e = 0; e < m; e++) {
            s[e] = 1 + (int)(rng() % n);
            d[e] = (rng() % 7 == 0) ? s[e] : 1 + (int)(rng() % n);
            w[e] = (rng() % 9 == 0) ? 0 : 1 + (int)(rng() % (trial % 3 == 0 ? 32767 : 6));
        }
        check_graph(true, n, s, d, w);
        // A: keep at most one self-loop per vertex in half of the trials
        if (trial % 2) {
            std::vector<char> seen(n + 1, 0);
            for (int e = 0; e < m; e++)
                if (s[e] == d[e]) {
                    if (seen[s[e]]) d[e] = (s[e] % n) + 1;
                    seen[s[e]] = 1;
                }
        }
        check_graph(false, n, s, d, w);
    }
    // invalid inputs
    HostCsr G;
    std::string err;
    int32_t s1[1] = {1}, d1[1] = {5}, w1[1] = {1}, wbad[1] = {40000};
    CHECK(bm_build_host_csr(false, 4, 1, s1, d1, w1, G, err) == 1);
    CHECK(bm_build_host_csr(false, 8, 1, s1, d1, wbad, G, err) == 1);
    CHECK(bm_build_host_csr(false, 0, 0, s1, d1, w1, G, err) == 1);
    CHECK(bm_build_host_csr(true, BM_MAX_N + 1, 0, s1, d1, w1, G, err) == 1);
    CHECK(bm_build_host_csr(true, 3, 0, nullptr, nullptr, nullptr, G, err) == 0 && G.m_out() == 0);
    printf("csr_check ok\n");
    return 0;
}
