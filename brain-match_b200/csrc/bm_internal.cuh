// bm_internal.cuh — device data layout and shared helpers of libbmcuda.
//
// HBM layout of one graph (ids 1..n, slot 0 unused):
//   out_ptr[n+2], in_ptr[n+2]   int32 row offsets (CSR of out-lists, CSC of in-lists)
//   out_ent, in_ent             uint32 packed entries: neighbour id in bits 0..16,
//                               weight in bits 17..31 (n <= 131071, w <= 32767);
//                               each list padded to a multiple of 4 entries with
//                               null entries (0), so every list is 16-byte aligned
//   self_w[n+1]                 self-loop weight (0 if none); self-loops are kept
//                               out of the lists and scored separately
// Graph A's device lists hold their entries in bank-spread order
// (bm_bank_spread_lists: fewer shared-memory bank conflicts in the row
// kernel's scatter), not sorted; every kernel only sums over them.  The host
// copy of A (ctx->hA_*) keeps them sorted by neighbour id.
// Graph B additionally holds
//   out_ent0, in_ent0           the entries with B ids, sorted by id (immutable)
//   out_twin0, in_twin0         index of the same edge in the other direction,
//                               in the sorted lists (immutable)
//   hash[2^k]                   open-addressing table (g*(n+1)+h) -> w of B edges
// and its live out_ent/in_ent carry neighbour ids relabelled into A space
// (id = pi^-1(B id)), so B'-out(x) = B-out(pi x) lists A vertices directly.
// When the mapping is set the live lists are rebuilt from the sorted ones in
// bank-spread order of their A ids (spread_relabel_kernel), with their own
// twins out_twin/in_twin and the position maps out_pos/in_pos; swaps relabel
// live entries in place through the live twins.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/bm_cuda.h"
#include "bm_csr.hpp"

struct DevGraph {
    int32_t n = 0;
    int64_t m_out = 0;   // out-list slots, including the null entries padding each list to 4
    int64_t m_in = 0;    // in-list slots
    int64_t m_real = 0;  // non-self edges
    int32_t* out_ptr = nullptr;
    int32_t* in_ptr = nullptr;
    uint32_t* out_ent = nullptr;
    uint32_t* in_ent = nullptr;
    int32_t* self_w = nullptr;
    // B only
    int32_t* out_twin = nullptr;   // twins of the live lists (rebuilt with them)
    int32_t* in_twin = nullptr;
    uint32_t* out_ent0 = nullptr;
    uint32_t* in_ent0 = nullptr;
    int32_t* out_twin0 = nullptr;  // twins of the id-sorted lists (immutable)
    int32_t* in_twin0 = nullptr;
    int32_t* out_pos = nullptr;    // id-sorted position -> live position
    int32_t* in_pos = nullptr;
    unsigned long long* hash = nullptr;
    int32_t hash_log2 = 0;
    // statistics
    int32_t max_deg = 0;
    int64_t max_wdeg = 0;
    int has_self = 0;
    bool loaded = false;
};

// Read-only view handed to kernels.
struct GView {
    const int32_t* out_ptr;
    const int32_t* in_ptr;
    const uint32_t* out_ent;
    const uint32_t* in_ent;
    const int32_t* self_w;
};

struct HashView {
    const unsigned long long* tab;
    int32_t log2;
    int32_t np1;  // n+1, key = g*(n+1)+h
};

struct bm_ctx {
    int device = -1;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    size_t smem_optin = 0;
    DevGraph g[2];
    int32_t n = 0;
    int32_t nvec = 0;               // n+1 rounded up to a multiple of 4 (vectorised per-vertex arrays)
    // mapping state (device)
    int32_t* pi = nullptr;
    int32_t* pinv = nullptr;
    int32_t* ov = nullptr;          // S(v): per-vertex non-self overlap
    // per A vertex x, the bounds of B's lists at its image pi x:
    // {in begin, in end, out begin, out end}; kept with pi by every kernel
    // that moves images (the row kernel's first-hop staging reads it)
    int4* ximg = nullptr;
    unsigned long long* d_score = nullptr;  // scratch for score reductions
    bool mapped = false;
    int64_t score = 0;              // tracked score
    // staging buffers (device) grown on demand
    void* stage = nullptr;
    size_t stage_bytes = 0;
    void* hstage = nullptr;         // pinned host staging
    size_t hstage_bytes = 0;
    void* flush_buf = nullptr;
    size_t flush_bytes = 0;
    void* tscr = nullptr;           // scratch of the delta-table top-K
    size_t tscr_bytes = 0;
    int64_t launches = 0;
    int32_t row_ctas = 0;           // CTAs per row (cluster size); 0 = auto
    int32_t row_threads = 512;
    // split rows (bm_rows.cu): per-row work estimate, slot partial sums,
    // self-resetting arrival counters and slice reductions
    int32_t row_split = 0;          // 0 = automatic slots, -1 = off, k > 0 = k slots
    int32_t semantics = 0;          // BM_SEMANTICS_EXACT or BM_SEMANTICS_REF_CPU (pairwise swap deltas)
    int32_t* rwork = nullptr;
    std::vector<int32_t> h_rwork;   // host copy (the split plan is made on the host)
    int4* slots = nullptr;          // slot table of a split launch (device)
    int4* h_slots = nullptr;        // its pinned host copy
    cudaEvent_t slots_ev = nullptr; // recorded after each upload of h_slots
    void* spart = nullptr;
    unsigned* scnt = nullptr;
    unsigned* rcnt = nullptr;       // inside the scnt allocation
    void* rpart = nullptr;
    int32_t split_n = 0;
    int32_t split_slots_max = 0;
    int split_active[2 * 9] = {};   // resident clusters per (threads, cluster size); 0 = not queried
    // tiered row launches: 0 = automatic, -1 = off, k > 0 = at most k rows in
    // the wider tier; the second stream and its fork/join events
    int32_t row_tiers = 0;
    cudaStream_t row_side = nullptr;
    cudaEvent_t row_fork = nullptr;
    cudaEvent_t row_join = nullptr;
    // bm_rows_best's copy-in, row launches and copy-out as one CUDA graph,
    // for one row count, valid while every buffer and setting it captured is
    // unchanged (bm_rows.cu)
    struct RowGraph {
        cudaGraphExec_t exec = nullptr;
        int32_t nrows = -1, n = -1, semantics = -1, row_tiers = 0, row_ctas = -1, row_threads = -1;
        const void *stage = nullptr, *hstage = nullptr, *pi = nullptr, *ov = nullptr, *ximg = nullptr, *a = nullptr,
                   *b = nullptr;
        int64_t launches = 0;  // kernels per replay
    } row_graph;
    // set while the row graph is captured: its launches write each row
    // result's row id last, after a system-scope fence (the host polls it)
    bool row_host_res = false;
    // host copy of A's adjacency (independence tests of batched swaps)
    std::vector<int32_t> hA_optr, hA_iptr;
    std::vector<uint32_t> hA_oent, hA_ient;
    // device address of the allocation-free chain entry point's static
    // scratch on this context's device (bm_noalloc_setup, at creation)
    unsigned char* noalloc_scratch = nullptr;
    // bound of the device-side waits (MMA completions of the tensor-core
    // scorer, the auction), SM clock cycles; 0 = each kernel's default
    int64_t wait_limit = 0;
    std::string err;
};

// Every device and pinned-host allocation or release the library makes goes
// through these wrappers, which count the calls (bm_alloc_count), so a test
// can show that an entry point allocates nothing.
cudaError_t bm_cuda_malloc_raw(void** p, size_t bytes);
cudaError_t bm_cuda_free(void* p);
cudaError_t bm_cuda_host_malloc_raw(void** p, size_t bytes);
cudaError_t bm_cuda_host_alloc(void** p, size_t bytes, unsigned flags);
cudaError_t bm_cuda_host_free(void* p);
template <class T>
inline cudaError_t bm_cuda_malloc(T** p, size_t bytes) { return bm_cuda_malloc_raw(reinterpret_cast<void**>(p), bytes); }
template <class T>
inline cudaError_t bm_cuda_host_malloc(T** p, size_t bytes) { return bm_cuda_host_malloc_raw(reinterpret_cast<void**>(p), bytes); }

// Look up the device address of the static scratch of bm_sa_run_noalloc on
// ctx's device (current) and keep it in the context.  Run once by
// bm_ctx_create: the lookup loads the module holding the array, the only step
// of that entry point that can reserve device memory.
bm_status bm_noalloc_setup(bm_ctx* ctx);

// Set the error string and return a status.
bm_status bm_fail(bm_ctx* ctx, bm_status s, const char* fmt, ...);
bm_status bm_cuda_fail(bm_ctx* ctx, cudaError_t e, const char* what);

#define BM_CUDA(ctx, call)                                            \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return bm_cuda_fail((ctx), _e, #call); \
    } while (0)

#define BM_LAUNCH_CHECK(ctx, name)                                      \
    do {                                                                \
        (ctx)->launches++;                                              \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return bm_cuda_fail((ctx), _e, name);    \
    } while (0)

// Ensure the device staging buffer holds `bytes`.
bm_status bm_stage(bm_ctx* ctx, size_t bytes);
bm_status bm_hstage(bm_ctx* ctx, size_t bytes);
bm_status bm_require_mapped(bm_ctx* ctx);

// Stamps of closed A neighbourhoods (host copy of A's lists): the test that
// keeps a batch of swaps independent (no shared vertex, no A edge between
// their endpoint sets), so that their deltas add up exactly.
struct BmMarks {
    std::vector<uint32_t> stamp;
    uint32_t cur = 0;
    void reset(int32_t n) {
        if (stamp.size() != (size_t)n + 1) { stamp.assign((size_t)n + 1, 0); cur = 0; }
        if (++cur == 0) { std::fill(stamp.begin(), stamp.end(), 0); cur = 1; }
    }
    bool marked(int32_t v) const { return stamp[(size_t)v] == cur; }
    void mark_closed(const bm_ctx* ctx, int32_t v) {
        stamp[(size_t)v] = cur;
        for (int32_t j = ctx->hA_optr[(size_t)v]; j < ctx->hA_optr[(size_t)v + 1]; j++)
            stamp[(size_t)bm_eid(ctx->hA_oent[(size_t)j])] = cur;
        for (int32_t j = ctx->hA_iptr[(size_t)v]; j < ctx->hA_iptr[(size_t)v + 1]; j++)
            stamp[(size_t)bm_eid(ctx->hA_ient[(size_t)j])] = cur;
    }
};

inline GView gview(const DevGraph& g) { return GView{g.out_ptr, g.in_ptr, g.out_ent, g.in_ent, g.self_w}; }
inline HashView hview(const DevGraph& g) { return HashView{g.hash, g.hash_log2, g.n + 1}; }

// ------------------------------------------------------------------ device

// B's edge weights live in an open-addressing table at most half full, so an
// empty slot ends every linear probe sequence; lookups are also bounded by
// the table size.  Most lookups are for absent edges, whose sequences have a
// long tail, so a probe step reads a whole 32-byte sector.
// One step of the linear probe sequence: the aligned group of four slots (one
// 32-byte sector) at slot index `grp` (a multiple of 4), from slot `from`
// of the group on.  Returns true when the lookup is settled (key found, *w
// its weight, or an empty slot met, *w = 0).
__device__ __forceinline__ bool bm_hash_group(const HashView& hv, unsigned long long key, unsigned long long grp,
                                              int from, int32_t* w) {
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(hv.tab + grp);
    const ulonglong2 a = __ldg(p), b = __ldg(p + 1);
    const unsigned long long v[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i < from) continue;
        if (v[i] == BM_HASH_EMPTY) { *w = 0; return true; }
        if ((v[i] >> 16) == key) { *w = (int32_t)(v[i] & 0xFFFFull); return true; }
    }
    return false;
}

// Weight of B edge g->h (B ids), 0 if absent: linear probing from the home
// slot, read a 32-byte group of four slots per step (tables hold at least
// 1,024 slots and start 256-byte aligned).
__device__ __forceinline__ int32_t bm_hash_get(const HashView& hv, int32_t g, int32_t h) {
    const unsigned long long key = (unsigned long long)g * (unsigned long long)hv.np1 + (unsigned long long)h;
    const unsigned long long mask = (1ull << hv.log2) - 1ull;
    const unsigned long long s0 = bm_hash_slot0(key, hv.log2);
    unsigned long long grp = s0 & ~3ull;
    int from = (int)(s0 & 3ull);
    int32_t w = 0;
    for (unsigned long long it = 0; it <= mask; it += 4) {
        if (bm_hash_group(hv, key, grp, from, &w)) return w;
        from = 0;
        grp = (grp + 4) & mask;
    }
    return 0;
}

// The same lookup reading one 16-byte slot pair per step: fewer registers,
// for kernels at their register limit that look up rarely.
__device__ __forceinline__ int32_t bm_hash_get_small(const HashView& hv, int32_t g, int32_t h) {
    const unsigned long long key = (unsigned long long)g * (unsigned long long)hv.np1 + (unsigned long long)h;
    const unsigned long long mask = (1ull << hv.log2) - 1ull;
    const unsigned long long s0 = bm_hash_slot0(key, hv.log2);
    unsigned long long base = s0 & ~1ull;
    bool skip_first = (s0 & 1ull) != 0;
    for (unsigned long long it = 0; it <= mask; it += 2) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(hv.tab + base));
        if (!skip_first) {
            if (v.x == BM_HASH_EMPTY) return 0;
            if ((v.x >> 16) == key) return (int32_t)(v.x & 0xFFFFull);
        }
        skip_first = false;
        if (v.y == BM_HASH_EMPTY) return 0;
        if ((v.y >> 16) == key) return (int32_t)(v.y & 0xFFFFull);
        base = (base + 2) & mask;
    }
    return 0;
}

// Weight of neighbour id `key` in a B row staged in shared memory (entries
// sorted by id, zero padding last), 0 if absent: a binary search.
__device__ __forceinline__ int32_t bm_row_weight(const uint32_t* row, int32_t len, int32_t key) {
    int32_t l = 0, h = len;
    while (l < h) {
        const int32_t mid = (l + h) >> 1;
        const uint32_t e = row[mid];
        if (e != 0u && bm_eid(e) < key) l = mid + 1; else h = mid;
    }
    if (l < len) {
        const uint32_t e = row[l];
        if (e != 0u && bm_eid(e) == key) return bm_ew(e);
    }
    return 0;
}

__device__ __forceinline__ int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }

// The list bounds of image g, as kept in ctx->ximg for the A vertex mapped to g.
__device__ __forceinline__ int4 bm_image_bounds(const int32_t* Bin_ptr, const int32_t* Bout_ptr, int32_t g) {
    return make_int4(Bin_ptr[g], Bin_ptr[g + 1], Bout_ptr[g], Bout_ptr[g + 1]);
}

// Kernel launchers implemented across the .cu files.
bm_status bm_launch_score(bm_ctx* ctx, int64_t* score_out);
// Recompute the score and hold the tracked score (the sum of accepted
// deltas) against it; the recomputed score is kept either way.
bm_status bm_check_score(bm_ctx* ctx);
bm_status bm_launch_relabel(bm_ctx* ctx);
// exact_only: score differences whatever the context's delta semantics (for
// callers that apply swaps regardless of their deltas and track the score)
bm_status bm_launch_pairs(bm_ctx* ctx, const int32_t* d_pairs, int64_t k, int64_t* d_out, bool exact_only = false);
// Allocate the split-row buffers for the current n and refresh the per-row
// work estimate (after the mapping is set); refresh alone after many swaps.
bm_status bm_rows_prepare(bm_ctx* ctx);
bm_status bm_rows_refresh_work(bm_ctx* ctx);
// h_rows: a host copy of the rows, when the caller has one; it lets the
// launch spread heavy rows over several clusters (split rows).
bm_status bm_launch_rows(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                         int64_t* d_full, bm_row_result* d_res, const int32_t* h_rows = nullptr);
// Same with a delta-table output: entry (u, v) of row u at d_tab[u * tab_ld + v]
// as int32, and with tab_sym also (v, u).
bm_status bm_launch_rows_ex(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                            int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym,
                            const int32_t* h_rows = nullptr);
// One-sided mode: for each row u, G_u(pi v) - S(u) + self-loop term at the
// columns v = d_cols[0..ncols), into d_colout[r * ncols + j] (int32): the gain
// of u alone taking v's image with every other vertex fixed.
bm_status bm_launch_rows_gen(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                             int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym,
                             const int32_t* d_cols, int32_t ncols, int32_t* d_colout, const int32_t* h_rows = nullptr);
bm_status bm_launch_apply(bm_ctx* ctx, const int32_t* d_pairs, int32_t k);
bm_status bm_rows_smem_check(bm_ctx* ctx);
bm_status bm_launch_kset(bm_ctx* ctx, int32_t k, const int32_t* d_sets, int64_t nsets, long long* d_best,
                         int32_t* d_perm, long long* d_all, int32_t* d_status);
bm_status bm_launch_apply_sets(bm_ctx* ctx, int32_t k, const int32_t* d_sets, const int32_t* d_perms, int32_t nsets);
