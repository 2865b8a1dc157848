// bm_table.cu — the exact swap-delta table and its top-K: a restatement of
// the score-lookup engine of src/best-swap/score-lookup.c (the table of every
// pair's delta, create_score_lookup :246-293; the max-heap of positive swaps,
// heap.c:79-164; the updates after a swap, update_lookup_and_heap :129-244).
//
// Differences, deliberate: entries are int32 exact deltas (the reference
// truncates them to short); the heap is replaced by a device-wide top-K with
// deterministic order (largest delta, then smallest u, then smallest v); and
// after a swap of a and b every row that can change is recomputed, namely the
// rows of {a, b} and of their A neighbours, rows and columns together, where
// the reference recomputes only the pairs involving a and b and so lets the
// rest of the table go stale.  (Every term of delta(u, v) is an A edge at u or
// v evaluated under pi; pi changes only at a and b, so delta(u, v) changes
// only if u or v is a, b or one of their A neighbours.)
//
// Top-K: three radix passes (11, 11 and 10 bits of an order-preserving key)
// build histograms of the upper triangle in shared memory, a one-block kernel
// picks each digit, then one pass gathers every entry above the threshold and
// counts the ties per row, and a second gathers the first ties in (u, v)
// order (each block owns a contiguous range of rows and starts at the row
// prefix of the tie counts), and one block sorts the K entries by rank.  The
// order-free passes give each block row pairs (u, n - u), equal in entries.
#include <algorithm>
#include <chrono>
#include <climits>
#include <vector>

#include "bm_internal.cuh"

namespace {

constexpr int kTabThreads = 256;
constexpr int kBins = 2048;
constexpr int kTopMax = 4096;
constexpr int kTabBlocks = 1024;  // blocks of the scan passes (contiguous row ranges)

struct TopState {
    uint32_t prefix;
    uint32_t mask;
    int32_t need;   // entries still to take below the fixed digits
    int32_t n_gt;   // entries strictly above the threshold
    int32_t k;      // entries selected
    int32_t gt_slot;
};

__device__ __forceinline__ uint32_t okey(int32_t d) { return (uint32_t)d ^ 0x80000000u; }

// Entries of the upper triangle in rows 1..u-1 (row i holds v = i+1..n).
__device__ __forceinline__ int64_t tri_before(int64_t u, int64_t n) { return (u - 1) * n - (u - 1) * u / 2; }

// First row u in [1, n] with tri_before(u) >= e.
__device__ __forceinline__ int32_t tri_row(int64_t e, int32_t n) {
    int32_t lo = 1, hi = n;
    while (lo < hi) {
        const int32_t mid = lo + ((hi - lo) >> 1);
        if (tri_before(mid, n) >= e) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ void block_rows(int32_t n, int32_t* lo, int32_t* hi) {
    // rows 1..n-1 split into contiguous ranges of about equal entry counts
    // (row u holds n - u entries), in block order
    if (n < 2) { *lo = *hi = 1; return; }
    const int64_t total = tri_before(n, n);
    const int64_t b = blockIdx.x, g = gridDim.x;
    *lo = tri_row(total * b / g, n);
    *hi = b + 1 == g ? n : tri_row(total * (b + 1) / g, n);
}

// Rows of this block for the order-free scans: pairs (u, n - u), whose
// lengths n - u and u add up to n, for u in an equal share of 1..(n-1)/2; the
// middle row of an even n goes to the last block.  Returns the pair count;
// row j of the block is pair_row(j).
struct PairRows {
    int32_t p0, np, n, mid;
    __device__ __forceinline__ int32_t rows() const { return 2 * np + mid; }
    __device__ __forceinline__ int32_t row(int32_t j) const {
        if (j == 2 * np) return n / 2;  // the middle row
        const int32_t u = p0 + (j >> 1);
        return (j & 1) ? n - u : u;
    }
};

__device__ __forceinline__ PairRows block_pairs(int32_t n) {
    PairRows r;
    r.n = n;
    const int64_t P = n > 1 ? (n - 1) / 2 : 0;
    const int64_t b = blockIdx.x, g = gridDim.x;
    const int64_t a = P * b / g, e = P * (b + 1) / g;
    r.p0 = 1 + (int32_t)a;
    r.np = (int32_t)(e - a);
    r.mid = (n > 1 && (n - 1) % 2 == 1 && b + 1 == g) ? 1 : 0;
    return r;
}

// Visit the upper triangle of this block's rows with 16-byte streaming loads
// (rows start 16-byte aligned: ld is a multiple of 4).  The group loop is
// uniform over the block; f(u, v, d, ok) sees every lane, ok marks v in (u, n].
// Any order: used by the passes that do not depend on it.
template <class F>
__device__ __forceinline__ void scan_upper(const int32_t* __restrict__ tab, int64_t ld, int32_t n, F&& f) {
    const PairRows pr = block_pairs(n);
    for (int32_t j = 0; j < pr.rows(); j++) {
        const int32_t u = pr.row(j);
        const int4* r4 = reinterpret_cast<const int4*>(tab + (size_t)u * (size_t)ld);
        const int32_t g0 = (u + 1) >> 2, g1 = n >> 2;
        for (int32_t gb = g0; gb <= g1; gb += 2 * kTabThreads) {
            const int32_t ga = gb + (int32_t)threadIdx.x, gc = ga + kTabThreads;
            const int4 qa = ga <= g1 ? __ldcs(r4 + ga) : make_int4(0, 0, 0, 0);
            const int4 qc = gc <= g1 ? __ldcs(r4 + gc) : make_int4(0, 0, 0, 0);
            const int32_t da[4] = {qa.x, qa.y, qa.z, qa.w}, dc[4] = {qc.x, qc.y, qc.z, qc.w};
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int32_t v = 4 * ga + c;
                f(u, v, da[c], ga <= g1 && v > u && v <= n);
            }
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int32_t v = 4 * gc + c;
                f(u, v, dc[c], gc <= g1 && v > u && v <= n);
            }
        }
    }
}

// Histogram of one digit over the entries whose fixed digits match.  Deltas
// crowd into a few bins, so each thread merges runs of equal bins in a
// register and adds a run with one shared-memory atomic.
__global__ void __launch_bounds__(kTabThreads) hist_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                           const TopState* st, int shift, int bits,
                                                           uint32_t* __restrict__ ghist) {
    __shared__ uint32_t h[kBins];
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t prefix = st->prefix, mask = st->mask, dm = (1u << bits) - 1u;
    uint32_t run_bin = 0, run_cnt = 0;
    scan_upper(tab, ld, n, [&](int32_t, int32_t, int32_t d, bool ok) {
        const uint32_t key = okey(d);
        if (ok && (key & mask) == prefix) {
            const uint32_t b = (key >> shift) & dm;
            if (b != run_bin) {
                if (run_cnt) atomicAdd(&h[run_bin], run_cnt);
                run_bin = b;
                run_cnt = 0;
            }
            run_cnt++;
        }
    });
    if (run_cnt) atomicAdd(&h[run_bin], run_cnt);
    __syncthreads();
    for (int i = threadIdx.x; i < kBins; i += blockDim.x)
        if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// Fix the next digit: the largest d with (entries above d) < need <= (entries
// at or above d).  One block of kSelThreads: per-thread sums of kBins /
// kSelThreads bins, a suffix scan, then the owning thread walks its bins.
constexpr int kSelThreads = 256;
__global__ void __launch_bounds__(kSelThreads) select_digit_kernel(uint32_t* ghist, TopState* st, int shift, int bits) {
    __shared__ uint32_t suf[kSelThreads + 1];
    constexpr int per = kBins / kSelThreads;
    const int nb = 1 << bits;
    const int t = threadIdx.x;
    const int32_t need = st->need;  // read before the owner thread rewrites it
    uint32_t mine = 0;
    for (int j = 0; j < per; j++) {
        const int b = t * per + j;
        if (b < nb) mine += ghist[b];
    }
    suf[t] = mine;
    if (t == 0) suf[kSelThreads] = 0;
    __syncthreads();
    // inclusive suffix sums: suf[t] = entries in the bins of threads t..end
    for (int o = 1; o < kSelThreads; o <<= 1) {
        const uint32_t x = (t + o < kSelThreads) ? suf[t + o] : 0;
        __syncthreads();
        suf[t] += x;
        __syncthreads();
    }
    const uint32_t above = suf[t + 1];  // entries in the bins of higher threads
    if (need > 0 && (int64_t)above < need && (int64_t)suf[t] >= need) {
        int32_t left = need - (int32_t)above;
        int d = min(nb, (t + 1) * per) - 1;
        while (d > t * per && (int32_t)ghist[d] < left) {
            left -= (int32_t)ghist[d];
            d--;
        }
        st->need = left;
        st->prefix |= (uint32_t)d << shift;
        st->mask |= ((1u << bits) - 1u) << shift;
    } else if (need > 0 && t == 0 && (int64_t)suf[0] < need) {
        // fewer entries than needed (cannot happen for k <= entries): take digit 0
        st->need = need - (int32_t)(suf[0] - ghist[0]);
        st->mask |= ((1u << bits) - 1u) << shift;
    }
    __syncthreads();
    for (int i = t; i < kBins; i += kSelThreads) ghist[i] = 0;
}

struct Sel {
    int32_t* u;
    int32_t* v;
    int32_t* d;
};

// Entries above the threshold (any order, atomic slots) and the count of
// ties per block.
// Entries above the threshold (any order, atomic slots), and the ties per
// row (each thread adds its count for a row when it moves to another row).
__global__ void __launch_bounds__(kTabThreads) gather_gt_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                                TopState* st, Sel sel, int32_t* __restrict__ rowtie) {
    const uint32_t T = st->prefix;
    const int32_t n_gt = st->k - st->need;
    int32_t cur = 0, eq = 0;
    scan_upper(tab, ld, n, [&](int32_t u, int32_t v, int32_t d, bool ok) {
        const uint32_t key = okey(d);
        if (ok && key > T) {
            const int32_t slot = atomicAdd(&st->gt_slot, 1);
            if (slot < n_gt) { sel.u[slot] = u; sel.v[slot] = v; sel.d[slot] = d; }
        } else if (ok && key == T) {
            if (u != cur) {
                if (eq) atomicAdd(&rowtie[cur], eq);
                cur = u;
                eq = 0;
            }
            eq++;
        }
    });
    if (eq) atomicAdd(&rowtie[cur], eq);
}

// In place exclusive scan of the per-row tie counts (m entries, one block of
// kScanThreads): rowtie[u] becomes the ties in rows before u.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) scan_rows_kernel(int32_t* rowtie, int32_t m) {
    __shared__ int32_t w[kScanThreads / 32];
    __shared__ int32_t carry;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int32_t base = 0; base < m; base += kScanThreads) {
        const int32_t i = base + t;
        const int32_t x = i < m ? rowtie[i] : 0;
        int32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) w[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            const int32_t wv = w[lane];
            int32_t wi = wv;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += y;
            }
            w[lane] = wi - wv;
        }
        __syncthreads();
        const int32_t c = carry;
        if (i < m) rowtie[i] = c + w[wid] + incl - x;
        __syncthreads();
        if (t == kScanThreads - 1) carry = c + w[wid] + incl;
        __syncthreads();
    }
}

// The first `need` ties in (u, v) order after the entries above the threshold.
__global__ void __launch_bounds__(kTabThreads) gather_eq_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                                const TopState* st, Sel sel,
                                                                const int32_t* __restrict__ rowoff) {
    __shared__ int32_t wcnt[kTabThreads / 32];
    __shared__ int32_t s_base;
    const int32_t take = st->need;
    const int32_t n_gt = st->k - take;
    const uint32_t T = st->prefix;
    int32_t lo, hi;
    block_rows(n, &lo, &hi);
    if (threadIdx.x == 0) s_base = rowoff[lo];
    __syncthreads();
    // uniform over the block: enough ties before it, or none in its rows
    if (s_base >= take || rowoff[hi] == s_base) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int32_t u = lo; u < hi; u++) {
        if (rowoff[u + 1] == rowoff[u]) continue;  // no ties in this row (uniform)
        const int32_t* row = tab + (size_t)u * (size_t)ld;
        for (int32_t v0 = u + 1; v0 <= n; v0 += blockDim.x) {
            const int32_t v = v0 + threadIdx.x;
            int32_t d = 0;
            bool eq = false;
            if (v <= n) {
                d = row[v];
                eq = okey(d) == T;
            }
            const uint32_t b = __ballot_sync(0xffffffffu, eq);
            if (lane == 0) wcnt[wid] = __popc(b);
            __syncthreads();
            if (eq) {
                int32_t pos = s_base + __popc(b & ((1u << lane) - 1u));
                for (int w = 0; w < wid; w++) pos += wcnt[w];
                if (pos < take) { sel.u[n_gt + pos] = u; sel.v[n_gt + pos] = v; sel.d[n_gt + pos] = d; }
            }
            __syncthreads();
            if (threadIdx.x == 0)
                for (int w = 0; w < kTabThreads / 32; w++) s_base += wcnt[w];
            __syncthreads();
            if (s_base >= take) return;
        }
    }
}

// Rank sort of the k selected entries: larger delta first, then smaller u, v
// (entries staged in shared memory).
__global__ void __launch_bounds__(1024) rank_sort_kernel(Sel sel, const TopState* st, int32_t* __restrict__ out_pairs,
                                                         long long* __restrict__ out_d) {
    __shared__ int32_t su[kTopMax], sv[kTopMax], sd[kTopMax];
    const int32_t k = st->k;
    for (int32_t i = threadIdx.x; i < k; i += blockDim.x) { su[i] = sel.u[i]; sv[i] = sel.v[i]; sd[i] = sel.d[i]; }
    __syncthreads();
    for (int32_t i = threadIdx.x; i < k; i += blockDim.x) {
        const int32_t d = sd[i], u = su[i], v = sv[i];
        int32_t rank = 0;
        for (int32_t j = 0; j < k; j++) {
            const int32_t d2 = sd[j], u2 = su[j], v2 = sv[j];
            rank += (d2 > d) || (d2 == d && (u2 < u || (u2 == u && v2 < v)));
        }
        out_pairs[2 * rank] = u;
        out_pairs[2 * rank + 1] = v;
        out_d[rank] = d;
    }
}

__global__ void iota_kernel(int32_t* rows, int32_t n) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rows[i] = i + 1;
}

// Scratch of the top-K: state, histogram, block offsets, selection.
struct TopScratch {
    TopState* st;
    uint32_t* hist;
    int32_t* rowtie;  // n + 2 entries: ties per row, then their exclusive prefix
    Sel sel;
};

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

bm_status top_scratch(bm_ctx* ctx, TopScratch* s, void** base_out) {
    const size_t b_st = al256(sizeof(TopState)), b_h = al256(sizeof(uint32_t) * kBins),
                 b_blk = al256(sizeof(int32_t) * ((size_t)ctx->n + 2)), b_sel = al256(sizeof(int32_t) * kTopMax);
    const size_t total = b_st + b_h + b_blk + 3 * b_sel;
    if (ctx->tscr_bytes < total) {
        bm_cuda_free(ctx->tscr);
        ctx->tscr = nullptr;
        ctx->tscr_bytes = 0;
        if (bm_cuda_malloc(&ctx->tscr, total) != cudaSuccess) {
            cudaGetLastError();
            return bm_fail(ctx, BM_OOM, "top-K scratch");
        }
        ctx->tscr_bytes = total;
    }
    char* p = (char*)ctx->tscr;
    s->st = (TopState*)p;
    s->hist = (uint32_t*)(p + b_st);
    s->rowtie = (int32_t*)(p + b_st + b_h);
    s->sel.u = (int32_t*)(p + b_st + b_h + b_blk);
    s->sel.v = (int32_t*)(p + b_st + b_h + b_blk + b_sel);
    s->sel.d = (int32_t*)(p + b_st + b_h + b_blk + 2 * b_sel);
    *base_out = p;
    return BM_OK;
}

bm_status check_table(bm_ctx* ctx, const void* tab, int64_t ld) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!tab) return bm_fail(ctx, BM_INVALID_ARG, "null table");
    if (ld < (int64_t)ctx->n + 1) return bm_fail(ctx, BM_INVALID_ARG, "table stride %lld below n + 1", (long long)ld);
    return bm_rows_smem_check(ctx);
}

}  // namespace

// ------------------------------------------------------------------ C ABI

static bm_status bm_table_topk_launch(bm_ctx* ctx, const int32_t* d_tab, int64_t ld, int32_t k, int32_t* d_pairs,
                                      long long* d_deltas, int32_t* d_count) {
    TopScratch S{};
    void* base = nullptr;
    bm_status s = top_scratch(ctx, &S, &base);
    if (s != BM_OK) return s;
    const int32_t n = ctx->n;
    const long long total = (long long)n * (n - 1) / 2;
    const int32_t keff = (int32_t)std::min<long long>(k, total);
    TopState h{0u, 0u, keff, 0, keff, 0};
    BM_CUDA(ctx, cudaMemcpyAsync(S.st, &h, sizeof(TopState), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(S.hist, 0, sizeof(uint32_t) * kBins, ctx->stream));
    if (keff > 0) {
        const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
        for (int p = 0; p < 3; p++) {
            hist_kernel<<<kTabBlocks, kTabThreads, 0, ctx->stream>>>(d_tab, ld, n, S.st, shifts[p], widths[p], S.hist);
            BM_LAUNCH_CHECK(ctx, "hist_kernel");
            select_digit_kernel<<<1, kSelThreads, 0, ctx->stream>>>(S.hist, S.st, shifts[p], widths[p]);
            BM_LAUNCH_CHECK(ctx, "select_digit_kernel");
        }
        BM_CUDA(ctx, cudaMemsetAsync(S.rowtie, 0, sizeof(int32_t) * ((size_t)n + 2), ctx->stream));
        gather_gt_kernel<<<kTabBlocks, kTabThreads, 0, ctx->stream>>>(d_tab, ld, n, S.st, S.sel, S.rowtie);
        BM_LAUNCH_CHECK(ctx, "gather_gt_kernel");
        scan_rows_kernel<<<1, kScanThreads, 0, ctx->stream>>>(S.rowtie, n + 2);
        BM_LAUNCH_CHECK(ctx, "scan_rows_kernel");
        gather_eq_kernel<<<kTabBlocks, kTabThreads, 0, ctx->stream>>>(d_tab, ld, n, S.st, S.sel, S.rowtie);
        BM_LAUNCH_CHECK(ctx, "gather_eq_kernel");
        rank_sort_kernel<<<1, 1024, 0, ctx->stream>>>(S.sel, S.st, d_pairs, d_deltas);
        BM_LAUNCH_CHECK(ctx, "rank_sort_kernel");
    }
    if (d_count) BM_CUDA(ctx, cudaMemcpyAsync(d_count, &S.st->k, sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_delta_table_dev(bm_ctx* ctx, int32_t* d_table, int64_t ld) {
    bm_status s = check_table(ctx, d_table, ld);
    if (s != BM_OK) return s;
    const int32_t n = ctx->n;
    if ((s = bm_stage(ctx, sizeof(int32_t) * (size_t)n)) != BM_OK) return s;
    int32_t* d_rows = (int32_t*)ctx->stage;
    iota_kernel<<<64, 256, 0, ctx->stream>>>(d_rows, n);
    BM_LAUNCH_CHECK(ctx, "iota_kernel");
    // row 0 is never written by the row kernel; keep it zero
    BM_CUDA(ctx, cudaMemsetAsync(d_table, 0, sizeof(int32_t) * (size_t)ld, ctx->stream));
    return bm_launch_rows_ex(ctx, d_rows, nullptr, n, nullptr, nullptr, d_table, ld, 0);
}

extern "C" bm_status bm_table_refresh_dev(bm_ctx* ctx, int32_t* d_table, int64_t ld, const int32_t* d_rows,
                                          int32_t nrows) {
    bm_status s = check_table(ctx, d_table, ld);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && !d_rows)) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    if (nrows == 0) return BM_OK;
    return bm_launch_rows_ex(ctx, d_rows, nullptr, nrows, nullptr, nullptr, d_table, ld, 1);
}

extern "C" bm_status bm_table_topk_dev(bm_ctx* ctx, const int32_t* d_table, int64_t ld, int32_t k, int32_t* d_pairs,
                                       int64_t* d_deltas, int32_t* d_count) {
    bm_status s = check_table(ctx, d_table, ld);
    if (s != BM_OK) return s;
    if (k < 1 || k > kTopMax) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 1..%d", k, kTopMax);
    if (!d_pairs || !d_deltas) return bm_fail(ctx, BM_INVALID_ARG, "bad output buffers");
    return bm_table_topk_launch(ctx, d_table, ld, k, d_pairs, (long long*)d_deltas, d_count);
}

extern "C" bm_status bm_table_topk(bm_ctx* ctx, const int32_t* d_table, int64_t ld, int32_t k, int32_t* pairs,
                                   int64_t* deltas, int32_t* count) {
    bm_status s = check_table(ctx, d_table, ld);
    if (s != BM_OK) return s;
    if (k < 1 || k > kTopMax) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 1..%d", k, kTopMax);
    if (!pairs || !deltas || !count) return bm_fail(ctx, BM_INVALID_ARG, "bad output buffers");
    const size_t pb = al256(sizeof(int32_t) * 2 * (size_t)k), db = al256(sizeof(long long) * (size_t)k);
    if ((s = bm_stage(ctx, pb + db + 256)) != BM_OK) return s;
    int32_t* d_p = (int32_t*)ctx->stage;
    long long* d_d = (long long*)((char*)ctx->stage + pb);
    int32_t* d_c = (int32_t*)((char*)ctx->stage + pb + db);
    if ((s = bm_table_topk_launch(ctx, d_table, ld, k, d_p, d_d, d_c)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(count, d_c, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int32_t c = *count;
    if (c > 0) {
        BM_CUDA(ctx, cudaMemcpyAsync(pairs, d_p, sizeof(int32_t) * 2 * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(deltas, d_d, sizeof(long long) * (size_t)c, cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return BM_OK;
}

extern "C" bm_status bm_search_table(bm_ctx* ctx, int32_t* d_table, int64_t ld, int32_t k, int64_t max_accepts,
                                     int32_t max_rounds, double time_budget_s, bm_progress* prog) {
    using clk = std::chrono::steady_clock;
    bm_status s = check_table(ctx, d_table, ld);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if (k < 1 || k > kTopMax) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 1..%d", k, kTopMax);
    const int32_t n = ctx->n;
    const size_t pb = al256(sizeof(int32_t) * 2 * (size_t)k), db = al256(sizeof(long long) * (size_t)k);
    const size_t rb = al256(sizeof(int32_t) * ((size_t)n + 1));
    if ((s = bm_stage(ctx, pb + db + 256 + rb + pb)) != BM_OK) return s;
    char* base = (char*)ctx->stage;
    int32_t* d_p = (int32_t*)base;
    long long* d_d = (long long*)(base + pb);
    int32_t* d_c = (int32_t*)(base + pb + db);
    int32_t* d_rows = (int32_t*)(base + pb + db + 256);
    int32_t* d_ap = (int32_t*)(base + pb + db + 256 + rb);
    std::vector<int32_t> h_p((size_t)2 * k), h_ap, rows;
    std::vector<long long> h_d((size_t)k);
    std::vector<uint32_t> touched((size_t)n + 1, 0);
    uint32_t stamp = 0;
    BmMarks mk;
    const auto t0 = clk::now();
    const int64_t acc0 = prog->accepts;
    int32_t rounds = 0;
    bm_status ret = BM_OK;
    prog->converged = 0;
    for (;;) {
        if (max_accepts >= 0 && prog->accepts - acc0 >= max_accepts) break;
        if (max_rounds >= 0 && rounds >= max_rounds) break;
        if (time_budget_s > 0 &&
            std::chrono::duration<double>(clk::now() - t0).count() >= time_budget_s) { ret = BM_TIMEOUT; break; }
        if ((s = bm_table_topk_launch(ctx, d_table, ld, k, d_p, d_d, d_c)) != BM_OK) return s;
        int32_t c = 0;
        BM_CUDA(ctx, cudaMemcpyAsync(&c, d_c, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (c > 0) {
            BM_CUDA(ctx, cudaMemcpyAsync(h_p.data(), d_p, sizeof(int32_t) * 2 * (size_t)c, cudaMemcpyDeviceToHost,
                                         ctx->stream));
            BM_CUDA(ctx, cudaMemcpyAsync(h_d.data(), d_d, sizeof(long long) * (size_t)c, cudaMemcpyDeviceToHost,
                                         ctx->stream));
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        rounds++;
        prog->launches++;
        if (c == 0 || h_d[0] <= 0) { prog->converged = 1; break; }
        // independent improving swaps in descending delta (the list is sorted)
        mk.reset(n);
        h_ap.clear();
        int64_t gain = 0;
        for (int32_t i = 0; i < c && h_d[(size_t)i] > 0; i++) {
            const int32_t u = h_p[2 * (size_t)i], v = h_p[2 * (size_t)i + 1];
            if (mk.marked(u) || mk.marked(v)) continue;
            mk.mark_closed(ctx, u);
            mk.mark_closed(ctx, v);
            h_ap.push_back(u);
            h_ap.push_back(v);
            gain += h_d[(size_t)i];
            if (max_accepts >= 0 && prog->accepts - acc0 + (int64_t)h_ap.size() / 2 >= max_accepts) break;
        }
        const int32_t na = (int32_t)(h_ap.size() / 2);
        BM_CUDA(ctx, cudaMemcpyAsync(d_ap, h_ap.data(), sizeof(int32_t) * h_ap.size(), cudaMemcpyHostToDevice,
                                     ctx->stream));
        if ((s = bm_launch_apply(ctx, d_ap, na)) != BM_OK) return s;
        ctx->score += gain;
        prog->accepts += na;
        // rows to refresh: the swapped vertices and their A neighbours
        if (++stamp == 0) { std::fill(touched.begin(), touched.end(), 0u); stamp = 1; }
        rows.clear();
        auto touch = [&](int32_t x) {
            if (touched[(size_t)x] != stamp) { touched[(size_t)x] = stamp; rows.push_back(x); }
        };
        for (int32_t x : h_ap) {
            touch(x);
            for (int32_t j = ctx->hA_optr[(size_t)x]; j < ctx->hA_optr[(size_t)x + 1]; j++)
                if (ctx->hA_oent[(size_t)j]) touch(bm_eid(ctx->hA_oent[(size_t)j]));
            for (int32_t j = ctx->hA_iptr[(size_t)x]; j < ctx->hA_iptr[(size_t)x + 1]; j++)
                if (ctx->hA_ient[(size_t)j]) touch(bm_eid(ctx->hA_ient[(size_t)j]));
        }
        BM_CUDA(ctx, cudaMemcpyAsync(d_rows, rows.data(), sizeof(int32_t) * rows.size(), cudaMemcpyHostToDevice,
                                     ctx->stream));
        if ((s = bm_launch_rows_ex(ctx, d_rows, nullptr, (int32_t)rows.size(), nullptr, nullptr, d_table, ld, 1,
                                   rows.data())) !=
            BM_OK)
            return s;
        prog->rows_done += (int64_t)rows.size();
        prog->evaluated += (int64_t)rows.size() * (n - 1);
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->seconds += std::chrono::duration<double>(clk::now() - t0).count();
    prog->sweeps += rounds;
    s = bm_check_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}
