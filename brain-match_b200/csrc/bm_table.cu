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
// a second gathers the first ties in (u, v) order (each block owns a
// contiguous range of rows), and one block sorts the K entries by rank.
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

__device__ __forceinline__ void block_rows(int32_t n, int32_t* lo, int32_t* hi) {
    // rows 1..n-1 (row u holds the entries v > u), split into contiguous ranges
    const int64_t rows = n > 1 ? n - 1 : 0;
    const int64_t per = (rows + gridDim.x - 1) / gridDim.x;
    const int64_t a = per * (int64_t)blockIdx.x, b = per * ((int64_t)blockIdx.x + 1);
    *lo = 1 + (int32_t)(a < rows ? a : rows);
    *hi = 1 + (int32_t)(b < rows ? b : rows);
}

__global__ void __launch_bounds__(kTabThreads) hist_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                           const TopState* st, int shift, int bits,
                                                           uint32_t* __restrict__ ghist) {
    __shared__ uint32_t h[kBins];
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint32_t prefix = st->prefix, mask = st->mask, dm = (1u << bits) - 1u;
    int32_t lo, hi;
    block_rows(n, &lo, &hi);
    for (int32_t u = lo; u < hi; u++) {
        const int32_t* row = tab + (size_t)u * (size_t)ld;
        for (int32_t v = u + 1 + threadIdx.x; v <= n; v += blockDim.x) {
            const uint32_t key = okey(row[v]);
            if ((key & mask) == prefix) atomicAdd(&h[(key >> shift) & dm], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kBins; i += blockDim.x)
        if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// Fix the next digit: the largest d with (entries above d) < need <= (entries at or above d).
__global__ void select_digit_kernel(uint32_t* ghist, TopState* st, int shift, int bits) {
    if (threadIdx.x == 0 && st->need > 0) {
        int32_t need = st->need;
        int d = (1 << bits) - 1;
        while (d > 0 && (int32_t)ghist[d] < need) {
            need -= (int32_t)ghist[d];
            d--;
        }
        st->need = need;
        st->prefix |= (uint32_t)d << shift;
        st->mask |= ((1u << bits) - 1u) << shift;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kBins; i += blockDim.x) ghist[i] = 0;
}

struct Sel {
    int32_t* u;
    int32_t* v;
    int32_t* d;
};

// Entries above the threshold (any order, atomic slots) and the count of
// ties per block.
__global__ void __launch_bounds__(kTabThreads) gather_gt_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                                TopState* st, Sel sel, int32_t* __restrict__ blk_eq) {
    __shared__ int32_t s_eq;
    if (threadIdx.x == 0) s_eq = 0;
    __syncthreads();
    const uint32_t T = st->prefix;
    const int32_t n_gt = st->k - st->need;
    int32_t lo, hi, eq = 0;
    block_rows(n, &lo, &hi);
    for (int32_t u = lo; u < hi; u++) {
        const int32_t* row = tab + (size_t)u * (size_t)ld;
        for (int32_t v = u + 1 + threadIdx.x; v <= n; v += blockDim.x) {
            const int32_t d = row[v];
            const uint32_t key = okey(d);
            if (key > T) {
                const int32_t slot = atomicAdd(&st->gt_slot, 1);
                if (slot < n_gt) { sel.u[slot] = u; sel.v[slot] = v; sel.d[slot] = d; }
            } else if (key == T) {
                eq++;
            }
        }
    }
    for (int o = 16; o; o >>= 1) eq += __shfl_xor_sync(0xffffffffu, eq, o);
    if ((threadIdx.x & 31) == 0 && eq) atomicAdd(&s_eq, eq);
    __syncthreads();
    if (threadIdx.x == 0) blk_eq[blockIdx.x] = s_eq;
}

__global__ void scan_blocks_kernel(int32_t* blk, int32_t nb) {
    if (threadIdx.x == 0) {
        int32_t run = 0;
        for (int32_t b = 0; b < nb; b++) {
            const int32_t c = blk[b];
            blk[b] = run;
            run += c;
        }
    }
}

// The first `need` ties in (u, v) order after the entries above the threshold.
__global__ void __launch_bounds__(kTabThreads) gather_eq_kernel(const int32_t* __restrict__ tab, int64_t ld, int32_t n,
                                                                const TopState* st, Sel sel,
                                                                const int32_t* __restrict__ blk_off) {
    __shared__ int32_t wcnt[kTabThreads / 32];
    __shared__ int32_t s_base;
    const int32_t take = st->need;
    const int32_t n_gt = st->k - take;
    const uint32_t T = st->prefix;
    if (threadIdx.x == 0) s_base = blk_off[blockIdx.x];
    __syncthreads();
    if (s_base >= take) return;  // uniform over the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t lo, hi;
    block_rows(n, &lo, &hi);
    for (int32_t u = lo; u < hi; u++) {
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

// Rank sort of the k selected entries: larger delta first, then smaller u, v.
__global__ void rank_sort_kernel(Sel sel, const TopState* st, int32_t* __restrict__ out_pairs,
                                 long long* __restrict__ out_d) {
    const int32_t k = st->k;
    for (int32_t i = threadIdx.x; i < k; i += blockDim.x) {
        const int32_t d = sel.d[i], u = sel.u[i], v = sel.v[i];
        int32_t rank = 0;
        for (int32_t j = 0; j < k; j++) {
            const int32_t d2 = sel.d[j], u2 = sel.u[j], v2 = sel.v[j];
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
    int32_t* blk;
    Sel sel;
};

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

bm_status top_scratch(bm_ctx* ctx, TopScratch* s, void** base_out) {
    const size_t b_st = al256(sizeof(TopState)), b_h = al256(sizeof(uint32_t) * kBins),
                 b_blk = al256(sizeof(int32_t) * kTabBlocks), b_sel = al256(sizeof(int32_t) * kTopMax);
    const size_t total = b_st + b_h + b_blk + 3 * b_sel;
    if (ctx->tscr_bytes < total) {
        cudaFree(ctx->tscr);
        ctx->tscr = nullptr;
        ctx->tscr_bytes = 0;
        if (cudaMalloc(&ctx->tscr, total) != cudaSuccess) {
            cudaGetLastError();
            return bm_fail(ctx, BM_OOM, "top-K scratch");
        }
        ctx->tscr_bytes = total;
    }
    char* p = (char*)ctx->tscr;
    s->st = (TopState*)p;
    s->hist = (uint32_t*)(p + b_st);
    s->blk = (int32_t*)(p + b_st + b_h);
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
            select_digit_kernel<<<1, 256, 0, ctx->stream>>>(S.hist, S.st, shifts[p], widths[p]);
            BM_LAUNCH_CHECK(ctx, "select_digit_kernel");
        }
        gather_gt_kernel<<<kTabBlocks, kTabThreads, 0, ctx->stream>>>(d_tab, ld, n, S.st, S.sel, S.blk);
        BM_LAUNCH_CHECK(ctx, "gather_gt_kernel");
        scan_blocks_kernel<<<1, 32, 0, ctx->stream>>>(S.blk, kTabBlocks);
        BM_LAUNCH_CHECK(ctx, "scan_blocks_kernel");
        gather_eq_kernel<<<kTabBlocks, kTabThreads, 0, ctx->stream>>>(d_tab, ld, n, S.st, S.sel, S.blk);
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
    int64_t full = 0;
    if ((s = bm_launch_score(ctx, &full)) != BM_OK) return s;
    if (full != ctx->score) {
        const int64_t tracked = ctx->score;
        ctx->score = full;
        prog->score = full;
        return bm_fail(ctx, BM_PARITY_FAIL, "tracked score %lld != recomputed score %lld", (long long)tracked,
                       (long long)full);
    }
    prog->score = ctx->score;
    return ret;
}
