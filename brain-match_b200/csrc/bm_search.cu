// bm_search.cu — host-driven schedules over the row and apply kernels.
//
// bm_sweep_parity reproduces the serial first-improvement loop of
// optimize_mapping (src/graph-alignment-optimized.c:513-580) exactly: rows in
// order, columns ascending, accept the first delta > 0, continue with the next
// column under the new mapping.  A batch of K consecutive rows is evaluated at
// once under the current mapping; rows before the first row with an improving
// column are exactly what the serial loop would have scanned, the first
// improving column of that row is the serial loop's next accept, and
// everything after it is discarded and re-evaluated after the swap.  K adapts
// (doubling while batches hold no accept, halving after one).
//
// bm_search_batched is the throughput schedule: best improving column per row
// (the row argmax of src/re-alignment-parallel.c:598-618), then a greedy
// independent subset (descending delta, ascending row; no shared vertex and
// no A edge between two chosen swaps, the independence rule of
// src/independent-hungarian/hungarianSubset.c:657-740) applied in one launch.
// Independent swaps do not change each other's deltas, so the tracked score
// stays exact.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "bm_internal.cuh"
#include "bm_rng.hpp"

namespace {

using clk = std::chrono::steady_clock;

double secs_since(clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); }

// Device + pinned staging for one schedule call.
struct SchedBufs {
    int32_t* d_rows = nullptr;
    int32_t* d_col = nullptr;
    bm_row_result* d_res = nullptr;
    int32_t* d_pairs = nullptr;
    int32_t* h_rows = nullptr;
    int32_t* h_col = nullptr;
    bm_row_result* h_res = nullptr;
    int32_t* h_pairs = nullptr;
};

bm_status sched_bufs(bm_ctx* ctx, int32_t kmax, SchedBufs* b) {
    const size_t rb = ((size_t)kmax * sizeof(int32_t) + 255) & ~(size_t)255;
    const size_t resb = ((size_t)kmax * sizeof(bm_row_result) + 255) & ~(size_t)255;
    const size_t pb = ((size_t)kmax * 2 * sizeof(int32_t) + 255) & ~(size_t)255;
    const size_t total = 2 * rb + resb + pb;
    bm_status s = bm_stage(ctx, total);
    if (s != BM_OK) return s;
    s = bm_hstage(ctx, total);
    if (s != BM_OK) return s;
    char* d = (char*)ctx->stage;
    char* h = (char*)ctx->hstage;
    b->d_rows = (int32_t*)d;  b->h_rows = (int32_t*)h;
    b->d_col = (int32_t*)(d + rb);  b->h_col = (int32_t*)(h + rb);
    b->d_res = (bm_row_result*)(d + 2 * rb);  b->h_res = (bm_row_result*)(h + 2 * rb);
    b->d_pairs = (int32_t*)(d + 2 * rb + resb);  b->h_pairs = (int32_t*)(h + 2 * rb + resb);
    return BM_OK;
}

bm_status eval_rows(bm_ctx* ctx, SchedBufs& b, int32_t k, bool with_col) {
    BM_CUDA(ctx, cudaMemcpyAsync(b.d_rows, b.h_rows, sizeof(int32_t) * k, cudaMemcpyHostToDevice, ctx->stream));
    if (with_col)
        BM_CUDA(ctx, cudaMemcpyAsync(b.d_col, b.h_col, sizeof(int32_t) * k, cudaMemcpyHostToDevice, ctx->stream));
    bm_status s = bm_launch_rows(ctx, b.d_rows, with_col ? b.d_col : nullptr, k, nullptr, b.d_res, b.h_rows);
    if (s != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(b.h_res, b.d_res, sizeof(bm_row_result) * k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

bm_status apply_pairs(bm_ctx* ctx, SchedBufs& b, int32_t k) {
    BM_CUDA(ctx, cudaMemcpyAsync(b.d_pairs, b.h_pairs, sizeof(int32_t) * 2 * k, cudaMemcpyHostToDevice, ctx->stream));
    return bm_launch_apply(ctx, b.d_pairs, k);
}

bm_status verify_score(bm_ctx* ctx) { return bm_check_score(ctx); }

bm_status load_order(bm_ctx* ctx, const int32_t* row_order, int32_t nrows, std::vector<int32_t>& order) {
    const int32_t n = ctx->n;
    if (!row_order) {
        order.resize((size_t)n);
        for (int32_t i = 0; i < n; i++) order[(size_t)i] = i + 1;
        return BM_OK;
    }
    if (nrows <= 0) return bm_fail(ctx, BM_INVALID_ARG, "empty row order");
    order.assign(row_order, row_order + nrows);
    for (int32_t i = 0; i < nrows; i++)
        if (order[(size_t)i] < 1 || order[(size_t)i] > n)
            return bm_fail(ctx, BM_INVALID_ARG, "row_order[%d] = %d outside 1..%d", i, order[(size_t)i], n);
    return BM_OK;
}

}  // namespace

extern "C" bm_status bm_apply_swaps(bm_ctx* ctx, const int32_t* pairs, const int64_t* deltas, int32_t k) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 0 || (k > 0 && !pairs)) return bm_fail(ctx, BM_INVALID_ARG, "bad swap buffers");
    if (k == 0) return BM_OK;
    const int32_t n = ctx->n;
    BmMarks mk;
    mk.reset(n);
    for (int32_t i = 0; i < k; i++) {
        const int32_t a = pairs[2 * i], b = pairs[2 * i + 1];
        if (a < 1 || a > n || b < 1 || b > n) return bm_fail(ctx, BM_INVALID_ARG, "swap %d: id outside 1..%d", i, n);
        if (k > 1) {
            if (a == b) return bm_fail(ctx, BM_INVALID_ARG, "swap %d: a == b in a batch", i);
            if (mk.marked(a) || mk.marked(b))
                return bm_fail(ctx, BM_INVALID_ARG, "swap %d (%d,%d) is not independent of an earlier swap", i, a, b);
            mk.mark_closed(ctx, a);
            mk.mark_closed(ctx, b);
        }
    }
    SchedBufs bufs;
    if ((s = sched_bufs(ctx, k, &bufs)) != BM_OK) return s;
    memcpy(bufs.h_pairs, pairs, sizeof(int32_t) * 2 * (size_t)k);
    if ((s = apply_pairs(ctx, bufs, k)) != BM_OK) return s;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (deltas)
        for (int32_t i = 0; i < k; i++) ctx->score += deltas[i];
    return BM_OK;
}

extern "C" bm_status bm_sweep_parity(bm_ctx* ctx, const int32_t* row_order, int32_t nrows, int64_t max_accepts,
                                     int32_t max_sweeps, double time_budget_s, bm_progress* prog) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    std::vector<int32_t> order;
    if ((s = load_order(ctx, row_order, nrows, order)) != BM_OK) return s;
    const int32_t nr = (int32_t)order.size();
    const int32_t n = ctx->n;
    const int32_t kmax = std::max(1, std::min(nr, ctx->num_sms));
    SchedBufs b;
    if ((s = sched_bufs(ctx, kmax, &b)) != BM_OK) return s;
    if ((s = bm_rows_refresh_work(ctx)) != BM_OK) return s;

    const auto t0 = clk::now();
    int32_t pos = prog->next_row_pos, col = prog->next_col;
    if (pos < 0 || pos >= nr) pos = 0;
    if (col < 1 || col > n) col = 1;
    bool pass_full = (pos == 0 && col == 1);
    int64_t pass_accepts = 0, accepts0 = prog->accepts;
    int32_t K = 1;
    prog->converged = 0;
    bm_status ret = BM_OK;
    for (;;) {
        if (max_accepts >= 0 && prog->accepts - accepts0 >= max_accepts) break;
        if (time_budget_s > 0 && secs_since(t0) >= time_budget_s) { ret = BM_TIMEOUT; break; }
        const int32_t k = std::min(K, nr - pos);
        for (int32_t i = 0; i < k; i++) {
            b.h_rows[i] = order[(size_t)(pos + i)];
            b.h_col[i] = (i == 0) ? col : 1;
        }
        if ((s = eval_rows(ctx, b, k, true)) != BM_OK) return s;
        prog->launches++;
        prog->evaluated += (int64_t)k * (n - 1);
        int32_t hit = -1;
        for (int32_t i = 0; i < k; i++)
            if (b.h_res[i].first_pos != 0) { hit = i; break; }
        if (hit >= 0) {
            const int32_t u = b.h_res[hit].row, v = b.h_res[hit].first_pos;
            b.h_pairs[0] = u;
            b.h_pairs[1] = v;
            if ((s = apply_pairs(ctx, b, 1)) != BM_OK) return s;
            ctx->score += b.h_res[hit].first_delta;
            prog->accepts++;
            pass_accepts++;
            prog->rows_done += hit;
            pos += hit;
            col = v + 1;
            if (col > n) { pos++; col = 1; prog->rows_done++; }
            K = std::max(1, K / 2);
        } else {
            prog->rows_done += k;
            pos += k;
            col = 1;
            K = std::min(kmax, K * 2);
        }
        if (pos >= nr) {
            pos = 0;
            col = 1;
            if (pass_full) prog->sweeps++;
            if (pass_full && pass_accepts == 0) { prog->converged = 1; break; }
            pass_full = true;
            pass_accepts = 0;
            if (max_sweeps >= 0 && prog->sweeps >= max_sweeps) break;
        }
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->next_row_pos = pos;
    prog->next_col = col;
    prog->seconds += secs_since(t0);
    s = verify_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}

extern "C" bm_status bm_search_batched(bm_ctx* ctx, const int32_t* row_order, int32_t nrows, int32_t rows_per_batch,
                                       int64_t max_accepts, int32_t max_sweeps, double time_budget_s,
                                       int64_t target_score, bm_progress* prog) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    std::vector<int32_t> order;
    if ((s = load_order(ctx, row_order, nrows, order)) != BM_OK) return s;
    const int32_t nr = (int32_t)order.size();
    const int32_t n = ctx->n;
    int32_t R = rows_per_batch > 0 ? rows_per_batch : 2 * ctx->num_sms;
    R = std::min(R, nr);
    SchedBufs b;
    if ((s = sched_bufs(ctx, R, &b)) != BM_OK) return s;
    if ((s = bm_rows_refresh_work(ctx)) != BM_OK) return s;
    std::vector<int32_t> cand;
    BmMarks mk;
    const auto t0 = clk::now();
    int32_t pos = prog->next_row_pos;
    if (pos < 0 || pos >= nr) pos = 0;
    bool pass_full = (pos == 0);
    int64_t pass_accepts = 0, accepts0 = prog->accepts;
    prog->converged = 0;
    bm_status ret = BM_OK;
    for (;;) {
        if (max_accepts >= 0 && prog->accepts - accepts0 >= max_accepts) break;
        if (target_score > 0 && ctx->score >= target_score) break;
        if (time_budget_s > 0 && secs_since(t0) >= time_budget_s) { ret = BM_TIMEOUT; break; }
        const int32_t k = std::min(R, nr - pos);
        for (int32_t i = 0; i < k; i++) b.h_rows[i] = order[(size_t)(pos + i)];
        if ((s = eval_rows(ctx, b, k, false)) != BM_OK) return s;
        prog->launches++;
        prog->evaluated += (int64_t)k * (n - 1);
        cand.clear();
        for (int32_t i = 0; i < k; i++)
            if (b.h_res[i].best_delta > 0) cand.push_back(i);
        std::sort(cand.begin(), cand.end(), [&](int32_t x, int32_t y) {
            if (b.h_res[x].best_delta != b.h_res[y].best_delta) return b.h_res[x].best_delta > b.h_res[y].best_delta;
            return x < y;
        });
        mk.reset(n);
        int32_t na = 0;
        int64_t gain = 0;
        for (int32_t i : cand) {
            const int32_t u = b.h_res[i].row, v = b.h_res[i].best;
            if (mk.marked(u) || mk.marked(v)) continue;
            mk.mark_closed(ctx, u);
            mk.mark_closed(ctx, v);
            b.h_pairs[2 * na] = u;
            b.h_pairs[2 * na + 1] = v;
            gain += b.h_res[i].best_delta;
            na++;
        }
        if (na > 0) {
            if ((s = apply_pairs(ctx, b, na)) != BM_OK) return s;
            ctx->score += gain;
            prog->accepts += na;
            pass_accepts += na;
        }
        prog->rows_done += k;
        pos += k;
        if (pos >= nr) {
            pos = 0;
            if (pass_full) prog->sweeps++;
            if (pass_full && pass_accepts == 0) { prog->converged = 1; break; }
            pass_full = true;
            pass_accepts = 0;
            if (max_sweeps >= 0 && prog->sweeps >= max_sweeps) break;
        }
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->next_row_pos = pos;
    prog->next_col = 1;
    prog->seconds += secs_since(t0);
    s = verify_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}

// ------------------------------------------------------------- k-set moves

extern "C" bm_status bm_apply_sets(bm_ctx* ctx, int32_t k, const int32_t* sets, const int32_t* perms,
                                   const int64_t* deltas, int32_t nsets) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 2 || k > 8) return bm_fail(ctx, BM_INVALID_ARG, "k must be 2..8");
    if (nsets < 0 || (nsets > 0 && (!sets || !perms))) return bm_fail(ctx, BM_INVALID_ARG, "bad set buffers");
    if (nsets == 0) return BM_OK;
    const int32_t n = ctx->n;
    BmMarks mk;
    mk.reset(n);
    for (int32_t i = 0; i < nsets; i++) {
        int used = 0;
        for (int a = 0; a < k; a++) {
            const int32_t v = sets[(size_t)i * k + a], p = perms[(size_t)i * k + a];
            if (v < 1 || v > n) return bm_fail(ctx, BM_INVALID_ARG, "set %d: id outside 1..%d", i, n);
            if (p < 0 || p >= k || (used >> p & 1)) return bm_fail(ctx, BM_INVALID_ARG, "set %d: not a permutation", i);
            used |= 1 << p;
            for (int b = 0; b < a; b++)
                if (sets[(size_t)i * k + b] == v) return bm_fail(ctx, BM_INVALID_ARG, "set %d repeats vertex %d", i, v);
            if (mk.marked(v))
                return bm_fail(ctx, BM_INVALID_ARG, "set %d is not independent of an earlier set", i);
        }
        for (int a = 0; a < k; a++) mk.mark_closed(ctx, sets[(size_t)i * k + a]);
    }
    const size_t b1 = ((size_t)nsets * k * sizeof(int32_t) + 255) & ~(size_t)255;
    if ((s = bm_stage(ctx, 2 * b1)) != BM_OK) return s;
    int32_t* d_sets = (int32_t*)ctx->stage;
    int32_t* d_perms = (int32_t*)((char*)ctx->stage + b1);
    BM_CUDA(ctx, cudaMemcpyAsync(d_sets, sets, sizeof(int32_t) * (size_t)nsets * k, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_perms, perms, sizeof(int32_t) * (size_t)nsets * k, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_apply_sets(ctx, k, d_sets, d_perms, nsets)) != BM_OK) return s;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (deltas)
        for (int32_t i = 0; i < nsets; i++) ctx->score += deltas[i];
    return BM_OK;
}

namespace {

// Candidate sets for bm_search_ksets: k distinct random vertices (mode 0), or
// for k == 3 a path u - x - y of A (mode 1: x a neighbour of u, y a neighbour
// of x).  Counter-based, so a (seed, launch, set) triple fixes the set.
void draw_set(const bm_ctx* ctx, int32_t k, int32_t mode, uint64_t seed, uint64_t launch, uint64_t idx, int32_t* out) {
    const int32_t n = ctx->n;
    uint64_t ctr = (launch << 32) ^ idx;
    uint32_t word[4];
    int have = 0;
    auto next = [&]() -> uint32_t {
        if (have == 0) {
            const uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0x6B657473u, 0u};
            const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
            bm_philox4x32_10(c, key, word);
            ctr += 1;
            have = 4;
        }
        return word[--have];
    };
    auto neighbour = [&](int32_t v, int32_t* w) -> bool {
        const int32_t d_out = ctx->hA_optr[(size_t)v + 1] - ctx->hA_optr[(size_t)v];
        const int32_t d_in = ctx->hA_iptr[(size_t)v + 1] - ctx->hA_iptr[(size_t)v];
        if (d_out + d_in == 0) return false;
        for (int tries = 0; tries < 8; tries++) {
            const uint32_t r = next() % (uint32_t)(d_out + d_in);
            const uint32_t e = (int32_t)r < d_out ? ctx->hA_oent[(size_t)ctx->hA_optr[(size_t)v] + r]
                                                   : ctx->hA_ient[(size_t)ctx->hA_iptr[(size_t)v] + (r - d_out)];
            if (e != 0) { *w = bm_eid(e); return true; }
        }
        return false;
    };
    for (;;) {
        int32_t m = 0;
        if (mode == 1 && k == 3) {
            const int32_t u = 1 + (int32_t)(next() % (uint32_t)n);
            int32_t x, y;
            if (neighbour(u, &x) && neighbour(x, &y) && y != u && y != x) {
                out[0] = u; out[1] = x; out[2] = y;
                return;
            }
            continue;
        }
        while (m < k) {
            const int32_t v = 1 + (int32_t)(next() % (uint32_t)n);
            bool dup = false;
            for (int32_t j = 0; j < m; j++) dup |= out[j] == v;
            if (!dup) out[m++] = v;
        }
        return;
    }
}

}  // namespace

extern "C" bm_status bm_search_ksets(bm_ctx* ctx, int32_t k, int32_t sets_per_launch, int32_t mode, uint64_t seed,
                                     int64_t max_launches, double time_budget_s, bm_progress* prog) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if (k < 2 || k > 8) return bm_fail(ctx, BM_INVALID_ARG, "k must be 2..8");
    if (mode == 1 && k != 3) return bm_fail(ctx, BM_INVALID_ARG, "path sets need k == 3");
    if (sets_per_launch < 1 || ctx->n < k) return bm_fail(ctx, BM_INVALID_ARG, "need sets_per_launch >= 1 and n >= k");
    const int64_t S = sets_per_launch;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t b_sets = al(sizeof(int32_t) * (size_t)(S * k)), b_best = al(sizeof(long long) * (size_t)S);
    const size_t total = 2 * b_sets + b_best + 256;
    if ((s = bm_stage(ctx, total)) != BM_OK) return s;
    if ((s = bm_hstage(ctx, total)) != BM_OK) return s;
    char* d = (char*)ctx->stage;
    char* h = (char*)ctx->hstage;
    int32_t* d_sets = (int32_t*)d;
    int32_t* d_perm = (int32_t*)(d + b_sets);
    long long* d_best = (long long*)(d + 2 * b_sets);
    int32_t* d_stat = (int32_t*)(d + 2 * b_sets + b_best);
    int32_t* h_sets = (int32_t*)h;
    int32_t* h_perm = (int32_t*)(h + b_sets);
    long long* h_best = (long long*)(h + 2 * b_sets);
    std::vector<int32_t> order((size_t)S), ap_sets, ap_perms;
    BmMarks mk;
    const auto t0 = clk::now();
    bm_status ret = BM_OK;
    for (int64_t l = 0; max_launches < 0 || l < max_launches; l++) {
        if (time_budget_s > 0 && secs_since(t0) >= time_budget_s) { ret = BM_TIMEOUT; break; }
        const uint64_t launch = (uint64_t)prog->launches;
        for (int64_t i = 0; i < S; i++) draw_set(ctx, k, mode, seed, launch, (uint64_t)i, h_sets + i * k);
        BM_CUDA(ctx, cudaMemcpyAsync(d_sets, h_sets, sizeof(int32_t) * (size_t)(S * k), cudaMemcpyHostToDevice, ctx->stream));
        BM_CUDA(ctx, cudaMemsetAsync(d_stat, 0, sizeof(int32_t), ctx->stream));
        if ((s = bm_launch_kset(ctx, k, d_sets, S, d_best, d_perm, nullptr, d_stat)) != BM_OK) return s;
        BM_CUDA(ctx, cudaMemcpyAsync(h_best, d_best, sizeof(long long) * (size_t)S, cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(h_perm, d_perm, sizeof(int32_t) * (size_t)(S * k), cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        prog->launches++;
        int64_t fact = 1;
        for (int i = 2; i <= k; i++) fact *= i;
        prog->evaluated += S * fact;
        // greedy independent subset of the improving sets
        int32_t cnt = 0;
        for (int64_t i = 0; i < S; i++)
            if (h_best[i] > 0) order[(size_t)cnt++] = (int32_t)i;
        std::sort(order.begin(), order.begin() + cnt, [&](int32_t x, int32_t y) {
            if (h_best[x] != h_best[y]) return h_best[x] > h_best[y];
            return x < y;
        });
        mk.reset(ctx->n);
        ap_sets.clear();
        ap_perms.clear();
        int64_t gain = 0;
        for (int32_t c = 0; c < cnt; c++) {
            const int32_t i = order[(size_t)c];
            bool free_ = true;
            for (int a = 0; a < k; a++) free_ &= !mk.marked(h_sets[i * k + a]);
            if (!free_) continue;
            for (int a = 0; a < k; a++) {
                mk.mark_closed(ctx, h_sets[i * k + a]);
                ap_sets.push_back(h_sets[i * k + a]);
                ap_perms.push_back(h_perm[i * k + a]);
            }
            gain += h_best[i];
        }
        const int32_t na = (int32_t)(ap_sets.size() / (size_t)k);
        if (na > 0) {
            BM_CUDA(ctx, cudaMemcpyAsync(d_sets, ap_sets.data(), sizeof(int32_t) * ap_sets.size(), cudaMemcpyHostToDevice, ctx->stream));
            BM_CUDA(ctx, cudaMemcpyAsync(d_perm, ap_perms.data(), sizeof(int32_t) * ap_perms.size(), cudaMemcpyHostToDevice, ctx->stream));
            if ((s = bm_launch_apply_sets(ctx, k, d_sets, d_perm, na)) != BM_OK) return s;
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            ctx->score += gain;
            prog->accepts += na;
        }
    }
    prog->seconds += secs_since(t0);
    s = verify_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}

// ------------------------------------------------------------- perturbation

// k disjoint swaps selected[i] <-> selected[i+k] over 2k distinct vertices, as
// random_swap_k_vertices (src/graph-re-alignment-gpu.cu:763-810; weighted
// variant src/graph-re-alignment-gpu-swap.cu:767-887): the first k vertices
// uniformly (mode 0) or with probability proportional to 7 * out-weight +
// 3 * in-weight of A (mode 1, the reference's 0.7/0.3 score in integers), the
// next k uniformly.  Draws come from Philox4x32-10 keyed by seed with
// `counter` as the stream position, instead of rand() seeded by the clock.
// Each swap's exact delta is computed and the swap applied in stream order,
// so the tracked score stays exact.
extern "C" bm_status bm_perturb(bm_ctx* ctx, int32_t k, int32_t mode, uint64_t seed, uint64_t counter,
                                int32_t* changed, int64_t* total_delta) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    const int32_t n = ctx->n;
    if (k < 1 || 2 * (int64_t)k > n) return bm_fail(ctx, BM_INVALID_ARG, "need 1 <= k and 2k <= n");
    if (mode != 0 && mode != 1) return bm_fail(ctx, BM_INVALID_ARG, "mode must be 0 (uniform) or 1 (weighted)");
    std::vector<int32_t> sel;
    std::vector<char> used((size_t)n + 1, 0);
    uint32_t word[4];
    int have = 0;
    uint64_t ctr = counter;
    auto next = [&]() -> uint32_t {
        if (have == 0) {
            const uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0x70657274u, 0u};
            const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
            bm_philox4x32_10(c, key, word);
            ctr++;
            have = 4;
        }
        return word[--have];
    };
    if (mode == 1) {
        std::vector<int64_t> cum((size_t)n + 1, 0);
        for (int32_t v = 1; v <= n; v++) {
            int64_t ow = 0, iw = 0;
            for (int32_t j = ctx->hA_optr[(size_t)v]; j < ctx->hA_optr[(size_t)v + 1]; j++) ow += bm_ew(ctx->hA_oent[(size_t)j]);
            for (int32_t j = ctx->hA_iptr[(size_t)v]; j < ctx->hA_iptr[(size_t)v + 1]; j++) iw += bm_ew(ctx->hA_ient[(size_t)j]);
            cum[(size_t)v] = cum[(size_t)v - 1] + 7 * ow + 3 * iw;
        }
        const int64_t total = cum[(size_t)n];
        while ((int32_t)sel.size() < k) {
            int32_t v;
            if (total > 0) {
                const uint64_t r64 = ((uint64_t)next() << 32) | next();
                const int64_t r = (int64_t)(r64 % (uint64_t)total);
                v = (int32_t)(std::upper_bound(cum.begin() + 1, cum.end(), r) - cum.begin());
            } else {
                v = 1 + (int32_t)(next() % (uint32_t)n);
            }
            if (used[(size_t)v]) {
                // weights of used vertices stay in the table; step to the next unused one
                int32_t w = v;
                do { w = w % n + 1; } while (used[(size_t)w]);
                v = w;
            }
            used[(size_t)v] = 1;
            sel.push_back(v);
        }
    }
    while ((int32_t)sel.size() < 2 * k) {
        const int32_t v = 1 + (int32_t)(next() % (uint32_t)n);
        if (used[(size_t)v]) continue;
        used[(size_t)v] = 1;
        sel.push_back(v);
    }
    const size_t pb = ((size_t)k * 2 * sizeof(int32_t) + 255) & ~(size_t)255;
    if ((s = bm_stage(ctx, pb + sizeof(int64_t) * (size_t)k)) != BM_OK) return s;
    int32_t* d_pairs = (int32_t*)ctx->stage;
    int64_t* d_delta = (int64_t*)((char*)ctx->stage + pb);
    std::vector<int32_t> pairs((size_t)2 * k);
    for (int32_t i = 0; i < k; i++) {
        pairs[(size_t)2 * i] = sel[(size_t)i];
        pairs[(size_t)2 * i + 1] = sel[(size_t)i + k];
    }
    BM_CUDA(ctx, cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(int32_t) * 2 * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    for (int32_t i = 0; i < k; i++) {
        // the swaps are applied whatever their deltas: score differences keep the tracked score
        if ((s = bm_launch_pairs(ctx, d_pairs + 2 * i, 1, d_delta + i, true)) != BM_OK) return s;
        if ((s = bm_launch_apply(ctx, d_pairs + 2 * i, 1)) != BM_OK) return s;
    }
    std::vector<int64_t> deltas((size_t)k);
    BM_CUDA(ctx, cudaMemcpyAsync(deltas.data(), d_delta, sizeof(int64_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int64_t sum = 0;
    for (int64_t d : deltas) sum += d;
    ctx->score += sum;
    if (changed)
        for (int32_t i = 0; i < 2 * k; i++) changed[i] = sel[(size_t)i];
    if (total_delta) *total_delta = sum;
    return BM_OK;
}

// Batched search with perturbation restarts, the driver pattern of
// src/graph-re-alignment-gpu.cu:1004-1028: when a pass finds no improving swap,
// perturb with k swaps and continue; the best mapping seen is kept and restored
// at the end.
extern "C" bm_status bm_search_restarts(bm_ctx* ctx, const int32_t* row_order, int32_t nrows, int32_t rows_per_batch,
                                        int32_t k_perturb, int32_t mode, uint64_t seed, int32_t max_restarts,
                                        double time_budget_s, bm_progress* prog, int64_t* best_score) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    const auto t0 = clk::now();
    std::vector<int32_t> best_pi((size_t)ctx->n + 1);
    int64_t best = ctx->score;
    BM_CUDA(ctx, cudaMemcpy(best_pi.data(), ctx->pi, sizeof(int32_t) * best_pi.size(), cudaMemcpyDeviceToHost));
    bm_status ret = BM_OK;
    for (int32_t r = 0;; r++) {
        const double left = time_budget_s > 0 ? time_budget_s - secs_since(t0) : 0;
        if (time_budget_s > 0 && left <= 0) { ret = BM_TIMEOUT; break; }
        bm_progress p = *prog;
        p.next_row_pos = 0;
        p.converged = 0;
        s = bm_search_batched(ctx, row_order, nrows, rows_per_batch, -1, -1, left, 0, &p);
        const double secs = prog->seconds;
        *prog = p;
        prog->seconds = secs;
        if (s == BM_TIMEOUT) { ret = BM_TIMEOUT; }
        else if (s != BM_OK) return s;
        if (ctx->score > best) {
            best = ctx->score;
            BM_CUDA(ctx, cudaMemcpy(best_pi.data(), ctx->pi, sizeof(int32_t) * best_pi.size(), cudaMemcpyDeviceToHost));
        }
        if (ret == BM_TIMEOUT || r >= max_restarts) break;
        if ((s = bm_perturb(ctx, k_perturb, mode, seed, (uint64_t)r << 20, nullptr, nullptr)) != BM_OK) return s;
    }
    if (ctx->score != best) {
        // restore the best mapping seen
        best_pi[0] = 0;
        if ((s = bm_set_mapping(ctx, best_pi.data())) != BM_OK) return s;
    }
    prog->score = ctx->score;
    prog->seconds += secs_since(t0);
    if (best_score) *best_score = best;
    return ret;
}

// The deterministic selection every rank of a sharded search runs on the same
// gathered candidate list: descending delta, then ascending position in the
// list; a candidate is taken when neither endpoint lies in the closed A
// neighbourhood of an endpoint already taken.
extern "C" bm_status bm_select_independent(bm_ctx* ctx, const int32_t* pairs, const int64_t* deltas, int32_t count,
                                           int32_t* chosen, int32_t* nchosen) {
    if (!ctx || count < 0 || (count > 0 && (!pairs || !deltas || !chosen)) || !nchosen) return BM_INVALID_ARG;
    if (!ctx->g[0].loaded) return bm_fail(ctx, BM_INVALID_ARG, "graph A not set");
    const int32_t n = ctx->n;
    std::vector<int32_t> order;
    for (int32_t i = 0; i < count; i++) {
        if (pairs[2 * i] < 1 || pairs[2 * i] > n || pairs[2 * i + 1] < 1 || pairs[2 * i + 1] > n)
            return bm_fail(ctx, BM_INVALID_ARG, "candidate %d: id outside 1..%d", i, n);
        if (deltas[i] > 0 && pairs[2 * i] != pairs[2 * i + 1]) order.push_back(i);
    }
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return deltas[a] > deltas[b]; });
    BmMarks mk;
    mk.reset(n);
    int32_t c = 0;
    for (int32_t i : order) {
        const int32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (mk.marked(u) || mk.marked(v)) continue;
        mk.mark_closed(ctx, u);
        mk.mark_closed(ctx, v);
        chosen[c++] = i;
    }
    *nchosen = c;
    return BM_OK;
}

// ------------------------------------------------ similarity-filtered pass
//
// The single pass of optimize_mapping in the reference's graph-alignment
// variant (src/graph-alignment.c:489-595): m1 and m2 run over the vertex list
// nodes[] (the variant's order of first appearance); the swap (m1, m2) is
// evaluated only when the similarity of the swapped images beats the current
// one (:545-553), and a positive delta is applied at once.  The engine
// evaluates K consecutive rows at a time under the current mapping (the row
// kernel, whole rows), then one CTA per row finds the first position p (from
// the row's start position on) whose vertex passes the filter with a positive
// delta; rows before the first row with such a position are what the serial
// pass scanned, that position is its next accept, and the rest is evaluated
// again after the swap (as bm_sweep_parity).  The similarity is computed in
// FP64 with the variant's operations in its order, each rounded on its own
// (no fused multiply-add), so the decisions are the variant's.

namespace {

constexpr int kSimThreads = 256;

// calculate_node_similarity (src/graph-alignment.c:274-284): -(0.7 x (5|d in|
// + 5|d out| + |d avg in| + |d avg out|) + 0.3 x |d rank|); a, b: five
// metrics (in, out, avg in, avg out, rank).
__device__ __forceinline__ double node_similarity(const double* a, const double* b) {
    double s = __dmul_rn(5.0, fabs(__dsub_rn(a[0], b[0])));
    s = __dadd_rn(s, __dmul_rn(5.0, fabs(__dsub_rn(a[1], b[1]))));
    s = __dadd_rn(s, fabs(__dsub_rn(a[2], b[2])));
    s = __dadd_rn(s, fabs(__dsub_rn(a[3], b[3])));
    const double o = fabs(__dsub_rn(a[4], b[4]));
    return -__dadd_rn(__dmul_rn(0.7, s), __dmul_rn(0.3, o));
}

// Per row r (u = rows[r]): the first position p >= start[r] of nodes[] with
// v = nodes[p] != u, delta(u, v) > 0 and the similarity filter passed; out_pos
// gets p (or nnodes when none), out_delta its delta.
__global__ void __launch_bounds__(kSimThreads) sim_first_kernel(const int64_t* __restrict__ full, int32_t n,
                                                                const int32_t* __restrict__ rows,
                                                                const int32_t* __restrict__ start,
                                                                const int32_t* __restrict__ nodes, int32_t nnodes,
                                                                const int32_t* __restrict__ pi,
                                                                const double* __restrict__ ma,
                                                                const double* __restrict__ mb, int32_t* out_pos,
                                                                long long* out_delta) {
    __shared__ int32_t s_best;
    const int r = blockIdx.x;
    const int32_t u = rows[r];
    const int64_t* row = full + (size_t)r * ((size_t)n + 1);
    const int32_t f1 = pi[u];
    if (threadIdx.x == 0) s_best = nnodes;
    __syncthreads();
    // positions in blocks of the CTA's width, so the first hit ends the scan
    for (int32_t p0 = start[r]; p0 < nnodes; p0 += kSimThreads) {
        const int32_t p = p0 + (int32_t)threadIdx.x;
        if (p < nnodes) {
            const int32_t v = nodes[p];
            if (v != u && row[v] > 0) {
                const int32_t f2 = pi[v];
                const double cur = __dadd_rn(node_similarity(ma + 5 * (size_t)u, mb + 5 * (size_t)f1),
                                             node_similarity(ma + 5 * (size_t)v, mb + 5 * (size_t)f2));
                const double swp = __dadd_rn(node_similarity(ma + 5 * (size_t)u, mb + 5 * (size_t)f2),
                                             node_similarity(ma + 5 * (size_t)v, mb + 5 * (size_t)f1));
                if (swp > cur) atomicMin(&s_best, p);
            }
        }
        __syncthreads();
        if (s_best < nnodes) break;
    }
    if (threadIdx.x == 0) {
        const int32_t p = s_best;
        out_pos[r] = p;
        out_delta[r] = p < nnodes ? (long long)row[nodes[p]] : 0;
    }
}

}  // namespace

extern "C" bm_status bm_sweep_similarity(bm_ctx* ctx, const int32_t* nodes, int32_t nnodes, const double* metrics_a,
                                         const double* metrics_b, int64_t max_accepts, double time_budget_s,
                                         bm_progress* prog) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog || !nodes || !metrics_a || !metrics_b || nnodes < 1)
        return bm_fail(ctx, BM_INVALID_ARG, "vertex list, metrics and progress are required");
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    const int32_t n = ctx->n;
    if (nnodes > n) return bm_fail(ctx, BM_INVALID_ARG, "%d listed vertices for n = %d", nnodes, n);
    {
        std::vector<char> seen((size_t)n + 1, 0);
        for (int32_t i = 0; i < nnodes; i++) {
            const int32_t v = nodes[i];
            if (v < 1 || v > n || seen[(size_t)v]) return bm_fail(ctx, BM_INVALID_ARG, "nodes[%d] = %d: bad or repeated", i, v);
            seen[(size_t)v] = 1;
        }
    }
    const int32_t kmax = std::max(1, std::min(nnodes, ctx->num_sms));
    // device copies: the list, both metric tables, whole rows and the per-row answers
    const size_t nb = ((size_t)nnodes * 4 + 255) & ~(size_t)255;
    const size_t mbytes = sizeof(double) * 5 * ((size_t)n + 1);
    const size_t fb = sizeof(int64_t) * (size_t)kmax * ((size_t)n + 1);
    const size_t small = 4 * (((size_t)kmax * 8 + 255) & ~(size_t)255);
    void* dev = nullptr;
    BM_CUDA(ctx, bm_cuda_malloc(&dev, nb + 2 * mbytes + fb + small));
    struct Free {
        void* p;
        ~Free() { bm_cuda_free(p); }
    } guard{dev};
    char* d = static_cast<char*>(dev);
    int32_t* d_nodes = reinterpret_cast<int32_t*>(d);
    double* d_ma = reinterpret_cast<double*>(d + nb);
    double* d_mb = reinterpret_cast<double*>(d + nb + mbytes);
    int64_t* d_full = reinterpret_cast<int64_t*>(d + nb + 2 * mbytes);
    char* sm = d + nb + 2 * mbytes + fb;
    const size_t sstep = ((size_t)kmax * 8 + 255) & ~(size_t)255;
    int32_t* d_rows = reinterpret_cast<int32_t*>(sm);
    int32_t* d_start = reinterpret_cast<int32_t*>(sm + sstep);
    int32_t* d_pos = reinterpret_cast<int32_t*>(sm + 2 * sstep);
    long long* d_delta = reinterpret_cast<long long*>(sm + 3 * sstep);
    BM_CUDA(ctx, cudaMemcpyAsync(d_nodes, nodes, sizeof(int32_t) * (size_t)nnodes, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_ma, metrics_a, mbytes, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_mb, metrics_b, mbytes, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_rows_refresh_work(ctx)) != BM_OK) return s;
    std::vector<int32_t> h_rows((size_t)kmax), h_start((size_t)kmax), h_pos((size_t)kmax);
    std::vector<long long> h_delta((size_t)kmax);
    const auto t0 = clk::now();
    int32_t pos = prog->next_row_pos, col = prog->next_col;  // row position; column position (0-based)
    if (pos < 0 || pos >= nnodes) pos = 0;
    if (col < 0 || col >= nnodes) col = 0;
    int64_t accepts0 = prog->accepts;
    int32_t K = 1;
    prog->converged = 0;
    bm_status ret = BM_OK;
    while (pos < nnodes) {
        if (max_accepts >= 0 && prog->accepts - accepts0 >= max_accepts) break;
        if (time_budget_s > 0 && secs_since(t0) >= time_budget_s) { ret = BM_TIMEOUT; break; }
        const int32_t k = std::min(K, nnodes - pos);
        for (int32_t i = 0; i < k; i++) {
            h_rows[(size_t)i] = nodes[pos + i];
            h_start[(size_t)i] = (i == 0) ? col : 0;
        }
        BM_CUDA(ctx, cudaMemcpyAsync(d_rows, h_rows.data(), sizeof(int32_t) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(d_start, h_start.data(), sizeof(int32_t) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
        if ((s = bm_launch_rows(ctx, d_rows, nullptr, k, d_full, nullptr, h_rows.data())) != BM_OK) return s;
        sim_first_kernel<<<k, kSimThreads, 0, ctx->stream>>>(d_full, n, d_rows, d_start, d_nodes, nnodes, ctx->pi, d_ma,
                                                             d_mb, d_pos, d_delta);
        BM_LAUNCH_CHECK(ctx, "sim_first_kernel");
        BM_CUDA(ctx, cudaMemcpyAsync(h_pos.data(), d_pos, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(h_delta.data(), d_delta, sizeof(long long) * (size_t)k, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        prog->launches++;
        prog->evaluated += (int64_t)k * (n - 1);
        int32_t hit = -1;
        for (int32_t i = 0; i < k; i++)
            if (h_pos[(size_t)i] < nnodes) { hit = i; break; }
        if (hit >= 0) {
            const int32_t u = h_rows[(size_t)hit], p = h_pos[(size_t)hit], v = nodes[p];
            const int32_t pr[2] = {u, v};
            BM_CUDA(ctx, cudaMemcpyAsync(d_rows, pr, sizeof pr, cudaMemcpyHostToDevice, ctx->stream));
            if ((s = bm_launch_apply(ctx, d_rows, 1)) != BM_OK) return s;
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            ctx->score += h_delta[(size_t)hit];
            prog->accepts++;
            prog->rows_done += hit;
            pos += hit;
            col = p + 1;
            if (col >= nnodes) { pos++; col = 0; prog->rows_done++; }
            K = std::max(1, K / 2);
        } else {
            prog->rows_done += k;
            pos += k;
            col = 0;
            K = std::min(kmax, K * 2);
        }
    }
    if (pos >= nnodes) { prog->sweeps++; pos = 0; col = 0; }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->next_row_pos = pos;
    prog->next_col = col;
    prog->seconds += secs_since(t0);
    s = verify_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}
