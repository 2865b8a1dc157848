// bm_assign.cu — re-assignment of an A-independent vertex subset by an optimal
// linear assignment: the method of src/independent-hungarian/hungarianSubset.c
// (random independent subset :657-740, one-sided gains one_side_swap_delta
// :414-459, optimal_assignment with the Hungarian method hungarian.c:144-334,
// apply and re-score :760-795).
//
// For a subset T = {t_0..t_{k-1}} with no A edge between two members, the
// score change of giving each t_i the old image of t_sigma(i) is exactly
// sum_i c[i][sigma(i)] with c[i][j] = G_{t_i}(pi t_j) - S(t_i) (+ self-loop
// terms), G_u(f) = sum over u's A entries of min(w, B at f and the neighbour's
// image): every A edge touches at most one member, so the moves do not
// interact.  The reference skips self-loops in the gains and re-scores; here
// they are included, so the delta is exact.
//
// On the device: the gains of a member against all images come from the row
// kernel in its one-sided mode (the first two 2-hop terms only), read at the
// members' columns; the assignment is solved by the auction algorithm
// (Bertsekas) with epsilon scaling on benefits multiplied by k + 1, which makes
// the final epsilon = 1 phase exactly optimal for integer benefits, in one CTA
// with prices, bids and owners in shared memory; apply_perm_kernel then moves
// every changed member at once (S updates of its A entries, relabelled B
// entries naming its new image, pi and pi^-1).
#include <algorithm>
#include <chrono>
#include <climits>
#include <numeric>
#include <vector>

#include "bm_internal.cuh"
#include "bm_rng.hpp"

namespace {

constexpr int kLapThreads = 1024;
constexpr int kLapMaxK = 4096;
constexpr int kLapIdBits = 13;  // person index in a bid key (k <= 4096 < 2^13)
constexpr int kPermThreads = 256;

// Bounded auction: `limit` SM clock cycles at most (by default kAuctionLimit,
// ~10 s); status 1 means it ran out.
constexpr long long kAuctionLimit = 20000000000ll;
__global__ void __launch_bounds__(kLapThreads) auction_kernel(const int32_t* __restrict__ a, int32_t k, long long eps0,
                                                              int32_t* __restrict__ assign, int32_t* __restrict__ status,
                                                              long long limit) {
    extern __shared__ unsigned long long lsm[];
    long long* price = reinterpret_cast<long long*>(lsm);
    unsigned long long* bid = lsm + k;
    int32_t* owner = reinterpret_cast<int32_t*>(lsm + 2 * k);
    int32_t* pobj = owner + k;
    int32_t* ulist = pobj + k;
    __shared__ int32_t s_nu;
    __shared__ int32_t s_fail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long scale = (long long)k + 1;
    const long long t0 = clock64();
    for (int32_t j = tid; j < k; j += kLapThreads) price[j] = 0;
    if (tid == 0) s_fail = 0;
    long long eps = eps0;
    for (;;) {  // epsilon phases
        for (int32_t i = tid; i < k; i += kLapThreads) { pobj[i] = -1; owner[i] = -1; }
        __syncthreads();
        for (;;) {  // auction rounds
            if (tid == 0) s_nu = 0;
            __syncthreads();
            for (int32_t i = tid; i < k; i += kLapThreads)
                if (pobj[i] < 0) ulist[atomicAdd(&s_nu, 1)] = i;
            for (int32_t j = tid; j < k; j += kLapThreads) bid[j] = 0ull;
            if (tid == 0 && clock64() - t0 > limit) s_fail = 1;
            __syncthreads();
            const int32_t nu = s_nu;
            if (nu == 0 || s_fail) break;
            // every unassigned person bids for its best object
            for (int32_t q = warp; q < nu; q += kLapThreads / 32) {
                const int32_t i = ulist[q];
                const int32_t* row = a + (size_t)i * (size_t)k;
                long long v1 = LLONG_MIN, v2 = LLONG_MIN;
                int32_t j1 = INT_MAX;
                for (int32_t j = lane; j < k; j += 32) {
                    const long long v = (long long)row[j] * scale - price[j];
                    if (v > v1) { v2 = v1; v1 = v; j1 = j; }
                    else if (v > v2) v2 = v;
                }
                for (int o = 16; o; o >>= 1) {
                    const long long ov1 = __shfl_xor_sync(0xffffffffu, v1, o);
                    const long long ov2 = __shfl_xor_sync(0xffffffffu, v2, o);
                    const int32_t oj1 = __shfl_xor_sync(0xffffffffu, j1, o);
                    if (ov1 > v1 || (ov1 == v1 && oj1 < j1)) {
                        v2 = max(v1, ov2);
                        v1 = ov1;
                        j1 = oj1;
                    } else {
                        v2 = max(v2, ov1);
                    }
                }
                if (lane == 0) {
                    if (v2 == LLONG_MIN) v2 = v1;  // a single object
                    const long long b = price[j1] + (v1 - v2) + eps;
                    if (b >= (1ll << (63 - kLapIdBits))) {
                        s_fail = 1;
                    } else {
                        const unsigned long long key = ((unsigned long long)b << kLapIdBits) |
                                                       (unsigned long long)((1 << kLapIdBits) - 1 - i);
                        atomicMax(&bid[j1], key);
                    }
                }
            }
            __syncthreads();
            // objects go to their highest bidder (the lowest person on ties)
            for (int32_t j = tid; j < k; j += kLapThreads) {
                const unsigned long long key = bid[j];
                if (!key) continue;
                const int32_t i = (1 << kLapIdBits) - 1 - (int32_t)(key & ((1ull << kLapIdBits) - 1));
                price[j] = (long long)(key >> kLapIdBits);
                const int32_t old = owner[j];
                if (old >= 0) pobj[old] = -1;
                owner[j] = i;
                pobj[i] = j;
            }
            __syncthreads();
        }
        if (s_fail || eps == 1) break;
        eps = max(1ll, eps / 5);
        __syncthreads();
    }
    __syncthreads();
    for (int32_t i = tid; i < k; i += kLapThreads) assign[i] = pobj[i];
    if (tid == 0) *status = s_fail;
}

struct PermArgs {
    GView A;
    const int32_t* Bout_ptr;
    const int32_t* Bin_ptr;
    uint32_t* Bout_ent;
    uint32_t* Bin_ent;
    const int32_t* Bout_twin;
    const int32_t* Bin_twin;
    HashView hb;
    int32_t* pi;
    int32_t* pinv;
    int32_t* ov;
    int4* ximg;
};

// One CTA per moved member u: old image g0, new image g1.  Members share no A
// edge, so every neighbour's image is fixed while the members move.
__global__ void __launch_bounds__(kPermThreads) apply_perm_kernel(PermArgs a, const int32_t* __restrict__ who,
                                                                  const int32_t* __restrict__ old_img,
                                                                  const int32_t* __restrict__ new_img) {
    const int32_t u = who[blockIdx.x], g0 = old_img[blockIdx.x], g1 = new_img[blockIdx.x];
    if (g0 == g1) return;
    for (int32_t j = a.A.out_ptr[u] + threadIdx.x; j < a.A.out_ptr[u + 1]; j += kPermThreads) {
        const uint32_t ent = a.A.out_ent[j];
        if (ent == 0) continue;
        const int32_t x = bm_eid(ent), w = bm_ew(ent);
        const int32_t gx = a.pi[x];
        const int32_t d = imin(w, bm_hash_get(a.hb, g1, gx)) - imin(w, bm_hash_get(a.hb, g0, gx));
        if (d) { atomicAdd(a.ov + u, d); atomicAdd(a.ov + x, d); }
    }
    for (int32_t j = a.A.in_ptr[u] + threadIdx.x; j < a.A.in_ptr[u + 1]; j += kPermThreads) {
        const uint32_t ent = a.A.in_ent[j];
        if (ent == 0) continue;
        const int32_t x = bm_eid(ent), w = bm_ew(ent);
        const int32_t gx = a.pi[x];
        const int32_t d = imin(w, bm_hash_get(a.hb, gx, g1)) - imin(w, bm_hash_get(a.hb, gx, g0));
        if (d) { atomicAdd(a.ov + u, d); atomicAdd(a.ov + x, d); }
    }
    // B entries naming the new image now name u (found through the twins)
    for (int dir = 0; dir < 2; dir++) {
        const int32_t* ptr = dir ? a.Bout_ptr : a.Bin_ptr;
        const int32_t* twin = dir ? a.Bout_twin : a.Bin_twin;
        uint32_t* other = dir ? a.Bin_ent : a.Bout_ent;
        for (int32_t j = ptr[g1] + threadIdx.x; j < ptr[g1 + 1]; j += kPermThreads) {
            const int32_t t = twin[j];
            if (t < 0) continue;
            other[t] = (other[t] & ~BM_ID_MASK) | (uint32_t)u;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a.pi[u] = g1;
        a.pinv[g1] = u;
        a.ximg[u] = bm_image_bounds(a.Bin_ptr, a.Bout_ptr, g1);
    }
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t lap_smem(int32_t k) { return (size_t)k * (8 + 8 + 4 + 4 + 4); }

bm_status lap_device(bm_ctx* ctx, const int32_t* d_a, int32_t k, int32_t* d_assign, int32_t* d_status,
                     long long max_abs) {
    const size_t smem = lap_smem(k);
    BM_CUDA(ctx, cudaFuncSetAttribute(auction_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long c = std::max(1ll, max_abs) * ((long long)k + 1);
    const long long eps0 = std::max(1ll, c / 5);
    auction_kernel<<<1, kLapThreads, smem, ctx->stream>>>(d_a, k, eps0, d_assign, d_status,
                                                          ctx->wait_limit > 0 ? (long long)ctx->wait_limit
                                                                              : kAuctionLimit);
    BM_LAUNCH_CHECK(ctx, "auction_kernel");
    return BM_OK;
}

// Subset checks: ids in 1..n, distinct, no A edge between two members.
bm_status check_subset(bm_ctx* ctx, const int32_t* subset, int32_t k, BmMarks& mk) {
    mk.reset(ctx->n);
    for (int32_t i = 0; i < k; i++)
        if (subset[i] < 1 || subset[i] > ctx->n)
            return bm_fail(ctx, BM_INVALID_ARG, "subset[%d] = %d outside 1..%d", i, subset[i], ctx->n);
    for (int32_t i = 0; i < k; i++) {
        if (mk.marked(subset[i]))
            return bm_fail(ctx, BM_INVALID_ARG, "subset[%d] = %d repeats or shares an A edge with another member", i,
                           subset[i]);
        mk.mark_closed(ctx, subset[i]);
    }
    return BM_OK;
}

// Gains, assignment and apply for a checked subset; *delta, *changed.
bm_status assign_subset(bm_ctx* ctx, const int32_t* subset, int32_t k, int64_t* delta, int32_t* changed) {
    const size_t sb = al256(sizeof(int32_t) * (size_t)k), cb = al256(sizeof(int32_t) * (size_t)k * (size_t)k);
    bm_status s;
    if ((s = bm_stage(ctx, 5 * sb + cb + 256)) != BM_OK) return s;
    char* base = (char*)ctx->stage;
    int32_t* d_sub = (int32_t*)base;
    int32_t* d_asg = (int32_t*)(base + sb);
    int32_t* d_old = (int32_t*)(base + 2 * sb);
    int32_t* d_new = (int32_t*)(base + 3 * sb);
    int32_t* d_who = (int32_t*)(base + 4 * sb);
    int32_t* d_cost = (int32_t*)(base + 5 * sb);
    int32_t* d_status = (int32_t*)(base + 5 * sb + cb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_sub, subset, sizeof(int32_t) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_rows_gen(ctx, d_sub, nullptr, k, nullptr, nullptr, nullptr, 0, 0, d_sub, k, d_cost)) != BM_OK)
        return s;
    // the largest |gain|, for the first epsilon
    std::vector<int32_t> cost((size_t)k * (size_t)k);
    BM_CUDA(ctx, cudaMemcpyAsync(cost.data(), d_cost, sizeof(int32_t) * cost.size(), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    long long mx = 1;
    for (int32_t c : cost) mx = std::max(mx, (long long)(c < 0 ? -(long long)c : c));
    if ((s = lap_device(ctx, d_cost, k, d_asg, d_status, mx)) != BM_OK) return s;
    std::vector<int32_t> asg((size_t)k), old((size_t)k), pi((size_t)ctx->n + 1);
    int32_t status = 0;
    BM_CUDA(ctx, cudaMemcpyAsync(asg.data(), d_asg, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(&status, d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(pi.data(), ctx->pi, sizeof(int32_t) * pi.size(), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int32_t i = 0; i < k; i++) old[(size_t)i] = pi[(size_t)subset[i]];  // old images of the members
    if (status) return bm_fail(ctx, BM_TIMEOUT, "auction did not finish within its bound");
    std::vector<int32_t> who, o_img, n_img;
    int64_t d = 0;
    std::vector<char> seen((size_t)k, 0);
    for (int32_t i = 0; i < k; i++) {
        const int32_t j = asg[(size_t)i];
        if (j < 0 || j >= k || seen[(size_t)j]) return bm_fail(ctx, BM_CUDA_ERROR, "auction returned no permutation");
        seen[(size_t)j] = 1;
        d += cost[(size_t)i * (size_t)k + (size_t)j];
        if (j != i) {
            who.push_back(subset[i]);
            o_img.push_back(old[(size_t)i]);
            n_img.push_back(old[(size_t)j]);
        }
    }
    const int32_t m = (int32_t)who.size();
    if (m > 0) {
        BM_CUDA(ctx, cudaMemcpyAsync(d_who, who.data(), sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(d_old, o_img.data(), sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(d_new, n_img.data(), sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
        const DevGraph& B = ctx->g[1];
        PermArgs pa{gview(ctx->g[0]), B.out_ptr, B.in_ptr, B.out_ent, B.in_ent, B.out_twin, B.in_twin, hview(B),
                    ctx->pi, ctx->pinv, ctx->ov, ctx->ximg};
        apply_perm_kernel<<<m, kPermThreads, 0, ctx->stream>>>(pa, d_who, d_old, d_new);
        BM_LAUNCH_CHECK(ctx, "apply_perm_kernel");
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    ctx->score += d;
    if (delta) *delta = d;
    if (changed) *changed = m;
    return BM_OK;
}

}  // namespace

extern "C" bm_status bm_lap_solve(bm_ctx* ctx, const int32_t* benefit, int32_t k, int32_t* assign, int64_t* total) {
    if (!ctx || !benefit || !assign) return BM_INVALID_ARG;
    if (k < 1 || k > kLapMaxK) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 1..%d", k, kLapMaxK);
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t cb = al256(sizeof(int32_t) * (size_t)k * (size_t)k), ab = al256(sizeof(int32_t) * (size_t)k);
    bm_status s = bm_stage(ctx, cb + ab + 256);
    if (s != BM_OK) return s;
    int32_t* d_a = (int32_t*)ctx->stage;
    int32_t* d_asg = (int32_t*)((char*)ctx->stage + cb);
    int32_t* d_st = (int32_t*)((char*)ctx->stage + cb + ab);
    long long mx = 1;
    for (size_t q = 0; q < (size_t)k * (size_t)k; q++) {
        const long long v = benefit[q];
        mx = std::max(mx, v < 0 ? -v : v);
    }
    if (mx > (1ll << 30)) return bm_fail(ctx, BM_INVALID_ARG, "benefits must stay within +-2^30");
    BM_CUDA(ctx, cudaMemcpyAsync(d_a, benefit, sizeof(int32_t) * (size_t)k * (size_t)k, cudaMemcpyHostToDevice,
                                 ctx->stream));
    if ((s = lap_device(ctx, d_a, k, d_asg, d_st, mx)) != BM_OK) return s;
    int32_t status = 0;
    BM_CUDA(ctx, cudaMemcpyAsync(assign, d_asg, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(&status, d_st, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (status) return bm_fail(ctx, BM_TIMEOUT, "auction did not finish within its bound");
    if (total) {
        int64_t t = 0;
        for (int32_t i = 0; i < k; i++) t += benefit[(size_t)i * (size_t)k + (size_t)assign[i]];
        *total = t;
    }
    return BM_OK;
}

extern "C" bm_status bm_subset_assign(bm_ctx* ctx, const int32_t* subset, int32_t k, int64_t* delta,
                                      int32_t* changed) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!subset || k < 1 || k > kLapMaxK) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 1..%d", k, kLapMaxK);
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    BmMarks mk;
    if ((s = check_subset(ctx, subset, k, mk)) != BM_OK) return s;
    return assign_subset(ctx, subset, k, delta, changed);
}

extern "C" bm_status bm_search_hungarian(bm_ctx* ctx, int32_t k, uint64_t seed, int32_t iterations,
                                         double time_budget_s, bm_progress* prog) {
    using clk = std::chrono::steady_clock;
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if (k < 2 || k > kLapMaxK) return bm_fail(ctx, BM_INVALID_ARG, "k = %d outside 2..%d", k, kLapMaxK);
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    const int32_t n = ctx->n;
    const auto t0 = clk::now();
    std::vector<uint64_t> keyv((size_t)n);
    std::vector<int32_t> order((size_t)n), subset;
    BmMarks mk;
    bm_status ret = BM_OK;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int32_t it = 0; iterations < 0 || it < iterations; it++) {
        if (time_budget_s > 0 && std::chrono::duration<double>(clk::now() - t0).count() >= time_budget_s) {
            ret = BM_TIMEOUT;
            break;
        }
        // a random order of the vertices (Philox keys, counter = vertex and
        // iteration), then greedily the members with disjoint closed A
        // neighbourhoods, the reference's random independent subset
        for (int32_t v = 1; v <= n; v++) {
            const uint32_t c[4] = {(uint32_t)v, (uint32_t)prog->launches, 0x48554E47u, 0u};
            uint32_t o[4];
            bm_philox4x32_10(c, key, o);
            keyv[(size_t)v - 1] = ((uint64_t)o[0] << 32) | o[1];
            order[(size_t)v - 1] = v;
        }
        std::sort(order.begin(), order.end(), [&](int32_t p, int32_t q) {
            const uint64_t a = keyv[(size_t)p - 1], b = keyv[(size_t)q - 1];
            return a != b ? a < b : p < q;
        });
        mk.reset(n);
        subset.clear();
        for (int32_t v : order) {
            if ((int32_t)subset.size() >= k) break;
            if (mk.marked(v)) continue;  // v is a member or next to one
            subset.push_back(v);
            mk.mark_closed(ctx, v);
        }
        int64_t d = 0;
        int32_t changed = 0;
        if ((s = assign_subset(ctx, subset.data(), (int32_t)subset.size(), &d, &changed)) != BM_OK) return s;
        prog->launches++;
        prog->accepts += changed;
        prog->rows_done += (int64_t)subset.size();
        prog->evaluated += (int64_t)subset.size() * (int64_t)subset.size();
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->seconds += std::chrono::duration<double>(clk::now() - t0).count();
    s = bm_check_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}
