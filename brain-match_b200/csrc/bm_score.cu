// bm_score.cu — full overlap score and per-vertex overlap, and the
// relabelling of B's lists into A space.
//
// score(pi) = sum over A entries (x->y, w) of min(w, w_B(pi x, pi y)), the sum
// of calculate_alignment_score (src/graph-alignment-optimized.c:292-307).
// One warp per A vertex u walks u's out-list (coalesced packed entries), looks
// up w_B(pi u, pi x) in B's hash table and adds min(w, w_B) to S(u) and S(x).
// Self-loops are scored from the two self-weight arrays.
#include "bm_internal.cuh"

namespace {

constexpr int kScoreThreads = 256;

__global__ void __launch_bounds__(kScoreThreads)
score_kernel(GView A, HashView hb, const int32_t* __restrict__ selfB, const int32_t* __restrict__ pi, int32_t n,
             int32_t* __restrict__ ov, unsigned long long* __restrict__ total) {
    __shared__ unsigned long long block_sum[kScoreThreads / 32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps_total = gridDim.x * (kScoreThreads / 32);
    unsigned long long mine = 0;
    for (int32_t u = 1 + blockIdx.x * (kScoreThreads / 32) + warp; u <= n; u += warps_total) {
        const int32_t fu = __ldg(pi + u);
        const int32_t b = __ldg(A.out_ptr + u), e = __ldg(A.out_ptr + u + 1);
        int32_t s = 0;
        for (int32_t j = b + lane; j < e; j += 32) {
            const uint32_t ent = __ldg(A.out_ent + j);
            if (ent == 0) continue;  // list padding
            const int32_t x = bm_eid(ent);
            const int32_t c = imin(bm_ew(ent), bm_hash_get(hb, fu, __ldg(pi + x)));
            if (c) atomicAdd(ov + x, c);
            s += c;
        }
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (s) atomicAdd(ov + u, s);
            int32_t self = imin(__ldg(A.self_w + u), __ldg(selfB + fu));
            mine += (unsigned long long)(s + self);
        }
    }
    if (lane == 0) block_sum[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kScoreThreads / 32; i++) t += block_sum[i];
        if (t) atomicAdd(total, t);
    }
}

__global__ void relabel_kernel(const uint32_t* __restrict__ ent0, uint32_t* __restrict__ ent,
                               const int32_t* __restrict__ pinv, int64_t m) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t e = __ldg(ent0 + j);
        ent[j] = bm_pack((uint32_t)__ldg(pinv + bm_eid(e)), (uint32_t)bm_ew(e));
    }
}

}  // namespace

bm_status bm_launch_score(bm_ctx* ctx, int64_t* score_out) {
    const int32_t n = ctx->n;
    BM_CUDA(ctx, cudaMemsetAsync(ctx->ov, 0, sizeof(int32_t) * (size_t)ctx->nvec, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(ctx->d_score, 0, sizeof(unsigned long long), ctx->stream));
    int blocks = ctx->num_sms * 8;
    int need = (n + (kScoreThreads / 32) - 1) / (kScoreThreads / 32);
    if (blocks > need) blocks = need > 0 ? need : 1;
    score_kernel<<<blocks, kScoreThreads, 0, ctx->stream>>>(gview(ctx->g[0]), hview(ctx->g[1]), ctx->g[1].self_w,
                                                            ctx->pi, n, ctx->ov, ctx->d_score);
    BM_LAUNCH_CHECK(ctx, "score_kernel");
    unsigned long long h = 0;
    BM_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_score, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *score_out = (int64_t)h;
    return BM_OK;
}

// Exact semantics: the tracked score must equal the recomputed one, and a
// mismatch is a failed self-check.  Reference-delta semantics: the tracked
// score sums calculate_swap_delta values, which are not score differences on
// graphs with self-loops, so the recomputed score replaces it, as the
// reference's loop re-scores after every accept
// (src/graph-alignment-optimized.c:571-576).
bm_status bm_check_score(bm_ctx* ctx) {
    int64_t full = 0;
    bm_status s = bm_launch_score(ctx, &full);
    if (s != BM_OK) return s;
    const int64_t tracked = ctx->score;
    ctx->score = full;
    if (full != tracked && ctx->semantics == BM_SEMANTICS_EXACT)
        return bm_fail(ctx, BM_PARITY_FAIL, "tracked score %lld != recomputed score %lld", (long long)tracked,
                       (long long)full);
    return BM_OK;
}

bm_status bm_launch_relabel(bm_ctx* ctx) {
    const DevGraph& B = ctx->g[1];
    int blocks = ctx->num_sms * 4;
    if (B.m_out > 0) {
        relabel_kernel<<<blocks, 256, 0, ctx->stream>>>(B.out_ent0, B.out_ent, ctx->pinv, B.m_out);
        BM_LAUNCH_CHECK(ctx, "relabel_kernel(out)");
    }
    if (B.m_in > 0) {
        relabel_kernel<<<blocks, 256, 0, ctx->stream>>>(B.in_ent0, B.in_ent, ctx->pinv, B.m_in);
        BM_LAUNCH_CHECK(ctx, "relabel_kernel(in)");
    }
    return BM_OK;
}
