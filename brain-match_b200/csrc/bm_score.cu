// bm_score.cu — full overlap score and per-vertex overlap, and the
// relabelling of B's lists into A space (with their bank-spread order and
// twins).
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

// One thread per B list g: the list's entries relabelled into A space
// (id = pi^-1(B id)) and written in bank-spread order of their A ids, the rule
// of bm_bank_spread_lists (position p takes, where it can, an entry of bank
// ((p >> 2) + 8 (p & 3)) mod 32, else the next bank up that still has
// entries), so the row kernel's scatter over these lists meets fewer
// shared-memory bank conflicts.  pos[j] = the live position of the entry at
// position j of the id-sorted list; padding stays last and in place.  tmp
// (one int32 per entry) holds each bank's entries while they are placed.
__global__ void spread_relabel_kernel(const int32_t* __restrict__ ptr, const uint32_t* __restrict__ ent0,
                                      const int32_t* __restrict__ pinv, int32_t n, uint32_t* __restrict__ ent,
                                      int32_t* __restrict__ pos, int32_t* __restrict__ tmp) {
    for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g <= n; g += gridDim.x * blockDim.x) {
        const int32_t lo = __ldg(ptr + g), hi = __ldg(ptr + g + 1);
        int32_t cnt = hi - lo;
        while (cnt > 0 && __ldg(ent0 + lo + cnt - 1) == 0u) cnt--;  // padding is last
        int32_t num[32], head[32], end[32];
        for (int b = 0; b < 32; b++) num[b] = 0;
        for (int32_t i = lo; i < lo + cnt; i++) num[__ldg(pinv + bm_eid(__ldg(ent0 + i))) & 31]++;
        int32_t s = lo;
        for (int b = 0; b < 32; b++) { head[b] = s; s += num[b]; end[b] = s; }
        for (int32_t i = lo; i < lo + cnt; i++) tmp[head[__ldg(pinv + bm_eid(__ldg(ent0 + i))) & 31]++] = i;
        for (int b = 0; b < 32; b++) head[b] = end[b] - num[b];
        for (int32_t p = 0; p < cnt; p++) {
            int b = ((p >> 2) + 8 * (p & 3)) & 31;
            while (head[b] == end[b]) b = (b + 1) & 31;
            const int32_t i = tmp[head[b]++];
            const uint32_t e = __ldg(ent0 + i);
            ent[lo + p] = bm_pack((uint32_t)__ldg(pinv + bm_eid(e)), (uint32_t)bm_ew(e));
            pos[i] = lo + p;
        }
        for (int32_t j = lo + cnt; j < hi; j++) { ent[j] = 0u; pos[j] = j; }
    }
}

// ximg[x] = the bounds of B's in- and out-lists at pi x, for every A vertex.
__global__ void image_bounds_kernel(const int32_t* __restrict__ pi, const int32_t* __restrict__ Bin_ptr,
                                    const int32_t* __restrict__ Bout_ptr, int32_t n, int4* __restrict__ ximg) {
    for (int32_t x = blockIdx.x * blockDim.x + threadIdx.x; x <= n; x += gridDim.x * blockDim.x)
        ximg[x] = x == 0 ? make_int4(0, 0, 0, 0) : bm_image_bounds(Bin_ptr, Bout_ptr, __ldg(pi + x));
}

// The twins of the live lists: the entry at live position pos_self[j] has its
// reverse-direction twin at live position pos_other[twin0[j]] (-1: padding).
__global__ void live_twins_kernel(const int32_t* __restrict__ twin0, const int32_t* __restrict__ pos_self,
                                  const int32_t* __restrict__ pos_other, int32_t* __restrict__ twin, int64_t m) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t t0 = __ldg(twin0 + j);
        twin[__ldg(pos_self + j)] = t0 < 0 ? -1 : __ldg(pos_other + t0);
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
    image_bounds_kernel<<<(ctx->n + 1 + 255) / 256, 256, 0, ctx->stream>>>(ctx->pi, B.in_ptr, B.out_ptr, ctx->n, ctx->ximg);
    BM_LAUNCH_CHECK(ctx, "image_bounds_kernel");
    if (B.m_out + B.m_in == 0) return BM_OK;
    const int blocks = (ctx->n + 1 + 127) / 128;
    // the live twin arrays serve as the placement scratch, then are rebuilt
    spread_relabel_kernel<<<blocks, 128, 0, ctx->stream>>>(B.out_ptr, B.out_ent0, ctx->pinv, ctx->n, B.out_ent,
                                                           B.out_pos, B.out_twin);
    BM_LAUNCH_CHECK(ctx, "spread_relabel_kernel(out)");
    spread_relabel_kernel<<<blocks, 128, 0, ctx->stream>>>(B.in_ptr, B.in_ent0, ctx->pinv, ctx->n, B.in_ent,
                                                           B.in_pos, B.in_twin);
    BM_LAUNCH_CHECK(ctx, "spread_relabel_kernel(in)");
    const int tb = ctx->num_sms * 4;
    if (B.m_out > 0) {
        live_twins_kernel<<<tb, 256, 0, ctx->stream>>>(B.out_twin0, B.out_pos, B.in_pos, B.out_twin, B.m_out);
        BM_LAUNCH_CHECK(ctx, "live_twins_kernel(out)");
    }
    if (B.m_in > 0) {
        live_twins_kernel<<<tb, 256, 0, ctx->stream>>>(B.in_twin0, B.in_pos, B.out_pos, B.in_twin, B.m_in);
        BM_LAUNCH_CHECK(ctx, "live_twins_kernel(in)");
    }
    return BM_OK;
}
