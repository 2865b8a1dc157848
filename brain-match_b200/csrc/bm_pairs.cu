// bm_pairs.cu — exact swap deltas for an arbitrary list of pairs.
//
// Follows calculate_swap_delta (src/graph-alignment-optimized.c:321-408) in
// score-difference form.  With f_u = pi u, f_v = pi v, S the per-vertex overlap
// and B self-loops kept out of the hash (so w_B(f, f) = 0 there):
//
//   delta(u,v) =   sum_{x in out(u)} min(w, B(f_v, pi x)) + sum_{x in in(u)} min(w, B(pi x, f_v))
//                + sum_{y in out(v)} min(w, B(f_u, pi y)) + sum_{y in in(v)} min(w, B(pi y, f_u))
//                - S(u) - S(v)
//                + sum over A entries between u and v of [min(w, B(f_u,f_v)) + min(w, B(f_v,f_u))]
//                + self-loop terms.
//
// Self-loop terms, with s_x the A self-loop weight of x, b_x = B(f_x, f_x),
// p = B(f_u, f_v), q = B(f_v, f_u): exact semantics
//   min(s_u, b_v) - min(s_u, b_u) + min(s_v, b_u) - min(s_v, b_v);
// reference-delta semantics (what calculate_swap_delta returns: its out- and
// in-edge loops, :327-388, each meet the self-loop of a swapped vertex and
// compare the image after the swap, p or q, with the old image's b_x)
//   min(s_u, p) + min(s_u, q) + min(s_v, p) + min(s_v, q) - 2 min(s_u, b_u) - 2 min(s_v, b_v).
//
// The last sum repairs the direct edges u->v and v->u that S(u) and S(v) both
// counted (the reference handles them at :390-405).  One warp per pair; every
// lookup of B is one probe sequence in the hash table (L2-resident).
#include "bm_internal.cuh"

namespace {

constexpr int kPairThreads = 256;

struct PairArgs {
    GView A;
    const int32_t* selfB;
    HashView hb;
    const int32_t* pi;
    const int32_t* ov;
    int32_t n;
    int has_self;  // self-loop terms needed (A and B have self-loops; A alone in reference-delta mode)
    int refcpu;    // reference-delta semantics
};

__device__ __forceinline__ int64_t pair_delta_warp(const PairArgs& a, int32_t u, int32_t v, int lane) {
    const int32_t fu = __ldg(a.pi + u), fv = __ldg(a.pi + v);
    int64_t s = 0;
    int32_t corr_w = 0;  // sum over direct A entries between u and v of min(w,p)+min(w,q)
    {
        const int32_t b = __ldg(a.A.out_ptr + u), e = __ldg(a.A.out_ptr + u + 1);
        for (int32_t j = b + lane; j < e; j += 32) {
            const uint32_t ent = __ldg(a.A.out_ent + j);
            if (ent == 0) continue;  // list padding
            const int32_t x = bm_eid(ent), w = bm_ew(ent);
            s += imin(w, bm_hash_get(a.hb, fv, __ldg(a.pi + x)));
            if (x == v) corr_w += imin(w, bm_hash_get(a.hb, fu, fv)) + imin(w, bm_hash_get(a.hb, fv, fu));
        }
    }
    {
        const int32_t b = __ldg(a.A.in_ptr + u), e = __ldg(a.A.in_ptr + u + 1);
        for (int32_t j = b + lane; j < e; j += 32) {
            const uint32_t ent = __ldg(a.A.in_ent + j);
            if (ent == 0) continue;
            const int32_t x = bm_eid(ent), w = bm_ew(ent);
            s += imin(w, bm_hash_get(a.hb, __ldg(a.pi + x), fv));
            if (x == v) corr_w += imin(w, bm_hash_get(a.hb, fu, fv)) + imin(w, bm_hash_get(a.hb, fv, fu));
        }
    }
    {
        const int32_t b = __ldg(a.A.out_ptr + v), e = __ldg(a.A.out_ptr + v + 1);
        for (int32_t j = b + lane; j < e; j += 32) {
            const uint32_t ent = __ldg(a.A.out_ent + j);
            if (ent == 0) continue;
            s += imin(bm_ew(ent), bm_hash_get(a.hb, fu, __ldg(a.pi + bm_eid(ent))));
        }
    }
    {
        const int32_t b = __ldg(a.A.in_ptr + v), e = __ldg(a.A.in_ptr + v + 1);
        for (int32_t j = b + lane; j < e; j += 32) {
            const uint32_t ent = __ldg(a.A.in_ent + j);
            if (ent == 0) continue;
            s += imin(bm_ew(ent), bm_hash_get(a.hb, __ldg(a.pi + bm_eid(ent)), fu));
        }
    }
    s += corr_w;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    s -= (int64_t)__ldg(a.ov + u) + (int64_t)__ldg(a.ov + v);
    if (a.has_self) {
        const int32_t su = __ldg(a.A.self_w + u), sv = __ldg(a.A.self_w + v);
        const int32_t bu = __ldg(a.selfB + fu), bv = __ldg(a.selfB + fv);
        if (a.refcpu) {
            const int32_t p = bm_hash_get(a.hb, fu, fv), q = bm_hash_get(a.hb, fv, fu);
            s += imin(su, p) + imin(su, q) + imin(sv, p) + imin(sv, q) - 2 * imin(su, bu) - 2 * imin(sv, bv);
        } else {
            s += imin(su, bv) - imin(su, bu) + imin(sv, bu) - imin(sv, bv);
        }
    }
    return s;
}

__global__ void __launch_bounds__(kPairThreads)
pairs_kernel(PairArgs a, const int32_t* __restrict__ pairs, int64_t k, int64_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps_total = (int64_t)gridDim.x * (kPairThreads / 32);
    for (int64_t i = (int64_t)blockIdx.x * (kPairThreads / 32) + (threadIdx.x >> 5); i < k; i += warps_total) {
        const int32_t u = __ldg(pairs + 2 * i), v = __ldg(pairs + 2 * i + 1);
        int64_t d = 0;
        // ids outside 1..n (device-pointer callers) and u == v give 0
        if (u != v && u >= 1 && u <= a.n && v >= 1 && v <= a.n) d = pair_delta_warp(a, u, v, lane);
        if (lane == 0) out[i] = d;
    }
}

}  // namespace

bm_status bm_launch_pairs(bm_ctx* ctx, const int32_t* d_pairs, int64_t k, int64_t* d_out, bool exact_only) {
    if (k <= 0) return BM_OK;
    PairArgs a;
    a.A = gview(ctx->g[0]);
    a.selfB = ctx->g[1].self_w;
    a.hb = hview(ctx->g[1]);
    a.pi = ctx->pi;
    a.ov = ctx->ov;
    a.n = ctx->n;
    a.refcpu = !exact_only && ctx->semantics == BM_SEMANTICS_REF_CPU;
    a.has_self = a.refcpu ? ctx->g[0].has_self : (ctx->g[0].has_self && ctx->g[1].has_self);
    int64_t blocks = (k + (kPairThreads / 32) - 1) / (kPairThreads / 32);
    int64_t cap = (int64_t)ctx->num_sms * 16;
    if (blocks > cap) blocks = cap;
    pairs_kernel<<<(unsigned)blocks, kPairThreads, 0, ctx->stream>>>(a, d_pairs, k, d_out);
    BM_LAUNCH_CHECK(ctx, "pairs_kernel");
    return BM_OK;
}

extern "C" bm_status bm_delta_pairs_dev(bm_ctx* ctx, const int32_t* d_pairs, int64_t k, int64_t* d_deltas) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 0 || (k > 0 && (!d_pairs || !d_deltas))) return bm_fail(ctx, BM_INVALID_ARG, "bad pair buffers");
    return bm_launch_pairs(ctx, d_pairs, k, d_deltas);
}

extern "C" bm_status bm_delta_pairs(bm_ctx* ctx, const int32_t* pairs, int64_t k, int64_t* deltas) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 0 || (k > 0 && (!pairs || !deltas))) return bm_fail(ctx, BM_INVALID_ARG, "bad pair buffers");
    if (k == 0) return BM_OK;
    for (int64_t i = 0; i < 2 * k; i++)
        if (pairs[i] < 1 || pairs[i] > ctx->n)
            return bm_fail(ctx, BM_INVALID_ARG, "pair entry %lld = %d outside 1..%d", (long long)i, pairs[i], ctx->n);
    const size_t in_bytes = sizeof(int32_t) * 2 * (size_t)k;
    const size_t in_al = (in_bytes + 255) & ~(size_t)255;
    s = bm_stage(ctx, in_al + sizeof(int64_t) * (size_t)k);
    if (s != BM_OK) return s;
    int32_t* d_pairs = (int32_t*)ctx->stage;
    int64_t* d_out = (int64_t*)((char*)ctx->stage + in_al);
    BM_CUDA(ctx, cudaMemcpyAsync(d_pairs, pairs, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    s = bm_launch_pairs(ctx, d_pairs, k, d_out);
    if (s != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(deltas, d_out, sizeof(int64_t) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}
