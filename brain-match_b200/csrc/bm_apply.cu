// bm_apply.cu — commit swaps pi(a) <-> pi(b) on the device.
//
// The reference swaps two mapping entries and re-scores the whole graph after
// every accept (src/graph-alignment-optimized.c:556-576).  Here one CTA per
// swap updates only what the swap changes:
//   * S(v) for a, b and their A neighbours: each A entry incident to a or b
//     changes its contribution from min(w, B(old ends)) to min(w, B(new ends));
//     the difference is added to both endpoints' S;
//   * the relabelled B lists: every B entry that names image pi(a) now names
//     A vertex b and vice versa; the entries are found through the twin index
//     of the reverse direction, so the update costs O(deg_B);
//   * pi and pi^-1.
// Swaps in one launch must be pairwise independent (no shared vertex and no A
// edge between their endpoint sets), so no entry is touched by two swaps and
// no swap reads a mapping entry that another one writes.
#include "bm_internal.cuh"

namespace {

constexpr int kApplyThreads = 256;

struct ApplyArgs {
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

__device__ __forceinline__ void relabel_twins(const int32_t* __restrict__ ptr, const int32_t* __restrict__ twin,
                                              uint32_t* __restrict__ other_ent, int32_t img, uint32_t new_id) {
    const int32_t b = ptr[img], e = ptr[img + 1];
    for (int32_t j = b + threadIdx.x; j < e; j += kApplyThreads) {
        const int32_t t = twin[j];
        if (t < 0) continue;  // list padding
        const uint32_t old = other_ent[t];
        other_ent[t] = (old & ~BM_ID_MASK) | new_id;
    }
}

__global__ void __launch_bounds__(kApplyThreads) apply_kernel(ApplyArgs a, const int32_t* __restrict__ pairs) {
    const int32_t sa = pairs[2 * blockIdx.x], sb = pairs[2 * blockIdx.x + 1];
    if (sa == sb) return;
    const int32_t fa = a.pi[sa], fb = a.pi[sb];
    // ---- S updates over A entries incident to sa or sb
    for (int side = 0; side < 2; side++) {
        const int32_t me = side ? sb : sa, other = side ? sa : sb;
        const int32_t fme = side ? fb : fa, fnew = side ? fa : fb;  // my image before / after
        // out-entries me -> x
        {
            const int32_t b = a.A.out_ptr[me], e = a.A.out_ptr[me + 1];
            for (int32_t j = b + threadIdx.x; j < e; j += kApplyThreads) {
                const uint32_t ent = a.A.out_ent[j];
                if (ent == 0) continue;  // list padding
                const int32_t x = bm_eid(ent), w = bm_ew(ent);
                if (x == other) {
                    // edge me -> other: (fme, fnew) before, (fnew, fme) after
                    const int32_t d = imin(w, bm_hash_get(a.hb, fnew, fme)) - imin(w, bm_hash_get(a.hb, fme, fnew));
                    if (d) { atomicAdd(a.ov + me, d); atomicAdd(a.ov + other, d); }
                } else {
                    const int32_t gx = a.pi[x];
                    const int32_t d = imin(w, bm_hash_get(a.hb, fnew, gx)) - imin(w, bm_hash_get(a.hb, fme, gx));
                    if (d) { atomicAdd(a.ov + me, d); atomicAdd(a.ov + x, d); }
                }
            }
        }
        // in-entries x -> me (the edge other -> me is handled as other's out-entry)
        {
            const int32_t b = a.A.in_ptr[me], e = a.A.in_ptr[me + 1];
            for (int32_t j = b + threadIdx.x; j < e; j += kApplyThreads) {
                const uint32_t ent = a.A.in_ent[j];
                if (ent == 0) continue;
                const int32_t x = bm_eid(ent), w = bm_ew(ent);
                if (x == other) continue;
                const int32_t gx = a.pi[x];
                const int32_t d = imin(w, bm_hash_get(a.hb, gx, fnew)) - imin(w, bm_hash_get(a.hb, gx, fme));
                if (d) { atomicAdd(a.ov + me, d); atomicAdd(a.ov + x, d); }
            }
        }
    }
    // ---- relabel B entries naming fa (now sb) and fb (now sa)
    relabel_twins(a.Bin_ptr, a.Bin_twin, a.Bout_ent, fa, (uint32_t)sb);
    relabel_twins(a.Bout_ptr, a.Bout_twin, a.Bin_ent, fa, (uint32_t)sb);
    relabel_twins(a.Bin_ptr, a.Bin_twin, a.Bout_ent, fb, (uint32_t)sa);
    relabel_twins(a.Bout_ptr, a.Bout_twin, a.Bin_ent, fb, (uint32_t)sa);
    __syncthreads();
    if (threadIdx.x == 0) {
        a.pi[sa] = fb;
        a.pi[sb] = fa;
        a.pinv[fa] = sb;
        a.pinv[fb] = sa;
        a.ximg[sa] = bm_image_bounds(a.Bin_ptr, a.Bout_ptr, fb);
        a.ximg[sb] = bm_image_bounds(a.Bin_ptr, a.Bout_ptr, fa);
    }
}

}  // namespace

bm_status bm_launch_apply(bm_ctx* ctx, const int32_t* d_pairs, int32_t k) {
    if (k <= 0) return BM_OK;
    const DevGraph& B = ctx->g[1];
    ApplyArgs a;
    a.A = gview(ctx->g[0]);
    a.Bout_ptr = B.out_ptr;
    a.Bin_ptr = B.in_ptr;
    a.Bout_ent = B.out_ent;
    a.Bin_ent = B.in_ent;
    a.Bout_twin = B.out_twin;
    a.Bin_twin = B.in_twin;
    a.hb = hview(B);
    a.pi = ctx->pi;
    a.pinv = ctx->pinv;
    a.ov = ctx->ov;
    a.ximg = ctx->ximg;
    apply_kernel<<<k, kApplyThreads, 0, ctx->stream>>>(a, d_pairs);
    BM_LAUNCH_CHECK(ctx, "apply_kernel");
    return BM_OK;
}
