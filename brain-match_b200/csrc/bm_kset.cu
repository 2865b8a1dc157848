// bm_kset.cu — exact deltas of permutations of small vertex sets (k <= 8):
// the 3-vertex moves of src/graph-re-alignment-gpu-3-swap.cu:43-305 (best of
// the non-identity permutations of a triple, applied by apply_permutation
// :925-956) and the permutation sets of
// src/graph-alignment-permset-parallel.c:304-363,625-746 (all k! permutations
// of a random k-subset, the best one applied).  The reference's group delta
// counts an edge inside the group twice and is repaired by a full re-score
// (:698-730); here the delta is exact.
//
// For a set T = {t_0..t_{k-1}} with images f_i = pi(t_i) and a permutation
// sigma (member i takes the image of member sigma(i)):
//
//   delta(sigma) = sum_i (g[i][sigma i] - S(t_i)) + sum over A entries e = (t_i -> t_j, w)
//                  inside T of [h(si, sj) + h(i, j) - h(si, j) - h(i, sj)] + self-loop terms
//
// with g[i][q] = G_{t_i}(f_q) = sum_{x in out(t_i)} min(w, B(f_q, pi x)) +
// sum_{x in in(t_i)} min(w, B(pi x, f_q)) (old images everywhere, so
// g[i][i] = S(t_i)), h(p, q) = min(w, B(f_p, f_q)) and h(p, p) = 0.  The first
// sum moves every member's external and internal edges as if the other end
// stayed; the second repairs each internal edge to its true new value.
//
// One CTA per set: the B rows of the members' images (out and in, B ids,
// sorted) are staged in shared memory, then the members' lists are scanned
// once with k-1 lookups per entry, binary searches in the staged rows (the
// hash for rows that do not fit), atomics into g in shared memory; then the
// k! permutations are enumerated in lexicographic order, each thread a
// contiguous block stepped by
// the lexicographic successor (the permutation packed in one register), and
// reduced to the best (largest delta, lowest index).
#include <climits>
#include <vector>

#include "bm_internal.cuh"

namespace {

constexpr int kKThreads = 256;
constexpr int kMaxK = 8;
constexpr int kMaxInternal = 256;

struct KsetArgs {
    GView A;
    HashView hb;
    const int32_t* selfB;
    int has_self;
    const int32_t* pi;
    const int32_t* ov;
    int32_t n;
    int32_t k;
    int32_t kfact;
    const int32_t* sets;
    int64_t nsets;
    long long* best_delta;
    int32_t* best_perm;  // nsets * k
    long long* all;      // nsets * kfact, optional
    int32_t* status;     // nonzero: some set was rejected (see bm_kset_eval)
    // B's rows in B ids (sorted by id): the gains' lookups are staged from them
    const int32_t* Bout_ptr;
    const int32_t* Bin_ptr;
    const uint32_t* Bout_ent0;
    const uint32_t* Bin_ent0;
};

constexpr int kKsetRowCap = 8192;  // B-row entries a set stages in shared memory (the rest: hash)

__device__ __forceinline__ void decode_perm(int32_t p, int k, int32_t* s) {
    int32_t avail[kMaxK];
    int32_t f = 1;
    for (int i = 0; i < k; i++) avail[i] = i;
    for (int i = 2; i < k; i++) f *= i;  // (k-1)!
    for (int i = 0; i < k; i++) {
        const int32_t idx = (k - 1 - i) > 0 ? p / f : 0;
        if (k - 1 - i > 0) p -= idx * f;
        s[i] = avail[idx];
        for (int j = idx; j < k - 1 - i; j++) avail[j] = avail[j + 1];
        if (k - 1 - i > 0) f /= (k - 1 - i);
    }
}

// The permutations [p0, p1) of K members, in lexicographic order, evaluated
// from the gain table g (shared), the internal entries and the self-loop
// terms; the best (largest delta, lowest index) is returned in bd, bp.  A
// permutation is held as K 4-bit fields of one register (field i = s[i]), so
// that the lexicographic successor is shifts and masks rather than indexed
// register arrays.
__device__ __forceinline__ uint32_t nib(uint32_t S, int i) { return (S >> (4 * i)) & 15u; }

template <int K>
__device__ void enumerate_perms(const KsetArgs& a, int64_t set, int32_t p0, int32_t p1, const int32_t* g,
                                const int32_t* Bsub, const int32_t* sA, const int32_t* sB, int32_t ni,
                                const int32_t* ie_i, const int32_t* ie_j, const int32_t* ie_w, long long& bd,
                                int32_t& bp) {
    int32_t s0[kMaxK];
    decode_perm(p0, K, s0);
    uint32_t S = 0;
#pragma unroll
    for (int i = 0; i < K; i++) S |= (uint32_t)s0[i] << (4 * i);
    long long base = 0;  // sum of g[i][i]
#pragma unroll
    for (int i = 0; i < K; i++) base += g[i * K + i];
    if constexpr (K >= 4) {
        // Without internal entries, self-loop terms or per-permutation output,
        // six consecutive permutations (p0 and p1 multiples of 6) share the
        // first K - 3 fields and order the last three values a < b < c as abc,
        // acb, bac, bca, cab, cba: one successor step per six, nine table reads.
        if (ni == 0 && !a.has_self && !a.all && p0 % 6 == 0 && p1 % 6 == 0) {
            const int32_t* g0 = g + (K - 3) * K;
            const int32_t* g1 = g + (K - 2) * K;
            const int32_t* g2 = g + (K - 1) * K;
            for (int32_t p = p0; p < p1; p += 6) {
                long long sp = -base;
#pragma unroll
                for (int i = 0; i < K - 3; i++) sp += g[i * K + (int)nib(S, i)];
                const int x = (int)nib(S, K - 3), y = (int)nib(S, K - 2), z = (int)nib(S, K - 1);
                const long long d6[6] = {sp + g0[x] + g1[y] + g2[z], sp + g0[x] + g1[z] + g2[y],
                                         sp + g0[y] + g1[x] + g2[z], sp + g0[y] + g1[z] + g2[x],
                                         sp + g0[z] + g1[x] + g2[y], sp + g0[z] + g1[y] + g2[x]};
#pragma unroll
                for (int q = 0; q < 6; q++)
                    if (d6[q] > bd) { bd = d6[q]; bp = p + q; }
                // the group's last permutation (suffix z y x), then its successor
                S = (S & ~(0xFFFu << (4 * (K - 3)))) |
                    ((uint32_t)z << (4 * (K - 3))) | ((uint32_t)y << (4 * (K - 2))) | ((uint32_t)x << (4 * (K - 1)));
                int piv = -1;
#pragma unroll
                for (int i = 0; i < K - 1; i++)
                    if (nib(S, i) < nib(S, i + 1)) piv = i;
                if (piv < 0) break;
                const uint32_t sv = nib(S, piv);
                int j = piv + 1;
#pragma unroll
                for (int jj = 1; jj < K; jj++)
                    if (jj > piv && nib(S, jj) > sv) j = jj;
                const uint32_t sj = nib(S, j);
                S = (S & ~((15u << (4 * piv)) | (15u << (4 * j)))) | (sj << (4 * piv)) | (sv << (4 * j));
                uint32_t R = 0;
#pragma unroll
                for (int i = 0; i < K; i++) {
                    const int src = (i > piv) ? (K - 1 - (i - piv - 1)) : i;
                    R |= nib(S, src) << (4 * i);
                }
                S = R;
            }
            return;
        }
    }
    for (int32_t p = p0; p < p1; p++) {
        long long d = -base;
#pragma unroll
        for (int i = 0; i < K; i++) d += g[i * K + (int)nib(S, i)];
        for (int32_t e = 0; e < ni; e++) {
            const int i = ie_i[e], j = ie_j[e], w = ie_w[e];
            const int si = (int)nib(S, i), sj = (int)nib(S, j);
            d += imin(w, Bsub[si * K + sj]) + imin(w, Bsub[i * K + j]) - imin(w, Bsub[si * K + j]) -
                 imin(w, Bsub[i * K + sj]);
        }
        if (a.has_self) {
#pragma unroll
            for (int i = 0; i < K; i++) d += imin(sA[i], sB[nib(S, i)]) - imin(sA[i], sB[i]);
        }
        if (a.all) a.all[set * a.kfact + p] = d;
        if (d > bd) { bd = d; bp = p; }
        // lexicographic successor: pivot = last i with s[i] < s[i+1]; swap it
        // with the last larger field after it; reverse the fields after it
        int piv = -1;
#pragma unroll
        for (int i = 0; i < K - 1; i++)
            if (nib(S, i) < nib(S, i + 1)) piv = i;
        if (piv < 0) break;
        const uint32_t sp = nib(S, piv);
        int j = piv + 1;
#pragma unroll
        for (int jj = 1; jj < K; jj++)
            if (jj > piv && nib(S, jj) > sp) j = jj;
        const uint32_t sj = nib(S, j);
        S = (S & ~((15u << (4 * piv)) | (15u << (4 * j)))) | (sj << (4 * piv)) | (sp << (4 * j));
        // reverse fields piv+1 .. K-1
        uint32_t R = 0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int src = (i > piv) ? (K - 1 - (i - piv - 1)) : i;
            R |= nib(S, src) << (4 * i);
        }
        S = R;
    }
}

__global__ void __launch_bounds__(kKThreads) kset_kernel(KsetArgs a) {
    extern __shared__ uint32_t rowbuf[];  // kKsetRowCap entries
    __shared__ int32_t r_off[2 * kMaxK], r_len[2 * kMaxK];  // row 2q: B-out(f_q), 2q+1: B-in(f_q); off -1: not staged
    __shared__ int32_t t[kMaxK], f[kMaxK], sA[kMaxK], sB[kMaxK];
    __shared__ int32_t g[kMaxK * kMaxK], Bsub[kMaxK * kMaxK];
    __shared__ int32_t n_int, bad;
    __shared__ int32_t ie_i[kMaxInternal], ie_j[kMaxInternal], ie_w[kMaxInternal];
    __shared__ long long red_d[kKThreads / 32];
    __shared__ int32_t red_p[kKThreads / 32];
    const int k = a.k, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int64_t set = blockIdx.x; set < a.nsets; set += gridDim.x) {
        if (tid == 0) { n_int = 0; bad = 0; }
        if (tid < k) {
            const int32_t v = a.sets[set * k + tid];
            t[tid] = v;
            if (v < 1 || v > a.n) bad = 1;
        }
        if (tid < k * k) g[tid] = 0;
        __syncthreads();
        if (tid == 0)
            for (int i = 0; i < k; i++)
                for (int j = i + 1; j < k; j++)
                    if (t[i] == t[j]) bad = 1;
        __syncthreads();
        if (bad) {
            if (tid < k) a.best_perm[set * k + tid] = tid;
            if (tid == 0) { a.best_delta[set] = 0; atomicOr(a.status, 1); }
            if (a.all)
                for (int32_t p = tid; p < a.kfact; p += kKThreads) a.all[set * a.kfact + p] = 0;
            __syncthreads();
            continue;
        }
        if (tid < k) {
            f[tid] = a.pi[t[tid]];
            sA[tid] = a.has_self ? a.A.self_w[t[tid]] : 0;
        }
        __syncthreads();
        if (tid < k) sB[tid] = a.has_self ? a.selfB[f[tid]] : 0;
        if (tid < k * k) {
            const int p = tid / k, q = tid % k;
            Bsub[tid] = (p == q) ? 0 : bm_hash_get(a.hb, f[p], f[q]);
        }
        // ---- stage the B rows of the members' images (out and in), in order,
        // while they fit
        if (tid == 0) {
            int32_t off = 0;
            for (int r = 0; r < 2 * k; r++) {
                const int32_t* ptr = (r & 1) ? a.Bin_ptr : a.Bout_ptr;
                const int32_t g0 = f[r >> 1];
                const int32_t len = ptr[g0 + 1] - ptr[g0];
                r_len[r] = len;
                r_off[r] = (off + len <= kKsetRowCap) ? off : -1;
                if (r_off[r] >= 0) off += len;
            }
        }
        __syncthreads();
        for (int r = 0; r < 2 * k; r++) {
            if (r_off[r] < 0) continue;
            const int32_t* ptr = (r & 1) ? a.Bin_ptr : a.Bout_ptr;
            const uint32_t* ent = ((r & 1) ? a.Bin_ent0 : a.Bout_ent0) + ptr[f[r >> 1]];
            for (int32_t j = tid; j < r_len[r]; j += kKThreads) rowbuf[r_off[r] + j] = ent[j];
        }
        __syncthreads();
        // ---- gains and internal entries: scan each member's out- and in-list
        for (int i = 0; i < k; i++) {
            for (int dir = 0; dir < 2; dir++) {
                const int32_t* ptr = dir ? a.A.in_ptr : a.A.out_ptr;
                const uint32_t* ent = dir ? a.A.in_ent : a.A.out_ent;
                const int32_t b = ptr[t[i]], e = ptr[t[i] + 1];
                for (int32_t j = b + tid; j < e; j += kKThreads) {
                    const uint32_t en = ent[j];
                    if (en == 0) continue;
                    const int32_t x = bm_eid(en), w = bm_ew(en);
                    const int32_t gx = a.pi[x];
                    if (dir == 0) {
                        for (int q = 0; q < k; q++)
                            if (t[q] == x) {
                                const int32_t slot = atomicAdd(&n_int, 1);
                                if (slot < kMaxInternal) { ie_i[slot] = i; ie_j[slot] = q; ie_w[slot] = w; }
                            }
                    }
                    for (int q = 0; q < k; q++) {
                        if (q == i) continue;
                        // out: B(f_q, pi x) in B-out(f_q); in: B(pi x, f_q) in B-in(f_q)
                        const int r = 2 * q + dir;
                        const int32_t bw = r_off[r] >= 0 ? bm_row_weight(rowbuf + r_off[r], r_len[r], gx)
                                           : (dir ? bm_hash_get(a.hb, gx, f[q]) : bm_hash_get(a.hb, f[q], gx));
                        const int32_t c = imin(w, bw);
                        if (c) atomicAdd(&g[i * k + q], c);
                    }
                }
            }
        }
        __syncthreads();
        if (tid < k) g[tid * k + tid] = a.ov[t[tid]];
        if (tid == 0 && n_int > kMaxInternal) { bad = 1; atomicOr(a.status, 2); }
        __syncthreads();
        const int32_t ni = bad ? 0 : n_int;
        // ---- enumerate permutations
        int32_t per = (a.kfact + kKThreads - 1) / kKThreads;
        if (k >= 4) per = (per + 5) / 6 * 6;  // whole groups of six (see enumerate_perms)
        const int32_t p0 = tid * per, p1 = min(a.kfact, p0 + per);
        long long bd = LLONG_MIN;
        int32_t bp = INT_MAX;
        if (!bad && p0 < p1) {
            switch (k) {
                case 2: enumerate_perms<2>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                case 3: enumerate_perms<3>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                case 4: enumerate_perms<4>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                case 5: enumerate_perms<5>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                case 6: enumerate_perms<6>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                case 7: enumerate_perms<7>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
                default: enumerate_perms<8>(a, set, p0, p1, g, Bsub, sA, sB, ni, ie_i, ie_j, ie_w, bd, bp); break;
            }
        }
        if (bad && a.all)
            for (int32_t p = tid; p < a.kfact; p += kKThreads) a.all[set * a.kfact + p] = 0;
        // ---- block argmax (largest delta, lowest index)
        for (int o = 16; o; o >>= 1) {
            const long long d2 = __shfl_xor_sync(0xffffffffu, bd, o);
            const int32_t p2 = __shfl_xor_sync(0xffffffffu, bp, o);
            if (d2 > bd || (d2 == bd && p2 < bp)) { bd = d2; bp = p2; }
        }
        if (lane == 0) { red_d[warp] = bd; red_p[warp] = bp; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < kKThreads / 32; w++)
                if (red_d[w] > red_d[0] || (red_d[w] == red_d[0] && red_p[w] < red_p[0])) {
                    red_d[0] = red_d[w];
                    red_p[0] = red_p[w];
                }
            if (bad) { red_d[0] = 0; red_p[0] = 0; }
            a.best_delta[set] = red_d[0];
            int32_t s[kMaxK];
            decode_perm(red_p[0], k, s);
            for (int i = 0; i < k; i++) a.best_perm[set * k + i] = s[i];
        }
        __syncthreads();
    }
}

// Apply permutations of independent sets: member i of set takes the image of
// member perm[i].  S updates of every A entry touching a member (entries
// inside a set once, from the out-lists), relabelled B entries, then pi.
struct ApplySetsArgs {
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
    int32_t k;
    const int32_t* sets;
    const int32_t* perms;
};

__global__ void __launch_bounds__(kKThreads) apply_sets_kernel(ApplySetsArgs a) {
    __shared__ int32_t t[kMaxK], f[kMaxK], fn[kMaxK];
    const int k = a.k;
    const int64_t set = blockIdx.x;
    if (threadIdx.x < k) {
        t[threadIdx.x] = a.sets[set * k + threadIdx.x];
        f[threadIdx.x] = a.pi[t[threadIdx.x]];
    }
    __syncthreads();
    if (threadIdx.x < k) fn[threadIdx.x] = f[a.perms[set * k + threadIdx.x]];
    __syncthreads();
    for (int i = 0; i < k; i++) {
        for (int dir = 0; dir < 2; dir++) {
            const int32_t* ptr = dir ? a.A.in_ptr : a.A.out_ptr;
            const uint32_t* ent = dir ? a.A.in_ent : a.A.out_ent;
            const int32_t b = ptr[t[i]], e = ptr[t[i] + 1];
            for (int32_t j = b + threadIdx.x; j < e; j += kKThreads) {
                const uint32_t en = ent[j];
                if (en == 0) continue;
                const int32_t x = bm_eid(en), w = bm_ew(en);
                int xq = -1;
                for (int q = 0; q < k; q++)
                    if (t[q] == x) xq = q;
                if (dir == 1 && xq >= 0) continue;  // inside the set: counted from the out-list
                const int32_t gx_old = a.pi[x];
                const int32_t gx_new = xq >= 0 ? fn[xq] : gx_old;
                int32_t d;
                if (dir == 0)
                    d = imin(w, bm_hash_get(a.hb, fn[i], gx_new)) - imin(w, bm_hash_get(a.hb, f[i], gx_old));
                else
                    d = imin(w, bm_hash_get(a.hb, gx_new, fn[i])) - imin(w, bm_hash_get(a.hb, gx_old, f[i]));
                if (d) { atomicAdd(a.ov + t[i], d); atomicAdd(a.ov + x, d); }
            }
        }
    }
    // image f[q] is now held by the member i with fn[i] == f[q]
    for (int i = 0; i < k; i++) {
        const int32_t img = fn[i];
        const uint32_t label = (uint32_t)t[i];
        for (int dir = 0; dir < 2; dir++) {
            const int32_t* ptr = dir ? a.Bout_ptr : a.Bin_ptr;
            const int32_t* twin = dir ? a.Bout_twin : a.Bin_twin;
            uint32_t* other = dir ? a.Bin_ent : a.Bout_ent;
            const int32_t b = ptr[img], e = ptr[img + 1];
            for (int32_t j = b + threadIdx.x; j < e; j += kKThreads) {
                const int32_t tw = twin[j];
                if (tw < 0) continue;
                other[tw] = (other[tw] & ~BM_ID_MASK) | label;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = 0; i < k; i++) {
            a.pi[t[i]] = fn[i];
            a.pinv[fn[i]] = t[i];
            a.ximg[t[i]] = bm_image_bounds(a.Bin_ptr, a.Bout_ptr, fn[i]);
        }
}

int32_t factorial(int k) {
    int32_t f = 1;
    for (int i = 2; i <= k; i++) f *= i;
    return f;
}

}  // namespace

bm_status bm_launch_kset(bm_ctx* ctx, int32_t k, const int32_t* d_sets, int64_t nsets, long long* d_best,
                         int32_t* d_perm, long long* d_all, int32_t* d_status) {
    if (nsets <= 0) return BM_OK;
    KsetArgs a;
    a.A = gview(ctx->g[0]);
    a.hb = hview(ctx->g[1]);
    a.selfB = ctx->g[1].self_w;
    a.has_self = ctx->g[0].has_self && ctx->g[1].has_self;
    a.pi = ctx->pi;
    a.ov = ctx->ov;
    a.n = ctx->n;
    a.k = k;
    a.kfact = factorial(k);
    a.Bout_ptr = ctx->g[1].out_ptr;
    a.Bin_ptr = ctx->g[1].in_ptr;
    a.Bout_ent0 = ctx->g[1].out_ent0;
    a.Bin_ent0 = ctx->g[1].in_ent0;
    a.sets = d_sets;
    a.nsets = nsets;
    a.best_delta = d_best;
    a.best_perm = d_perm;
    a.all = d_all;
    a.status = d_status;
    int64_t blocks = nsets < (int64_t)ctx->num_sms * 8 ? nsets : (int64_t)ctx->num_sms * 8;
    kset_kernel<<<(unsigned)blocks, kKThreads, sizeof(uint32_t) * kKsetRowCap, ctx->stream>>>(a);
    BM_LAUNCH_CHECK(ctx, "kset_kernel");
    return BM_OK;
}

bm_status bm_launch_apply_sets(bm_ctx* ctx, int32_t k, const int32_t* d_sets, const int32_t* d_perms, int32_t nsets) {
    if (nsets <= 0) return BM_OK;
    const DevGraph& B = ctx->g[1];
    ApplySetsArgs a;
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
    a.k = k;
    a.sets = d_sets;
    a.perms = d_perms;
    apply_sets_kernel<<<nsets, kKThreads, 0, ctx->stream>>>(a);
    BM_LAUNCH_CHECK(ctx, "apply_sets_kernel");
    return BM_OK;
}

extern "C" bm_status bm_kset_eval(bm_ctx* ctx, int32_t k, const int32_t* sets, int64_t nsets, int64_t* best_delta,
                                  int32_t* best_perm, int64_t* all_deltas) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 2 || k > kMaxK) return bm_fail(ctx, BM_INVALID_ARG, "k must be 2..%d", kMaxK);
    if (nsets < 0 || (nsets > 0 && (!sets || !best_delta || !best_perm)))
        return bm_fail(ctx, BM_INVALID_ARG, "bad set buffers");
    if (nsets == 0) return BM_OK;
    for (int64_t i = 0; i < nsets; i++)
        for (int a = 0; a < k; a++) {
            const int32_t v = sets[i * k + a];
            if (v < 1 || v > ctx->n) return bm_fail(ctx, BM_INVALID_ARG, "set %lld: id %d outside 1..%d", (long long)i, v, ctx->n);
            for (int b = 0; b < a; b++)
                if (sets[i * k + b] == v) return bm_fail(ctx, BM_INVALID_ARG, "set %lld repeats vertex %d", (long long)i, v);
        }
    const int32_t kf = factorial(k);
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t b_sets = al(sizeof(int32_t) * (size_t)(nsets * k));
    const size_t b_best = al(sizeof(long long) * (size_t)nsets);
    const size_t b_perm = al(sizeof(int32_t) * (size_t)(nsets * k));
    const size_t b_stat = 256;
    const size_t b_all = all_deltas ? al(sizeof(long long) * (size_t)nsets * (size_t)kf) : 0;
    if ((s = bm_stage(ctx, b_sets + b_best + b_perm + b_stat + b_all)) != BM_OK) return s;
    char* base = (char*)ctx->stage;
    int32_t* d_sets = (int32_t*)base;
    long long* d_best = (long long*)(base + b_sets);
    int32_t* d_perm = (int32_t*)(base + b_sets + b_best);
    int32_t* d_stat = (int32_t*)(base + b_sets + b_best + b_perm);
    long long* d_all = all_deltas ? (long long*)(base + b_sets + b_best + b_perm + b_stat) : nullptr;
    BM_CUDA(ctx, cudaMemcpyAsync(d_sets, sets, sizeof(int32_t) * (size_t)(nsets * k), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_stat, 0, sizeof(int32_t), ctx->stream));
    if ((s = bm_launch_kset(ctx, k, d_sets, nsets, d_best, d_perm, d_all, d_stat)) != BM_OK) return s;
    int32_t hstat = 0;
    BM_CUDA(ctx, cudaMemcpyAsync(best_delta, d_best, sizeof(long long) * (size_t)nsets, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(best_perm, d_perm, sizeof(int32_t) * (size_t)(nsets * k), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(&hstat, d_stat, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (all_deltas)
        BM_CUDA(ctx, cudaMemcpyAsync(all_deltas, d_all, sizeof(long long) * (size_t)nsets * (size_t)kf,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (hstat & 2)
        return bm_fail(ctx, BM_UNSUPPORTED, "a set has more than %d A entries between its members", kMaxInternal);
    return BM_OK;
}

extern "C" bm_status bm_kset_eval_dev(bm_ctx* ctx, int32_t k, const int32_t* d_sets, int64_t nsets,
                                      int64_t* d_best_delta, int32_t* d_best_perm, int32_t* d_status) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (k < 2 || k > kMaxK) return bm_fail(ctx, BM_INVALID_ARG, "k must be 2..%d", kMaxK);
    if (nsets < 0 || (nsets > 0 && (!d_sets || !d_best_delta || !d_best_perm || !d_status)))
        return bm_fail(ctx, BM_INVALID_ARG, "bad set buffers");
    return bm_launch_kset(ctx, k, d_sets, nsets, (long long*)d_best_delta, d_best_perm, nullptr, d_status);
}
