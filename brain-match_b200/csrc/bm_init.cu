// bm_init.cu — greedy-similarity initial matching on the device.
//
// The algorithm of src/greedy-match.c:
//   features  per vertex: in-degree, out-degree, the number of distinct
//             vertices reachable in two out-steps and the number that reach
//             it in two in-steps (compute_vertex_features /
//             compute_2hop_metrics :213-293); duplicate edges count, as the
//             reference's adjacency lists keep them;
//   sort      both graphs' vertices by descending feature sum (:295-300,
//             :478-479), ties by ascending id;
//   greedy    each A vertex in that order takes the unmatched B vertex at the
//             smallest L1 feature distance, the first in B's sorted order on
//             ties (:442-447, :483-510).
// The result equals bm_greedy_match of the host library (bm_host.h), which
// restates the same steps on the CPU.
//
// Kernels: reach2_kernel gives each vertex to one CTA (taken from a counter,
// so hubs do not hold up a static share), which marks 2-hop targets in an
// n-bit shared-memory bitmap and counts them with popc; greedy_kernel is one
// CTA of 1024 threads looping over the A vertices, each step a block-wide
// argmin over the unmatched B vertices on a packed (distance, position) key.
#include <algorithm>
#include <climits>
#include <numeric>
#include <vector>

#include "bm_internal.cuh"

namespace {

constexpr int kReachThreads = 256;
constexpr int kGreedyThreads = 1024;

struct Adj {
    const int32_t* ptr;  // n+2
    const int32_t* idx;  // neighbour ids
};

__global__ void __launch_bounds__(kReachThreads) reach2_kernel(Adj out, Adj in, int32_t n, int* next,
                                                               int4* __restrict__ feat) {
    extern __shared__ uint32_t bits[];
    __shared__ int s_v;
    __shared__ int s_cnt;
    const uint32_t nw = (uint32_t)(n + 32) / 32u;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = kReachThreads / 32;
    for (;;) {
        if (tid == 0) s_v = atomicAdd(next, 1) + 1;
        __syncthreads();
        const int32_t v = s_v;
        if (v > n) break;
        int counts[2];
        for (int dir = 0; dir < 2; dir++) {
            const Adj a = dir == 0 ? out : in;
            for (uint32_t i = tid; i < nw; i += kReachThreads) bits[i] = 0u;
            if (tid == 0) s_cnt = 0;
            __syncthreads();
            // warps take the first-step neighbours x, lanes stream x's list
            for (int32_t j = a.ptr[v] + warp; j < a.ptr[v + 1]; j += nwarps) {
                const int32_t x = a.idx[j];
                for (int32_t k = a.ptr[x] + lane; k < a.ptr[x + 1]; k += 32) {
                    const int32_t y = a.idx[k];
                    atomicOr(&bits[y >> 5], 1u << (y & 31));
                }
            }
            __syncthreads();
            int c = 0;
            for (uint32_t i = tid; i < nw; i += kReachThreads) c += __popc(bits[i]);
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) atomicAdd(&s_cnt, c);
            __syncthreads();
            counts[dir] = s_cnt;
            __syncthreads();
        }
        if (tid == 0)
            feat[v] = make_int4(in.ptr[v + 1] - in.ptr[v], out.ptr[v + 1] - out.ptr[v], counts[0], counts[1]);
    }
}

__device__ __forceinline__ long long l1(const int4& a, const int4& b) {
    return llabs((long long)a.x - b.x) + llabs((long long)a.y - b.y) + llabs((long long)a.z - b.z) +
           llabs((long long)a.w - b.w);
}

// fa, ida: A vertices in sorted order (features, ids); fb, idb: the same for
// B.  pi[ida[i]] = idb[j] for the position j chosen at step i.
__global__ void __launch_bounds__(kGreedyThreads) greedy_kernel(const int4* __restrict__ fa,
                                                                const int32_t* __restrict__ ida,
                                                                const int4* __restrict__ fb,
                                                                const int32_t* __restrict__ idb, int32_t n,
                                                                int32_t* __restrict__ pi) {
    extern __shared__ uint32_t used[];
    __shared__ unsigned long long s_best[kGreedyThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t nw = (uint32_t)(n + 31) / 32u;
    for (uint32_t i = tid; i < nw; i += kGreedyThreads) used[i] = 0u;
    __syncthreads();
    for (int32_t i = 0; i < n; i++) {
        const int4 a = fa[i];
        // key = distance << 17 | position: the smallest distance, then the
        // first position (n <= 131071 < 2^17; distances stay below 2^46)
        unsigned long long best = ~0ull;
#pragma unroll 4
        for (int32_t j = tid; j < n; j += kGreedyThreads) {
            const int4 b = fb[j];
            const bool free_j = !((used[j >> 5] >> (j & 31)) & 1u);
            const unsigned long long key = ((unsigned long long)l1(a, b) << 17) | (unsigned long long)j;
            if (free_j && key < best) best = key;
        }
        for (int o = 16; o; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
            best = t < best ? t : best;
        }
        if (lane == 0) s_best[warp] = best;
        __syncthreads();
        if (warp == 0) {
            best = s_best[lane];
            for (int o = 16; o; o >>= 1) {
                const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
                best = t < best ? t : best;
            }
            if (lane == 0 && best != ~0ull) {
                const int32_t j = (int32_t)(best & 0x1FFFFull);
                used[j >> 5] |= 1u << (j & 31);
                pi[ida[i]] = idb[j];
            }
        }
        __syncthreads();
    }
}

// Plain CSR (ids only) of one direction of an edge list, on the host.
void build_adj(int32_t n, int64_t m, const int32_t* from, const int32_t* to, std::vector<int32_t>& ptr,
               std::vector<int32_t>& idx) {
    ptr.assign((size_t)n + 2, 0);
    for (int64_t e = 0; e < m; e++) ptr[(size_t)from[e] + 1]++;
    for (int32_t i = 1; i <= n + 1; i++) ptr[(size_t)i] += ptr[(size_t)i - 1];
    idx.resize((size_t)std::max<int64_t>(m, 1));
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t e = 0; e < m; e++) idx[(size_t)fill[(size_t)from[e]]++] = to[e];
}

struct DevBuf {
    std::vector<void*> p;
    ~DevBuf() { for (void* x : p) bm_cuda_free(x); }
    template <typename T>
    bool get(T** out, size_t count) {
        void* d = nullptr;
        if (bm_cuda_malloc(&d, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        p.push_back(d);
        *out = static_cast<T*>(d);
        return true;
    }
};

// Features (n+1 int4: in, out, reach2, canreach2) of one graph on the device.
bm_status graph_features(bm_ctx* ctx, DevBuf& mem, int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                         std::vector<int4>& feat) {
    std::vector<int32_t> optr, oidx, iptr, iidx;
    build_adj(n, m, src, dst, optr, oidx);
    build_adj(n, m, dst, src, iptr, iidx);
    int32_t *d_optr, *d_oidx, *d_iptr, *d_iidx;
    int* d_next;
    int4* d_feat;
    if (!mem.get(&d_optr, optr.size()) || !mem.get(&d_oidx, oidx.size()) || !mem.get(&d_iptr, iptr.size()) ||
        !mem.get(&d_iidx, iidx.size()) || !mem.get(&d_next, 1) || !mem.get(&d_feat, (size_t)n + 1))
        return bm_fail(ctx, BM_OOM, "greedy matching: device allocation failed");
    BM_CUDA(ctx, cudaMemcpyAsync(d_optr, optr.data(), sizeof(int32_t) * optr.size(), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_oidx, oidx.data(), sizeof(int32_t) * oidx.size(), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_iptr, iptr.data(), sizeof(int32_t) * iptr.size(), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_iidx, iidx.data(), sizeof(int32_t) * iidx.size(), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_next, 0, sizeof(int), ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_feat, 0, sizeof(int4) * ((size_t)n + 1), ctx->stream));
    const size_t smem = sizeof(uint32_t) * (((size_t)n + 32) / 32);
    if (smem > 48 * 1024)
        BM_CUDA(ctx, cudaFuncSetAttribute(reach2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    reach2_kernel<<<ctx->num_sms * 4, kReachThreads, smem, ctx->stream>>>(Adj{d_optr, d_oidx}, Adj{d_iptr, d_iidx}, n,
                                                                         d_next, d_feat);
    BM_LAUNCH_CHECK(ctx, "reach2_kernel");
    feat.resize((size_t)n + 1);
    BM_CUDA(ctx, cudaMemcpyAsync(feat.data(), d_feat, sizeof(int4) * ((size_t)n + 1), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    return BM_OK;
}

}  // namespace

extern "C" bm_status bm_greedy_match_dev(bm_ctx* ctx, int32_t n, int64_t mA, const int32_t* srcA,
                                         const int32_t* dstA, int64_t mB, const int32_t* srcB, const int32_t* dstB,
                                         int32_t* pi) {
    if (!ctx || !pi) return BM_INVALID_ARG;
    if (n < 1 || n > BM_MAX_N) return bm_fail(ctx, BM_INVALID_ARG, "n = %d outside 1..%d", n, BM_MAX_N);
    if (mA < 0 || mB < 0 || mA >= INT32_MAX || mB >= INT32_MAX || (mA > 0 && (!srcA || !dstA)) ||
        (mB > 0 && (!srcB || !dstB)))
        return bm_fail(ctx, BM_INVALID_ARG, "bad edge arrays");
    const int32_t* ends[4] = {srcA, dstA, srcB, dstB};
    const int64_t ms[4] = {mA, mA, mB, mB};
    for (int q = 0; q < 4; q++)
        for (int64_t e = 0; e < ms[q]; e++)
            if (ends[q][e] < 1 || ends[q][e] > n)
                return bm_fail(ctx, BM_INVALID_ARG, "edge endpoint %d outside 1..%d", ends[q][e], n);
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    DevBuf mem;
    std::vector<int4> fa, fb;
    bm_status s;
    if ((s = graph_features(ctx, mem, n, mA, srcA, dstA, fa)) != BM_OK) return s;
    if ((s = graph_features(ctx, mem, n, mB, srcB, dstB, fb)) != BM_OK) return s;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // both graphs' vertices by descending feature sum, ties by id
    auto order = [&](const std::vector<int4>& f, std::vector<int32_t>& ids, std::vector<int4>& sorted) {
        ids.resize((size_t)n);
        std::iota(ids.begin(), ids.end(), 1);
        auto total = [&](int32_t v) {
            const int4& x = f[(size_t)v];
            return (long long)x.x + x.y + x.z + x.w;
        };
        std::stable_sort(ids.begin(), ids.end(), [&](int32_t p, int32_t q) { return total(p) > total(q); });
        sorted.resize((size_t)n);
        for (int32_t i = 0; i < n; i++) sorted[(size_t)i] = f[(size_t)ids[(size_t)i]];
    };
    std::vector<int32_t> ida, idb;
    std::vector<int4> sfa, sfb;
    order(fa, ida, sfa);
    order(fb, idb, sfb);
    int4 *d_fa, *d_fb;
    int32_t *d_ida, *d_idb, *d_pi;
    if (!mem.get(&d_fa, (size_t)n) || !mem.get(&d_fb, (size_t)n) || !mem.get(&d_ida, (size_t)n) ||
        !mem.get(&d_idb, (size_t)n) || !mem.get(&d_pi, (size_t)n + 1))
        return bm_fail(ctx, BM_OOM, "greedy matching: device allocation failed");
    BM_CUDA(ctx, cudaMemcpyAsync(d_fa, sfa.data(), sizeof(int4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_fb, sfb.data(), sizeof(int4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_ida, ida.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_idb, idb.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_pi, 0, sizeof(int32_t) * ((size_t)n + 1), ctx->stream));
    const size_t smem = sizeof(uint32_t) * (((size_t)n + 31) / 32);
    greedy_kernel<<<1, kGreedyThreads, smem, ctx->stream>>>(d_fa, d_ida, d_fb, d_idb, n, d_pi);
    BM_LAUNCH_CHECK(ctx, "greedy_kernel");
    BM_CUDA(ctx, cudaMemcpyAsync(pi, d_pi, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}
