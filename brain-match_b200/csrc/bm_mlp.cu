// bm_mlp.cu — learned swap-partner proposals.
//
// A 24 -> 128 -> 128 -> 1 MLP scores candidate partners v of a vertex u; the
// top-K partners of each row are then checked by the exact int64 delta (pairs
// kernel) and only improving, independent swaps are applied.  The model has
// no counterpart in the reference, whose only guided proposal is the
// degree-weighted random swap of src/graph-re-alignment-gpu-swap.cu:767-887;
// uniform random partners stay available as the yardstick of its hit rate.
//
// Numerics: inputs, weights and hidden activations are rounded to BF16;
// products accumulate in FP32 (SIMT FMA for training, tcgen05 MMA with TMEM
// accumulators for bulk row scoring); master weights and AdamW moments are
// FP32.  The oracle holds an FP64 replica with the same roundings.
//
// Per-vertex table T[v] (12 floats, A space, current mapping):
//   0 log1p out-degree      1 log1p in-degree
//   2 log1p out-weight      3 log1p in-weight
//   4 log1p S(v)            5 log1p(weighted degree - S(v))   (local deficit)
//   6 log1p #A entries of v whose B counterpart under pi is missing
//   7 0
//   8 log1p B out-degree of pi(v)   9 log1p B in-degree of pi(v)   10, 11: 0
// Pair features of a swap (u, v), a = T[u], b = T[v]:
//   x0..6 = a0..6, x7 = a8 + a9, x8..14 = b0..6, x15 = b8 + b9,
//   x16 = |a0 - b8|, x17 = |a1 - b9|, x18 = |b0 - a8|, x19 = |b1 - a9|
//     (degrees of each vertex against the B degrees of its new image),
//   x20 = [B(pi u, pi v) > 0], x21 = [B(pi v, pi u) > 0],
//   x22 = |a4 - b4|, x23 = a5 + b5.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "bm_internal.cuh"
#include "bm_rng.hpp"

#define BM_MLP_IN 24
#define BM_MLP_H 128
#define BM_FT 12

namespace {

constexpr int kNW1 = BM_MLP_IN * BM_MLP_H;
constexpr int kOffB1 = kNW1;
constexpr int kOffW2 = kOffB1 + BM_MLP_H;
constexpr int kOffB2 = kOffW2 + BM_MLP_H * BM_MLP_H;
constexpr int kOffW3 = kOffB2 + BM_MLP_H;
constexpr int kOffB3 = kOffW3 + BM_MLP_H;
constexpr int kNParams = kOffB3 + 1;

// Weight image of the tensor-core kernels: W1, W2 and the output row w3 as
// BF16 in the K-major, no-swizzle operand layout, then the FP32 epilogue
// vectors b1, b2, w3 (BF16-rounded), b3, then W2 transposed (the B operand of
// the backward product dH2 . W2^T of the training kernel).
constexpr int kImgW1 = 128 * 32 * 2;   // N=128 hidden x K=32 (24 inputs + 8 zero)
constexpr int kImgW2 = 128 * 128 * 2;  // N=128 out x K=128 in
constexpr int kImgW3 = 16 * 128 * 2;   // N=16 x K=128: w3 in row 0, zeros elsewhere
constexpr int kImgEp = (3 * BM_MLP_H + 4) * 4;
constexpr int kImgW2T = 128 * 128 * 2;  // N=128 in x K=128 out
constexpr int kImgOffW2T = kImgW1 + kImgW2 + kImgW3 + kImgEp;
// The row scorer's image follows, with the biases folded into the products:
// each layer's input gets two constant-one columns (K = 24, 25 of layer 1's
// 32; K = 128, 129 of a 144-wide hidden input), and the weights' matching
// columns hold the bias as a pair of BF16 values, hi = bf16(b) and
// lo = bf16(b - hi), so the FP32 accumulator receives b to about 2^-16.
constexpr int kHK = 144;                   // hidden input width of the scorer's layer 2
constexpr int kImgW1S = 128 * 32 * 2;      // N=128 hidden x K=32
constexpr int kImgW2S = 128 * kHK * 2;     // N=128 out x K=144
constexpr int kImgOffS = kImgOffW2T + kImgW2T;
constexpr int kImgBytes = kImgOffS + kImgW1S + kImgW2S;

}  // namespace

struct bm_mlp {
    bm_ctx* ctx = nullptr;
    int device = 0;
    int32_t n = 0;
    float* d_w = nullptr;      // FP32 master parameters
    float* d_m = nullptr;      // AdamW first moment
    float* d_v = nullptr;      // AdamW second moment
    float* d_g = nullptr;      // gradient of the last batch
    float* d_loss = nullptr;
    float* d_tab = nullptr;    // per-vertex table [(n+1) * 12]
    float2* d_bdeg = nullptr;  // per B vertex: log1p out-degree, log1p in-degree
    unsigned char* d_img = nullptr;
    bool img_dirty = true;
    float* d_sc = nullptr;     // row scores [rows x n]
    size_t sc_cap = 0;
    int32_t* d_flag = nullptr; // error flag of the tensor-core kernel
    int64_t step = 0;
    int32_t backend = 0;       // 0 tensor cores, 1 SIMT
    // record store: BF16 features and float targets (ring buffer)
    uint16_t* d_rx = nullptr;
    float* d_ry = nullptr;
    int64_t rcap = 0, rsize = 0, rhead = 0;
    // minibatch and search scratch
    uint16_t* d_bx = nullptr;
    float* d_by = nullptr;
    int32_t bcap = 0;
    void* d_scr = nullptr;
    size_t scr_bytes = 0;
};

namespace {

using clk = std::chrono::steady_clock;
double secs_since(clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); }

__host__ __device__ __forceinline__ float bf16r(float x) {
    // round to nearest even BF16, returned widened to float
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return x;  // inf / nan unchanged
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

__device__ __forceinline__ float bf16_to_float(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// ------------------------------------------------------------------ features

__global__ void bdeg_kernel(const int32_t* __restrict__ optr, const uint32_t* __restrict__ oent,
                            const int32_t* __restrict__ iptr, const uint32_t* __restrict__ ient, int32_t n,
                            float2* __restrict__ bdeg) {
    for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g <= n; g += gridDim.x * blockDim.x) {
        int32_t dout = 0, din = 0;
        if (g >= 1) {
            for (int32_t j = optr[g]; j < optr[g + 1]; j++) dout += oent[j] != 0;
            for (int32_t j = iptr[g]; j < iptr[g + 1]; j++) din += ient[j] != 0;
        }
        bdeg[g] = make_float2(log1pf((float)dout), log1pf((float)din));
    }
}

// One warp per A vertex.  Row 0 of the table stays zero.
__global__ void vertex_table_kernel(GView A, HashView hb, const int32_t* __restrict__ pi,
                                    const int32_t* __restrict__ ov, const float2* __restrict__ bdeg, int32_t n,
                                    float* __restrict__ tab) {
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int32_t u = 1 + blockIdx.x * wpb + (threadIdx.x >> 5); u <= n; u += gridDim.x * wpb) {
        const int32_t fu = pi[u];
        int32_t dout = 0, din = 0, miss = 0;
        long long wout = 0, win = 0;
        for (int32_t j = A.out_ptr[u] + lane; j < A.out_ptr[u + 1]; j += 32) {
            const uint32_t e = A.out_ent[j];
            if (!e) continue;
            dout++;
            wout += bm_ew(e);
            miss += bm_hash_get(hb, fu, pi[bm_eid(e)]) == 0;
        }
        for (int32_t j = A.in_ptr[u] + lane; j < A.in_ptr[u + 1]; j += 32) {
            const uint32_t e = A.in_ent[j];
            if (!e) continue;
            din++;
            win += bm_ew(e);
            miss += bm_hash_get(hb, pi[bm_eid(e)], fu) == 0;
        }
        for (int o = 16; o; o >>= 1) {
            dout += __shfl_xor_sync(0xffffffffu, dout, o);
            din += __shfl_xor_sync(0xffffffffu, din, o);
            miss += __shfl_xor_sync(0xffffffffu, miss, o);
            wout += __shfl_xor_sync(0xffffffffu, wout, o);
            win += __shfl_xor_sync(0xffffffffu, win, o);
        }
        if (lane == 0) {
            float* t = tab + (size_t)u * BM_FT;
            const long long s = ov[u];
            const float2 bd = bdeg[fu];
            const long long def = wout + win - s;
            t[0] = log1pf((float)dout);
            t[1] = log1pf((float)din);
            t[2] = log1pf((float)wout);
            t[3] = log1pf((float)win);
            t[4] = log1pf((float)s);
            t[5] = log1pf((float)(def > 0 ? def : 0));
            t[6] = log1pf((float)miss);
            t[7] = 0.f;
            t[8] = bd.x;
            t[9] = bd.y;
            t[10] = 0.f;
            t[11] = 0.f;
        }
    }
}

// The 24 features of swap (u, v) from the two table rows and the two B
// adjacency bits, before rounding.
__device__ __forceinline__ void pair_features_raw(const float* a, const float* b, bool b_uv, bool b_vu, float* x) {
#pragma unroll
    for (int i = 0; i < 7; i++) {
        x[i] = a[i];
        x[8 + i] = b[i];
    }
    x[7] = a[8] + a[9];
    x[15] = b[8] + b[9];
    x[16] = fabsf(a[0] - b[8]);
    x[17] = fabsf(a[1] - b[9]);
    x[18] = fabsf(b[0] - a[8]);
    x[19] = fabsf(b[1] - a[9]);
    x[20] = b_uv ? 1.f : 0.f;
    x[21] = b_vu ? 1.f : 0.f;
    x[22] = fabsf(a[4] - b[4]);
    x[23] = a[5] + b[5];
}

// Same, rounded to BF16 (nearest even).
__device__ __forceinline__ void pair_features(const float* a, const float* b, bool b_uv, bool b_vu, float* x) {
    pair_features_raw(a, b, b_uv, b_vu, x);
#pragma unroll
    for (int i = 0; i < BM_MLP_IN; i++) x[i] = bf16r(x[i]);
}

struct FeatSrc {
    const float* tab;
    const int32_t* pi;
    HashView hb;
};

__device__ __forceinline__ void pair_features_lookup(const FeatSrc& F, int32_t u, int32_t v, float* x) {
    float a[BM_FT], b[BM_FT];
#pragma unroll
    for (int i = 0; i < BM_FT; i++) {
        a[i] = F.tab[(size_t)u * BM_FT + i];
        b[i] = F.tab[(size_t)v * BM_FT + i];
    }
    const int32_t fu = F.pi[u], fv = F.pi[v];
    pair_features(a, b, bm_hash_get(F.hb, fu, fv) > 0, bm_hash_get(F.hb, fv, fu) > 0, x);
}

__global__ void pair_features_kernel(FeatSrc F, const int32_t* __restrict__ pairs, int64_t k, float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        float x[BM_MLP_IN];
        const int32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (u == v) {
            for (int j = 0; j < BM_MLP_IN; j++) x[j] = 0.f;
        } else {
            pair_features_lookup(F, u, v, x);
        }
        for (int j = 0; j < BM_MLP_IN; j++) out[i * BM_MLP_IN + j] = x[j];
    }
}

// ------------------------------------------------- SIMT forward / backward

constexpr int kTile = 32;  // pairs per tile
constexpr int kMT = 128;   // threads = hidden width

struct MlpSmem {
    float w1[BM_MLP_IN * BM_MLP_H];  // BF16-rounded
    float w2[BM_MLP_H * BM_MLP_H];   // BF16-rounded
    float b1[BM_MLP_H], b2[BM_MLP_H], w3[BM_MLP_H];
    float x[kTile][BM_MLP_IN];
    float h1[kTile][BM_MLP_H];
    float h2[kTile][BM_MLP_H];
    float out[kTile];
    int valid[kTile];
};

struct GradSmem {
    MlpSmem f;
    float gw2[BM_MLP_H * BM_MLP_H];  // block partial of dW2 (thread j owns column j)
    float dh2[kTile][BM_MLP_H];
    float dout[kTile];
};

__device__ void load_weights(MlpSmem& s, const float* __restrict__ w) {
    for (int i = threadIdx.x; i < kNW1; i += blockDim.x) s.w1[i] = bf16r(w[i]);
    for (int i = threadIdx.x; i < BM_MLP_H * BM_MLP_H; i += blockDim.x) s.w2[i] = bf16r(w[kOffW2 + i]);
    for (int i = threadIdx.x; i < BM_MLP_H; i += blockDim.x) {
        s.b1[i] = w[kOffB1 + i];
        s.b2[i] = w[kOffB2 + i];
        s.w3[i] = bf16r(w[kOffW3 + i]);
    }
}

// Forward of one tile of np pairs (x filled); thread j = hidden unit j.
__device__ void tile_forward(MlpSmem& s, int np, float b3) {
    const int j = threadIdx.x;
    for (int p = 0; p < np; p++) {
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < BM_MLP_IN; i++) acc = fmaf(s.x[p][i], s.w1[i * BM_MLP_H + j], acc);
        s.h1[p][j] = bf16r(fmaxf(acc + s.b1[j], 0.f));
    }
    __syncthreads();
    for (int p = 0; p < np; p++) {
        float acc = 0.f;
        for (int i = 0; i < BM_MLP_H; i++) acc = fmaf(s.h1[p][i], s.w2[i * BM_MLP_H + j], acc);
        s.h2[p][j] = bf16r(fmaxf(acc + s.b2[j], 0.f));
    }
    __syncthreads();
    const int lane = j & 31, warp = j >> 5;
    for (int p = warp; p < np; p += kMT / 32) {
        float acc = 0.f;
        for (int i = lane; i < BM_MLP_H; i += 32) acc = fmaf(s.h2[p][i], s.w3[i], acc);
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) s.out[p] = acc + b3;
    }
    __syncthreads();
}

// Input of pair q: explicit float features (xin, k x 24), BF16 records
// (xbf, k x 24), a pair list, or rows x all partners (q -> u = rows[q / n],
// v = q % n + 1).  Returns false for u == v.
struct PairSrc {
    const float* xin;
    const uint16_t* xbf;
    const int32_t* pairs;
    const int32_t* rows;
    int32_t n;             // partners per row: all vertices, or cands' row length
    const int32_t* cands;  // [rows][n] partner lists; null = partners 1..n
};

__device__ __forceinline__ bool load_pair(const FeatSrc& F, const PairSrc& P, int64_t q, float* x) {
    if (P.xin) {
        for (int i = 0; i < BM_MLP_IN; i++) x[i] = bf16r(P.xin[q * BM_MLP_IN + i]);
        return true;
    }
    if (P.xbf) {
        for (int i = 0; i < BM_MLP_IN; i++) x[i] = bf16_to_float(P.xbf[q * BM_MLP_IN + i]);
        return true;
    }
    int32_t u, v;
    if (P.pairs) {
        u = P.pairs[2 * q];
        v = P.pairs[2 * q + 1];
    } else {
        u = P.rows[q / P.n];
        v = P.cands ? P.cands[q] : (int32_t)(q % P.n) + 1;
    }
    if (u == v) {
        for (int i = 0; i < BM_MLP_IN; i++) x[i] = 0.f;
        return false;
    }
    pair_features_lookup(F, u, v, x);
    return true;
}

__global__ void __launch_bounds__(kMT) mlp_score_kernel(FeatSrc F, PairSrc P, const float* __restrict__ w, int64_t k,
                                                        float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    MlpSmem& s = *reinterpret_cast<MlpSmem*>(sm_raw);
    load_weights(s, w);
    const float b3 = w[kOffB3];
    __syncthreads();
    for (int64_t t0 = (int64_t)blockIdx.x * kTile; t0 < k; t0 += (int64_t)gridDim.x * kTile) {
        const int np = (int)min((int64_t)kTile, k - t0);
        if (threadIdx.x < np) {
            float x[BM_MLP_IN];
            s.valid[threadIdx.x] = load_pair(F, P, t0 + threadIdx.x, x);
            for (int i = 0; i < BM_MLP_IN; i++) s.x[threadIdx.x][i] = x[i];
        }
        __syncthreads();
        tile_forward(s, np, b3);
        if (threadIdx.x < np) out[t0 + threadIdx.x] = s.valid[threadIdx.x] ? s.out[threadIdx.x] : -INFINITY;
        __syncthreads();
    }
}

// Loss mean((out - y)^2) over k pairs and its gradient, added into g (zeroed
// by the caller); the loss is added into *loss.
__global__ void __launch_bounds__(kMT) mlp_grad_kernel(FeatSrc F, PairSrc P, const float* __restrict__ w,
                                                       const float* __restrict__ y, int64_t k, float* __restrict__ g,
                                                       float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    GradSmem& G = *reinterpret_cast<GradSmem*>(sm_raw);
    MlpSmem& s = G.f;
    load_weights(s, w);
    for (int i = threadIdx.x; i < BM_MLP_H * BM_MLP_H; i += blockDim.x) G.gw2[i] = 0.f;
    const float b3 = w[kOffB3];
    __syncthreads();
    const int j = threadIdx.x;
    float gw1[BM_MLP_IN];
#pragma unroll
    for (int i = 0; i < BM_MLP_IN; i++) gw1[i] = 0.f;
    float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, lsum = 0.f;
    const float scale = 2.0f / (float)k;
    for (int64_t t0 = (int64_t)blockIdx.x * kTile; t0 < k; t0 += (int64_t)gridDim.x * kTile) {
        const int np = (int)min((int64_t)kTile, k - t0);
        if (j < np) {
            float x[BM_MLP_IN];
            load_pair(F, P, t0 + j, x);
            for (int i = 0; i < BM_MLP_IN; i++) s.x[j][i] = x[i];
        }
        __syncthreads();
        tile_forward(s, np, b3);
        if (j < np) {
            const float r = s.out[j] - y[t0 + j];
            G.dout[j] = scale * r;
            lsum += r * r;
        }
        __syncthreads();
        for (int p = 0; p < np; p++) {
            const float d = G.dout[p];
            gw3 = fmaf(d, s.h2[p][j], gw3);
            const float dh = s.h2[p][j] > 0.f ? d * s.w3[j] : 0.f;
            G.dh2[p][j] = dh;
            gb2 += dh;
            if (j == 0) gb3 += d;
        }
        __syncthreads();
        for (int i = 0; i < BM_MLP_H; i++) {
            float acc = G.gw2[i * BM_MLP_H + j];
            for (int p = 0; p < np; p++) acc = fmaf(s.h1[p][i], G.dh2[p][j], acc);
            G.gw2[i * BM_MLP_H + j] = acc;
        }
        for (int p = 0; p < np; p++) {
            if (s.h1[p][j] > 0.f) {
                float acc = 0.f;
                for (int q = 0; q < BM_MLP_H; q++) acc = fmaf(s.w2[j * BM_MLP_H + q], G.dh2[p][q], acc);
                gb1 += acc;
#pragma unroll
                for (int i = 0; i < BM_MLP_IN; i++) gw1[i] = fmaf(s.x[p][i], acc, gw1[i]);
            }
        }
        __syncthreads();
    }
    for (int i = 0; i < BM_MLP_H; i++) {
        const float v = G.gw2[i * BM_MLP_H + j];
        if (v != 0.f) atomicAdd(&g[kOffW2 + i * BM_MLP_H + j], v);
    }
#pragma unroll
    for (int i = 0; i < BM_MLP_IN; i++)
        if (gw1[i] != 0.f) atomicAdd(&g[i * BM_MLP_H + j], gw1[i]);
    atomicAdd(&g[kOffB1 + j], gb1);
    atomicAdd(&g[kOffB2 + j], gb2);
    atomicAdd(&g[kOffW3 + j], gw3);
    if (j == 0) atomicAdd(&g[kOffB3], gb3);
    for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((j & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum / (float)k);
}

__global__ void adamw_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                             const float* __restrict__ g, int n, float lr, float b1, float b2, float eps, float wd,
                             float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * w[i]);
    }
}

// Training target of an exact delta: sign(d) * log1p(|d|) / 8.
__host__ __device__ __forceinline__ float delta_target(long long d) {
    const double a = log1p((double)(d < 0 ? -d : d)) / 8.0;
    return (float)(d < 0 ? -a : a);
}

// ------------------------------------------------------------ record store

// Append k records (features of pair i under the current mapping, target of
// delta i) at ring positions (head + i) mod cap.
__global__ void append_records_kernel(FeatSrc F, const int32_t* __restrict__ pairs, const long long* __restrict__ d,
                                      int64_t k, int64_t head, int64_t cap, uint16_t* __restrict__ rx,
                                      float* __restrict__ ry) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = pairs[2 * i], v = pairs[2 * i + 1];
        float x[BM_MLP_IN];
        if (u == v) {
            for (int j = 0; j < BM_MLP_IN; j++) x[j] = 0.f;
        } else {
            pair_features_lookup(F, u, v, x);
        }
        const int64_t slot = (head + i) % cap;
        for (int j = 0; j < BM_MLP_IN; j++) rx[slot * BM_MLP_IN + j] = (uint16_t)(__float_as_uint(x[j]) >> 16);
        ry[slot] = delta_target(d[i]);
    }
}

// Records from whole rows of exact deltas (full[r * (n+1) + v]): per row up to
// `per_row` records: the improving partners (evenly spaced over them in id
// order when there are more than half of per_row) and uniform random partners
// for the rest.  One block per row writes pairs and deltas at r * per_row;
// unused slots get (u, u) and delta 0 and are dropped by the caller's count.
constexpr int kHarvThreads = 256;
__global__ void __launch_bounds__(kHarvThreads) harvest_kernel(const long long* __restrict__ full,
                                                               const int32_t* __restrict__ rows, int32_t n,
                                                               int32_t per_row, uint64_t seed, int32_t* __restrict__ pairs,
                                                               long long* __restrict__ deltas) {
    __shared__ uint32_t wcnt[kHarvThreads / 32];
    __shared__ uint32_t s_npos, s_base;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int32_t r = blockIdx.x;
    const int32_t u = rows[r];
    const long long* row = full + (size_t)r * ((size_t)n + 1);
    int32_t* pr = pairs + (size_t)r * per_row * 2;
    long long* dr = deltas + (size_t)r * per_row;
    if (tid == 0) { s_npos = 0; s_base = 0; }
    __syncthreads();
    uint32_t cnt = 0;
    for (int32_t v = 1 + tid; v <= n; v += kHarvThreads) cnt += (v != u && row[v] > 0);
    atomicAdd(&s_npos, cnt);
    __syncthreads();
    const uint32_t npos = s_npos;
    const uint32_t P = min(npos, (uint32_t)per_row / 2u);
    for (int32_t c0 = 1; c0 <= n; c0 += kHarvThreads) {
        const int32_t v = c0 + tid;
        const bool pos = v <= n && v != u && row[v] > 0;
        const uint32_t b = __ballot_sync(0xffffffffu, pos);
        if (lane == 0) wcnt[wid] = (uint32_t)__popc(b);
        __syncthreads();
        if (pos) {
            uint32_t q = s_base + (uint32_t)__popc(b & ((1u << lane) - 1u));
            for (int w = 0; w < wid; w++) q += wcnt[w];
            // take positive number q when floor((q+1)P/npos) > floor(qP/npos)
            const uint64_t a0 = (uint64_t)q * P / npos, a1 = (uint64_t)(q + 1) * P / npos;
            if (a1 > a0) {
                pr[2 * a0] = u;
                pr[2 * a0 + 1] = v;
                dr[a0] = row[v];
            }
        }
        __syncthreads();
        if (tid == 0)
            for (int w = 0; w < kHarvThreads / 32; w++) s_base += wcnt[w];
        __syncthreads();
    }
    for (int32_t j = (int32_t)P + tid; j < per_row; j += kHarvThreads) {
        int32_t v = u;
        if (n > 1) {
            const uint32_t c[4] = {(uint32_t)j, (uint32_t)u, 0x48525653u, 0u};
            const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
            uint32_t o[4];
            bm_philox4x32_10(c, key, o);
            v = 1 + (int32_t)(o[0] % (uint32_t)(n - 1));
            if (v >= u) v++;  // uniform over partners other than u
        }
        pr[2 * j] = u;
        pr[2 * j + 1] = v;
        dr[j] = row[v];
    }
}

// Minibatch gather: B random records of the store (Philox, counter = step).
__global__ void gather_batch_kernel(const uint16_t* __restrict__ rx, const float* __restrict__ ry, int64_t size,
                                    int32_t B, uint64_t seed, uint64_t step, uint16_t* __restrict__ bx,
                                    float* __restrict__ by) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
        const uint32_t c[4] = {(uint32_t)i, (uint32_t)step, (uint32_t)(step >> 32), 0x42415443u};
        const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        uint32_t o[4];
        bm_philox4x32_10(c, key, o);
        const int64_t q = (int64_t)((((uint64_t)o[1] << 32) | o[0]) % (uint64_t)size);
        for (int j = 0; j < BM_MLP_IN; j++) bx[(size_t)i * BM_MLP_IN + j] = rx[q * BM_MLP_IN + j];
        by[i] = ry[q];
    }
}

// --------------------------------------------- tensor-core row scoring kernel
//
// One CTA per SM (768 threads, all 512 TMEM columns) scores whole rows: for
// row u, candidates v = 1..n in tiles of 128, one candidate per TMEM lane.
// The tiles of the CTA's rows flow through a pipeline of three roles; each
// role has two groups of four warps, group g taking the tiles t = g mod 2, so
// that two tiles are in flight in every role.  Tile t holds TMEM slot
// D[t & 3] (128 columns: layer 1's accumulators, then layer 2's over them,
// then the output layer's operand and accumulator) and shared-memory slots
// X[t & 1], H[t & 1].  A group ends each step with a named barrier over its
// warps, after which its first thread issues the MMAs that consume what the
// group wrote:
//   F  (warps 0-7)    build tile t's BF16 features (K padded to 32, the bias
//                     inputs in columns 24, 25) into X, then layer 1 (two K=16
//                     MMAs, M=N=128) into D;
//   E1 (warps 8-15)   read layer 1 back (tcgen05.ld 32x32b; the bias is
//                     already in it), write bf16(relu(.)) (cvt.rn.relu.bf16x2)
//                     into H, then layer 2 (nine K=16 MMAs over H, K=144 with
//                     the bias inputs in columns 128, 129) into the same D;
//   E2 (warps 16-23)  read layer 2 back, write bf16(relu(.)) as the output
//                     layer's A operand into columns 0..63 of D (two BF16 per
//                     column; each quarter is written after it was read), run
//                     the output layer (eight K=16 MMAs, N=16, A in tensor
//                     memory, w3 in row 0 of B) into columns 64..79, read the
//                     output column back and add b3.  Neither h2 nor the
//                     output layer touches shared memory, whose bandwidth the
//                     N=128 MMAs already use up.
// mbarriers, one per TMEM slot and kind: d1full, d2full, d3full (the commits
// after each layer; d1full(t) also frees X for tile t+2, d2full(t) H for tile
// t+2) and dfree (an E2 group's 128 threads: the slot is free for tile t+4).
// Use k of a slot waits for phase k & 1; no barrier can run two phases ahead
// of a waiter, since each completion needs the waiter's own earlier step.
// Every wait is bounded (the context's wait limit); a wait that runs out
// raises the CTA's abort flag, which every other wait checks, and each group
// leaves its loop together (its waits are combined over its barrier); the
// issuing threads then wait (default bound) for their last commits before
// the columns are freed.

constexpr int kTcThreads = 768;                        // F 0-7, E1 8-15, E2 16-23 (two groups each)
constexpr uint32_t kSmW1 = 0;                          // W1 (bias columns 24, 25), 8 KB
constexpr uint32_t kSmW2 = kSmW1 + kImgW1S;            // 8192: W2, K = 144 (bias columns 128, 129), 36 KB
constexpr uint32_t kSmW3 = kSmW2 + kImgW2S;            // 45056: the output layer's B (N=16, K=128), then b3 (FP32)
constexpr uint32_t kSmH = 50 * 1024;                   // H[2]: h1 operands, K = 144, 36 KB each
constexpr uint32_t kSmHBytes = 128 * kHK * 2;
constexpr uint32_t kSmX = kSmH + 2 * kSmHBytes;        // 122880: X[2]: feature operands, K = 32, 8 KB each
constexpr uint32_t kSmXBytes = 128 * 32 * 2;
constexpr uint32_t kSmBits = kSmX + 2 * kSmXBytes;     // 141312: each F group's two candidate bitmaps
static_assert(kSmW3 + kImgW3 + 16 <= kSmH && kSmH % 1024 == 0 && kSmX % 1024 == 0 && kSmBits % 16 == 0,
              "operand layout");
constexpr uint32_t kBf16One2 = 0x3F803F80u;         // two BF16 ones, packed

__host__ __device__ constexpr uint32_t bits_words(int32_t n) { return (uint32_t)(n + 32) / 32u; }
__host__ __device__ constexpr uint32_t tc_bits_bytes(int32_t n) { return (2u * bits_words(n) * 4u + 15u) & ~15u; }
__host__ __device__ constexpr uint32_t tc_tail(int32_t n) { return kSmBits + 2u * tc_bits_bytes(n); }
// two F groups' candidate bitmaps, then 16 mbarriers, the TMEM base slot and
// the abort flag (at least 138 KB in all: one CTA per SM)
__host__ __device__ constexpr uint32_t tc_smem_bytes(int32_t n) { return tc_tail(n) + 144u; }

// Byte offset of element (row r, k) in a K-major no-swizzle operand with
// kcols columns: 8-row x 8-element core matrices of 128 contiguous bytes,
// K-adjacent core matrices 128 bytes apart (the descriptor's leading byte
// offset), 8-row groups kcols/8 * 128 bytes apart (its stride byte offset).
__host__ __device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k, uint32_t kcols) {
    return (r >> 3) * (kcols / 8u) * 128u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // SM100 shared-memory matrix descriptor: start >> 4 (bits 0-13), leading
    // byte offset >> 4 (16-29), stride byte offset >> 4 (32-45), version 1
    // (bits 46-47), base offset 0, layout "no swizzle" (bits 61-63 = 0).
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bit 4), A and B BF16
// (bits 7 and 10), both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at
// bit 24.  A and B have the same type, as kind::f16 requires.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}
constexpr uint32_t kIdesc128 = idesc_bf16(128, 128);
constexpr uint32_t kIdesc16 = idesc_bf16(128, 16);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// The same with the A operand in tensor memory (M rows in lanes 0..127, K
// along the columns, two 16-bit elements per column, lower K in the low half).
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Two FP32 values to packed BF16 (round to nearest even), lo in the low half.
__device__ __forceinline__ uint32_t cvt_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
// Same with ReLU applied (negative results become +0).
__device__ __forceinline__ uint32_t cvt_relu_bf16x2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive 32-bit columns of this thread's TMEM lane, without waiting:
// the registers are valid after tmem_wait_ld().
__device__ __forceinline__ void tmem_ld32_async(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's TMEM lane from registers;
// complete after tmem_wait_st().
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* r) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};"
        :
        : "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
          "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// One 32-bit column of this thread's TMEM lane.
__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return r;
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier: try_wait suspends the thread
// until the phase completes or a hardware time slice passes; the loop gives up
// once `limit` SM clock cycles (by default kWaitLimit, about two seconds) have
// passed, checked before every try, and returns false.
constexpr long long kWaitLimit = 4000000000ll;
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit = kWaitLimit) {
    const long long t0 = clock64();
    for (;;) {
        if (clock64() - t0 >= limit) return false;
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
}

__global__ void prep_image_kernel(const float* __restrict__ w, unsigned char* __restrict__ img) {
    // the training image: W1, W2, W3, the epilogue vectors, W2^T
    unsigned short* w1 = reinterpret_cast<unsigned short*>(img);
    unsigned short* w2 = reinterpret_cast<unsigned short*>(img + kImgW1);
    unsigned short* w3 = reinterpret_cast<unsigned short*>(img + kImgW1 + kImgW2);
    float* ep = reinterpret_cast<float*>(img + kImgW1 + kImgW2 + kImgW3);
    unsigned short* w2t = reinterpret_cast<unsigned short*>(img + kImgOffW2T);
    unsigned short* s1 = reinterpret_cast<unsigned short*>(img + kImgOffS);
    unsigned short* s2 = reinterpret_cast<unsigned short*>(img + kImgOffS + kImgW1S);
    const int n1 = 128 * 32, n2 = 128 * 128, n3 = 16 * 128;
    const int nt = n1 + n2 + n3 + 3 * 128 + 4 + n2;  // the training image
    const int total = nt + n1 + 128 * kHK;
    // a bias as the BF16 pair (hi, lo) of a folded column
    auto hi = [](float b) { return bf16r(b); };
    auto lo = [](float b) { return bf16r(b - bf16r(b)); };
    auto put = [](unsigned short* p, float v) { *p = (unsigned short)(__float_as_uint(v) >> 16); };
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t < n1) {
            const int j = t / 32, i = t % 32;  // hidden j (N), input i (K)
            const float v = i < BM_MLP_IN ? bf16r(w[i * BM_MLP_H + j]) : 0.f;
            w1[kmajor_off(j, i, 32) / 2] = (unsigned short)(__float_as_uint(v) >> 16);
        } else if (t < n1 + n2) {
            const int q = t - n1, j = q / 128, i = q % 128;  // out j (N), in i (K)
            const float v = bf16r(w[kOffW2 + i * BM_MLP_H + j]);
            w2[kmajor_off(j, i, 128) / 2] = (unsigned short)(__float_as_uint(v) >> 16);
        } else if (t < n1 + n2 + n3) {
            const int q = t - n1 - n2, j = q / 128, i = q % 128;  // row j (N = 16), in i (K)
            const float v = j == 0 ? bf16r(w[kOffW3 + i]) : 0.f;
            w3[kmajor_off(j, i, 128) / 2] = (unsigned short)(__float_as_uint(v) >> 16);
        } else if (t < n1 + n2 + n3 + 3 * 128 + 4) {
            const int q = t - n1 - n2 - n3;
            if (q < 128) ep[q] = w[kOffB1 + q];
            else if (q < 256) ep[q] = w[kOffB2 + q - 128];
            else if (q < 384) ep[q] = bf16r(w[kOffW3 + q - 256]);
            else ep[q] = (q == 384) ? w[kOffB3] : 0.f;
        } else if (t < nt) {
            const int q = t - (n1 + n2 + n3 + 3 * 128 + 4), i = q / 128, j = q % 128;  // in i (N), out j (K)
            const float v = bf16r(w[kOffW2 + i * BM_MLP_H + j]);
            w2t[kmajor_off(i, j, 128) / 2] = (unsigned short)(__float_as_uint(v) >> 16);
        } else if (t < nt + n1) {
            const int q = t - nt, j = q / 32, i = q % 32;  // hidden j (N), input i (K)
            const float b = w[kOffB1 + j];
            const float v = i < BM_MLP_IN ? bf16r(w[i * BM_MLP_H + j]) : i == 24 ? hi(b) : i == 25 ? lo(b) : 0.f;
            put(s1 + kmajor_off(j, i, 32) / 2, v);
        } else {
            const int q = t - nt - n1, j = q / kHK, i = q % kHK;  // out j (N), in i (K)
            const float b = w[kOffB2 + j];
            const float v = i < 128 ? bf16r(w[kOffW2 + i * BM_MLP_H + j]) : i == 128 ? hi(b) : i == 129 ? lo(b) : 0.f;
            put(s2 + kmajor_off(j, i, kHK) / 2, v);
        }
    }
}

struct TcArgs {
    const unsigned char* img;
    const float* tab;
    const int32_t* rows;
    int32_t nrows;
    int32_t n;
    const int32_t* b_optr;  // B lists with ids relabelled to A space (B'-out, B'-in)
    const uint32_t* b_oent;
    const int32_t* b_iptr;
    const uint32_t* b_ient;
    const int32_t* pi;
    float* scores;  // [nrows x span], row r at r * span: partner v at v - 1, or list entry i at i
    int32_t* flag;
    long long wait_limit;  // bound of each MMA-completion wait, SM cycles
    const int32_t* cands;  // [nrows x span] partner lists (never u itself); null = partners 1..n
    int32_t span;          // n, or the lists' length
};

// Candidate v's vertex record (12 floats).
struct CandRec {
    float4 q[3];
};
__device__ __forceinline__ CandRec load_cand(const TcArgs& a, int32_t v) {
    CandRec c;
    if (v <= a.n) {
        const float4* t4 = reinterpret_cast<const float4*>(a.tab + (size_t)v * BM_FT);
        c.q[0] = t4[0]; c.q[1] = t4[1]; c.q[2] = t4[2];
    } else {
        c.q[0] = c.q[1] = c.q[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    return c;
}

// Features of candidate v of row u into row `row` of the X operand at xs.
__device__ __forceinline__ void build_features(const TcArgs& a, const float* ta, const uint32_t* bits_out,
                                               const uint32_t* bits_in, int32_t u, int32_t v, const CandRec& cr,
                                               unsigned char* xs, int row) {
    float x[BM_MLP_IN];
    if (v <= a.n && v != u) {
        float tb[BM_FT];
        const float4 q0 = cr.q[0], q1 = cr.q[1], q2 = cr.q[2];
        tb[0] = q0.x; tb[1] = q0.y; tb[2] = q0.z; tb[3] = q0.w;
        tb[4] = q1.x; tb[5] = q1.y; tb[6] = q1.z; tb[7] = q1.w;
        tb[8] = q2.x; tb[9] = q2.y; tb[10] = q2.z; tb[11] = q2.w;
        const bool buv = (bits_out[v >> 5] >> (v & 31)) & 1u;
        const bool bvu = (bits_in[v >> 5] >> (v & 31)) & 1u;
        pair_features_raw(ta, tb, buv, bvu, x);
    } else {
#pragma unroll
        for (int i = 0; i < BM_MLP_IN; i++) x[i] = 0.f;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        uint4 q = make_uint4(kBf16One2, 0u, 0u, 0u);  // columns 24, 25: the bias inputs
        if (c < 3) {
            q.x = cvt_bf16x2(x[8 * c + 0], x[8 * c + 1]);
            q.y = cvt_bf16x2(x[8 * c + 2], x[8 * c + 3]);
            q.z = cvt_bf16x2(x[8 * c + 4], x[8 * c + 5]);
            q.w = cvt_bf16x2(x[8 * c + 6], x[8 * c + 7]);
        }
        *reinterpret_cast<uint4*>(xs + kmajor_off(row, 8 * c, 32)) = q;
    }
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// Bounded wait of one role: gives up when the wait limit passes or another
// role raised the abort flag (both checked before every try).
__device__ __forceinline__ bool role_wait(uint32_t mbar, uint32_t parity, long long limit, volatile int* abort) {
    const long long t0 = clock64();
    for (;;) {
        if (*abort || clock64() - t0 >= limit) return false;
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
}

// Named barrier `id` over one role's four warps (128 threads), AND of v.
__device__ __forceinline__ bool role_bar_and(uint32_t id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %2, 0;\n\t"
        "bar.red.and.pred p, %1, 128, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"(id), "r"((uint32_t)v)
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void role_bar(uint32_t id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

__global__ void __launch_bounds__(kTcThreads, 1) mlp_rows_tc_kernel(TcArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int role = warp >> 3;                 // 0 F, 1 E1, 2 E2
    const int grp = (warp >> 2) & 1;            // the tiles t = grp mod 2
    const int gtid = tid & 127;                 // thread in the group = TMEM lane / tile row
    const bool leader = gtid == 0;
    const uint32_t gbar = 1u + 2u * (uint32_t)role + (uint32_t)grp;  // the group's named barrier
    const uint32_t nw = bits_words(a.n);
    const uint32_t tail = tc_tail(a.n);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + tail);  // four of each kind below, one per TMEM slot
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + tail + 128);
    volatile int* abort = reinterpret_cast<volatile int*>(sm + tail + 132);
    auto bar = [&](int k, int q) { return smem_u32(&bars[4 * k + q]); };
    constexpr int D1FULL = 0, D2FULL = 1, D3FULL = 2, DFREE = 3;
    auto par = [](int32_t t) { return (uint32_t)(t >> 2) & 1u; };  // phase of tile t on its slot's barrier

    {  // the scorer image (W1, W2); the training image's output-layer B (w3 in
       // row 0) and b3 (FP32, from its epilogue vectors); the constant columns
       // of both H (128, 129: the bias inputs of layer 2; 130..143 zero)
        const uint4* src = reinterpret_cast<const uint4*>(a.img + kImgOffS);
        for (int i = tid; i < (kImgW1S + kImgW2S) / 16; i += kTcThreads) reinterpret_cast<uint4*>(sm)[i] = src[i];
        const uint4* w3src = reinterpret_cast<const uint4*>(a.img + kImgW1 + kImgW2);
        if (tid < kImgW3 / 16) reinterpret_cast<uint4*>(sm + kSmW3)[tid] = w3src[tid];
        const float* ep = reinterpret_cast<const float*>(a.img + kImgW1 + kImgW2 + kImgW3);
        if (tid == 0) *reinterpret_cast<float*>(sm + kSmW3 + kImgW3) = ep[384];
        if (tid < 256) {
            unsigned char* h = sm + kSmH + (tid >> 7) * kSmHBytes;
            const int row = tid & 127;
            *reinterpret_cast<uint4*>(h + kmajor_off(row, 128, kHK)) = make_uint4(kBf16One2, 0u, 0u, 0u);
            *reinterpret_cast<uint4*>(h + kmajor_off(row, 136, kHK)) = make_uint4(0u, 0u, 0u, 0u);
        }
    }
    if (tid == 0) {
        for (int k = 0; k < 4; k++)
            for (int q = 0; q < 4; q++) mbar_init(bar(k, q), k == DFREE ? 128u : 1u);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // the CTA's tiles: rows blockIdx.x, blockIdx.x + gridDim.x, ...; tiles of 128 candidates
    const int32_t tpr = (a.span + 127) / 128;
    const int32_t my_rows = a.nrows > (int32_t)blockIdx.x ? (a.nrows - 1 - (int32_t)blockIdx.x) / (int32_t)gridDim.x + 1 : 0;
    const int32_t T = my_rows * tpr;
    auto tile_row = [&](int32_t t, int32_t& r, int32_t& v0) {
        const int32_t ri = t / tpr;
        r = (int32_t)blockIdx.x + ri * (int32_t)gridDim.x;
        v0 = 1 + (t - ri * tpr) * 128;
    };
    const long long lim = a.wait_limit;
    bool ok = true;
    uint32_t last_bar = 0, last_par = 0;  // this thread's last commit (the issuing threads)
    const uint32_t lb = (uint32_t)((warp & 3) * 32) << 16;  // the warp's TMEM lanes

    if (role == 0) {
        // ---- F: features, then layer 1
        uint32_t* bits_out = reinterpret_cast<uint32_t*>(sm + kSmBits + grp * tc_bits_bytes(a.n));
        uint32_t* bits_in = bits_out + nw;
        const uint32_t sW1 = smem_u32(sm + kSmW1);
        const uint32_t sX = smem_u32(sm + kSmX + grp * kSmXBytes);
        float ta[BM_FT];
        int32_t u = 0, cur_r = -1;
        for (int32_t t = grp; t < T; t += 2) {
            const int q = t & 3;
            int32_t r, v0;
            tile_row(t, r, v0);
            bool w = true;
            if (t >= 2) w = role_wait(bar(D1FULL, (t - 2) & 3), par(t - 2), lim, abort);  // X free
            if (!role_bar_and(gbar, w)) { ok = false; break; }
            if (r != cur_r) {
                // a new row: its bitmaps of the v with B(pi u, pi v) > 0
                // (B'-out of u) and B(pi v, pi u) > 0 (B'-in of u), and its record
                cur_r = r;
                u = a.rows[r];
                for (uint32_t i = gtid; i < 2 * nw; i += 128) bits_out[i] = 0u;
                role_bar(gbar);
                const int32_t fu = a.pi[u];
                for (int32_t j = a.b_optr[fu] + gtid; j < a.b_optr[fu + 1]; j += 128) {
                    const uint32_t e = a.b_oent[j];
                    if (e) atomicOr(&bits_out[bm_eid(e) >> 5], 1u << (bm_eid(e) & 31));
                }
                for (int32_t j = a.b_iptr[fu] + gtid; j < a.b_iptr[fu + 1]; j += 128) {
                    const uint32_t e = a.b_ient[j];
                    if (e) atomicOr(&bits_in[bm_eid(e) >> 5], 1u << (bm_eid(e) & 31));
                }
#pragma unroll
                for (int i = 0; i < BM_FT; i++) ta[i] = a.tab[(size_t)u * BM_FT + i];
                role_bar(gbar);
            }
            // candidate: partner v0 + gtid, or list entry v0 - 1 + gtid (past the list: none)
            const int32_t ci = v0 - 1 + gtid;
            const int32_t v = a.cands ? (ci < a.span ? __ldg(a.cands + (size_t)r * a.span + ci) : a.n + 1) : v0 + gtid;
            build_features(a, ta, bits_out, bits_in, u, v, load_cand(a, v), sm + kSmX + grp * kSmXBytes, gtid);
            proxy_fence();
            // the TMEM slot is waited for only now: the features are built
            // while tile t - 4 still holds it
            w = true;
            if (t >= 4) w = role_wait(bar(DFREE, q), par(t - 4), lim, abort);
            if (!role_bar_and(gbar, w)) { ok = false; break; }
            if (leader) {
                tc_fence_after();
#pragma unroll
                for (int k = 0; k < 2; k++)
                    mma_bf16(tmem + 128u * q, smem_desc(sX + 256u * k, 128u, 512u), smem_desc(sW1 + 256u * k, 128u, 512u),
                             kIdesc128, k > 0);
                mma_commit(bar(D1FULL, q));
                last_bar = bar(D1FULL, q);
                last_par = par(t);
            }
        }
    } else if (role == 1) {
        // ---- E1: layer-1 epilogue into H, then layer 2
        unsigned char* h = sm + kSmH + grp * kSmHBytes;
        const uint32_t sH = smem_u32(h), sW2 = smem_u32(sm + kSmW2);
        for (int32_t t = grp; t < T; t += 2) {
            const int q = t & 3;
            bool w = role_wait(bar(D1FULL, q), par(t), lim, abort);
            if (w && t >= 2) w = role_wait(bar(D2FULL, (t - 2) & 3), par(t - 2), lim, abort);  // H free
            if (!role_bar_and(gbar, w)) { ok = false; break; }
            tc_fence_after();
#pragma unroll
            for (int c4 = 0; c4 < 4; c4++) {
                uint32_t d[32];
                tmem_ld32_async(tmem + 128u * q + 32u * c4 + lb, d);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    uint4 o;
                    o.x = cvt_relu_bf16x2(__uint_as_float(d[8 * c + 0]), __uint_as_float(d[8 * c + 1]));
                    o.y = cvt_relu_bf16x2(__uint_as_float(d[8 * c + 2]), __uint_as_float(d[8 * c + 3]));
                    o.z = cvt_relu_bf16x2(__uint_as_float(d[8 * c + 4]), __uint_as_float(d[8 * c + 5]));
                    o.w = cvt_relu_bf16x2(__uint_as_float(d[8 * c + 6]), __uint_as_float(d[8 * c + 7]));
                    *reinterpret_cast<uint4*>(h + kmajor_off(gtid, 32 * c4 + 8 * c, kHK)) = o;
                }
            }
            proxy_fence();
            tc_fence_before();
            role_bar(gbar);
            if (leader) {
                tc_fence_after();
#pragma unroll
                for (int k = 0; k < kHK / 16; k++)
                    mma_bf16(tmem + 128u * q, smem_desc(sH + 256u * k, 128u, kHK / 8 * 128u),
                             smem_desc(sW2 + 256u * k, 128u, kHK / 8 * 128u), kIdesc128, k > 0);
                mma_commit(bar(D2FULL, q));
                last_bar = bar(D2FULL, q);
                last_par = par(t);
            }
        }
    } else {
        // ---- E2: h2 = bf16(relu(D2)) into columns 0..63 of the tile's slot,
        // the output layer, its column back + b3
        const uint32_t sW3 = smem_u32(sm + kSmW3);
        const float b3 = *reinterpret_cast<const float*>(sm + kSmW3 + kImgW3);
        int32_t cur_r = -1, u = 0;
        for (int32_t t = grp; t < T; t += 2) {
            const int q = t & 3;
            int32_t r, v0;
            tile_row(t, r, v0);
            if (r != cur_r) { cur_r = r; u = a.rows[r]; }
            bool w = role_wait(bar(D2FULL, q), par(t), lim, abort);
            if (!role_bar_and(gbar, w)) { ok = false; break; }
            tc_fence_after();
            const uint32_t d2 = tmem + 128u * q + lb;
#pragma unroll
            for (int c4 = 0; c4 < 4; c4++) {
                // columns 32 c4 .. 32 c4 + 31 in, packed into 16 c4 .. 16 c4 + 15
                // (columns already read)
                uint32_t d[32], hh[16];
                tmem_ld32_async(d2 + 32u * c4, d);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 16; c++) hh[c] = cvt_relu_bf16x2(__uint_as_float(d[2 * c]), __uint_as_float(d[2 * c + 1]));
                tmem_st16(d2 + 16u * c4, hh);
            }
            tmem_wait_st();
            tc_fence_before();
            role_bar(gbar);
            if (leader) {
                tc_fence_after();
                const uint32_t dq = tmem + 128u * q;
#pragma unroll
                for (int k = 0; k < 8; k++)
                    mma_bf16_ts(dq + 64u, dq + 8u * k, smem_desc(sW3 + 256u * k, 128u, 2048u), kIdesc16, k > 0);
                mma_commit(bar(D3FULL, q));
                last_bar = bar(D3FULL, q);
                last_par = par(t);
            }
            w = role_wait(bar(D3FULL, q), par(t), lim, abort);
            if (!role_bar_and(gbar, w)) { ok = false; break; }
            tc_fence_after();
            const float o = __uint_as_float(tmem_ld1(d2 + 64u)) + b3;
            tc_fence_before();
            mbar_arrive(bar(DFREE, q));  // the slot is free for tile t + 4
            const int32_t ci = v0 - 1 + gtid;
            if (ci < a.span) a.scores[(size_t)r * a.span + ci] = (a.cands || ci + 1 != u) ? o : -INFINITY;
        }
    }
    if (!ok) {
        *abort = 1;
        atomicExch(a.flag, 1);
    }
    tc_fence_before();
    __syncthreads();
    // after an abort the issuing threads let their MMAs in flight finish
    // before the columns are freed (the default bound, whatever bound the
    // waits above were given); otherwise every commit has been waited on
    if (*abort && last_bar) mbar_wait(last_bar, last_par);
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// Make this thread's generic shared-memory writes visible to the tensor cores
// and order its earlier tcgen05 accesses before the barrier.
__device__ __forceinline__ void tc_handoff() {
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// ------------------------------------------- tensor-core training kernel
//
// Loss mean((out - y)^2) over k records and its gradient, with every matrix
// product of the forward and backward passes on the tensor cores (tcgen05
// MMA, BF16 operands in shared memory, FP32 accumulators in TMEM).  One CTA
// (128 threads, one record per thread and TMEM lane) takes tiles of 128
// records; per tile:
//   1. X = the records' features (K padded to 32) and X^T;
//   2. layer 1: D1 = X . W1 (TMEM columns 0..127); h1 = bf16(relu(D1 + b1))
//      into H (record rows) and H1^T (hidden rows);
//   3. layer 2: D2 = H . W2 (columns 128..255); h2 = bf16(relu(D2 + b2)) into
//      H2^T (over H), the output o = h2 . w3 + b3, r = o - y, dout = 2 r / k,
//      dh2 = bf16(h2 > 0 ? dout w3 : 0) into dH2 (record rows) and dH2^T;
//   4. dH1 = dH2 . W2^T (columns 0..127) and dW2 += H1^T . dH2 (columns
//      256..383, accumulated over the CTA's tiles); meanwhile thread j sums row
//      j of dH2^T (db2) and dout . row j of H2^T (dw3);
//   5. dh1 = bf16(h1 > 0 ? dH1 : 0) into dH1^T (over dH2);
//   6. dW1^T += dH1^T . X^T (N = 32, columns 384..415); thread j sums row j of
//      dH1^T (db1).
// At the end each CTA reads its dW2 and dW1^T accumulators back and adds them,
// with its bias and w3 sums, into the FP32 gradient (atomics).  Rounding: as
// the SIMT kernel, plus dh2 and dh1 rounded to BF16 (they are MMA operands);
// the bias sums use the rounded values.
//
// Operands whose K index is the record (H1^T, H2^T, dH2^T, dH1^T, X^T) are
// written by each thread as its own K column, one 16-bit element per store.
// Their core matrices are 144 bytes apart along K (the descriptor's leading
// byte offset) instead of 128, so the four groups of eight lanes of a warp
// store into distinct banks; the 8-row groups are 16 x 144 = 2,304 bytes
// apart.
constexpr int kTrThreads = 128;
constexpr uint32_t kTLbo = 144, kTSbo = 16 * kTLbo;  // transposed operands
constexpr uint32_t kTBytes128 = 16 * kTSbo;          // 128 rows: 36,864 bytes
__host__ __device__ __forceinline__ uint32_t tmajor_off(uint32_t r, uint32_t k) {
    return (r >> 3) * kTSbo + (k >> 3) * kTLbo + (r & 7u) * 16u + (k & 7u) * 2u;
}
constexpr uint32_t kTrW1 = 0;                          // W1 image (8 KB)
constexpr uint32_t kTrW2 = kTrW1 + kImgW1;             // 8192: W2 image (32 KB)
constexpr uint32_t kTrW2T = kTrW2 + kImgW2;            // 40960: W2^T image (32 KB)
constexpr uint32_t kTrXT = kTrW2T + kImgW2T;           // 73728: X^T, feature rows 0..23 (row group 3 holds
                                                       //   b1, b2, w3, b3 and the tile's dout; it only feeds
                                                       //   the unused columns 24..31 of dW1^T)
constexpr uint32_t kTrEp = kTrXT + 3 * kTSbo;          // 80640
constexpr uint32_t kTrDout = kTrEp + ((kImgEp + 15) & ~15);
constexpr uint32_t kTrH = kTrXT + 4 * kTSbo;           // 82944: h1 (record rows), then h2^T
constexpr uint32_t kTrH1T = kTrH + kTBytes128;         // 119808: h1^T
constexpr uint32_t kTrD = kTrH1T + kTBytes128;         // 156672: X, then dh2 (record rows), then dh1^T
constexpr uint32_t kTrDT = kTrD + kTBytes128;          // 193536: dh2^T
constexpr uint32_t kTrBars = kTrDT + kTBytes128;       // 230400: four mbarriers, then the TMEM base slot
constexpr uint32_t kTrSmem = kTrBars + 48;
static_assert(kTrDout + 128 * 4 <= kTrH, "epilogue vectors in X^T's spare row group");
static_assert(kTrXT % 1024 == 0 && kTrH % 16 == 0 && kTrH1T % 16 == 0 && kTrD % 16 == 0 && kTrDT % 16 == 0,
              "training operand alignment");
static_assert(kTrSmem <= 227 * 1024, "training kernel shared memory");
constexpr uint32_t kIdesc32 = idesc_bf16(128, 32);

struct TrArgs {
    const unsigned char* img;
    const float* xin;      // k x 24 float features, or
    const uint16_t* xbf;   // k x 24 BF16 records
    const float* y;
    int64_t k;
    float* g;              // gradient (zeroed by the caller), FP32, parameter order
    float* loss;           // += mean squared error
    int32_t* flag;
    long long wait_limit;
};

__device__ __forceinline__ uint16_t bf16_bits(float x) { return (uint16_t)(cvt_bf16x2(x, 0.f) & 0xFFFFu); }

// Element (row r, this thread's record p) of a transposed operand.
__device__ __forceinline__ void st_t(unsigned char* base, uint32_t r, uint32_t p, uint16_t v) {
    *reinterpret_cast<uint16_t*>(base + tmajor_off(r, p)) = v;
}

// Sum of row j of a transposed operand (128 BF16 values).
__device__ __forceinline__ float row_sum_t(const unsigned char* base, uint32_t j) {
    float s = 0.f;
#pragma unroll 4
    for (int c = 0; c < 16; c++) {
        const uint4 q = *reinterpret_cast<const uint4*>(base + tmajor_off(j, 8 * c));
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int e = 0; e < 4; e++) s += __uint_as_float(w[e] << 16) + __uint_as_float(w[e] & 0xFFFF0000u);
    }
    return s;
}

// Row j of a transposed operand dotted with the tile's dout.
__device__ __forceinline__ float row_dot_t(const unsigned char* base, uint32_t j, const float* dout) {
    float s = 0.f;
#pragma unroll 4
    for (int c = 0; c < 16; c++) {
        const uint4 q = *reinterpret_cast<const uint4*>(base + tmajor_off(j, 8 * c));
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            s = fmaf(__uint_as_float(w[e] << 16), dout[8 * c + 2 * e], s);
            s = fmaf(__uint_as_float(w[e] & 0xFFFF0000u), dout[8 * c + 2 * e + 1], s);
        }
    }
    return s;
}

__global__ void __launch_bounds__(kTrThreads, 1) mlp_train_tc_kernel(TrArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kTrBars);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kTrBars + 32);
    uint32_t bar[4];
#pragma unroll
    for (int b = 0; b < 4; b++) bar[b] = smem_u32(&bars[b]);
    const float* ep = reinterpret_cast<const float*>(sm + kTrEp);  // b1 [0..127], b2 [128..], w3 [256..], b3 [384]
    float* dsm = reinterpret_cast<float*>(sm + kTrDout);
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.img);
        for (int i = tid; i < (kImgW1 + kImgW2) / 16; i += kTrThreads) reinterpret_cast<uint4*>(sm + kTrW1)[i] = src[i];
        for (int i = tid; i < kImgW2T / 16; i += kTrThreads)
            reinterpret_cast<uint4*>(sm + kTrW2T)[i] = src[kImgOffW2T / 16 + i];
        for (int i = tid; i < kImgEp / 16; i += kTrThreads)
            reinterpret_cast<uint4*>(sm + kTrEp)[i] = src[(kImgW1 + kImgW2 + kImgW3) / 16 + i];
    }
    if (tid == 0) {
        for (int b = 0; b < 4; b++) mbar_init(bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_handoff();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lb = (uint32_t)(warp * 32) << 16;
    const uint32_t tD1 = tmem, tD2 = tmem + 128u, tW2 = tmem + 256u, tW1 = tmem + 384u;
    const uint32_t sXT = smem_u32(sm + kTrXT), sH = smem_u32(sm + kTrH), sH1T = smem_u32(sm + kTrH1T),
                   sD = smem_u32(sm + kTrD), sDT = smem_u32(sm + kTrDT), sW1 = smem_u32(sm + kTrW1),
                   sW2 = smem_u32(sm + kTrW2), sW2T = smem_u32(sm + kTrW2T);
    const uint32_t p = (uint32_t)tid;
    const float scale = 2.0f / (float)a.k;
    const int64_t tiles = (a.k + 127) / 128;
    float gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, lsum = 0.f;
    uint32_t phase = 0, last_bar = 0, last_par = 0;
    bool ok = true, first = true;
    auto wait = [&](int b) -> bool { return __syncthreads_and(mbar_wait(bar[b], phase, a.wait_limit)); };
    auto commit = [&](int b) {
        if (tid == 0) mma_commit(bar[b]);
        last_bar = bar[b];
        last_par = phase;
    };
    for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int64_t q = t * 128 + tid;
        const bool valid = q < a.k;
        // ---- 1. features: X (record rows, K = 32, in D's space) and X^T
        {
            float x[BM_MLP_IN];
            if (valid && a.xbf) {
                const uint4* r4 = reinterpret_cast<const uint4*>(a.xbf + q * BM_MLP_IN);
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const uint4 v4 = r4[c];
                    const uint32_t w[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        x[8 * c + 2 * e] = __uint_as_float(w[e] << 16);
                        x[8 * c + 2 * e + 1] = __uint_as_float(w[e] & 0xFFFF0000u);
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < BM_MLP_IN; i++) x[i] = valid ? a.xin[q * BM_MLP_IN + i] : 0.f;
            }
#pragma unroll
            for (int c = 0; c < 4; c++) {
                uint4 o = make_uint4(0u, 0u, 0u, 0u);
                if (c < 3) {
                    o.x = cvt_bf16x2(x[8 * c + 0], x[8 * c + 1]);
                    o.y = cvt_bf16x2(x[8 * c + 2], x[8 * c + 3]);
                    o.z = cvt_bf16x2(x[8 * c + 4], x[8 * c + 5]);
                    o.w = cvt_bf16x2(x[8 * c + 6], x[8 * c + 7]);
                }
                *reinterpret_cast<uint4*>(sm + kTrD + kmajor_off(p, 8 * c, 32)) = o;
            }
#pragma unroll
            for (int f = 0; f < BM_MLP_IN; f++) st_t(sm + kTrXT, (uint32_t)f, p, bf16_bits(x[f]));
        }
        const float yv = valid ? a.y[q] : 0.f;
        tc_handoff();
        // ---- 2. layer 1
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < 2; s++)
                mma_bf16(tD1, smem_desc(sD + 256u * s, 128u, 512u), smem_desc(sW1 + 256u * s, 128u, 512u), kIdesc128,
                         s > 0);
        }
        commit(0);
        if (!wait(0)) { ok = false; break; }
        tc_fence_after();
        uint32_t m1[4];  // h1 > 0, one bit per hidden unit
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float d[32];
            tmem_ld32(tD1 + lb + 32u * c, d);
            uint32_t hb[16];
            m1[c] = 0u;
#pragma unroll
            for (int e = 0; e < 16; e++) {
                hb[e] = cvt_relu_bf16x2(d[2 * e] + ep[32 * c + 2 * e], d[2 * e + 1] + ep[32 * c + 2 * e + 1]);
                if (hb[e] & 0xFFFFu) m1[c] |= 1u << (2 * e);
                if (hb[e] >> 16) m1[c] |= 1u << (2 * e + 1);
            }
#pragma unroll
            for (int qd = 0; qd < 4; qd++)
                *reinterpret_cast<uint4*>(sm + kTrH + kmajor_off(p, 32 * c + 8 * qd, 128)) =
                    make_uint4(hb[4 * qd], hb[4 * qd + 1], hb[4 * qd + 2], hb[4 * qd + 3]);
#pragma unroll
            for (int e = 0; e < 16; e++) {
                st_t(sm + kTrH1T, (uint32_t)(32 * c + 2 * e), p, (uint16_t)(hb[e] & 0xFFFFu));
                st_t(sm + kTrH1T, (uint32_t)(32 * c + 2 * e + 1), p, (uint16_t)(hb[e] >> 16));
            }
        }
        tc_handoff();
        // ---- 3. layer 2; h2^T over H; output, loss, dh2
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < 8; s++)
                mma_bf16(tD2, smem_desc(sH + 256u * s, 128u, 2048u), smem_desc(sW2 + 256u * s, 128u, 2048u),
                         kIdesc128, s > 0);
        }
        commit(1);
        if (!wait(1)) { ok = false; break; }
        tc_fence_after();
        float o = ep[384];
        uint32_t m2[4];  // h2 > 0
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float d[32];
            tmem_ld32(tD2 + lb + 32u * c, d);
            m2[c] = 0u;
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const uint32_t h = cvt_relu_bf16x2(d[2 * e] + ep[128 + 32 * c + 2 * e],
                                                   d[2 * e + 1] + ep[128 + 32 * c + 2 * e + 1]);
                const float h0 = __uint_as_float(h << 16), h1v = __uint_as_float(h & 0xFFFF0000u);
                o = fmaf(h0, ep[256 + 32 * c + 2 * e], o);
                o = fmaf(h1v, ep[256 + 32 * c + 2 * e + 1], o);
                if (h & 0xFFFFu) m2[c] |= 1u << (2 * e);
                if (h >> 16) m2[c] |= 1u << (2 * e + 1);
                st_t(sm + kTrH, (uint32_t)(32 * c + 2 * e), p, (uint16_t)(h & 0xFFFFu));
                st_t(sm + kTrH, (uint32_t)(32 * c + 2 * e + 1), p, (uint16_t)(h >> 16));
            }
        }
        const float r = valid ? o - yv : 0.f;
        const float dout = scale * r;
        lsum += r * r;
        dsm[tid] = dout;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            uint32_t db[16];
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const int j = 32 * c + 2 * e;
                const float d0 = ((m2[c] >> (2 * e)) & 1u) ? dout * ep[256 + j] : 0.f;
                const float d1 = ((m2[c] >> (2 * e + 1)) & 1u) ? dout * ep[256 + j + 1] : 0.f;
                db[e] = cvt_bf16x2(d0, d1);
                st_t(sm + kTrDT, (uint32_t)j, p, (uint16_t)(db[e] & 0xFFFFu));
                st_t(sm + kTrDT, (uint32_t)(j + 1), p, (uint16_t)(db[e] >> 16));
            }
#pragma unroll
            for (int qd = 0; qd < 4; qd++)
                *reinterpret_cast<uint4*>(sm + kTrD + kmajor_off(p, 32 * c + 8 * qd, 128)) =
                    make_uint4(db[4 * qd], db[4 * qd + 1], db[4 * qd + 2], db[4 * qd + 3]);
        }
        tc_handoff();
        // ---- 4. dH1 = dH2 . W2^T and dW2 += H1^T . dH2
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < 8; s++)
                mma_bf16(tD1, smem_desc(sD + 256u * s, 128u, 2048u), smem_desc(sW2T + 256u * s, 128u, 2048u),
                         kIdesc128, s > 0);
#pragma unroll
            for (int s = 0; s < 8; s++)
                mma_bf16(tW2, smem_desc(sH1T + 2u * kTLbo * s, kTLbo, kTSbo),
                         smem_desc(sDT + 2u * kTLbo * s, kTLbo, kTSbo), kIdesc128, (first && s == 0) ? 0u : 1u);
        }
        commit(2);
        gb2 += row_sum_t(sm + kTrDT, p);
        gw3 += row_dot_t(sm + kTrH, p, dsm);
        if (tid == 0) {
            float sd = 0.f;
            for (int i = 0; i < 128; i++) sd += dsm[i];
            gb3 += sd;
        }
        if (!wait(2)) { ok = false; break; }
        tc_fence_after();
        // ---- 5. dh1^T over dH2 (dead after step 4)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            float d[32];
            tmem_ld32(tD1 + lb + 32u * c, d);
#pragma unroll
            for (int e = 0; e < 32; e++)
                st_t(sm + kTrD, (uint32_t)(32 * c + e), p, ((m1[c] >> e) & 1u) ? bf16_bits(d[e]) : (uint16_t)0);
        }
        tc_handoff();
        // ---- 6. dW1^T += dH1^T . X^T
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < 8; s++)
                mma_bf16(tW1, smem_desc(sD + 2u * kTLbo * s, kTLbo, kTSbo), smem_desc(sXT + 2u * kTLbo * s, kTLbo, kTSbo),
                         kIdesc32, (first && s == 0) ? 0u : 1u);
        }
        commit(3);
        gb1 += row_sum_t(sm + kTrD, p);
        if (!wait(3)) { ok = false; break; }
        tc_fence_after();
        first = false;
        phase ^= 1u;
    }
    if (ok && !first) {
        // this CTA's weight-gradient accumulators: row tid of dW2 (input unit
        // tid) and of dW1^T (hidden unit tid)
#pragma unroll 1
        for (int c = 0; c < 4; c++) {
            float d[32];
            tmem_ld32(tW2 + lb + 32u * c, d);
#pragma unroll
            for (int e = 0; e < 32; e++)
                if (d[e] != 0.f) atomicAdd(&a.g[kOffW2 + tid * BM_MLP_H + 32 * c + e], d[e]);
        }
        {
            float d[32];
            tmem_ld32(tW1 + lb, d);
#pragma unroll
            for (int f = 0; f < BM_MLP_IN; f++)
                if (d[f] != 0.f) atomicAdd(&a.g[f * BM_MLP_H + tid], d[f]);
        }
        atomicAdd(&a.g[kOffB1 + tid], gb1);
        atomicAdd(&a.g[kOffB2 + tid], gb2);
        atomicAdd(&a.g[kOffW3 + tid], gw3);
        if (tid == 0) atomicAdd(&a.g[kOffB3], gb3);
        for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0 && lsum != 0.f) atomicAdd(a.loss, lsum / (float)a.k);
    }
    if (!ok && tid == 0) atomicExch(a.flag, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        // let the MMAs in flight finish before the columns are freed (the
        // default bound, whatever bound the waits above were given)
        if (!ok) mbar_wait(last_bar, last_par);
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// ------------------------------------------------------------------ top-K
//
// For each row of scores, the K largest (ties: lower partner id first),
// written sorted.  Scores map to order-preserving 32-bit keys; an MSB-first
// radix select (four 8-bit digits) finds the K-th largest key T, then one
// ordered pass gathers every key above T and the first ties equal to T.

__device__ __forceinline__ uint32_t order_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

constexpr int kTopThreads = 256;
constexpr int kMaxTopK = 64;

__global__ void __launch_bounds__(kTopThreads) topk_kernel(const float* __restrict__ scores, int32_t n, int32_t K,
                                                           int32_t* __restrict__ out_v, float* __restrict__ out_s) {
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_prefix, s_need;
    __shared__ uint32_t wcnt[kTopThreads / 32];
    __shared__ uint32_t s_gt, s_eq;
    __shared__ uint32_t sel_key[kMaxTopK];
    __shared__ int32_t sel_v[kMaxTopK];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const float* row = scores + (size_t)blockIdx.x * n;
    const int32_t keff = min(K, n);
    if (tid == 0) { s_prefix = 0; s_need = (uint32_t)keff; s_gt = 0; s_eq = 0; }
    uint32_t mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        hist[tid] = 0;
        __syncthreads();
        const uint32_t prefix = s_prefix;
        for (int32_t i = tid; i < n; i += kTopThreads) {
            const uint32_t k = order_key(row[i]);
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (tid == 0 && keff > 0) {
            uint32_t need = s_need, d = 255;
            while (d > 0 && hist[d] < need) {
                need -= hist[d];
                d--;
            }
            s_need = need;
            s_prefix = prefix | (d << shift);
        }
        mask |= 255u << shift;
        __syncthreads();
    }
    const uint32_t T = s_prefix;
    const uint32_t take_eq = keff > 0 ? s_need : 0u;
    const uint32_t n_gt = (uint32_t)keff - take_eq;
    for (int32_t c0 = 0; c0 < n && keff > 0; c0 += kTopThreads) {
        const int32_t i = c0 + tid;
        uint32_t k = 0;
        bool eq = false;
        if (i < n) {
            k = order_key(row[i]);
            eq = k == T;
            if (k > T) {
                const uint32_t slot = atomicAdd(&s_gt, 1u);
                if (slot < n_gt) { sel_key[slot] = k; sel_v[slot] = i + 1; }
            }
        }
        const uint32_t beq = __ballot_sync(0xffffffffu, eq);
        if (lane == 0) wcnt[wid] = (uint32_t)__popc(beq);
        __syncthreads();
        if (eq) {
            uint32_t before = s_eq + (uint32_t)__popc(beq & ((1u << lane) - 1u));
            for (int w = 0; w < wid; w++) before += wcnt[w];
            if (before < take_eq) { sel_key[n_gt + before] = k; sel_v[n_gt + before] = i + 1; }
        }
        __syncthreads();
        if (tid == 0)
            for (int w = 0; w < kTopThreads / 32; w++) s_eq += wcnt[w];
        __syncthreads();
    }
    // rank sort of the selection: larger key first, then smaller id
    if (tid < keff) {
        const uint32_t k = sel_key[tid];
        const int32_t v = sel_v[tid];
        int rank = 0;
        for (int j = 0; j < keff; j++) {
            const uint32_t k2 = sel_key[j];
            rank += (k2 > k) || (k2 == k && sel_v[j] < v);
        }
        out_v[(size_t)blockIdx.x * K + rank] = v;
        out_s[(size_t)blockIdx.x * K + rank] = row[v - 1];
    }
    for (int j = keff + tid; j < K; j += kTopThreads) {
        out_v[(size_t)blockIdx.x * K + j] = 0;
        out_s[(size_t)blockIdx.x * K + j] = -INFINITY;
    }
}

// S distinct partners other than u for every row: u's other n - 1 ids taken
// along an arithmetic progression modulo n - 1 with a random start and a
// random step coprime to n - 1 (Philox, counter = row id, call), so each
// listed partner is uniform and no two repeat.  One warp per row; S <= n - 1.
__global__ void sample_cands_kernel(const int32_t* __restrict__ rows, int32_t nrows, int32_t S, int32_t n, uint64_t seed,
                                    uint64_t call, int32_t* __restrict__ cands) {
    const int32_t warps = (int32_t)(gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t m = (uint32_t)(n - 1);
    for (int32_t i = (int32_t)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < nrows; i += warps) {
        const int32_t u = rows[i];
        uint32_t start = 0, step = 1;
        if (lane == 0 && m > 1) {
            const uint32_t c[4] = {(uint32_t)i, (uint32_t)u, (uint32_t)call, 0x53414D50u};
            const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
            uint32_t o[4];
            bm_philox4x32_10(c, key, o);
            start = o[0] % m;
            step = 1u + o[1] % (m - 1u);
            auto gcd = [](uint32_t x, uint32_t y) {
                while (y) { const uint32_t t = x % y; x = y; y = t; }
                return x;
            };
            while (gcd(step, m) != 1u) step = step + 1u < m ? step + 1u : 1u;
        }
        start = __shfl_sync(0xffffffffu, start, 0);
        step = __shfl_sync(0xffffffffu, step, 0);
        for (int32_t j = lane; j < S; j += 32) {
            const uint32_t idx = (uint32_t)(((uint64_t)start + (uint64_t)j * step) % m);
            int32_t v = 1 + (int32_t)idx;
            if (v >= u) v++;
            cands[(size_t)i * S + j] = v;
        }
    }
}

// pairs (u, partner) of every row's K proposals; an empty slot gives (u, u).
// topv holds partner ids, or, with cands, positions + 1 in the rows' S-long
// partner lists.  With `uniform` set, partners are uniform random ids other
// than u instead (Philox, counter = row id, slot, call).
__global__ void proposal_pairs_kernel(const int32_t* __restrict__ rows, const int32_t* __restrict__ topv, int32_t nrows,
                                      int32_t K, int32_t n, int32_t uniform, uint64_t seed, uint64_t call,
                                      int32_t* __restrict__ pairs, const int32_t* __restrict__ cands, int32_t S) {
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrows * K; i += gridDim.x * blockDim.x) {
        const int32_t u = rows[i / K];
        int32_t v;
        if (uniform) {
            v = u;
            if (n > 1) {
                const uint32_t c[4] = {(uint32_t)(i % K), (uint32_t)u, (uint32_t)call, 0x554E4946u};
                const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
                uint32_t o[4];
                bm_philox4x32_10(c, key, o);
                v = 1 + (int32_t)(o[0] % (uint32_t)(n - 1));
                if (v >= u) v++;
            }
        } else if (cands) {
            v = topv[i] > 0 ? cands[(size_t)(i / K) * S + (topv[i] - 1)] : u;
        } else {
            v = topv[i] > 0 ? topv[i] : u;
        }
        pairs[2 * i] = u;
        pairs[2 * i + 1] = v;
    }
}

FeatSrc feat_src(bm_ctx* ctx, bm_mlp* M) { return FeatSrc{M->d_tab, ctx->pi, hview(ctx->g[1])}; }

int simt_grid(bm_ctx* ctx, int64_t k, int per_sm) {
    const int64_t blocks = (k + kTile - 1) / kTile;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)ctx->num_sms * per_sm));
}


bm_status set_attrs(bm_mlp* M) {
    bm_ctx* ctx = M->ctx;
    BM_CUDA(ctx, cudaFuncSetAttribute(mlp_score_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(MlpSmem)));
    BM_CUDA(ctx, cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sizeof(GradSmem)));
    const uint32_t tcs = tc_smem_bytes(M->n);
    if (tcs > ctx->smem_optin)
        return bm_fail(ctx, BM_UNSUPPORTED, "tensor-core scoring needs %u bytes of shared memory", tcs);
    BM_CUDA(ctx, cudaFuncSetAttribute(mlp_rows_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tcs));
    if (kTrSmem > ctx->smem_optin)
        return bm_fail(ctx, BM_UNSUPPORTED, "tensor-core training needs %u bytes of shared memory", kTrSmem);
    BM_CUDA(ctx, cudaFuncSetAttribute(mlp_train_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTrSmem));
    return BM_OK;
}

bm_status mlp_check(bm_mlp* M) {
    if (!M || !M->ctx) return BM_INVALID_ARG;
    bm_status s = bm_require_mapped(M->ctx);
    if (s != BM_OK) return s;
    if (M->ctx->n != M->n) return bm_fail(M->ctx, BM_INVALID_ARG, "the graphs changed since the model was created");
    return BM_OK;
}

bm_status check_ids(bm_ctx* ctx, const int32_t* ids, int64_t cnt, const char* what) {
    for (int64_t i = 0; i < cnt; i++)
        if (ids[i] < 1 || ids[i] > ctx->n)
            return bm_fail(ctx, BM_INVALID_ARG, "%s[%lld] = %d outside 1..%d", what, (long long)i, ids[i], ctx->n);
    return BM_OK;
}

bm_status scratch(bm_mlp* M, size_t bytes) {
    if (bytes <= M->scr_bytes) return BM_OK;
    bm_cuda_free(M->d_scr);
    M->d_scr = nullptr;
    M->scr_bytes = 0;
    if (bm_cuda_malloc(&M->d_scr, bytes) != cudaSuccess) {
        cudaGetLastError();
        return bm_fail(M->ctx, BM_OOM, "model scratch of %zu bytes", bytes);
    }
    M->scr_bytes = bytes;
    return BM_OK;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

bm_status launch_table(bm_mlp* M) {
    bm_ctx* ctx = M->ctx;
    vertex_table_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(gview(ctx->g[0]), hview(ctx->g[1]), ctx->pi, ctx->ov,
                                                                    M->d_bdeg, ctx->n, M->d_tab);
    BM_LAUNCH_CHECK(ctx, "vertex_table_kernel");
    return BM_OK;
}

bm_status launch_score_simt(bm_mlp* M, PairSrc P, int64_t k, float* d_out) {
    bm_ctx* ctx = M->ctx;
    if (k <= 0) return BM_OK;
    mlp_score_kernel<<<simt_grid(ctx, k, 2), kMT, sizeof(MlpSmem), ctx->stream>>>(feat_src(ctx, M), P, M->d_w, k,
                                                                                 d_out);
    BM_LAUNCH_CHECK(ctx, "mlp_score_kernel");
    return BM_OK;
}

// Gradient of the loss over k records into M->d_g and M->d_loss: on the
// tensor cores (backend 0, records given as features) or the SIMT kernel.
bm_status launch_grad(bm_mlp* M, PairSrc P, const float* d_y, int64_t k) {
    bm_ctx* ctx = M->ctx;
    BM_CUDA(ctx, cudaMemsetAsync(M->d_g, 0, sizeof(float) * (size_t)kNParams, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(M->d_loss, 0, sizeof(float), ctx->stream));
    if (M->backend == 0 && (P.xin || P.xbf)) {
        if (M->img_dirty) {
            prep_image_kernel<<<64, 256, 0, ctx->stream>>>(M->d_w, M->d_img);
            BM_LAUNCH_CHECK(ctx, "prep_image_kernel");
            M->img_dirty = false;
        }
        TrArgs a{M->d_img, P.xin, P.xbf, d_y, k, M->d_g, M->d_loss, M->d_flag,
                 ctx->wait_limit > 0 ? (long long)ctx->wait_limit : kWaitLimit};
        const int64_t tiles = (k + 127) / 128;
        const int grid = (int)std::min<int64_t>(tiles, ctx->num_sms);
        mlp_train_tc_kernel<<<grid, kTrThreads, kTrSmem, ctx->stream>>>(a);
        BM_LAUNCH_CHECK(ctx, "mlp_train_tc_kernel");
        return BM_OK;
    }
    mlp_grad_kernel<<<simt_grid(ctx, k, 1), kMT, sizeof(GradSmem), ctx->stream>>>(feat_src(ctx, M), P, M->d_w, d_y, k,
                                                                                  M->d_g, M->d_loss);
    BM_LAUNCH_CHECK(ctx, "mlp_grad_kernel");
    return BM_OK;
}

bm_status launch_adamw(bm_mlp* M, float lr, float wd) {
    bm_ctx* ctx = M->ctx;
    M->step++;
    const float c1 = (float)(1.0 - std::pow(0.9, (double)M->step));
    const float c2 = (float)(1.0 - std::pow(0.999, (double)M->step));
    adamw_kernel<<<64, 256, 0, ctx->stream>>>(M->d_w, M->d_m, M->d_v, M->d_g, kNParams, lr, 0.9f, 0.999f, 1e-8f, wd,
                                              c1, c2);
    BM_LAUNCH_CHECK(ctx, "adamw_kernel");
    M->img_dirty = true;
    return BM_OK;
}

// Scores of rows x all partners into M->d_sc (row r at r * n).
// Scores of rows x all partners into M->d_sc (row r at r * n), or, with
// d_cands, of rows x their S listed partners (row r at r * S).
bm_status launch_row_scores(bm_mlp* M, const int32_t* d_rows, int32_t nrows, const int32_t* d_cands = nullptr,
                            int32_t S = 0) {
    bm_ctx* ctx = M->ctx;
    const int32_t span = d_cands ? S : M->n;
    const size_t need = (size_t)nrows * (size_t)span;
    if (need > M->sc_cap) {
        bm_cuda_free(M->d_sc);
        M->d_sc = nullptr;
        M->sc_cap = 0;
        if (bm_cuda_malloc(&M->d_sc, sizeof(float) * need) != cudaSuccess) {
            cudaGetLastError();
            return bm_fail(ctx, BM_OOM, "row score buffer of %zu floats", need);
        }
        M->sc_cap = need;
    }
    if (M->backend == 1) {
        PairSrc P{nullptr, nullptr, nullptr, d_rows, span, d_cands};
        return launch_score_simt(M, P, (int64_t)nrows * span, M->d_sc);
    }
    if (M->img_dirty) {
        prep_image_kernel<<<64, 256, 0, ctx->stream>>>(M->d_w, M->d_img);
        BM_LAUNCH_CHECK(ctx, "prep_image_kernel");
        M->img_dirty = false;
    }
    const DevGraph& B = ctx->g[1];
    TcArgs a{M->d_img, M->d_tab, d_rows, nrows, M->n, B.out_ptr, B.out_ent, B.in_ptr, B.in_ent, ctx->pi, M->d_sc,
             M->d_flag, ctx->wait_limit > 0 ? (long long)ctx->wait_limit : kWaitLimit, d_cands, span};
    const int grid = std::min(nrows, ctx->num_sms);
    mlp_rows_tc_kernel<<<grid, kTcThreads, tc_smem_bytes(M->n), ctx->stream>>>(a);
    BM_LAUNCH_CHECK(ctx, "mlp_rows_tc_kernel");
    return BM_OK;
}

bm_status launch_topk(bm_mlp* M, int32_t nrows, int32_t K, int32_t* d_v, float* d_s, int32_t span = 0) {
    bm_ctx* ctx = M->ctx;
    topk_kernel<<<nrows, kTopThreads, 0, ctx->stream>>>(M->d_sc, span > 0 ? span : M->n, K, d_v, d_s);
    BM_LAUNCH_CHECK(ctx, "topk_kernel");
    return BM_OK;
}

bm_status check_flag(bm_mlp* M) {
    bm_ctx* ctx = M->ctx;
    int32_t f = 0;
    BM_CUDA(ctx, cudaMemcpyAsync(&f, M->d_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (f) {
        BM_CUDA(ctx, cudaMemsetAsync(M->d_flag, 0, sizeof(int32_t), ctx->stream));
        return bm_fail(ctx, BM_TIMEOUT, "tensor-core kernel: an MMA completion wait ran out");
    }
    return BM_OK;
}

bm_status ensure_records(bm_mlp* M, int64_t cap) {
    if (M->rcap >= cap) return BM_OK;
    bm_ctx* ctx = M->ctx;
    uint16_t* nx = nullptr;
    float* ny = nullptr;
    if (bm_cuda_malloc(&nx, sizeof(uint16_t) * BM_MLP_IN * (size_t)cap) != cudaSuccess ||
        bm_cuda_malloc(&ny, sizeof(float) * (size_t)cap) != cudaSuccess) {
        cudaGetLastError();
        bm_cuda_free(nx);
        bm_cuda_free(ny);
        return bm_fail(ctx, BM_OOM, "record store of %lld records", (long long)cap);
    }
    // keep the existing records in ring order, oldest first
    if (M->rsize > 0) {
        const int64_t first = (M->rhead - M->rsize + M->rcap) % M->rcap;
        const int64_t a = std::min(M->rsize, M->rcap - first);
        BM_CUDA(ctx, cudaMemcpyAsync(nx, M->d_rx + first * BM_MLP_IN, sizeof(uint16_t) * BM_MLP_IN * a,
                                     cudaMemcpyDeviceToDevice, ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(ny, M->d_ry + first, sizeof(float) * a, cudaMemcpyDeviceToDevice, ctx->stream));
        if (a < M->rsize) {
            BM_CUDA(ctx, cudaMemcpyAsync(nx + a * BM_MLP_IN, M->d_rx, sizeof(uint16_t) * BM_MLP_IN * (M->rsize - a),
                                         cudaMemcpyDeviceToDevice, ctx->stream));
            BM_CUDA(ctx, cudaMemcpyAsync(ny + a, M->d_ry, sizeof(float) * (M->rsize - a), cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        }
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    bm_cuda_free(M->d_rx);
    bm_cuda_free(M->d_ry);
    M->d_rx = nx;
    M->d_ry = ny;
    M->rhead = M->rsize;
    M->rcap = cap;
    return BM_OK;
}

// Append k device records (pairs, exact deltas) with features of the current
// mapping.
bm_status append_records(bm_mlp* M, const int32_t* d_pairs, const long long* d_deltas, int64_t k) {
    bm_ctx* ctx = M->ctx;
    if (k <= 0) return BM_OK;
    if (M->rcap == 0) {
        bm_status s = ensure_records(M, std::max<int64_t>(k, 1 << 20));
        if (s != BM_OK) return s;
    }
    // a batch larger than the store keeps only its last rcap records
    if (k > M->rcap) {
        d_pairs += 2 * (k - M->rcap);
        d_deltas += (k - M->rcap);
        k = M->rcap;
    }
    const int blocks = (int)std::min<int64_t>((k + 255) / 256, (int64_t)ctx->num_sms * 8);
    append_records_kernel<<<blocks, 256, 0, ctx->stream>>>(feat_src(ctx, M), d_pairs, d_deltas, k, M->rhead, M->rcap,
                                                           M->d_rx, M->d_ry);
    BM_LAUNCH_CHECK(ctx, "append_records_kernel");
    M->rhead = (M->rhead + k) % M->rcap;
    M->rsize = std::min(M->rcap, M->rsize + k);
    return BM_OK;
}

bm_status fit_steps(bm_mlp* M, int32_t steps, int32_t batch, float lr, float wd, uint64_t seed, float* loss) {
    bm_ctx* ctx = M->ctx;
    if (M->rsize == 0) return bm_fail(ctx, BM_INVALID_ARG, "no training records collected");
    if (batch > M->bcap) {
        bm_cuda_free(M->d_bx);
        bm_cuda_free(M->d_by);
        M->d_bx = nullptr;
        M->d_by = nullptr;
        M->bcap = 0;
        if (bm_cuda_malloc(&M->d_bx, sizeof(uint16_t) * BM_MLP_IN * (size_t)batch) != cudaSuccess ||
            bm_cuda_malloc(&M->d_by, sizeof(float) * (size_t)batch) != cudaSuccess) {
            cudaGetLastError();
            return bm_fail(ctx, BM_OOM, "minibatch of %d records", batch);
        }
        M->bcap = batch;
    }
    for (int32_t s = 0; s < steps; s++) {
        gather_batch_kernel<<<(batch + 255) / 256, 256, 0, ctx->stream>>>(M->d_rx, M->d_ry, M->rsize, batch, seed,
                                                                          (uint64_t)M->step, M->d_bx, M->d_by);
        BM_LAUNCH_CHECK(ctx, "gather_batch_kernel");
        PairSrc P{nullptr, M->d_bx, nullptr, nullptr, M->n};
        bm_status st = launch_grad(M, P, M->d_by, batch);
        if (st != BM_OK) return st;
        if ((st = launch_adamw(M, lr, wd)) != BM_OK) return st;
    }
    if (loss) {
        float l = 0.f;
        BM_CUDA(ctx, cudaMemcpyAsync(&l, M->d_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *loss = l;
    }
    return check_flag(M);
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" void bm_mlp_destroy(bm_mlp* M) {
    if (!M) return;
    // the context may already be gone: synchronise the device, not its stream
    cudaSetDevice(M->device);
    cudaDeviceSynchronize();
    bm_cuda_free(M->d_w); bm_cuda_free(M->d_m); bm_cuda_free(M->d_v); bm_cuda_free(M->d_g); bm_cuda_free(M->d_loss);
    bm_cuda_free(M->d_tab); bm_cuda_free(M->d_bdeg); bm_cuda_free(M->d_img); bm_cuda_free(M->d_sc); bm_cuda_free(M->d_flag);
    bm_cuda_free(M->d_rx); bm_cuda_free(M->d_ry); bm_cuda_free(M->d_bx); bm_cuda_free(M->d_by); bm_cuda_free(M->d_scr);
    delete M;
}

extern "C" bm_status bm_mlp_create(bm_ctx* ctx, uint64_t seed, bm_mlp** out) {
    if (!ctx || !out) return BM_INVALID_ARG;
    *out = nullptr;
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    bm_mlp* M = new (std::nothrow) bm_mlp();
    if (!M) return BM_OOM;
    M->ctx = ctx;
    M->device = ctx->device;
    M->n = ctx->n;
    // Glorot-uniform weights from Philox (counter = parameter index), zero biases
    std::vector<float> w((size_t)kNParams, 0.f);
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    auto init = [&](int off, int fan_in, int fan_out, int count) {
        const double lim = std::sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < count; i++) {
            const uint32_t c[4] = {(uint32_t)(off + i), 0u, 0x6D6C7000u, 0u};
            uint32_t o[4];
            bm_philox4x32_10(c, key, o);
            w[(size_t)off + i] = (float)((bm_u01(o[0], o[1]) * 2.0 - 1.0) * lim);
        }
    };
    init(0, BM_MLP_IN, BM_MLP_H, kNW1);
    init(kOffW2, BM_MLP_H, BM_MLP_H, BM_MLP_H * BM_MLP_H);
    init(kOffW3, BM_MLP_H, 1, BM_MLP_H);
    const size_t pb = sizeof(float) * (size_t)kNParams;
    const size_t tb = sizeof(float) * ((size_t)ctx->n + 1) * BM_FT;
    if (bm_cuda_malloc(&M->d_w, pb) || bm_cuda_malloc(&M->d_m, pb) || bm_cuda_malloc(&M->d_v, pb) || bm_cuda_malloc(&M->d_g, pb) ||
        bm_cuda_malloc(&M->d_loss, 256) || bm_cuda_malloc(&M->d_tab, tb) ||
        bm_cuda_malloc(&M->d_bdeg, sizeof(float2) * ((size_t)ctx->n + 1)) || bm_cuda_malloc(&M->d_img, kImgBytes) ||
        bm_cuda_malloc(&M->d_flag, 256)) {
        cudaGetLastError();
        bm_mlp_destroy(M);
        return bm_fail(ctx, BM_OOM, "bm_mlp_create: device allocation failed");
    }
    if (cudaMemcpy(M->d_w, w.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(M->d_m, 0, pb) != cudaSuccess || cudaMemset(M->d_v, 0, pb) != cudaSuccess ||
        cudaMemset(M->d_g, 0, pb) != cudaSuccess || cudaMemset(M->d_tab, 0, tb) != cudaSuccess ||
        cudaMemset(M->d_flag, 0, 256) != cudaSuccess || cudaMemset(M->d_loss, 0, 256) != cudaSuccess) {
        bm_mlp_destroy(M);
        return bm_fail(ctx, BM_CUDA_ERROR, "bm_mlp_create: initialisation failed");
    }
    if ((s = set_attrs(M)) != BM_OK) {
        bm_mlp_destroy(M);
        return s;
    }
    const DevGraph& B = ctx->g[1];
    bdeg_kernel<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(B.out_ptr, B.out_ent0, B.in_ptr, B.in_ent0, ctx->n,
                                                           M->d_bdeg);
    ctx->launches++;
    if (cudaGetLastError() != cudaSuccess) {
        bm_mlp_destroy(M);
        return bm_fail(ctx, BM_CUDA_ERROR, "bdeg_kernel launch failed");
    }
    if ((s = launch_table(M)) != BM_OK || cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        bm_mlp_destroy(M);
        return s != BM_OK ? s : bm_fail(ctx, BM_CUDA_ERROR, "bm_mlp_create: feature table failed");
    }
    *out = M;
    return BM_OK;
}

extern "C" int32_t bm_mlp_num_params(void) { return kNParams; }

extern "C" bm_status bm_mlp_set_backend(bm_mlp* M, int32_t backend) {
    if (!M || backend < 0 || backend > 1) return BM_INVALID_ARG;
    M->backend = backend;
    return BM_OK;
}

extern "C" bm_status bm_mlp_refresh_features(bm_mlp* M) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    if ((s = launch_table(M)) != BM_OK) return s;
    BM_CUDA(M->ctx, cudaStreamSynchronize(M->ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_get_features(bm_mlp* M, float* table) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    if (!table) return bm_fail(M->ctx, BM_INVALID_ARG, "null table");
    BM_CUDA(M->ctx, cudaMemcpyAsync(table, M->d_tab, sizeof(float) * ((size_t)M->n + 1) * BM_FT,
                                    cudaMemcpyDeviceToHost, M->ctx->stream));
    BM_CUDA(M->ctx, cudaStreamSynchronize(M->ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_get_params(bm_mlp* M, float* w) {
    if (!M || !w) return BM_INVALID_ARG;
    BM_CUDA(M->ctx, cudaMemcpyAsync(w, M->d_w, sizeof(float) * (size_t)kNParams, cudaMemcpyDeviceToHost,
                                    M->ctx->stream));
    BM_CUDA(M->ctx, cudaStreamSynchronize(M->ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_set_params(bm_mlp* M, const float* w) {
    if (!M || !w) return BM_INVALID_ARG;
    BM_CUDA(M->ctx, cudaMemcpyAsync(M->d_w, w, sizeof(float) * (size_t)kNParams, cudaMemcpyHostToDevice,
                                    M->ctx->stream));
    BM_CUDA(M->ctx, cudaStreamSynchronize(M->ctx->stream));
    M->img_dirty = true;
    return BM_OK;
}

extern "C" bm_status bm_mlp_pair_features(bm_mlp* M, const int32_t* pairs, int64_t k, float* feats) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (k < 0 || (k > 0 && (!pairs || !feats))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (k == 0) return BM_OK;
    if ((s = check_ids(ctx, pairs, 2 * k, "pairs")) != BM_OK) return s;
    const size_t pbytes = al256(sizeof(int32_t) * 2 * (size_t)k);
    if ((s = scratch(M, pbytes + sizeof(float) * (size_t)k * BM_MLP_IN)) != BM_OK) return s;
    int32_t* d_p = (int32_t*)M->d_scr;
    float* d_f = (float*)((char*)M->d_scr + pbytes);
    BM_CUDA(ctx, cudaMemcpyAsync(d_p, pairs, sizeof(int32_t) * 2 * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    const int blocks = (int)std::min<int64_t>((k + 255) / 256, (int64_t)ctx->num_sms * 8);
    pair_features_kernel<<<blocks, 256, 0, ctx->stream>>>(feat_src(ctx, M), d_p, k, d_f);
    BM_LAUNCH_CHECK(ctx, "pair_features_kernel");
    BM_CUDA(ctx, cudaMemcpyAsync(feats, d_f, sizeof(float) * (size_t)k * BM_MLP_IN, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_score_pairs(bm_mlp* M, const int32_t* pairs, int64_t k, float* scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (k < 0 || (k > 0 && (!pairs || !scores))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (k == 0) return BM_OK;
    if ((s = check_ids(ctx, pairs, 2 * k, "pairs")) != BM_OK) return s;
    const size_t pbytes = al256(sizeof(int32_t) * 2 * (size_t)k);
    if ((s = scratch(M, pbytes + sizeof(float) * (size_t)k)) != BM_OK) return s;
    int32_t* d_p = (int32_t*)M->d_scr;
    float* d_o = (float*)((char*)M->d_scr + pbytes);
    BM_CUDA(ctx, cudaMemcpyAsync(d_p, pairs, sizeof(int32_t) * 2 * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    PairSrc P{nullptr, nullptr, d_p, nullptr, M->n};
    if ((s = launch_score_simt(M, P, k, d_o)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(scores, d_o, sizeof(float) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_score_features(bm_mlp* M, const float* x, int64_t k, float* scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (k < 0 || (k > 0 && (!x || !scores))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (k == 0) return BM_OK;
    const size_t xb = al256(sizeof(float) * (size_t)k * BM_MLP_IN);
    if ((s = scratch(M, xb + sizeof(float) * (size_t)k)) != BM_OK) return s;
    float* d_x = (float*)M->d_scr;
    float* d_o = (float*)((char*)M->d_scr + xb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_x, x, sizeof(float) * (size_t)k * BM_MLP_IN, cudaMemcpyHostToDevice, ctx->stream));
    PairSrc P{d_x, nullptr, nullptr, nullptr, M->n};
    if ((s = launch_score_simt(M, P, k, d_o)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(scores, d_o, sizeof(float) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_score_rows(bm_mlp* M, const int32_t* rows, int32_t nrows, float* scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (nrows < 0 || (nrows > 0 && (!rows || !scores))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (nrows == 0) return BM_OK;
    if ((s = check_ids(ctx, rows, nrows, "rows")) != BM_OK) return s;
    if ((s = scratch(M, sizeof(int32_t) * (size_t)nrows)) != BM_OK) return s;
    int32_t* d_r = (int32_t*)M->d_scr;
    BM_CUDA(ctx, cudaMemcpyAsync(d_r, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = launch_row_scores(M, d_r, nrows)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(scores, M->d_sc, sizeof(float) * (size_t)nrows * M->n, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    return check_flag(M);
}

extern "C" bm_status bm_mlp_score_rows_dev(bm_mlp* M, const int32_t* d_rows, int32_t nrows, float* d_scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (nrows < 0 || (nrows > 0 && (!d_rows || !d_scores))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (nrows == 0) return BM_OK;
    if ((s = launch_row_scores(M, d_rows, nrows)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(d_scores, M->d_sc, sizeof(float) * (size_t)nrows * M->n, cudaMemcpyDeviceToDevice,
                                 ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_mlp_score_candidates(bm_mlp* M, const int32_t* rows, int32_t nrows, const int32_t* cands,
                                             int32_t S, float* scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (nrows < 0 || S < 1 || (nrows > 0 && (!rows || !cands || !scores)))
        return bm_fail(ctx, BM_INVALID_ARG, "bad buffers or S < 1");
    if (nrows == 0) return BM_OK;
    if ((s = check_ids(ctx, rows, nrows, "rows")) != BM_OK) return s;
    for (int64_t i = 0; i < (int64_t)nrows * S; i++) {
        const int32_t v = cands[i];
        if (v < 1 || v > ctx->n || v == rows[i / S])
            return bm_fail(ctx, BM_INVALID_ARG, "candidate %lld = %d is outside 1..%d or its row's vertex", (long long)i,
                           v, ctx->n);
    }
    const size_t rb = al256(sizeof(int32_t) * (size_t)nrows);
    if ((s = scratch(M, rb + sizeof(int32_t) * (size_t)nrows * (size_t)S)) != BM_OK) return s;
    int32_t* d_r = (int32_t*)M->d_scr;
    int32_t* d_c = (int32_t*)((char*)M->d_scr + rb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_r, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_c, cands, sizeof(int32_t) * (size_t)nrows * S, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = launch_row_scores(M, d_r, nrows, d_c, S)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(scores, M->d_sc, sizeof(float) * (size_t)nrows * S, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    return check_flag(M);
}

extern "C" bm_status bm_mlp_status(bm_mlp* M) {
    if (!M || !M->ctx) return BM_INVALID_ARG;
    return check_flag(M);
}

extern "C" bm_status bm_mlp_rows_topk(bm_mlp* M, const int32_t* rows, int32_t nrows, int32_t K, int32_t* partners,
                                      float* scores) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (K < 1 || K > kMaxTopK) return bm_fail(ctx, BM_INVALID_ARG, "K = %d outside 1..%d", K, kMaxTopK);
    if (nrows < 0 || (nrows > 0 && (!rows || !partners))) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    if (nrows == 0) return BM_OK;
    if ((s = check_ids(ctx, rows, nrows, "rows")) != BM_OK) return s;
    const size_t rb = al256(sizeof(int32_t) * (size_t)nrows);
    const size_t vb = al256(sizeof(int32_t) * (size_t)nrows * K);
    if ((s = scratch(M, rb + 2 * vb)) != BM_OK) return s;
    int32_t* d_r = (int32_t*)M->d_scr;
    int32_t* d_v = (int32_t*)((char*)M->d_scr + rb);
    float* d_s = (float*)((char*)M->d_scr + rb + vb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_r, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = launch_row_scores(M, d_r, nrows)) != BM_OK) return s;
    if ((s = launch_topk(M, nrows, K, d_v, d_s)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(partners, d_v, sizeof(int32_t) * (size_t)nrows * K, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    if (scores)
        BM_CUDA(ctx, cudaMemcpyAsync(scores, d_s, sizeof(float) * (size_t)nrows * K, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    return check_flag(M);
}

extern "C" bm_status bm_mlp_gradients(bm_mlp* M, const float* x, const float* y, int64_t k, float* grads,
                                      float* loss) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (k <= 0 || !x || !y || !grads) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    const size_t xb = al256(sizeof(float) * (size_t)k * BM_MLP_IN);
    if ((s = scratch(M, xb + sizeof(float) * (size_t)k)) != BM_OK) return s;
    float* d_x = (float*)M->d_scr;
    float* d_y = (float*)((char*)M->d_scr + xb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_x, x, sizeof(float) * (size_t)k * BM_MLP_IN, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_y, y, sizeof(float) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    PairSrc P{d_x, nullptr, nullptr, nullptr, M->n};
    if ((s = launch_grad(M, P, d_y, k)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(grads, M->d_g, sizeof(float) * (size_t)kNParams, cudaMemcpyDeviceToHost, ctx->stream));
    float l = 0.f;
    BM_CUDA(ctx, cudaMemcpyAsync(&l, M->d_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = l;
    return check_flag(M);
}

extern "C" bm_status bm_mlp_adamw_step(bm_mlp* M, const float* x, const float* y, int64_t k, float lr,
                                       float weight_decay, float* loss) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (k <= 0 || !x || !y) return bm_fail(ctx, BM_INVALID_ARG, "bad buffers");
    const size_t xb = al256(sizeof(float) * (size_t)k * BM_MLP_IN);
    if ((s = scratch(M, xb + sizeof(float) * (size_t)k)) != BM_OK) return s;
    float* d_x = (float*)M->d_scr;
    float* d_y = (float*)((char*)M->d_scr + xb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_x, x, sizeof(float) * (size_t)k * BM_MLP_IN, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(d_y, y, sizeof(float) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
    PairSrc P{d_x, nullptr, nullptr, nullptr, M->n};
    if ((s = launch_grad(M, P, d_y, k)) != BM_OK) return s;
    if ((s = launch_adamw(M, lr, weight_decay)) != BM_OK) return s;
    float l = 0.f;
    BM_CUDA(ctx, cudaMemcpyAsync(&l, M->d_loss, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = l;
    return check_flag(M);
}

extern "C" bm_status bm_mlp_collect_rows(bm_mlp* M, const int32_t* rows, int32_t nrows, int32_t per_row, uint64_t seed,
                                         int64_t* nrecords) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    bm_ctx* ctx = M->ctx;
    if (nrows < 0 || (nrows > 0 && !rows) || per_row < 2) return bm_fail(ctx, BM_INVALID_ARG, "bad arguments");
    if ((s = check_ids(ctx, rows, nrows, "rows")) != BM_OK) return s;
    if ((s = launch_table(M)) != BM_OK) return s;
    // rows in chunks so that the whole-row deltas stay below ~256 MB
    const int32_t chunk = (int32_t)std::max<int64_t>(1, std::min<int64_t>(nrows, (256ll << 20) / (8ll * (M->n + 1))));
    const size_t rb = al256(sizeof(int32_t) * (size_t)chunk);
    const size_t fb = al256(sizeof(long long) * (size_t)chunk * ((size_t)M->n + 1));
    const size_t pb = al256(sizeof(int32_t) * 2 * (size_t)chunk * per_row);
    const size_t db = al256(sizeof(long long) * (size_t)chunk * per_row);
    if ((s = scratch(M, rb + fb + pb + db)) != BM_OK) return s;
    char* base = (char*)M->d_scr;
    int32_t* d_r = (int32_t*)base;
    long long* d_full = (long long*)(base + rb);
    int32_t* d_p = (int32_t*)(base + rb + fb);
    long long* d_d = (long long*)(base + rb + fb + pb);
    for (int32_t r0 = 0; r0 < nrows; r0 += chunk) {
        const int32_t c = std::min(chunk, nrows - r0);
        BM_CUDA(ctx, cudaMemcpyAsync(d_r, rows + r0, sizeof(int32_t) * (size_t)c, cudaMemcpyHostToDevice, ctx->stream));
        if ((s = bm_launch_rows(ctx, d_r, nullptr, c, (int64_t*)d_full, nullptr)) != BM_OK) return s;
        harvest_kernel<<<c, kHarvThreads, 0, ctx->stream>>>(d_full, d_r, M->n, per_row, seed + (uint64_t)r0, d_p, d_d);
        BM_LAUNCH_CHECK(ctx, "harvest_kernel");
        if ((s = append_records(M, d_p, d_d, (int64_t)c * per_row)) != BM_OK) return s;
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    if (nrecords) *nrecords = M->rsize;
    return BM_OK;
}

extern "C" bm_status bm_mlp_reserve_records(bm_mlp* M, int64_t capacity) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    if (capacity < 1) return bm_fail(M->ctx, BM_INVALID_ARG, "capacity must be positive");
    return ensure_records(M, capacity);
}

extern "C" bm_status bm_mlp_clear_records(bm_mlp* M) {
    if (!M) return BM_INVALID_ARG;
    M->rsize = 0;
    M->rhead = 0;
    return BM_OK;
}

extern "C" bm_status bm_mlp_fit(bm_mlp* M, int32_t steps, int32_t batch, float lr, float weight_decay, uint64_t seed,
                                float* loss) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    if (steps < 0 || batch < 1) return bm_fail(M->ctx, BM_INVALID_ARG, "bad steps or batch");
    return fit_steps(M, steps, batch, lr, weight_decay, seed, loss);
}

// ------------------------------------------------------------ learned search

extern "C" bm_status bm_search_learned(bm_ctx* ctx, bm_mlp* M, const int32_t* row_order, int32_t nrows,
                                       const bm_learned_params* p, bm_progress* prog, bm_learned_stats* st) {
    bm_status s = mlp_check(M);
    if (s != BM_OK) return s;
    if (M->ctx != ctx) return bm_fail(ctx, BM_INVALID_ARG, "model belongs to another context");
    if (!p || !prog || !st) return bm_fail(ctx, BM_INVALID_ARG, "params, progress and stats are required");
    const int32_t n = ctx->n;
    const int32_t K = p->topk > 0 ? p->topk : 64;
    if (K > kMaxTopK) return bm_fail(ctx, BM_INVALID_ARG, "topk %d above %d", K, kMaxTopK);
    std::vector<int32_t> order;
    if (row_order) {
        if (nrows <= 0) return bm_fail(ctx, BM_INVALID_ARG, "empty row order");
        if ((s = check_ids(ctx, row_order, nrows, "row_order")) != BM_OK) return s;
        order.assign(row_order, row_order + nrows);
    } else {
        order.resize((size_t)n);
        for (int32_t i = 0; i < n; i++) order[(size_t)i] = i + 1;
    }
    const int32_t nr = (int32_t)order.size();
    const int32_t R = std::min(nr, p->rows_per_batch > 0 ? p->rows_per_batch : 2 * ctx->num_sms);
    if (p->sample < 0) return bm_fail(ctx, BM_INVALID_ARG, "sample must be 0 (all partners) or a partner count");
    // sampled scoring: the model scores S random partners per row (distinct,
    // never u) and proposes the top K of them; S >= n - 1 scores every partner
    const int32_t S = (!p->uniform && p->sample > 0 && p->sample < n - 1) ? std::max(p->sample, K) : 0;
    const int64_t RK = (int64_t)R * K;
    const size_t rb = al256(sizeof(int32_t) * (size_t)R);
    const size_t vb = al256(sizeof(int32_t) * (size_t)RK);
    const size_t pb = al256(sizeof(int32_t) * 2 * (size_t)RK);
    const size_t db = al256(sizeof(long long) * (size_t)RK);
    const size_t cb = al256(sizeof(int32_t) * (size_t)R * (size_t)S);
    if ((s = scratch(M, rb + 2 * vb + pb + db + pb + cb)) != BM_OK) return s;
    char* base = (char*)M->d_scr;
    int32_t* d_r = (int32_t*)base;
    int32_t* d_tv = (int32_t*)(base + rb);
    float* d_ts = (float*)(base + rb + vb);
    int32_t* d_p = (int32_t*)(base + rb + 2 * vb);
    long long* d_d = (long long*)(base + rb + 2 * vb + pb);
    int32_t* d_ap = (int32_t*)(base + rb + 2 * vb + pb + db);
    int32_t* d_c = S ? (int32_t*)(base + rb + 2 * vb + pb + db + pb) : nullptr;
    std::vector<int32_t> h_p((size_t)2 * RK), h_ap((size_t)2 * R);
    std::vector<long long> h_d((size_t)RK);
    std::vector<int32_t> cand;
    std::vector<int64_t> cand_d;
    std::vector<int32_t> cand_v;
    BmMarks mk;
    const auto t0 = clk::now();
    const int32_t refresh = p->refresh_batches > 0 ? p->refresh_batches : 1;
    int64_t batch = 0, pass_accepts = 0;
    int32_t pos = 0;
    prog->converged = 0;
    bm_status ret = BM_OK;
    const int64_t accepts0 = prog->accepts;
    for (;;) {
        if (p->max_accepts >= 0 && prog->accepts - accepts0 >= p->max_accepts) break;
        if (p->target_score > 0 && ctx->score >= p->target_score) break;
        if (p->time_budget_s > 0 && secs_since(t0) >= p->time_budget_s) { ret = BM_TIMEOUT; break; }
        const int32_t k = std::min(R, nr - pos);
        auto ta = clk::now();
        if (batch % refresh == 0 && !p->uniform) {
            if ((s = launch_table(M)) != BM_OK) return s;
        }
        BM_CUDA(ctx, cudaMemcpyAsync(d_r, order.data() + pos, sizeof(int32_t) * (size_t)k, cudaMemcpyHostToDevice,
                                     ctx->stream));
        if (!p->uniform && S) {
            sample_cands_kernel<<<(int)std::min<int64_t>(((int64_t)k * 32 + 255) / 256, 4096), 256, 0, ctx->stream>>>(
                d_r, k, S, n, p->seed, (uint64_t)batch, d_c);
            BM_LAUNCH_CHECK(ctx, "sample_cands_kernel");
            if ((s = launch_row_scores(M, d_r, k, d_c, S)) != BM_OK) return s;
            if ((s = launch_topk(M, k, K, d_tv, d_ts, S)) != BM_OK) return s;
        } else if (!p->uniform) {
            if ((s = launch_row_scores(M, d_r, k)) != BM_OK) return s;
            if ((s = launch_topk(M, k, K, d_tv, d_ts)) != BM_OK) return s;
        }
        proposal_pairs_kernel<<<(int)std::min<int64_t>((k * (int64_t)K + 255) / 256, 4096), 256, 0, ctx->stream>>>(
            d_r, d_tv, k, K, n, p->uniform, p->seed, (uint64_t)batch, d_p, d_c, S);
        BM_LAUNCH_CHECK(ctx, "proposal_pairs_kernel");
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        st->t_propose += secs_since(ta);
        if (!p->uniform && (s = check_flag(M)) != BM_OK) return s;
        ta = clk::now();
        const int64_t kk = (int64_t)k * K;
        if ((s = bm_launch_pairs(ctx, d_p, kk, (int64_t*)d_d)) != BM_OK) return s;
        BM_CUDA(ctx, cudaMemcpyAsync(h_p.data(), d_p, sizeof(int32_t) * 2 * (size_t)kk, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        BM_CUDA(ctx, cudaMemcpyAsync(h_d.data(), d_d, sizeof(long long) * (size_t)kk, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        // records of this batch, under the mapping the deltas were computed for
        if (p->train_every > 0 && !p->uniform) {
            if ((s = append_records(M, d_p, d_d, kk)) != BM_OK) return s;
        }
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        st->t_exact += secs_since(ta);
        st->proposals += kk;
        prog->evaluated += kk;
        // per row: the best improving proposal
        cand.clear();
        cand_d.clear();
        cand_v.clear();
        for (int32_t i = 0; i < k; i++) {
            int64_t best = 0;
            int32_t bv = 0;
            for (int32_t j = 0; j < K; j++) {
                const int64_t d = h_d[(size_t)i * K + j];
                const int32_t v = h_p[2 * ((size_t)i * K + j) + 1];
                if (d > 0 && v != order[(size_t)(pos + i)]) st->hits++;
                if (d > best || (d == best && d > 0 && v < bv)) { best = d; bv = v; }
            }
            if (best > 0) {
                cand.push_back(order[(size_t)(pos + i)]);
                cand_v.push_back(bv);
                cand_d.push_back(best);
            }
        }
        std::vector<int32_t> idx(cand.size());
        for (size_t i = 0; i < idx.size(); i++) idx[i] = (int32_t)i;
        std::sort(idx.begin(), idx.end(), [&](int32_t x, int32_t y) {
            if (cand_d[(size_t)x] != cand_d[(size_t)y]) return cand_d[(size_t)x] > cand_d[(size_t)y];
            return x < y;
        });
        mk.reset(n);
        int32_t na = 0;
        int64_t gain = 0;
        for (int32_t i : idx) {
            const int32_t u = cand[(size_t)i], v = cand_v[(size_t)i];
            if (mk.marked(u) || mk.marked(v)) continue;
            mk.mark_closed(ctx, u);
            mk.mark_closed(ctx, v);
            h_ap[2 * (size_t)na] = u;
            h_ap[2 * (size_t)na + 1] = v;
            gain += cand_d[(size_t)i];
            na++;
        }
        if (na > 0) {
            BM_CUDA(ctx, cudaMemcpyAsync(d_ap, h_ap.data(), sizeof(int32_t) * 2 * (size_t)na, cudaMemcpyHostToDevice,
                                         ctx->stream));
            if ((s = bm_launch_apply(ctx, d_ap, na)) != BM_OK) return s;
            ctx->score += gain;
            prog->accepts += na;
            pass_accepts += na;
        }
        if (p->train_every > 0 && !p->uniform && (batch + 1) % p->train_every == 0) {
            ta = clk::now();
            if ((s = fit_steps(M, 1, p->train_batch > 0 ? p->train_batch : 4096, p->lr, p->weight_decay,
                               p->seed ^ 0x5452414E49ull, nullptr)) != BM_OK)
                return s;
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            st->train_steps++;
            st->t_train += secs_since(ta);
        }
        batch++;
        prog->launches++;
        prog->rows_done += k;
        pos += k;
        if (pos >= nr) {
            pos = 0;
            prog->sweeps++;
            if (pass_accepts <= (int64_t)std::max(0, p->fallback_accepts)) {
                // the proposals found (almost) nothing in a whole pass: an exact pass judges
                if (p->exact_fallback) {
                    ta = clk::now();
                    bm_progress ex;
                    memset(&ex, 0, sizeof(ex));
                    const double left = p->time_budget_s > 0 ? p->time_budget_s - secs_since(t0) : 0.0;
                    if (p->time_budget_s > 0 && left <= 0) { ret = BM_TIMEOUT; break; }
                    s = bm_search_batched(ctx, order.data(), nr, R, -1, 1, left, p->target_score, &ex);
                    st->t_exact += secs_since(ta);
                    st->exact_passes++;
                    prog->accepts += ex.accepts;
                    prog->evaluated += ex.evaluated;
                    if (s != BM_OK && s != BM_TIMEOUT) return s;
                    if (s == BM_TIMEOUT) { ret = BM_TIMEOUT; break; }
                    if (ex.accepts == 0 || ex.converged) { prog->converged = 1; break; }
                } else if (pass_accepts == 0) {
                    prog->converged = 1;
                    break;
                }
            }
            pass_accepts = 0;
            if (p->max_sweeps >= 0 && prog->sweeps >= p->max_sweeps) break;
        }
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->next_row_pos = pos;
    prog->seconds += secs_since(t0);
    s = bm_check_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    return ret;
}
