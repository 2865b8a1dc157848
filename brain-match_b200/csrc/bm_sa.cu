// bm_sa.cu — batched simulated-annealing chains over many graph pairs.
//
// Follows the annealing of src/best-swap/score-lookup.c:346-408: a proposal is
// a random pair (nodeM1, nodeM2), accepted if delta >= 0 or u < exp(delta/T),
// with the geometric schedule T_i = Tmax * exp(ln(Tmin/Tmax) * i / iters).
// Differences, deliberate: the deltas are exact int64 (pair form of
// bm_pairs.cu) instead of an int16 lookup table; the RNG is Philox4x32-10
// keyed per chain with the step as counter (instead of xoshiro256** seeded
// from time), and exp is the project's own bm_exp, so a chain replays bit for
// bit on the CPU; every chain ends on its final mapping and score, like the
// reference's return value (:407).
//
// One CTA runs one chain.  Each iteration evaluates the K proposals of steps
// s..s+K-1 under the current mapping with the whole CTA (their list entries
// are spread over all warps, so a proposal touching a hub does not stall the
// others); the first accepted one in step order is applied and the rest are
// discarded, so the chain is exactly the one-at-a-time chain for every K (the
// step counter moves past the accepted proposal, or by K when none is
// accepted).  K starts at the tuned value and then follows the chain's
// acceptances (up to 64), so long runs of rejections are evaluated 64 at a
// time; the chain's mapping lives in shared memory when it fits.  A launch advances every chain by at most `chunk` proposals;
// the launch is captured once in a CUDA graph and replayed until all chains
// finish.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cooperative_groups.h>

#include "bm_internal.cuh"
#include "bm_rng.hpp"

namespace cg = cooperative_groups;

namespace {

struct PairDev {
    int32_t n;
    int32_t has_self;
    const int32_t* Aout_ptr;
    const int32_t* Ain_ptr;
    const uint32_t* Aout_ent;
    const uint32_t* Ain_ent;
    const int32_t* selfA;
    const int32_t* selfB;
    HashView hb;
    // B's rows (sorted by neighbour id, zero padding at the end), searched
    // for the edges of a whole A list at once
    const int32_t* Bout_ptr;
    const int32_t* Bin_ptr;
    const uint32_t* Bout_ent;
    const uint32_t* Bin_ent;
};

struct ChainDev {
    int32_t pair;
    int32_t status;
    int32_t* pi;    // n+1
    int32_t* ov;    // n+1, per-vertex overlap (scratch)
    uint64_t key;
    uint64_t step;  // next proposal index
    long long score;
    long long accepts;
};

struct SaArgs {
    const PairDev* pairs;
    ChainDev* chains;
    int32_t nchains;
    int32_t K;        // proposals per iteration at the start (1..kSaMaxInitialK); adapts up to kSaMaxK
    int32_t pi_smem;  // 1: the chain's mapping is kept in shared memory
    uint64_t steps;
    uint64_t chunk;
    double t0;
    double log_ratio;
};

constexpr int kSaThreads = 512;     // threads per CTA of the allocation-free entry point (bm_sa_run tunes 256 or 512)
constexpr int kSaMaxK = 64;         // proposals per iteration, adaptive up to this
constexpr int kSaMaxInitialK = 16;  // largest settable starting K
constexpr int kSaItem = 128;        // list entries per work item (four per lane)
constexpr int kSaRowCap = 512;      // B row entries a warp stages in shared memory (longer rows: hash)
constexpr int kSaUnitTable = 4096;  // items per iteration with an item -> list table (else binary search)

constexpr int kSaApplyRowCap = 4096;  // entries per staged row in the swap apply (4 rows)

// Dynamic shared memory of the chain kernel: the warps' B-row buffers (two
// per warp), which the swap apply reuses for its four staged rows (at least
// 64 KB), then the chain's mapping when it fits.
__host__ __device__ constexpr size_t sa_dyn_base(int threads) {
    return sizeof(uint32_t) * kSaRowCap * 2 * (size_t)(threads / 32) > sizeof(uint32_t) * 4 * kSaApplyRowCap
               ? sizeof(uint32_t) * kSaRowCap * 2 * (size_t)(threads / 32)
               : sizeof(uint32_t) * 4 * kSaApplyRowCap;
}

// Apply the swap pi(a) <-> pi(b) of one chain with the whole CTA: S updates of
// every A entry incident to a or b (as apply_kernel in bm_apply.cu), then pi.
// Every lookup is in one of four B rows (out and in of pi a and pi b), staged
// in `stage` (4 x kSaApplyRowCap entries of shared memory; longer rows use
// the hash).  `pi` is the working copy (shared or global memory), `gpi` the
// chain's mapping in global memory, updated too.
template <int CL>
__device__ void chain_apply_block(const PairDev& P, int32_t* pi, int32_t* gpi, int32_t* ov, int32_t sa, int32_t sb,
                                  uint32_t* stage, int crank) {
    const int32_t fa = pi[sa], fb = pi[sb];
    // rows: 0 = out(fa), 1 = out(fb), 2 = in(fa), 3 = in(fb)
    int32_t rlen[4];
    bool rst[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int32_t g = (r & 1) ? fb : fa;
        const int32_t* ptr = (r < 2) ? P.Bout_ptr : P.Bin_ptr;
        const uint32_t* ent = (r < 2) ? P.Bout_ent : P.Bin_ent;
        const int32_t b = __ldg(ptr + g);
        rlen[r] = __ldg(ptr + g + 1) - b;
        rst[r] = rlen[r] <= kSaApplyRowCap;
        if (rst[r])
            for (int32_t j = threadIdx.x; j < rlen[r]; j += blockDim.x) stage[r * kSaApplyRowCap + j] = __ldg(ent + b + j);
    }
    __syncthreads();
    // B(g, h) for g in {fa, fb} (rows 0, 1) and B(h, g) (rows 2, 3)
    auto bout = [&](int32_t g, int32_t h) -> int32_t {
        const bool a = g == fa;
        const int32_t len = a ? rlen[0] : rlen[1];
        const bool st = a ? rst[0] : rst[1];
        return st ? bm_row_weight(stage + (a ? 0 : kSaApplyRowCap), len, h) : bm_hash_get(P.hb, g, h);
    };
    auto bin = [&](int32_t h, int32_t g) -> int32_t {
        const bool a = g == fa;
        const int32_t len = a ? rlen[2] : rlen[3];
        const bool st = a ? rst[2] : rst[3];
        return st ? bm_row_weight(stage + (a ? 2 : 3) * kSaApplyRowCap, len, h) : bm_hash_get(P.hb, h, g);
    };
    for (int side = 0; side < 2; side++) {
        const int32_t me = side ? sb : sa, other = side ? sa : sb;
        const int32_t fme = side ? fb : fa, fnew = side ? fa : fb;
        {
            const int32_t b = __ldg(P.Aout_ptr + me), e = __ldg(P.Aout_ptr + me + 1);
            for (int32_t j = b + (int32_t)threadIdx.x + crank * (int32_t)blockDim.x; j < e; j += CL * (int32_t)blockDim.x) {
                const uint32_t ent = __ldg(P.Aout_ent + j);
                if (ent == 0) continue;
                const int32_t x = bm_eid(ent), w = bm_ew(ent);
                if (x == other) {
                    const int32_t d = imin(w, bout(fnew, fme)) - imin(w, bout(fme, fnew));
                    if (d) { atomicAdd(ov + me, d); atomicAdd(ov + other, d); }
                } else {
                    const int32_t gx = pi[x];
                    const int32_t d = imin(w, bout(fnew, gx)) - imin(w, bout(fme, gx));
                    if (d) { atomicAdd(ov + me, d); atomicAdd(ov + x, d); }
                }
            }
        }
        {
            const int32_t b = __ldg(P.Ain_ptr + me), e = __ldg(P.Ain_ptr + me + 1);
            for (int32_t j = b + (int32_t)threadIdx.x + crank * (int32_t)blockDim.x; j < e; j += CL * (int32_t)blockDim.x) {
                const uint32_t ent = __ldg(P.Ain_ent + j);
                if (ent == 0) continue;
                const int32_t x = bm_eid(ent), w = bm_ew(ent);
                if (x == other) continue;
                const int32_t gx = pi[x];
                const int32_t d = imin(w, bin(gx, fnew)) - imin(w, bin(gx, fme));
                if (d) { atomicAdd(ov + me, d); atomicAdd(ov + x, d); }
            }
        }
    }
    // every read of the mapping (both CTAs of a pair) before it changes
    if constexpr (CL > 1) cg::this_cluster().sync(); else __syncthreads();
    if (threadIdx.x == 0) {
        if (pi != gpi || crank == 0) {
            pi[sa] = fb;
            pi[sb] = fa;
        }
        if (gpi != pi && crank == 0) {
            gpi[sa] = fb;
            gpi[sb] = fa;
        }
    }
    // the mapping and the overlap updates of both CTAs seen by both
    if constexpr (CL > 1) cg::this_cluster().sync(); else __syncthreads();
}

// One CTA runs one chain.  Each iteration draws the proposals of steps
// s..s+K-1 and evaluates all of them at once under the current mapping.
// Each entry of the four A lists of a proposal (out(u), in(u), out(v),
// in(v)) contributes (the per-pair identity of bm_pairs.cu)
//   out(u): min(w, B(pi v, pi x))   in(u): min(w, B(pi x, pi v))
//   out(v): min(w, B(pi u, pi x))   in(v): min(w, B(pi x, pi u))
// so every entry of one list looks up the same B row (B-out or B-in of pi v
// or pi u).  The lists are cut into items of kSaItem entries; warp w takes
// items w, w + 16, ..., stages the item's B row in its shared buffer with
// coalesced loads, and each lane binary-searches pi x in it (rows longer
// than the buffer use the hash).  For an entry of u whose other end is v,
// the direct-edge repair min(w, B(pi u, pi v)) + min(w, B(pi v, pi u)) is
// added; the item sums meet in a per-proposal shared counter, then
//   delta = sum - S(u) - S(v) + self-loop terms.
// The first accepted proposal in step order is applied and the rest are
// discarded, so the chain is the one-at-a-time chain for every K.  K adapts
// to the acceptance rate: it doubles (up to kSaMaxK) after an iteration with
// no acceptance and drops to max(a.K, 2 (j + 1)) after the j-th proposal is
// accepted; a function of the chain's own history, so replays are exact.
template <int CL, int THREADS>
__device__ __forceinline__ void sa_chain_body(const SaArgs& a) {
    extern __shared__ __align__(16) uint32_t s_dyn[];
    // CL CTAs (a cluster) run one chain: they draw the same proposals, split
    // the evaluation's items and the swap apply's list entries, and read each
    // other's per-proposal sums through distributed shared memory
    const int c = blockIdx.x / CL;
    const int crank = CL > 1 ? (int)cg::this_cluster().block_rank() : 0;
    if (c >= a.nchains) return;
    constexpr int kSeg = 4 * kSaMaxK;
    constexpr int kW = THREADS / 32;
    __shared__ bm_proposal s_prop[kSaMaxK];
    __shared__ int32_t s_sum[kSaMaxK];
    __shared__ long long s_d[kSaMaxK];
    __shared__ int32_t s_seglen[kSeg];             // entries per list
    __shared__ int32_t s_segbase[kSeg];            // offset of each list in its CSR
    __shared__ int32_t s_upre[kSeg + 1];           // unit prefix over the lists
    __shared__ uint8_t s_unit_seg[kSaUnitTable];   // unit -> list (when the units fit)
    __shared__ int32_t s_wsum[kW];
    __shared__ int32_t s_first;
    ChainDev& ch = a.chains[c];
    const PairDev P = a.pairs[ch.pair];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int32_t* gpi = ch.pi;
    int32_t* pi = gpi;
    uint32_t* rowbuf = s_dyn + (size_t)warp * 2 * kSaRowCap;  // this warp's two B-row buffers
    if (a.pi_smem) {
        int32_t* s_pi = reinterpret_cast<int32_t*>(s_dyn + sa_dyn_base(THREADS) / sizeof(uint32_t));
        for (int32_t i = tid; i <= P.n; i += blockDim.x) s_pi[i] = gpi[i];
        pi = s_pi;
    }
    int32_t* ov = ch.ov;
    uint64_t step = ch.step;
    const uint64_t end = min(a.steps, step + a.chunk);
    long long score = ch.score, accepts = ch.accepts;
    int K = min(max(a.K, 1), kSaMaxK);
    if (tid == 0) s_first = kSaMaxK;
    __syncthreads();
    while (step < end) {
        const int nseg = 4 * K;
        // ---- proposals (each list's thread draws its own proposal) and list lengths
        int32_t units = 0;
        if (tid < nseg) {
            const int w = tid >> 2, kind = tid & 3;
            const uint64_t sidx = step + (uint64_t)w;
            int32_t len = 0, base = 0;
            if (sidx < end) {
                const bm_proposal pr = bm_sa_proposal(ch.key, sidx, P.n);
                if (kind == 0) { s_prop[w] = pr; s_sum[w] = 0; }
                const int32_t me = kind < 2 ? pr.u : pr.v;
                const int32_t* ptr = (kind & 1) ? P.Ain_ptr : P.Aout_ptr;
                base = __ldg(ptr + me);
                len = __ldg(ptr + me + 1) - base;
            }
            s_seglen[tid] = len;
            s_segbase[tid] = base;
            units = (len + kSaItem - 1) / kSaItem;
        }
        // ---- exclusive block scan of the unit counts
        int32_t incl = units;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        int32_t woff = 0, U = 0;
#pragma unroll
        for (int w = 0; w < kW; w++) {
            const int32_t x = s_wsum[w];
            woff += (w < warp) ? x : 0;
            U += x;
        }
        const int32_t excl = woff + incl - units;
        if (tid < nseg) s_upre[tid] = excl;
        if (tid == 0) s_upre[nseg] = U;
        const bool table = U <= kSaUnitTable;
        if (table && tid < nseg)
            for (int32_t x = excl; x < excl + units; x++) s_unit_seg[x] = (uint8_t)tid;
        __syncthreads();
        // ---- evaluate: warp w takes items w, w + kW, ... through a three-stage
        // pipeline: the B-row bounds and A entries of item i + 2 kW are
        // loaded, the B row of item i + kW is copied (cp.async) into the
        // warp's other buffer, and item i is searched, all at once
        {
            struct Stage {
                int32_t item, w, kind, g, rb, rl;
                uint32_t ent[kSaItem / 32];
            };
            auto fetch = [&](int32_t item, Stage& st) {
                st.item = item;
                st.rb = 0;
                st.rl = 0;
                st.w = 0;
                st.kind = 0;
                st.g = 0;
#pragma unroll
                for (int k = 0; k < kSaItem / 32; k++) st.ent[k] = 0u;
                if (item >= U) return;
                int32_t lo;
                if (table) {
                    lo = s_unit_seg[item];
                } else {
                    lo = 0;
                    int32_t hi = nseg;  // last list with s_upre[list] <= item
                    while (hi - lo > 1) {
                        const int32_t mid = (lo + hi) >> 1;
                        if (s_upre[mid] <= item) lo = mid; else hi = mid;
                    }
                }
                st.w = lo >> 2;
                st.kind = lo & 3;
                const bool out = !(st.kind & 1);
                const int32_t e0 = (item - s_upre[lo]) * kSaItem, len = s_seglen[lo], base = s_segbase[lo];
                const uint32_t* alist = out ? P.Aout_ent : P.Ain_ent;
#pragma unroll
                for (int k = 0; k < kSaItem / 32; k++) {
                    const int32_t off = e0 + lane + 32 * k;
                    if (off < len) st.ent[k] = __ldg(alist + base + off);
                }
                const bm_proposal& pr = s_prop[st.w];
                st.g = st.kind < 2 ? pi[pr.v] : pi[pr.u];
                const int32_t* rptr = out ? P.Bout_ptr : P.Bin_ptr;
                st.rb = __ldg(rptr + st.g);
                st.rl = __ldg(rptr + st.g + 1) - st.rb;
            };
            // B rows start on 16-byte boundaries (rows are padded to multiples of 4)
            auto copy_row = [&](const Stage& st, int buf) {
                if (st.item < U && st.rl <= kSaRowCap) {
                    const uint32_t* rent = !(st.kind & 1) ? P.Bout_ent : P.Bin_ent;
                    const uint32_t dst0 = (uint32_t)__cvta_generic_to_shared(rowbuf + (size_t)buf * kSaRowCap);
                    for (int32_t j = 4 * lane; j < st.rl; j += 128)
                        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst0 + 4u * (uint32_t)j),
                                     "l"(rent + st.rb + j) : "memory");
                }
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            constexpr int kStride = CL * kW;  // the chain's warps over all its CTAs
            const int gw = crank * kW + warp;
            Stage cur, nxt, far;
            fetch(gw, cur);
            fetch(gw + kStride, nxt);
            copy_row(cur, 0);
            int buf = 0;
            for (int32_t item = gw; item < U; item += kStride) {
                copy_row(nxt, buf ^ 1);
                fetch(item + 2 * kStride, far);
                asm volatile("cp.async.wait_group 1;" ::: "memory");  // this item's row has landed
                __syncwarp();
                const uint32_t* row = rowbuf + (size_t)buf * kSaRowCap;
                const bool out = !(cur.kind & 1);
                const bool staged = cur.rl <= kSaRowCap;
                const bm_proposal pr = s_prop[cur.w];
                int32_t val = 0;
#pragma unroll
                for (int k = 0; k < kSaItem / 32; k++) {
                    if (cur.ent[k] == 0) continue;
                    const int32_t x = bm_eid(cur.ent[k]), wa = bm_ew(cur.ent[k]);
                    const int32_t gx = pi[x];
                    int32_t wb = 0;
                    if (staged) {
                        // first row slot whose id is >= gx (zero padding sorts last)
                        int32_t l = 0, h = cur.rl;
                        while (l < h) {
                            const int32_t mid = (l + h) >> 1;
                            const uint32_t e = row[mid];
                            if (e != 0u && bm_eid(e) < gx) l = mid + 1; else h = mid;
                        }
                        if (l < cur.rl) {
                            const uint32_t e = row[l];
                            if (e != 0u && bm_eid(e) == gx) wb = bm_ew(e);
                        }
                    } else {
                        wb = out ? bm_hash_get(P.hb, cur.g, gx) : bm_hash_get(P.hb, gx, cur.g);
                    }
                    val += imin(wa, wb);
                    if (cur.kind < 2 && x == pr.v) {
                        const int32_t fu = pi[pr.u], fv = pi[pr.v];
                        val += imin(wa, bm_hash_get(P.hb, fu, fv)) + imin(wa, bm_hash_get(P.hb, fv, fu));
                    }
                }
                // an item lies in one list, hence one proposal: warp sum, one atomic
#pragma unroll
                for (int o = 16; o; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
                if (lane == 0 && val) atomicAdd(&s_sum[cur.w], val);
                __syncwarp();  // this buffer is rewritten two items on
                cur = nxt;
                nxt = far;
                buf ^= 1;
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            __syncwarp();
        }
        __syncthreads();
        if constexpr (CL > 1) cg::this_cluster().sync();  // every CTA's sums are complete
        // ---- deltas and acceptance, one thread per proposal; the first
        // accepted one in step order wins (each CTA of a pair decides alike)
        if (tid < K && step + (uint64_t)tid < end) {
            const bm_proposal pr = s_prop[tid];
            long long sum = s_sum[tid];
            if constexpr (CL > 1) {
#pragma unroll
                for (int q = 1; q < CL; q++) sum += *cg::this_cluster().map_shared_rank(s_sum + tid, (crank + q) % CL);
            }
            long long d = sum - (long long)ov[pr.u] - (long long)ov[pr.v];
            if (P.has_self) {
                const int32_t fu = pi[pr.u], fv = pi[pr.v];
                const int32_t su = __ldg(P.selfA + pr.u), sv = __ldg(P.selfA + pr.v);
                const int32_t bu = __ldg(P.selfB + fu), bv = __ldg(P.selfB + fv);
                d += imin(su, bv) - imin(su, bu) + imin(sv, bu) - imin(sv, bv);
            }
            s_d[tid] = d;
            if (bm_sa_accept(d, pr.uni, bm_sa_temperature(a.t0, a.log_ratio, step + (uint64_t)tid, a.steps)))
                atomicMin(&s_first, tid);
        }
        __syncthreads();
        const int first = s_first;
        if (first < K) {
            const bm_proposal pr = s_prop[first];
            score += s_d[first];
            accepts++;
            step += (uint64_t)first + 1;
            K = min(kSaMaxK, max(a.K, 2 * (first + 1)));
            chain_apply_block<CL>(P, pi, gpi, ov, pr.u, pr.v, s_dyn, crank);  // ends with a (cluster) barrier
            if (tid == 0) s_first = kSaMaxK;
        } else {
            step = min(end, step + (uint64_t)K);
            K = min(kSaMaxK, 2 * K);
            // the other CTA's reads of these sums end before they are reset
            if constexpr (CL > 1) cg::this_cluster().sync();
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && crank == 0) {
        ch.step = step;
        ch.score = score;
        ch.accepts = accepts;
    }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) sa_chain_kernel(SaArgs a) { sa_chain_body<1, THREADS>(a); }

// One chain per pair of CTAs (a cluster of two on two SMs), for batches with
// fewer chains than half the SMs.
template <int THREADS>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1) sa_chain_kernel_pair(SaArgs a) {
    sa_chain_body<2, THREADS>(a);
}

// Initial S(v) and score of every chain: a warp per (chain, A vertex).
__global__ void sa_init_kernel(const PairDev* pairs, ChainDev* chains, int32_t nchains) {
    const int c = blockIdx.y;
    if (c >= nchains) return;
    ChainDev& ch = chains[c];
    const PairDev P = pairs[ch.pair];
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int32_t u = 1 + blockIdx.x * wpb + (threadIdx.x >> 5); u <= P.n; u += gridDim.x * wpb) {
        const int32_t fu = ch.pi[u];
        int32_t s = 0;
        for (int32_t j = __ldg(P.Aout_ptr + u) + lane; j < __ldg(P.Aout_ptr + u + 1); j += 32) {
            const uint32_t ent = __ldg(P.Aout_ent + j);
            if (ent == 0) continue;
            const int32_t x = bm_eid(ent);
            const int32_t cc = imin(bm_ew(ent), bm_hash_get(P.hb, fu, ch.pi[x]));
            if (cc) atomicAdd(ch.ov + x, cc);
            s += cc;
        }
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (s) atomicAdd(ch.ov + u, s);
            const long long t = (long long)s + imin(__ldg(P.selfA + u), __ldg(P.selfB + fu));
            if (t) atomicAdd(reinterpret_cast<unsigned long long*>(&ch.score), (unsigned long long)t);
        }
    }
}

}  // namespace

// ------------------------------------------------------------------ batches

struct bm_batch {
    bm_ctx* ctx = nullptr;
    int device = 0;  // kept so that destruction does not need the context
    struct Pair {
        int32_t n = 0;
        int64_t m_real_a = 0;
        int32_t* d[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // Aoptr, Aiptr, selfA, selfB, Boptr, Biptr
        uint32_t* e[4] = {nullptr, nullptr, nullptr, nullptr};                 // Aoent, Aient, Boent, Bient
        unsigned long long* hash = nullptr;
        int hlog2 = 0;
        int has_self = 0;
    };
    std::vector<Pair> pairs;
    PairDev* d_pairs = nullptr;
    bool dirty = true;
};

static PairDev pair_dev(const bm_batch::Pair& p) {
    return PairDev{p.n, p.has_self, p.d[0], p.d[1], p.e[0], p.e[1], p.d[2], p.d[3], HashView{p.hash, p.hlog2, p.n + 1},
                   p.d[4], p.d[5], p.e[2], p.e[3]};
}

static void free_pair(bm_batch::Pair& p) {
    for (auto* x : p.d) bm_cuda_free(x);
    for (auto* x : p.e) bm_cuda_free(x);
    bm_cuda_free(p.hash);
    p = bm_batch::Pair();
}

extern "C" bm_status bm_batch_create(bm_ctx* ctx, bm_batch** out) {
    if (!ctx || !out) return BM_INVALID_ARG;
    *out = new (std::nothrow) bm_batch();
    if (!*out) return BM_OOM;
    (*out)->ctx = ctx;
    (*out)->device = ctx->device;
    return BM_OK;
}

extern "C" void bm_batch_destroy(bm_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    for (auto& p : b->pairs) free_pair(p);
    bm_cuda_free(b->d_pairs);
    delete b;
}

template <typename T>
static bm_status up(bm_ctx* ctx, T** d, const std::vector<T>& h) {
    BM_CUDA(ctx, bm_cuda_malloc((void**)d, sizeof(T) * (h.empty() ? 1 : h.size())));
    if (!h.empty()) BM_CUDA(ctx, cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return BM_OK;
}

extern "C" bm_status bm_batch_add_pair(bm_batch* b, int32_t n, int64_t mA, const int32_t* srcA, const int32_t* dstA,
                                       const int32_t* wA, int64_t mB, const int32_t* srcB, const int32_t* dstB,
                                       const int32_t* wB, int32_t* pair_index) {
    if (!b) return BM_INVALID_ARG;
    bm_ctx* ctx = b->ctx;
    HostCsr HA, HB;
    std::string err;
    if (bm_build_host_csr(false, n, mA, srcA, dstA, wA, HA, err) != 0) return bm_fail(ctx, BM_INVALID_ARG, "A: %s", err.c_str());
    if (bm_build_host_csr(true, n, mB, srcB, dstB, wB, HB, err) != 0) return bm_fail(ctx, BM_INVALID_ARG, "B: %s", err.c_str());
    if (n < 2) return bm_fail(ctx, BM_INVALID_ARG, "annealing needs n >= 2");
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    bm_batch::Pair p;
    p.n = n;
    p.m_real_a = HA.m_real;
    bm_status s;
    if ((s = up(ctx, &p.d[0], HA.optr)) != BM_OK || (s = up(ctx, &p.d[1], HA.iptr)) != BM_OK ||
        (s = up(ctx, &p.d[2], HA.self)) != BM_OK || (s = up(ctx, &p.d[3], HB.self)) != BM_OK ||
        (s = up(ctx, &p.e[0], HA.oent)) != BM_OK || (s = up(ctx, &p.e[1], HA.ient)) != BM_OK ||
        (s = up(ctx, &p.d[4], HB.optr)) != BM_OK || (s = up(ctx, &p.d[5], HB.iptr)) != BM_OK ||
        (s = up(ctx, &p.e[2], HB.oent)) != BM_OK || (s = up(ctx, &p.e[3], HB.ient)) != BM_OK ||
        (s = up(ctx, &p.hash, HB.htab)) != BM_OK) {
        free_pair(p);
        return s;
    }
    p.hlog2 = HB.hlog2;
    p.has_self = HA.has_self && HB.has_self;
    b->pairs.push_back(p);
    b->dirty = true;
    if (pair_index) *pair_index = (int32_t)b->pairs.size() - 1;
    return BM_OK;
}

// ------------------------------------------------------------- autotuning

namespace {

struct Tuning {
    int32_t candidates = 8;
    int32_t threads_unused = 0;
};

std::string tune_cache_path() {
    const char* p = getenv("BM_TUNE_CACHE");
    if (p && *p) return p;
    const char* h = getenv("HOME");
    return std::string(h && *h ? h : "/tmp") + "/.bm_b200_tune.txt";
}

// One line per key: "<device name>|<total n>|<chains> <candidates>"
bool tune_lookup(const std::string& key, int32_t* cand) {
    FILE* f = fopen(tune_cache_path().c_str(), "r");
    if (!f) return false;
    char line[512];
    bool found = false;
    while (fgets(line, sizeof line, f)) {
        char* sp = strrchr(line, ' ');
        if (!sp) continue;
        *sp = 0;
        if (key == line) { *cand = atoi(sp + 1); found = true; }
    }
    fclose(f);
    return found;
}

void tune_store(const std::string& key, int32_t cand) {
    FILE* f = fopen(tune_cache_path().c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %d\n", key.c_str(), cand);
    fclose(f);
}

}  // namespace

namespace {

// Dynamic shared memory of a chain: the warps' B-row buffers, plus the
// chain's mapping when it fits (the largest n + 1 ints of the launch), else
// the mapping stays in global memory.  Sets the kernel's dynamic
// shared-memory limit; called before any stream capture.
bm_status chain_smem(bm_ctx* ctx, SaArgs& args, int32_t n_max, int32_t threads, size_t* smem) {
    const size_t need = sizeof(int32_t) * ((size_t)n_max + 1);
    const size_t base = sa_dyn_base(threads);
    *smem = base;
    args.pi_smem = 0;
    if (base + need + 16384 <= ctx->smem_optin) {
        args.pi_smem = 1;
        *smem += need;
    }
    if (threads == 256) {
        BM_CUDA(ctx, cudaFuncSetAttribute(sa_chain_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
        BM_CUDA(ctx, cudaFuncSetAttribute(sa_chain_kernel_pair<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
    } else {
        BM_CUDA(ctx, cudaFuncSetAttribute(sa_chain_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
        BM_CUDA(ctx, cudaFuncSetAttribute(sa_chain_kernel_pair<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
    }
    return BM_OK;
}

// One launch of the chains: a CTA per chain, or a pair of CTAs per chain, of
// 256 or 512 threads.
void launch_chains(const SaArgs& args, int32_t ctas_per_chain, int32_t threads, size_t smem, cudaStream_t stream) {
    if (threads == 256) {
        if (ctas_per_chain == 2)
            sa_chain_kernel_pair<256><<<args.nchains * 2, 256, smem, stream>>>(args);
        else
            sa_chain_kernel<256><<<args.nchains, 256, smem, stream>>>(args);
    } else {
        if (ctas_per_chain == 2)
            sa_chain_kernel_pair<512><<<args.nchains * 2, 512, smem, stream>>>(args);
        else
            sa_chain_kernel<512><<<args.nchains, 512, smem, stream>>>(args);
    }
}

}  // namespace

extern "C" bm_status bm_sa_run(bm_batch* b, int32_t nchains, const int32_t* chain_pair, const uint64_t* chain_key,
                               const int32_t* init_pi, const bm_sa_params* prm, int32_t* final_pi,
                               int64_t* final_score, int64_t* accepts, bm_sa_stats* stats) {
    if (!b || !prm || nchains < 1 || !chain_pair || !chain_key || !init_pi) return BM_INVALID_ARG;
    bm_ctx* ctx = b->ctx;
    if (prm->steps < 0 || !(prm->t0 > 0) || !(prm->t_end > 0))
        return bm_fail(ctx, BM_INVALID_ARG, "need steps >= 0 and positive temperatures");
    if (prm->candidates < 0 || prm->candidates > 16)
        return bm_fail(ctx, BM_INVALID_ARG, "candidates must be 0 (tuned) or 1..16");
    if (prm->threads_per_cta != 0 && prm->threads_per_cta != 256 && prm->threads_per_cta != 512)
        return bm_fail(ctx, BM_INVALID_ARG, "threads_per_cta must be 0, 256 or 512");
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    const int32_t np = (int32_t)b->pairs.size();
    // chain layout and validation
    std::vector<int64_t> off((size_t)nchains + 1, 0);
    for (int32_t c = 0; c < nchains; c++) {
        if (chain_pair[c] < 0 || chain_pair[c] >= np) return bm_fail(ctx, BM_INVALID_ARG, "chain %d: bad pair", c);
        const int32_t n = b->pairs[(size_t)chain_pair[c]].n;
        off[(size_t)c + 1] = off[(size_t)c] + (int64_t)n + 1;
    }
    for (int32_t c = 0; c < nchains; c++) {
        const int32_t n = b->pairs[(size_t)chain_pair[c]].n;
        const int32_t* p = init_pi + off[(size_t)c];
        std::vector<char> seen((size_t)n + 1, 0);
        for (int32_t i = 1; i <= n; i++) {
            const int32_t f = p[i];
            if (f < 1 || f > n || seen[(size_t)f]) return bm_fail(ctx, BM_INVALID_ARG, "chain %d: pi is not a bijection", c);
            seen[(size_t)f] = 1;
        }
    }
    // pair table
    if (b->dirty) {
        std::vector<PairDev> hp((size_t)np);
        for (int32_t i = 0; i < np; i++) {
            const auto& p = b->pairs[(size_t)i];
            hp[(size_t)i] = pair_dev(p);
        }
        bm_cuda_free(b->d_pairs);
        b->d_pairs = nullptr;
        BM_CUDA(ctx, bm_cuda_malloc(&b->d_pairs, sizeof(PairDev) * (size_t)np));
        BM_CUDA(ctx, cudaMemcpy(b->d_pairs, hp.data(), sizeof(PairDev) * (size_t)np, cudaMemcpyHostToDevice));
        b->dirty = false;
    }
    // per-chain state: mapping (input/output) and the per-vertex overlap (scratch)
    const int64_t tot = off[(size_t)nchains];
    int32_t* d_pi = nullptr;
    int32_t* d_ov = nullptr;
    ChainDev* d_ch = nullptr;
    BM_CUDA(ctx, bm_cuda_malloc(&d_pi, sizeof(int32_t) * (size_t)tot));
    BM_CUDA(ctx, bm_cuda_malloc(&d_ov, sizeof(int32_t) * (size_t)tot));
    BM_CUDA(ctx, bm_cuda_malloc(&d_ch, sizeof(ChainDev) * (size_t)nchains));
    struct Guard {
        void* p[3];
        ~Guard() { for (void* x : p) bm_cuda_free(x); }
    } guard{{d_pi, d_ov, d_ch}};
    BM_CUDA(ctx, cudaMemcpyAsync(d_pi, init_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_ov, 0, sizeof(int32_t) * (size_t)tot, ctx->stream));
    std::vector<ChainDev> hc((size_t)nchains);
    for (int32_t c = 0; c < nchains; c++) {
        hc[(size_t)c] = ChainDev{chain_pair[c], 0, d_pi + off[(size_t)c], d_ov + off[(size_t)c], chain_key[c], 0ull, 0, 0};
    }
    BM_CUDA(ctx, cudaMemcpyAsync(d_ch, hc.data(), sizeof(ChainDev) * (size_t)nchains, cudaMemcpyHostToDevice, ctx->stream));
    {
        dim3 g(64, (unsigned)nchains);
        sa_init_kernel<<<g, 256, 0, ctx->stream>>>(b->d_pairs, d_ch, nchains);
        BM_LAUNCH_CHECK(ctx, "sa_init_kernel");
    }
    SaArgs args;
    args.pairs = b->d_pairs;
    args.chains = d_ch;
    args.nchains = nchains;
    args.steps = (uint64_t)prm->steps;
    args.t0 = prm->t0;
    args.log_ratio = log(prm->t_end / prm->t0);
    args.chunk = prm->chunk > 0 ? (uint64_t)prm->chunk : (uint64_t)65536;
    const int32_t kmax = kSaMaxInitialK;
    int32_t K = prm->candidates;
    if (K > kmax) return bm_fail(ctx, BM_INVALID_ARG, "candidates %d above this build's limit %d", K, kmax);
    int32_t n_max = 0;
    for (int32_t c = 0; c < nchains; c++) n_max = std::max(n_max, b->pairs[(size_t)chain_pair[c]].n);
    // CTAs per chain: a pair when the chains fill at most half the SMs (the
    // tuner may keep one); a fixed K keeps the pair rule and 512 threads
    int32_t CLc = (2 * nchains <= ctx->num_sms) ? 2 : 1;
    int32_t TH = prm->threads_per_cta ? prm->threads_per_cta : 512;
    if (K == 0) {
        int64_t ntot = 0;
        for (int32_t c = 0; c < nchains; c++) ntot += b->pairs[(size_t)chain_pair[c]].n;
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, ctx->device);
        const std::string key = std::string(prop.name) + "|" + std::to_string(ntot) + "|" + std::to_string(nchains);
        int32_t tuned = 0;
        if (tune_lookup(key, &tuned)) {
            K = tuned & 0xFF;
            CLc = ((tuned >> 8) & 0xF) == 2 ? 2 : 1;
            TH = ((tuned >> 12) & 1) ? 256 : 512;
            if (CLc == 2 && 2 * nchains > ctx->num_sms) CLc = 1;
            if (K < 1 || K > kmax) K = 8;
        } else {
            // time a short prefix of the real run for each (K, CTAs per
            // chain, threads per CTA) and keep the fastest; the chain depends
            // on none of them, so the prefix is simply replayed by the real
            // run below
            float best_ms = 1e30f;
            int32_t best_k = 8, best_cl = 1, best_th = 512;
            std::vector<ChainDev> snap = hc;
            const int32_t max_cl = (2 * nchains <= ctx->num_sms) ? 2 : 1;
            for (int32_t trial = 0; trial < 10 * max_cl; trial++) {
                const int32_t cand = 1 << (trial % 5), cl = 1 + trial / 10, th = ((trial / 5) & 1) ? 256 : 512;
                if (cand > kmax) continue;
                SaArgs t = args;
                size_t tsmem = 0;
                {
                    bm_status st = chain_smem(ctx, t, n_max, th, &tsmem);
                    if (st != BM_OK) return st;
                }
                BM_CUDA(ctx, cudaMemcpyAsync(d_pi, init_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyHostToDevice, ctx->stream));
                BM_CUDA(ctx, cudaMemsetAsync(d_ov, 0, sizeof(int32_t) * (size_t)tot, ctx->stream));
                BM_CUDA(ctx, cudaMemcpyAsync(d_ch, snap.data(), sizeof(ChainDev) * (size_t)nchains, cudaMemcpyHostToDevice, ctx->stream));
                sa_init_kernel<<<dim3(64, (unsigned)nchains), 256, 0, ctx->stream>>>(b->d_pairs, d_ch, nchains);
                BM_LAUNCH_CHECK(ctx, "sa_init_kernel");
                t.K = cand;
                t.chunk = std::min<uint64_t>(4096, args.steps > 0 ? args.steps : 1);
                struct Events {
                    cudaEvent_t a = nullptr, b = nullptr;
                    ~Events() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
                } ev;
                BM_CUDA(ctx, cudaEventCreate(&ev.a));
                BM_CUDA(ctx, cudaEventCreate(&ev.b));
                BM_CUDA(ctx, cudaEventRecord(ev.a, ctx->stream));
                launch_chains(t, cl, th, tsmem, ctx->stream);
                BM_LAUNCH_CHECK(ctx, "sa_chain_kernel(tune)");
                BM_CUDA(ctx, cudaEventRecord(ev.b, ctx->stream));
                BM_CUDA(ctx, cudaEventSynchronize(ev.b));
                float ms = 0;
                cudaEventElapsedTime(&ms, ev.a, ev.b);
                if (ms < best_ms) { best_ms = ms; best_k = cand; best_cl = cl; best_th = th; }
            }
            K = best_k;
            CLc = best_cl;
            TH = best_th;
            tune_store(key, K | (CLc << 8) | ((TH == 256 ? 1 : 0) << 12));
            // restart from the initial state
            BM_CUDA(ctx, cudaMemcpyAsync(d_pi, init_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyHostToDevice, ctx->stream));
            BM_CUDA(ctx, cudaMemsetAsync(d_ov, 0, sizeof(int32_t) * (size_t)tot, ctx->stream));
            BM_CUDA(ctx, cudaMemcpyAsync(d_ch, snap.data(), sizeof(ChainDev) * (size_t)nchains, cudaMemcpyHostToDevice, ctx->stream));
            sa_init_kernel<<<dim3(64, (unsigned)nchains), 256, 0, ctx->stream>>>(b->d_pairs, d_ch, nchains);
            BM_LAUNCH_CHECK(ctx, "sa_init_kernel");
        }
    }
    size_t smem = 0;
    {
        bm_status st = chain_smem(ctx, args, n_max, TH, &smem);
        if (st != BM_OK) return st;
    }
    // capture one chunk launch in a graph and replay it
    const uint64_t launches = args.steps == 0 ? 0 : (args.steps + args.chunk - 1) / args.chunk;
    const auto t0 = std::chrono::steady_clock::now();
    if (launches > 0) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        args.K = K;
        BM_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        launch_chains(args, CLc, TH, smem, ctx->stream);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
        if (ce != cudaSuccess) return bm_cuda_fail(ctx, ce, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&exec, graph, 0);
        if (ce != cudaSuccess) { cudaGraphDestroy(graph); return bm_cuda_fail(ctx, ce, "cudaGraphInstantiate"); }
        for (uint64_t l = 0; l < launches; l++) {
            ce = cudaGraphLaunch(exec, ctx->stream);
            if (ce != cudaSuccess) break;
            ctx->launches++;
        }
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return bm_cuda_fail(ctx, ce, "cudaGraphLaunch");
    }
    BM_CUDA(ctx, cudaMemcpyAsync(hc.data(), d_ch, sizeof(ChainDev) * (size_t)nchains, cudaMemcpyDeviceToHost, ctx->stream));
    if (final_pi)
        BM_CUDA(ctx, cudaMemcpyAsync(final_pi, d_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int32_t c = 0; c < nchains; c++) {
        if (final_score) final_score[c] = hc[(size_t)c].score;
        if (accepts) accepts[c] = hc[(size_t)c].accepts;
    }
    if (stats) {
        stats->candidates = K;
        stats->ctas_per_chain = CLc;
        stats->threads_per_cta = TH;
        stats->launches = (int64_t)launches;
        stats->seconds = secs;
    }
    return BM_OK;
}

extern "C" int64_t bm_sa_layout_size(bm_batch* b, int32_t nchains, const int32_t* chain_pair) {
    if (!b || !chain_pair || nchains < 0) return -1;
    int64_t tot = 0;
    for (int32_t c = 0; c < nchains; c++) {
        if (chain_pair[c] < 0 || chain_pair[c] >= (int32_t)b->pairs.size()) return -1;
        tot += b->pairs[(size_t)chain_pair[c]].n + 1;
    }
    return tot;
}

// --------------------------------------------------- allocation-free variant
//
// bm_sa_run_noalloc runs the same chains as bm_sa_run without allocating any
// device memory.  It is for callers that cannot call cudaMalloc/cudaFree while
// they run: a process whose device memory is owned by its own pool allocator
// under a fixed budget, or a serving path that must not pay the implicit
// device-wide synchronisation of cudaFree while other streams are busy.
//
// Its scratch is the file-scope array below: the pair table, the chain states,
// and every chain's mapping and per-vertex overlap.  Host code must not use the
// symbol's name as a device address: bm_ctx_create looks the address up with
// cudaGetSymbolAddress, with the context's device current, and keeps it in the
// context.  That lookup loads the module that holds the array (the runtime
// loads modules lazily), so the array is reserved on a device when the first
// context on it is created and stays reserved until the process exits; the
// entry point itself never reserves it.  A device reset (cudaDeviceReset)
// unloads the module and invalidates every context on the device: create a new
// context after one.  All calls share the array and it keeps the last call's
// contents, so each call rewrites what it reads and clears the overlap arrays;
// calls whose work overlaps on the GPU (two host threads, or two contexts on
// one device) race and must be serialised by the caller.

namespace {

constexpr int64_t kNoAllocMaxPairs = 256;
constexpr int64_t kNoAllocMaxChains = 1024;
constexpr int64_t kNoAllocMaxInts = 1 << 20;  // sum over chains of (n + 1)
constexpr size_t kNoAllocPairBytes = 128;
constexpr size_t kNoAllocChainBytes = 64;
constexpr size_t kNoAllocOffChains = kNoAllocMaxPairs * kNoAllocPairBytes;
constexpr size_t kNoAllocOffPi = kNoAllocOffChains + kNoAllocMaxChains * kNoAllocChainBytes;
constexpr size_t kNoAllocOffOv = kNoAllocOffPi + sizeof(int32_t) * kNoAllocMaxInts;
constexpr size_t kNoAllocBytes = kNoAllocOffOv + sizeof(int32_t) * kNoAllocMaxInts;  // 8,486,912 bytes
static_assert(sizeof(PairDev) <= kNoAllocPairBytes, "pair slot too small");
static_assert(sizeof(ChainDev) <= kNoAllocChainBytes, "chain slot too small");

}  // namespace

static __device__ __align__(256) unsigned char g_sa_noalloc_scratch[kNoAllocBytes];

bm_status bm_noalloc_setup(bm_ctx* ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sa_noalloc_scratch);
    if (e != cudaSuccess) return bm_cuda_fail(ctx, e, "cudaGetSymbolAddress(g_sa_noalloc_scratch)");
    ctx->noalloc_scratch = static_cast<unsigned char*>(p);
    // the runtime also loads each kernel's code on its first use: load the
    // entry point's two kernels here, so its first call loads nothing
    cudaFuncAttributes fa;
    BM_CUDA(ctx, cudaFuncGetAttributes(&fa, sa_init_kernel));
    BM_CUDA(ctx, cudaFuncGetAttributes(&fa, sa_chain_kernel<kSaThreads>));
    BM_CUDA(ctx, cudaFuncGetAttributes(&fa, sa_chain_kernel_pair<kSaThreads>));  // its smem limit is set by every chain call
    return BM_OK;
}

extern "C" bm_status bm_sa_run_noalloc(bm_batch* b, int32_t nchains, const int32_t* chain_pair,
                                       const uint64_t* chain_key, const int32_t* init_pi,
                                       const bm_sa_params* prm, int32_t* final_pi, int64_t* final_score,
                                       int64_t* accepts) {
    if (!b || !prm || nchains < 1 || !chain_pair || !chain_key || !init_pi) return BM_INVALID_ARG;
    bm_ctx* ctx = b->ctx;
    const int64_t np = (int64_t)b->pairs.size();
    if (np > kNoAllocMaxPairs)
        return bm_fail(ctx, BM_INVALID_ARG, "batch holds %lld pairs; the allocation-free entry point takes at most %lld",
                       (long long)np, (long long)kNoAllocMaxPairs);
    if (nchains > kNoAllocMaxChains)
        return bm_fail(ctx, BM_INVALID_ARG, "%d chains; the allocation-free entry point takes at most %lld", nchains,
                       (long long)kNoAllocMaxChains);
    if (prm->steps < 0 || !(prm->t0 > 0) || !(prm->t_end > 0))
        return bm_fail(ctx, BM_INVALID_ARG, "need steps >= 0 and positive temperatures");
    int64_t tot = 0;
    for (int32_t c = 0; c < nchains; c++) {
        if (chain_pair[c] < 0 || chain_pair[c] >= np) return bm_fail(ctx, BM_INVALID_ARG, "chain %d: bad pair", c);
        tot += (int64_t)b->pairs[(size_t)chain_pair[c]].n + 1;
    }
    if (tot > kNoAllocMaxInts)
        return bm_fail(ctx, BM_INVALID_ARG,
                       "chains need %lld mapping entries; the allocation-free entry point holds at most %lld",
                       (long long)tot, (long long)kNoAllocMaxInts);
    // bijection check with a fixed bitset (n <= 131071)
    {
        uint64_t seen[(BM_MAX_N + 64) / 64];
        int64_t o = 0;
        for (int32_t c = 0; c < nchains; c++) {
            const int32_t n = b->pairs[(size_t)chain_pair[c]].n;
            memset(seen, 0, sizeof(uint64_t) * (size_t)((n + 64) / 64));
            for (int32_t i = 1; i <= n; i++) {
                const int32_t f = init_pi[o + i];
                if (f < 1 || f > n || ((seen[f >> 6] >> (f & 63)) & 1ull))
                    return bm_fail(ctx, BM_INVALID_ARG, "chain %d: pi is not a bijection", c);
                seen[f >> 6] |= 1ull << (f & 63);
            }
            o += n + 1;
        }
    }
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    const int32_t kmax = kSaMaxInitialK;
    int32_t K = prm->candidates == 0 ? std::min(8, kmax) : prm->candidates;
    if (K < 1 || K > kmax) return bm_fail(ctx, BM_INVALID_ARG, "candidates must be 0 or 1..%d", kmax);
    int32_t n_max = 0;
    for (int32_t c = 0; c < nchains; c++) n_max = std::max(n_max, b->pairs[(size_t)chain_pair[c]].n);
    unsigned char* base = ctx->noalloc_scratch;  // resolved when the context was created
    if (!base) return bm_fail(ctx, BM_CUDA_ERROR, "the context holds no address of the static scratch");
    bm_status st = BM_OK;
    PairDev* d_pairs = reinterpret_cast<PairDev*>(base);
    ChainDev* d_ch = reinterpret_cast<ChainDev*>(base + kNoAllocOffChains);
    int32_t* d_pi = reinterpret_cast<int32_t*>(base + kNoAllocOffPi);
    int32_t* d_ov = reinterpret_cast<int32_t*>(base + kNoAllocOffOv);
    // pair table and chain states, staged through small host arrays on the stack
    {
        PairDev hp[16];
        for (int64_t i0 = 0; i0 < np; i0 += 16) {
            const int64_t k = std::min<int64_t>(16, np - i0);
            for (int64_t j = 0; j < k; j++) {
                const auto& p = b->pairs[(size_t)(i0 + j)];
                hp[j] = pair_dev(p);
            }
            BM_CUDA(ctx, cudaMemcpyAsync(d_pairs + i0, hp, sizeof(PairDev) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        ChainDev hc[32];
        int64_t o = 0;
        for (int32_t c0 = 0; c0 < nchains; c0 += 32) {
            const int32_t k = std::min(32, nchains - c0);
            for (int32_t j = 0; j < k; j++) {
                const int32_t c = c0 + j;
                hc[j] = ChainDev{chain_pair[c], 0, d_pi + o, d_ov + o, chain_key[c], 0ull, 0, 0};
                o += (int64_t)b->pairs[(size_t)chain_pair[c]].n + 1;
            }
            BM_CUDA(ctx, cudaMemcpyAsync(d_ch + c0, hc, sizeof(ChainDev) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
    }
    BM_CUDA(ctx, cudaMemcpyAsync(d_pi, init_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemsetAsync(d_ov, 0, sizeof(int32_t) * (size_t)tot, ctx->stream));
    sa_init_kernel<<<dim3(64, (unsigned)nchains), 256, 0, ctx->stream>>>(d_pairs, d_ch, nchains);
    BM_LAUNCH_CHECK(ctx, "sa_init_kernel");
    SaArgs args;
    args.pairs = d_pairs;
    args.chains = d_ch;
    args.nchains = nchains;
    args.steps = (uint64_t)prm->steps;
    args.t0 = prm->t0;
    args.log_ratio = log(prm->t_end / prm->t0);
    args.chunk = prm->chunk > 0 ? (uint64_t)prm->chunk : (uint64_t)65536;
    args.K = K;
    size_t smem = 0;
    if ((st = chain_smem(ctx, args, n_max, kSaThreads, &smem)) != BM_OK) return st;
    const uint64_t launches = args.steps == 0 ? 0 : (args.steps + args.chunk - 1) / args.chunk;
    for (uint64_t l = 0; l < launches; l++) {
        sa_chain_kernel<kSaThreads><<<nchains, kSaThreads, smem, ctx->stream>>>(args);
        BM_LAUNCH_CHECK(ctx, "sa_chain_kernel");
    }
    if (final_pi)
        BM_CUDA(ctx, cudaMemcpyAsync(final_pi, d_pi, sizeof(int32_t) * (size_t)tot, cudaMemcpyDeviceToHost, ctx->stream));
    {
        ChainDev hc[32];
        for (int32_t c0 = 0; c0 < nchains; c0 += 32) {
            const int32_t k = std::min(32, nchains - c0);
            BM_CUDA(ctx, cudaMemcpyAsync(hc, d_ch + c0, sizeof(ChainDev) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            for (int32_t j = 0; j < k; j++) {
                if (final_score) final_score[c0 + j] = hc[j].score;
                if (accepts) accepts[c0 + j] = hc[j].accepts;
            }
        }
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}
