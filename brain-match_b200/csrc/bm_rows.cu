// bm_rows.cu — exact swap deltas of whole rows: delta(u, v) for one u and
// every v, the m2 sweep of one m1 row of optimize_mapping
// (src/graph-alignment-optimized.c:542-579), with the per-row reductions the
// schedules need (first improving column, best column, count).
//
// Instead of walking the neighbourhoods of u and v for every pair (about 650
// scattered probes per pair at the full-scale workload), a row is computed by
// scattering 2-hop sums into an accumulator acc[v] in shared memory:
//
//   T1  x in out_A(u), weight a:  for (v, b) in B'-in(x):   acc[v] += min(a, b)
//   T2  x in in_A(u),  weight a:  for (v, b) in B'-out(x):  acc[v] += min(a, b)
//   T3  (y, b) in B'-out(u):      for (v, w) in A-in(y):    acc[v] += min(w, b)
//   T4  (y, b) in B'-in(u):       for (v, w) in A-out(y):   acc[v] += min(w, b)
//   C   x in out_A(u) or in_A(u), weight a:  acc[x] += min(a, B(pi u, pi x)) + min(a, B(pi x, pi u))
//       (through shared memory: B's row and column at pi u are written into
//       the empty accumulator and read back, no per-entry lookups)
//
// where B'-out(x) = B-out(pi x) with neighbour ids relabelled into A space
// (maintained by the apply kernel).  Then
//   delta(u, v) = acc[v] - S(u) - S(v) + self-loop terms     (v != u)
// which is exactly score(after swap) - score(before) (see bm_pairs.cu for the
// per-pair form of the same identity).  T1+T2 are the new contributions of u
// moved to pi v, T3+T4 those of v moved to pi u, C repairs the direct edges.
//
// Work per row is the number of 2-hop entries (about 10 per delta at the
// full-scale workload) and every list is read as a coalesced stream.  Load
// balance: first-hop items are cut into units of kSeg second-hop entries; the
// units of a row are dealt round-robin to the CTAs of a thread-block cluster
// (1..8 CTAs per row) and to their warps.  Each CTA scatters into its own
// accumulator; after a cluster barrier each CTA sums one slice of v across the
// cluster's accumulators through distributed shared memory and finalises it.
#include <cooperative_groups.h>

#include <climits>

#include "bm_internal.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int kItemChunk = 1024;  // first-hop items staged per pass
constexpr int kSeg = 512;         // second-hop entries per work unit
constexpr int kMaxCluster = 8;
constexpr int kSideCap = 4096;    // A entries of u whose corrections go through shared memory
constexpr int kMaxUnits = 4096;   // units per chunk with a unit -> item table (else binary search)

struct RowArgs {
    const int32_t* Aout_ptr;
    const int32_t* Ain_ptr;
    const uint32_t* Aout_ent;
    const uint32_t* Ain_ent;
    const int32_t* Bout_ptr;
    const int32_t* Bin_ptr;
    const uint32_t* Bout_ent;  // live: ids in A space
    const uint32_t* Bin_ent;
    const int32_t* selfA;
    const int32_t* selfB;
    int has_self;
    HashView hb;
    const int32_t* pi;
    const int32_t* ov;
    int32_t n;
    const int32_t* rows;
    const int32_t* col_lo;
    int32_t nrows;
    int64_t* full;
    bm_row_result* res;
    int32_t* tab;      // delta table: entry (u, v) at u * tab_ld + v (int32; |delta| < 2^31 checked)
    int64_t tab_ld;
    int32_t tab_sym;   // also write entry (v, u)
    // one-sided mode: only T1 + T2 (u's own edges moved to pi v, everything
    // else fixed), read at the columns cols[0..ncols): colout[r * ncols + j] =
    // G_u(pi cols[j]) - S(u) + self-loop term
    int32_t half;
    const int32_t* cols;
    int32_t ncols;
    int32_t* colout;
};

struct Partial {
    int32_t first_v;
    int32_t best_v;
    int32_t npos;
    int32_t pad;
    long long first_d;
    long long best_d;
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline int32_t nvec_of(int32_t n) { return (n + 1 + 3) & ~3; }

__host__ __device__ inline size_t rows_smem_bytes(int32_t n) {
    return align16(sizeof(int32_t) * (size_t)nvec_of(n))  // acc
           + sizeof(void*) * kItemChunk                  // item base
           + sizeof(int32_t) * kItemChunk * 2            // len, cap
           + sizeof(int32_t) * (kItemChunk + 4)          // unit prefix
           + sizeof(int16_t) * kMaxUnits                 // unit -> item
           + sizeof(int32_t) * 32                        // scan scratch + unit counter
           + sizeof(Partial) * (kMaxCluster + 32);       // cluster partials + warp partials
}

__device__ __forceinline__ void better_first(int32_t& v, long long& d, int32_t v2, long long d2) {
    if (v2 < v) { v = v2; d = d2; }
}

__device__ __forceinline__ void better_best(int32_t& v, long long& d, int32_t v2, long long d2) {
    if (d2 > d || (d2 == d && v2 < v)) { v = v2; d = d2; }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 2) rows_kernel(RowArgs a) {
    constexpr int NW = THREADS / 32;
    constexpr int IPT = kItemChunk / THREADS;  // items built per thread
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const int r = blockIdx.x / CL;
    const int32_t n = a.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const int32_t nv = nvec_of(n);
    int32_t* acc = (int32_t*)smem;
    unsigned char* p = smem + align16(sizeof(int32_t) * (size_t)nv);
    const uint32_t** it_base = (const uint32_t**)p;
    p += sizeof(void*) * kItemChunk;
    int32_t* it_len = (int32_t*)p;
    int32_t* it_cap = it_len + kItemChunk;
    int32_t* it_upre = it_cap + kItemChunk;
    int16_t* unit_item = reinterpret_cast<int16_t*>(it_upre + kItemChunk + 4);
    int32_t* scan_tmp = reinterpret_cast<int32_t*>(unit_item + kMaxUnits);  // [0..15] warp offsets, [31] unit counter
    int* unit_ctr = scan_tmp + 31;
    Partial* parts = (Partial*)(scan_tmp + 32);  // [kMaxCluster] cluster partials
    Partial* wparts = parts + kMaxCluster;       // [32] warp partials

    const int32_t u = (r < a.nrows) ? __ldg(a.rows + r) : 0;
    const bool valid = (u >= 1 && u <= n);

    {
        int4* acc4 = reinterpret_cast<int4*>(acc);
        for (int32_t i = tid; i < (nv >> 2); i += THREADS) acc4[i] = make_int4(0, 0, 0, 0);
    }
    __syncthreads();

    int32_t fu = 0;
    if (valid) {
        fu = __ldg(a.pi + u);
        const int32_t ao = __ldg(a.Aout_ptr + u), d1 = __ldg(a.Aout_ptr + u + 1) - ao;
        const int32_t ai = __ldg(a.Ain_ptr + u), d2 = __ldg(a.Ain_ptr + u + 1) - ai;
        const int32_t bo = __ldg(a.Bout_ptr + fu), d3 = __ldg(a.Bout_ptr + fu + 1) - bo;
        const int32_t bi = __ldg(a.Bin_ptr + fu), d4 = __ldg(a.Bin_ptr + fu + 1) - bi;
        const int32_t F = a.half ? d1 + d2 : d1 + d2 + d3 + d4;
        const int32_t dA = d1 + d2;
        // ---- direct-edge corrections C, for A entries (x, w) of u:
        //   acc[x] += min(w, B(pi u, pi x)) + min(w, B(pi x, pi u)).
        // The B weights at pi u are written packed (out | in << 16) into the
        // still-empty accumulator, read back for u's A entries into a side
        // buffer (the item table's storage), cleared, then added.  Rows with
        // more than kSideCap A entries use hash lookups, spread over the
        // cluster's CTAs.
        const bool side_path = dA <= kSideCap;
        if (!a.half && side_path && crank == 0) {
            int32_t* side = reinterpret_cast<int32_t*>(it_base);
            for (int32_t j = tid; j < d3; j += THREADS) {
                const uint32_t e = __ldg(a.Bout_ent + bo + j);
                if (e) atomicAdd(acc + bm_eid(e), bm_ew(e));
            }
            for (int32_t j = tid; j < d4; j += THREADS) {
                const uint32_t e = __ldg(a.Bin_ent + bi + j);
                if (e) atomicAdd(acc + bm_eid(e), bm_ew(e) << 16);
            }
            __syncthreads();
            for (int32_t j = tid; j < dA; j += THREADS) {
                const uint32_t e = (j < d1) ? __ldg(a.Aout_ent + ao + j) : __ldg(a.Ain_ent + ai + (j - d1));
                int32_t c = 0;
                if (e) {
                    const uint32_t pq = (uint32_t)acc[bm_eid(e)];
                    const int32_t w = bm_ew(e);
                    c = imin(w, (int32_t)(pq & 0xFFFFu)) + imin(w, (int32_t)(pq >> 16));
                }
                side[j] = c;
            }
            __syncthreads();
            for (int32_t j = tid; j < d3; j += THREADS) {
                const uint32_t e = __ldg(a.Bout_ent + bo + j);
                if (e) acc[bm_eid(e)] = 0;
            }
            for (int32_t j = tid; j < d4; j += THREADS) {
                const uint32_t e = __ldg(a.Bin_ent + bi + j);
                if (e) acc[bm_eid(e)] = 0;
            }
            __syncthreads();
            for (int32_t j = tid; j < dA; j += THREADS) {
                const int32_t c = side[j];
                if (c) {
                    const uint32_t e = (j < d1) ? __ldg(a.Aout_ent + ao + j) : __ldg(a.Ain_ent + ai + (j - d1));
                    atomicAdd(acc + bm_eid(e), c);
                }
            }
            __syncthreads();
        }
        for (int32_t c0 = 0; c0 < F; c0 += kItemChunk) {
            const int32_t cnt = min(kItemChunk, F - c0);
            // ---- build this thread's IPT consecutive items (null padding
            // entries give empty items)
            int32_t tsum = 0;
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                const int32_t li = tid * IPT + k;
                const int32_t i = c0 + li;
                if (li >= cnt) break;
                const uint32_t* base = a.Aout_ent;
                int32_t len = 0, cap = 0;
                if (i < d1 + d2) {
                    const uint32_t ent = (i < d1) ? __ldg(a.Aout_ent + ao + i) : __ldg(a.Ain_ent + ai + (i - d1));
                    if (ent != 0) {
                        const int32_t x = bm_eid(ent), w = bm_ew(ent);
                        const int32_t g = __ldg(a.pi + x);
                        if (i < d1) {
                            const int32_t o = __ldg(a.Bin_ptr + g);
                            base = a.Bin_ent + o;
                            len = __ldg(a.Bin_ptr + g + 1) - o;
                        } else {
                            const int32_t o = __ldg(a.Bout_ptr + g);
                            base = a.Bout_ent + o;
                            len = __ldg(a.Bout_ptr + g + 1) - o;
                        }
                        cap = w;
                        if (!a.half && !side_path && (i % CL) == crank) {
                            const int32_t c = imin(w, bm_hash_get(a.hb, fu, g)) + imin(w, bm_hash_get(a.hb, g, fu));
                            if (c) atomicAdd(acc + x, c);
                        }
                    }
                } else {
                    const bool outb = i < d1 + d2 + d3;
                    const uint32_t ent = outb ? __ldg(a.Bout_ent + bo + (i - d1 - d2))
                                              : __ldg(a.Bin_ent + bi + (i - d1 - d2 - d3));
                    if (ent != 0) {
                        const int32_t y = bm_eid(ent);
                        if (outb) {
                            const int32_t o = __ldg(a.Ain_ptr + y);
                            base = a.Ain_ent + o;
                            len = __ldg(a.Ain_ptr + y + 1) - o;
                        } else {
                            const int32_t o = __ldg(a.Aout_ptr + y);
                            base = a.Aout_ent + o;
                            len = __ldg(a.Aout_ptr + y + 1) - o;
                        }
                        cap = bm_ew(ent);
                    }
                }
                it_base[li] = base;
                it_len[li] = len;
                it_cap[li] = cap;
                tsum += (len + kSeg - 1) / kSeg;
            }
            // ---- exclusive scan of units over the block
            int32_t incl = tsum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (lane == 31) scan_tmp[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                int32_t wv = (lane < NW) ? scan_tmp[lane] : 0;
                int32_t wi = wv;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                    if (lane >= o) wi += t;
                }
                if (lane < NW) scan_tmp[lane] = wi - wv;  // exclusive warp offsets
                if (lane == 0) *unit_ctr = 0;
            }
            __syncthreads();
            {
                int32_t run = scan_tmp[warp] + incl - tsum;
#pragma unroll
                for (int k = 0; k < IPT; k++) {
                    const int32_t li = tid * IPT + k;
                    if (li >= cnt) break;
                    it_upre[li] = run;
                    run += (it_len[li] + kSeg - 1) / kSeg;
                }
                if (tid * IPT < cnt && (tid + 1) * IPT >= cnt) it_upre[cnt] = run;
            }
            __syncthreads();
            // ---- unit -> item table (one shared load per unit instead of a
            // binary search), when the chunk's units fit
            const int32_t U = it_upre[cnt];
            const bool table = U <= kMaxUnits;
            if (table) {
#pragma unroll
                for (int k = 0; k < IPT; k++) {
                    const int32_t li = tid * IPT + k;
                    if (li >= cnt) break;
                    for (int32_t x = it_upre[li]; x < it_upre[li + 1]; x++) unit_item[x] = (int16_t)li;
                }
                __syncthreads();
            }
            // ---- scatter: this CTA owns units crank, crank+CL, ...; its warps
            // take them one at a time from a shared counter.  A unit is at most
            // kSeg entries of one list, read as 16-byte vectors (lists are
            // padded to multiples of 4 entries and start 16-byte aligned).  The
            // loop is software-pipelined: the next unit's loads are issued
            // before the current unit's shared-memory atomics.
            auto grab = [&]() -> int32_t {
                int32_t k = 0;
                if (lane == 0) k = atomicAdd(unit_ctr, 1);
                return crank + CL * __shfl_sync(0xffffffffu, k, 0);
            };
            auto load_unit = [&](int32_t unit, uint4 (&q)[kSeg / 128], int32_t& cap) {
                int32_t it;
                if (table) {
                    it = unit_item[unit];
                } else {
                    int32_t lo = 0, hi = cnt;  // last i with it_upre[i] <= unit
                    while (hi - lo > 1) {
                        const int32_t mid = (lo + hi) >> 1;
                        if (it_upre[mid] <= unit) lo = mid; else hi = mid;
                    }
                    it = lo;
                }
                cap = it_cap[it];
                const int32_t s0 = (unit - it_upre[it]) * kSeg;
                const int32_t nq = (min(it_len[it], s0 + kSeg) - s0) >> 2;
                const uint4* b4 = reinterpret_cast<const uint4*>(it_base[it] + s0);
#pragma unroll
                for (int t = 0; t < kSeg / 128; t++) {
                    const int qi = lane + 32 * t;
                    q[t] = (qi < nq) ? __ldg(b4 + qi) : make_uint4(0u, 0u, 0u, 0u);
                }
            };
            uint4 qa[kSeg / 128], qb[kSeg / 128];
            int32_t capa = 0, capb = 0;
            int32_t ua = grab();
            if (ua < U) load_unit(ua, qa, capa);
            while (ua < U) {
                const int32_t ub = grab();
                if (ub < U) load_unit(ub, qb, capb);
#pragma unroll
                for (int t = 0; t < kSeg / 128; t++) {
                    const uint32_t e4[4] = {qa[t].x, qa[t].y, qa[t].z, qa[t].w};
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        if (e4[c] != 0) atomicAdd(acc + bm_eid(e4[c]), imin(capa, bm_ew(e4[c])));
                }
#pragma unroll
                for (int t = 0; t < kSeg / 128; t++) qa[t] = qb[t];
                capa = capb;
                ua = ub;
            }
            __syncthreads();
        }
    }
    cluster.sync();

    // ---- finalise this CTA's slice of v, four consecutive v per thread
    const int32_t groups = nv >> 2;
    const int32_t gslice = (groups + CL - 1) / CL;
    const int32_t glo = crank * gslice;
    const int32_t ghi = min(groups, glo + gslice);
    const int32_t collo = (valid && a.col_lo) ? __ldg(a.col_lo + r) : 1;
    int32_t first_v = INT_MAX, best_v = INT_MAX, npos = 0;
    long long first_d = 0, best_d = LLONG_MIN;
    const long long ovu = valid ? (long long)__ldg(a.ov + u) : 0;
    int32_t sAu = 0, sBu = 0;
    if (valid && a.has_self) { sAu = __ldg(a.selfA + u); sBu = __ldg(a.selfB + fu); }
    int64_t* frow = a.full ? a.full + (size_t)r * ((size_t)n + 1) : nullptr;
    const int4* ov4 = reinterpret_cast<const int4*>(a.ov);
    if (a.cols && valid) {
        // one-sided mode: the requested columns, split over the cluster's CTAs
        for (int32_t j = crank * THREADS + tid; j < a.ncols; j += CL * THREADS) {
            const int32_t v = __ldg(a.cols + j);
            int32_t sum = acc[v];
            for (int q = 1; q < CL; q++) sum += *cluster.map_shared_rank(acc + v, (crank + q) % CL);
            long long c = (long long)sum - ovu;
            if (a.has_self) c += imin(sAu, __ldg(a.selfB + __ldg(a.pi + v))) - imin(sAu, sBu);
            a.colout[(size_t)r * (size_t)a.ncols + j] = (int32_t)c;
        }
    }
    for (int32_t gi = glo + tid; gi < ghi && !a.cols; gi += THREADS) {
        int4 s4 = reinterpret_cast<const int4*>(acc)[gi];
        for (int q = 1; q < CL; q++) {
            const int4 t4 = *reinterpret_cast<const int4*>(cluster.map_shared_rank(acc + 4 * gi, (crank + q) % CL));
            s4.x += t4.x; s4.y += t4.y; s4.z += t4.z; s4.w += t4.w;
        }
        const int4 o4 = __ldg(ov4 + gi);
        const int32_t sv[4] = {s4.x, s4.y, s4.z, s4.w};
        const int32_t ovv[4] = {o4.x, o4.y, o4.z, o4.w};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int32_t v = 4 * gi + c;
            if (v > n) break;
            long long d = 0;
            if (valid && v != u && v >= 1) {
                d = (long long)sv[c] - ovu - (long long)ovv[c];
                if (a.has_self) {
                    const int32_t sAv = __ldg(a.selfA + v), sBv = __ldg(a.selfB + __ldg(a.pi + v));
                    d += imin(sAu, sBv) - imin(sAu, sBu) + imin(sAv, sBu) - imin(sAv, sBv);
                }
                if (v >= collo) {
                    if (d > 0) {
                        npos++;
                        if (v < first_v) { first_v = v; first_d = d; }
                    }
                    better_best(best_v, best_d, v, d);
                }
            }
            if (frow) frow[v] = d;
            if (a.tab && valid) {
                a.tab[(size_t)u * (size_t)a.tab_ld + (size_t)v] = (int32_t)d;
                if (a.tab_sym && v >= 1 && v != u) a.tab[(size_t)v * (size_t)a.tab_ld + (size_t)u] = (int32_t)d;
            }
        }
    }
    if (a.res) {
        // warp, then block reduction
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const int32_t fv2 = __shfl_xor_sync(0xffffffffu, first_v, o);
            const long long fd2 = __shfl_xor_sync(0xffffffffu, first_d, o);
            const int32_t bv2 = __shfl_xor_sync(0xffffffffu, best_v, o);
            const long long bd2 = __shfl_xor_sync(0xffffffffu, best_d, o);
            npos += __shfl_xor_sync(0xffffffffu, npos, o);
            better_first(first_v, first_d, fv2, fd2);
            better_best(best_v, best_d, bv2, bd2);
        }
        if (lane == 0) wparts[warp] = Partial{first_v, best_v, npos, 0, first_d, best_d};
        __syncthreads();
        if (tid == 0) {
            Partial t = wparts[0];
            for (int w = 1; w < NW; w++) {
                better_first(t.first_v, t.first_d, wparts[w].first_v, wparts[w].first_d);
                better_best(t.best_v, t.best_d, wparts[w].best_v, wparts[w].best_d);
                t.npos += wparts[w].npos;
            }
            *cluster.map_shared_rank(parts + crank, 0) = t;
        }
    }
    cluster.sync();
    if (a.res && crank == 0 && tid == 0) {
        Partial t = parts[0];
        for (int q = 1; q < CL; q++) {
            better_first(t.first_v, t.first_d, parts[q].first_v, parts[q].first_d);
            better_best(t.best_v, t.best_d, parts[q].best_v, parts[q].best_d);
            t.npos += parts[q].npos;
        }
        bm_row_result out;
        out.row = u;
        out.first_pos = (t.first_v == INT_MAX) ? 0 : t.first_v;
        out.first_delta = (t.first_v == INT_MAX) ? 0 : t.first_d;
        out.best = (t.best_v == INT_MAX) ? 0 : t.best_v;
        out.best_delta = (t.best_v == INT_MAX) ? 0 : t.best_d;
        out.npos = t.npos;
        a.res[r] = out;
    }
}

template <int THREADS>
bm_status launch_rows_t(bm_ctx* ctx, const RowArgs& args, int cl, size_t smem) {
    static bool configured[64] = {false};
    auto kern = rows_kernel<THREADS>;
    if (!configured[ctx->device & 63]) {
        BM_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem_optin));
        configured[ctx->device & 63] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(args.nrows * cl), 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BM_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, args));
    BM_LAUNCH_CHECK(ctx, "rows_kernel");
    return BM_OK;
}

template <int THREADS>
bm_status max_clusters_t(bm_ctx* ctx, int cl, size_t smem, int* out) {
    auto kern = rows_kernel<THREADS>;
    BM_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem_optin));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(cl * 64), 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BM_CUDA(ctx, cudaOccupancyMaxActiveClusters(out, kern, &cfg));
    return BM_OK;
}

}  // namespace

bm_status bm_rows_smem_check(bm_ctx* ctx) {
    const size_t smem = rows_smem_bytes(ctx->n);
    if (smem > ctx->smem_optin)
        return bm_fail(ctx, BM_UNSUPPORTED, "row kernel needs %zu B of shared memory for n=%d; the device allows %zu",
                       smem, ctx->n, ctx->smem_optin);
    // Accumulator bound: |acc| <= 4 * max weighted degree of A must fit int32.
    if (ctx->g[0].max_wdeg * 4 >= (int64_t)INT_MAX)
        return bm_fail(ctx, BM_UNSUPPORTED, "weighted degree %lld too large for the row kernel's int32 accumulators",
                       (long long)ctx->g[0].max_wdeg);
    return BM_OK;
}

bm_status bm_launch_rows(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows, int64_t* d_full,
                         bm_row_result* d_res) {
    return bm_launch_rows_ex(ctx, d_rows, d_col_lo, nrows, d_full, d_res, nullptr, 0, 0);
}

bm_status bm_launch_rows_ex(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                            int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym) {
    return bm_launch_rows_gen(ctx, d_rows, d_col_lo, nrows, d_full, d_res, d_tab, tab_ld, tab_sym, nullptr, 0, nullptr);
}

bm_status bm_launch_rows_gen(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                             int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym,
                             const int32_t* d_cols, int32_t ncols, int32_t* d_colout) {
    if (nrows <= 0) return BM_OK;
    bm_status st = bm_rows_smem_check(ctx);
    if (st != BM_OK) return st;
    const size_t smem = rows_smem_bytes(ctx->n);
    const DevGraph& A = ctx->g[0];
    const DevGraph& B = ctx->g[1];
    RowArgs args;
    args.Aout_ptr = A.out_ptr;
    args.Ain_ptr = A.in_ptr;
    args.Aout_ent = A.out_ent;
    args.Ain_ent = A.in_ent;
    args.Bout_ptr = B.out_ptr;
    args.Bin_ptr = B.in_ptr;
    args.Bout_ent = B.out_ent;
    args.Bin_ent = B.in_ent;
    args.selfA = A.self_w;
    args.selfB = B.self_w;
    args.has_self = A.has_self && B.has_self;
    args.hb = hview(B);
    args.pi = ctx->pi;
    args.ov = ctx->ov;
    args.n = ctx->n;
    args.rows = d_rows;
    args.col_lo = d_col_lo;
    args.full = d_full;
    args.res = d_res;
    args.tab = d_tab;
    args.tab_ld = tab_ld;
    args.tab_sym = tab_sym;
    args.half = d_cols ? 1 : 0;
    args.cols = d_cols;
    args.ncols = ncols;
    args.colout = d_colout;
    int cl = ctx->row_ctas;
    if (cl == 0) {
        // two CTAs fit per SM: the largest cluster size with nrows*cl <= 2*SMs
        cl = 1;
        while (cl < kMaxCluster && (int64_t)nrows * cl * 2 <= (int64_t)ctx->num_sms * 2) cl *= 2;
    }
    // grid.x is limited to 2^31-1; chunk very long row lists
    const int32_t max_rows_per_launch = 1 << 20;
    for (int32_t r0 = 0; r0 < nrows; r0 += max_rows_per_launch) {
        RowArgs ar = args;
        ar.nrows = min(max_rows_per_launch, nrows - r0);
        ar.rows = d_rows + r0;
        ar.col_lo = d_col_lo ? d_col_lo + r0 : nullptr;
        ar.full = d_full ? d_full + (size_t)r0 * ((size_t)ctx->n + 1) : nullptr;
        ar.res = d_res ? d_res + r0 : nullptr;
        ar.colout = d_colout ? d_colout + (size_t)r0 * (size_t)ncols : nullptr;
        st = (ctx->row_threads == 256) ? launch_rows_t<256>(ctx, ar, cl, smem) : launch_rows_t<512>(ctx, ar, cl, smem);
        if (st != BM_OK) return st;
    }
    return BM_OK;
}

extern "C" bm_status bm_delta_rows_dev(bm_ctx* ctx, const int32_t* d_rows, int32_t nrows, int64_t* d_deltas) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && (!d_rows || !d_deltas))) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    return bm_launch_rows(ctx, d_rows, nullptr, nrows, d_deltas, nullptr);
}

extern "C" bm_status bm_rows_best_dev(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                                      bm_row_result* d_out) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && (!d_rows || !d_out))) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    return bm_launch_rows(ctx, d_rows, d_col_lo, nrows, nullptr, d_out);
}

static bm_status check_rows(bm_ctx* ctx, const int32_t* rows, int32_t nrows) {
    for (int32_t i = 0; i < nrows; i++)
        if (rows[i] < 1 || rows[i] > ctx->n)
            return bm_fail(ctx, BM_INVALID_ARG, "row %d = %d outside 1..%d", i, rows[i], ctx->n);
    return BM_OK;
}

extern "C" bm_status bm_delta_rows(bm_ctx* ctx, const int32_t* rows, int32_t nrows, int64_t* deltas) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && (!rows || !deltas))) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    if (nrows == 0) return BM_OK;
    if ((s = check_rows(ctx, rows, nrows)) != BM_OK) return s;
    const size_t in_al = (sizeof(int32_t) * (size_t)nrows + 255) & ~(size_t)255;
    const size_t out_bytes = sizeof(int64_t) * (size_t)nrows * ((size_t)ctx->n + 1);
    if ((s = bm_stage(ctx, in_al + out_bytes)) != BM_OK) return s;
    int32_t* d_rows = (int32_t*)ctx->stage;
    int64_t* d_out = (int64_t*)((char*)ctx->stage + in_al);
    BM_CUDA(ctx, cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_rows(ctx, d_rows, nullptr, nrows, d_out, nullptr)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(deltas, d_out, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_rows_best(bm_ctx* ctx, const int32_t* rows, const int32_t* col_lo, int32_t nrows,
                                  bm_row_result* out) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && (!rows || !out))) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    if (nrows == 0) return BM_OK;
    if ((s = check_rows(ctx, rows, nrows)) != BM_OK) return s;
    const size_t rb = (sizeof(int32_t) * (size_t)nrows + 255) & ~(size_t)255;
    const size_t ob = sizeof(bm_row_result) * (size_t)nrows;
    if ((s = bm_stage(ctx, 2 * rb + ob)) != BM_OK) return s;
    int32_t* d_rows = (int32_t*)ctx->stage;
    int32_t* d_col = (int32_t*)((char*)ctx->stage + rb);
    bm_row_result* d_out = (bm_row_result*)((char*)ctx->stage + 2 * rb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if (col_lo)
        BM_CUDA(ctx, cudaMemcpyAsync(d_col, col_lo, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_rows(ctx, d_rows, col_lo ? d_col : nullptr, nrows, nullptr, d_out)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_rows_max_active_clusters(bm_ctx* ctx, int32_t ctas_per_row, int32_t threads, int32_t* out) {
    if (!ctx || !out) return BM_INVALID_ARG;
    const size_t smem = rows_smem_bytes(ctx->n > 0 ? ctx->n : 1);
    int v = 0;
    bm_status s = (threads == 256) ? max_clusters_t<256>(ctx, ctas_per_row, smem, &v)
                                   : max_clusters_t<512>(ctx, ctas_per_row, smem, &v);
    *out = v;
    return s;
}
