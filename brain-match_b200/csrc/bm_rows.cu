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
// balance: the second-hop lists of a chunk of first-hop items form one stream
// of 16-byte quads; the warps of all CTAs of a thread-block cluster (1..8 CTAs
// per row) claim ranges of kGrain quads from a counter in the cluster's first
// CTA, and each lane walks its quads with a cursor on the list they fall in.
// Each CTA scatters into its own accumulator; after a cluster barrier each CTA
// sums one slice of v across the cluster's accumulators through distributed
// shared memory and finalises it.
//
// Split rows.  A heavy row (a hub: up to 19 chunks of 1,024 first-hop items
// and 7M 2-hop entries) is bound by its chunk count and its cluster's width.
// When the caller holds the rows on the host, the launcher plans slots there
// from a per-row work estimate kept beside the mapping: row r gets c_r
// consecutive cluster slots, and slot j of c_r takes the first-hop items j,
// j + c_r, j + 2 c_r, ...  Split rows meet in global memory: each slot
// cluster writes its slice sums, the last slot to arrive (a self-resetting
// counter) finalises the slice, and the last slice to arrive writes the row's
// reduction.  Nothing waits on another cluster.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "bm_internal.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int kItemChunk = 1024;  // first-hop items staged per pass
constexpr int kGrain = 512;       // quads (4 second-hop entries each) per claimed range
constexpr int kMaxCluster = 8;
constexpr int kFinBatch = 2;     // groups of four columns a thread finalises per pass
constexpr int kSideCap = 4096;    // A entries of u whose corrections go through shared memory
constexpr int kItemCost = 32;     // work estimate: entries charged per first-hop item

struct Partial {
    int32_t first_v;
    int32_t best_v;
    int32_t npos;
    int32_t pad;
    long long first_d;
    long long best_d;
};

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
    int has_self;  // self-loop terms needed (A and B have self-loops; A alone in reference-delta mode)
    int refcpu;    // reference-delta semantics (selects the REFCPU instantiation)
    HashView hb;
    const int32_t* pi;
    const int32_t* ov;
    const int4* ximg;  // per A vertex x, the bounds of B's lists at pi x
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
    // split rows: slots[s] = {row, part, parts, 0} of cluster slot s (the
    // parts of a row are consecutive slots); null = one slot per row
    int32_t nslots;
    const int4* slots;
    int4* spart;        // [nslots][nvec / 4] slice sums of each slot cluster
    unsigned* scnt;     // [nrows][kMaxCluster] slot arrivals per slice (self-resetting)
    unsigned* rcnt;     // [nrows] slice arrivals per row (self-resetting)
    Partial* rpart;     // [nrows][kMaxCluster] slice reductions
    // tiered launches: slot s takes the row whose work estimate ranks
    // rank_lo + s among the launch's rows (descending, ties by position);
    // null = slot s takes row s
    const int32_t* rank_work;
    int32_t rank_lo;
    // results in host memory polled by the caller: each row id is written
    // last, after a system-scope fence, as the row's completion flag
    int32_t host_res;
};

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

__host__ __device__ inline int32_t nvec_of(int32_t n) { return (n + 1 + 3) & ~3; }

__host__ __device__ inline size_t rows_smem_bytes(int32_t n) {
    return align16(sizeof(int32_t) * ((size_t)nvec_of(n) + 32))  // acc + one sink slot per lane
           + sizeof(void*) * kItemChunk                  // item base
           + sizeof(int32_t) * kItemChunk * 2            // len, cap
           + sizeof(int32_t) * (kItemChunk + 4)          // quad prefix
           + sizeof(int32_t) * 32                        // scan scratch + range counters
           + sizeof(Partial) * (kMaxCluster + 32)        // cluster partials + warp partials
           + sizeof(int32_t) * 4;                        // split plan of this slot
}

__device__ __forceinline__ void better_first(int32_t& v, long long& d, int32_t v2, long long d2) {
    if (v2 < v) { v = v2; d = d2; }
}

__device__ __forceinline__ void better_best(int32_t& v, long long& d, int32_t v2, long long d2) {
    if (d2 > d || (d2 == d && v2 < v)) { v = v2; d = d2; }
}

__device__ __forceinline__ Partial ld_partial(const Partial* p) {
    const int4* q = reinterpret_cast<const int4*>(p);
    const int4 x = __ldcg(q), y = __ldcg(q + 1);
    Partial t;
    t.first_v = x.x; t.best_v = x.y; t.npos = x.z; t.pad = x.w;
    t.first_d = ((long long)(unsigned)y.y << 32) | (unsigned)y.x;
    t.best_d = ((long long)(unsigned)y.w << 32) | (unsigned)y.z;
    return t;
}

__device__ __forceinline__ bm_row_result row_result(int32_t u, const Partial& t) {
    bm_row_result out;
    out.row = u;
    out.first_pos = (t.first_v == INT_MAX) ? 0 : t.first_v;
    out.first_delta = (t.first_v == INT_MAX) ? 0 : t.first_d;
    out.best = (t.best_v == INT_MAX) ? 0 : t.best_v;
    out.best_delta = (t.best_v == INT_MAX) ? 0 : t.best_d;
    out.npos = t.npos;
    return out;
}

// REFCPU: reference-delta semantics (a separate instantiation, so the exact
// one carries none of its code or registers)
template <int THREADS, bool REFCPU>
__global__ void __launch_bounds__(THREADS, 2) rows_kernel(RowArgs a) {
    constexpr int NW = THREADS / 32;
    constexpr int IPT = kItemChunk / THREADS;  // items built per thread
    extern __shared__ __align__(16) unsigned char smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const int slot = blockIdx.x / CL;
    const int32_t n = a.n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    const int32_t nv = nvec_of(n);
    int32_t* acc = (int32_t*)smem;
    unsigned char* p = smem + align16(sizeof(int32_t) * ((size_t)nv + 32));
    const uint32_t** it_base = (const uint32_t**)p;
    p += sizeof(void*) * kItemChunk;
    int32_t* it_len = (int32_t*)p;
    int32_t* it_cap = it_len + kItemChunk;
    int32_t* it_upre = it_cap + kItemChunk;  // quad prefix of the items
    int32_t* scan_tmp = it_upre + kItemChunk + 4;  // [0..15] warp offsets, [29..30] range counters
    Partial* parts = (Partial*)(scan_tmp + 32);  // [kMaxCluster] cluster partials
    Partial* wparts = parts + kMaxCluster;       // [32] warp partials
    int32_t* plan = reinterpret_cast<int32_t*>(wparts + 32);  // row, part, parts, last-arrival flag

    // zeroing the accumulator and prefetching the per-vertex arrays; in rank
    // mode this overlaps the loads of the rows' work estimates
    auto zero_and_prefetch = [&]() {
        {
            int4* acc4 = reinterpret_cast<int4*>(acc);
            for (int32_t i = tid; i < (nv >> 2); i += THREADS) acc4[i] = make_int4(0, 0, 0, 0);
        }
        {
            // the per-vertex arrays every row reads at random (pi, S(v), A's two
            // CSR pointer arrays, the image list bounds) are prefetched into L2
            // once per launch, one 128-byte line per thread spread over the grid,
            // so the dependent loads of the first-hop staging and the finalise
            // pass hit L2.  The image bounds (four int32 per vertex) count as four
            // segments of `lines` lines.
            const int32_t lines = (int32_t)((sizeof(int32_t) * ((size_t)nv + 4) + 127) / 128);
            const int32_t total = 8 * lines;
            for (int32_t j = tid * (int32_t)gridDim.x + (int32_t)blockIdx.x; j < total; j += THREADS * (int32_t)gridDim.x) {
                const int32_t k = j / lines, l = j - k * lines;
                const int32_t seg = k < 4 ? 0 : (k - 4) * lines * 32;  // ints before this segment of the bounds
                const int32_t* arr = k == 0 ? a.pi : k == 1 ? a.ov : k == 2 ? a.Aout_ptr : k == 3 ? a.Ain_ptr
                                   : reinterpret_cast<const int32_t*>(a.ximg) + seg;
                const int32_t lim = (k == 0) ? n + 1 : (k == 1) ? nv : (k < 4) ? n + 2 : 4 * (n + 1) - seg;
                const int32_t e = l * 32;
                if (e < lim) asm volatile("prefetch.global.L2 [%0];" :: "l"(arr + e));
            }
        }
    };
    // plan[0..2]: row, part of the row, parts of the row.  Read back from
    // shared memory where needed (short register live ranges).
    if (a.rank_work) {
        // rank the launch's rows (at most kItemChunk) by their work estimate;
        // it_len is free until the first item chunk is staged
        int32_t* wr = it_len;
        if (tid == 0) { plan[0] = -1; plan[1] = 0; plan[2] = 1; }
        int32_t w0 = -1;
        if (tid < a.nrows) {
            const int32_t u0 = __ldg(a.rows + tid);
            w0 = (u0 >= 1 && u0 <= n) ? __ldg(a.rank_work + u0) : -1;
        }
        zero_and_prefetch();
        if (tid < a.nrows) wr[tid] = w0;
        for (int32_t j = tid + THREADS; j < a.nrows; j += THREADS) {
            const int32_t uj = __ldg(a.rows + j);
            wr[j] = (uj >= 1 && uj <= n) ? __ldg(a.rank_work + uj) : -1;
        }
        __syncthreads();
        const int32_t want = a.rank_lo + slot;
        for (int32_t j = tid; j < a.nrows; j += THREADS) {
            const int32_t wj = wr[j];
            int32_t rk = 0;
            for (int32_t k = 0; k < a.nrows; k++) {
                const int32_t wk = wr[k];
                rk += (wk > wj || (wk == wj && k < j)) ? 1 : 0;
            }
            if (rk == want) plan[0] = j;
        }
    } else {
        if (tid == 0) {
            if (a.slots) {
                const int4 d = __ldg(a.slots + slot);
                plan[0] = d.x; plan[1] = d.y; plan[2] = d.z;
            } else {
                plan[0] = slot; plan[1] = 0; plan[2] = 1;
            }
        }
        zero_and_prefetch();
    }
    auto P = [&](int k) -> int32_t { return *reinterpret_cast<volatile int32_t*>(plan + k); };
    // Quad ranges are shared out across the whole cluster from counters in
    // CTA 0's shared memory (one per chunk parity), so a CTA that shares its
    // SM or also runs the corrections simply takes fewer ranges.
    int* cctr = scan_tmp + 29;
    if (crank == 0 && tid == 0) { cctr[0] = 0; cctr[1] = 0; }
    cluster.sync();
    const int32_t u = (P(0) < 0 || P(0) >= a.nrows) ? 0 : __ldg(a.rows + P(0));
    const bool valid = (u >= 1 && u <= n);

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
        if (!a.half && side_path && crank == 0 && P(1) == 0) {
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
        // a split row's slot j of c takes the first-hop items j, j + c, ...
        // (j and c are read back from shared memory where they are used)
        const int32_t Fs = (F - P(1) + P(2) - 1) / P(2);
        for (int32_t c0 = 0; c0 < Fs; c0 += kItemChunk) {
            const int32_t cnt = min(kItemChunk, Fs - c0);
            const int ci = c0 / kItemChunk;
            if (crank == 0 && tid == 0) cctr[(ci + 1) & 1] = 0;  // next chunk's counter (unused until the chunk barrier)
            // 32-bit shared::cluster address of CTA 0's counter for this chunk
            uint32_t gctr;
            asm volatile("mapa.shared::cluster.u32 %0, %1, 0;"
                         : "=r"(gctr) : "r"((uint32_t)__cvta_generic_to_shared(cctr + (ci & 1))));
            // ---- build this thread's IPT consecutive items (null padding
            // entries give empty items)
            int32_t tsum = 0;
#pragma unroll
            for (int k = 0; k < IPT; k++) {
                const int32_t li = tid * IPT + k;
                const int32_t i = P(1) + P(2) * (c0 + li);
                if (li >= cnt) break;
                const uint32_t* base = a.Aout_ent;
                int32_t len = 0, cap = 0;
                if (i < d1 + d2) {
                    const uint32_t ent = (i < d1) ? __ldg(a.Aout_ent + ao + i) : __ldg(a.Ain_ent + ai + (i - d1));
                    if (ent != 0) {
                        // the list bounds at pi x come from the per-vertex
                        // image record: one load instead of pi x, then its bounds
                        const int32_t x = bm_eid(ent), w = bm_ew(ent);
                        const int4 xb = __ldg(a.ximg + x);
                        if (i < d1) {
                            base = a.Bin_ent + xb.x;
                            len = xb.y - xb.x;
                        } else {
                            base = a.Bout_ent + xb.z;
                            len = xb.w - xb.z;
                        }
                        cap = w;
                        if (!a.half && !side_path && (i % CL) == crank) {
                            const int32_t g = __ldg(a.pi + x);
                            const int32_t c = imin(w, bm_hash_get_small(a.hb, fu, g)) + imin(w, bm_hash_get_small(a.hb, g, fu));
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
                tsum += len >> 2;  // quads (lists are padded to multiples of 4 entries)
            }
            // ---- exclusive scan of quads over the block
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
            }
            __syncthreads();
            {
                int32_t run = scan_tmp[warp] + incl - tsum;
#pragma unroll
                for (int k = 0; k < IPT; k++) {
                    const int32_t li = tid * IPT + k;
                    if (li >= cnt) break;
                    it_upre[li] = run;
                    run += it_len[li] >> 2;
                }
                if (tid * IPT < cnt && (tid + 1) * IPT >= cnt) it_upre[cnt] = run;
            }
            __syncthreads();
            // ---- scatter: the chunk's second-hop lists form one stream of
            // Q quads (16-byte vectors; lists are padded to multiples of four
            // entries and start 16-byte aligned).  Warps of every CTA of the
            // cluster claim ranges of kGrain quads from the cluster counter;
            // lane l of a warp handles quads q0 + l + 32 j of its range, and
            // keeps a cursor on the item (list) its quads fall in, which only
            // moves forward.  Two quads per lane are loaded while the two
            // before them are scattered.  Quads past the range are sinks with
            // cap 0 (each lane its own slot past the accumulator).
            const int32_t Q = it_upre[cnt];
            auto claim = [&]() -> int32_t {
                int32_t k = 0;
                if (lane == 0) asm volatile("atom.shared::cluster.add.u32 %0, [%1], 1;" : "=r"(k) : "r"(gctr));
                return k;
            };
            auto claimed = [&](int32_t k) -> int32_t { return __shfl_sync(0xffffffffu, k, 0); };
            int32_t it = 0, st = 0, en = 0, capv = 0;
            const uint4* bp = nullptr;
            const uint32_t sink = (uint32_t)(nv + lane);
            auto fetch = [&](int32_t qq, int32_t qhi, uint4& out, int32_t& capo) {
                if (qq < qhi) {
                    while (qq >= en) {
                        ++it;
                        st = en;
                        en = it_upre[it + 1];
                        bp = reinterpret_cast<const uint4*>(it_base[it]);
                        capv = it_cap[it];
                    }
                    out = __ldg(bp + (qq - st));
                    capo = capv;
                } else {
                    out = make_uint4(sink, sink, sink, sink);
                    capo = 0;
                }
            };
            auto scatter4 = [&](const uint4& q4, int32_t cw) {
                const uint32_t e4[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
                for (int c = 0; c < 4; c++) atomicAdd(acc + bm_eid(e4[c]), imin(cw, bm_ew(e4[c])));
            };
            int32_t g = claimed(claim());
            while ((int64_t)g * kGrain < Q) {
                const int32_t qlo = g * kGrain, qhi = min(Q, qlo + kGrain);
                const int32_t knext = claim();
                // cursor: the item holding quad qlo + lane (binary search), set
                // one item back so the first fetch loads its pointer and cap
                {
                    int32_t lo = 0, hi = cnt;  // last i with it_upre[i] <= q
                    const int32_t q = min(qlo + lane, qhi - 1);
                    while (hi - lo > 1) {
                        const int32_t mid = (lo + hi) >> 1;
                        if (it_upre[mid] <= q) lo = mid; else hi = mid;
                    }
                    it = lo - 1;
                    en = it_upre[lo];
                    st = en;
                }
                uint4 qa[2], qb[2];
                int32_t ca[2], cb[2];
                int32_t q = qlo + lane;
                fetch(q, qhi, qa[0], ca[0]);
                fetch(q + 32, qhi, qa[1], ca[1]);
                for (; q < qhi; q += 128) {
                    fetch(q + 64, qhi, qb[0], cb[0]);
                    fetch(q + 96, qhi, qb[1], cb[1]);
                    scatter4(qa[0], ca[0]);
                    scatter4(qa[1], ca[1]);
                    if (q + 64 >= qhi) break;
                    fetch(q + 128, qhi, qa[0], ca[0]);
                    fetch(q + 160, qhi, qa[1], ca[1]);
                    scatter4(qb[0], cb[0]);
                    scatter4(qb[1], cb[1]);
                }
                g = claimed(knext);
            }
            if (c0 + kItemChunk < Fs) cluster.sync(); else __syncthreads();
        }
    }
    if (REFCPU && valid && crank == 0 && P(1) == 0) {
        // reference-delta semantics: calculate_swap_delta meets the self-loop
        // of u and of the partner v in its out- and in-edge loops
        // (src/graph-alignment-optimized.c:327-388) and compares the images
        // after the swap, B(pi u, pi v) and B(pi v, pi u).  Those are the
        // entries of B's row and column at pi u, so each adds
        // min(s_u, b) + min(s_v, b) at its v; the old-image terms are added
        // per column in the finalise pass.
        const int32_t fu = __ldg(a.pi + u), su = __ldg(a.selfA + u);
        const int32_t bo = __ldg(a.Bout_ptr + fu), d3 = __ldg(a.Bout_ptr + fu + 1) - bo;
        const int32_t bi = __ldg(a.Bin_ptr + fu), d4 = __ldg(a.Bin_ptr + fu + 1) - bi;
        for (int32_t j = tid; j < d3 + d4; j += THREADS) {
            const uint32_t e = (j < d3) ? __ldg(a.Bout_ent + bo + j) : __ldg(a.Bin_ent + bi + (j - d3));
            if (e) {
                const int32_t v = bm_eid(e), b = bm_ew(e);
                const int32_t c = imin(su, b) + imin(__ldg(a.selfA + v), b);
                if (c) atomicAdd(acc + v, c);
            }
        }
    }
    cluster.sync();

    // ---- finalise this CTA's slice of v, four consecutive v per thread
    const int32_t groups = nv >> 2;
    const int32_t gslice = (groups + CL - 1) / CL;
    const int32_t glo = crank * gslice;
    const int32_t ghi = min(groups, glo + gslice);
    const int r = P(0), sj = P(1), sc = P(2);
    const bool idle = r < 0 || r >= a.nrows;
    const int32_t collo = (valid && a.col_lo) ? __ldg(a.col_lo + r) : 1;
    int32_t first_v = INT_MAX, best_v = INT_MAX, npos = 0;
    long long first_d = 0, best_d = LLONG_MIN;
    const long long ovu = valid ? (long long)__ldg(a.ov + u) : 0;
    int32_t sAu = 0, sBu = 0;
    if (valid && a.has_self) { sAu = __ldg(a.selfA + u); sBu = __ldg(a.selfB + fu); }
    int64_t* frow = (a.full && !idle) ? a.full + (size_t)r * ((size_t)n + 1) : nullptr;
    const int4* ov4 = reinterpret_cast<const int4*>(a.ov);
    auto cluster_sum = [&](int32_t gi) -> int4 {
        int4 s4 = reinterpret_cast<const int4*>(acc)[gi];
        for (int q = 1; q < CL; q++) {
            const int rk = crank + q < CL ? crank + q : crank + q - CL;  // (crank + q) mod CL
            const int4 t4 = *reinterpret_cast<const int4*>(cluster.map_shared_rank(acc + 4 * gi, rk));
            s4.x += t4.x; s4.y += t4.y; s4.z += t4.z; s4.w += t4.w;
        }
        return s4;
    };
    // split row: publish this slot's slice sums; the last slot to arrive for
    // the slice finalises it from all the row's slot sums
    bool fin = !idle;
    if (sc > 1) {
        int4* mine = a.spart + (size_t)slot * (size_t)groups;
        for (int32_t gi = glo + tid; gi < ghi; gi += THREADS) mine[gi] = cluster_sum(gi);
        __threadfence();
        __syncthreads();
        if (tid == 0) {
            const unsigned old = atomicInc(a.scnt + (size_t)r * kMaxCluster + crank, (unsigned)(sc - 1));
            plan[3] = (old == (unsigned)(sc - 1)) ? 1 : 0;
        }
        __syncthreads();
        fin = plan[3] != 0;
        if (fin) __threadfence();
    }
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
    auto finish_group = [&](int32_t gi, const int4 s4) {
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
                    if constexpr (REFCPU)
                        d += -2 * imin(sAu, sBu) - 2 * imin(sAv, sBv);
                    else
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
    };
    if (fin && !a.cols) {
        if (sc > 1) {
            for (int32_t gi = glo + tid; gi < ghi; gi += THREADS) {
                int4 s4 = make_int4(0, 0, 0, 0);
                const int4* base = a.spart + (size_t)(slot - sj) * (size_t)groups + gi;
                for (int q = 0; q < sc; q++) {
                    const int4 t4 = __ldcg(base + (size_t)q * (size_t)groups);
                    s4.x += t4.x; s4.y += t4.y; s4.z += t4.z; s4.w += t4.w;
                }
                finish_group(gi, s4);
            }
        } else {
            // a thread's groups (kFinBatch per pass) are read from the other
            // CTAs' accumulators together, so the remote loads overlap
            for (int32_t g0 = glo + tid; g0 < ghi; g0 += kFinBatch * THREADS) {
                int4 sb[kFinBatch];
#pragma unroll
                for (int b = 0; b < kFinBatch; b++) {
                    const int32_t gi = g0 + b * THREADS;
                    sb[b] = gi < ghi ? reinterpret_cast<const int4*>(acc)[gi] : make_int4(0, 0, 0, 0);
                }
#pragma unroll
                for (int q = 1; q < kMaxCluster; q++) {
                    if (q >= CL) break;
                    const int rk = crank + q < CL ? crank + q : crank + q - CL;  // (crank + q) mod CL
#pragma unroll
                    for (int b = 0; b < kFinBatch; b++) {
                        const int32_t gi = g0 + b * THREADS;
                        if (gi < ghi) {
                            const int4 t4 = *reinterpret_cast<const int4*>(cluster.map_shared_rank(acc + 4 * gi, rk));
                            sb[b].x += t4.x; sb[b].y += t4.y; sb[b].z += t4.z; sb[b].w += t4.w;
                        }
                    }
                }
#pragma unroll
                for (int b = 0; b < kFinBatch; b++) {
                    const int32_t gi = g0 + b * THREADS;
                    if (gi < ghi) finish_group(gi, sb[b]);
                }
            }
        }
    }
    if (a.res && fin) {
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
            if (sc > 1) {
                // split row: the last slice to arrive combines the slices
                Partial* rp = a.rpart + (size_t)r * kMaxCluster;
                rp[crank] = t;
                __threadfence();
                const unsigned old = atomicInc(a.rcnt + r, (unsigned)(CL - 1));
                if (old == (unsigned)(CL - 1)) {
                    __threadfence();
                    Partial c = ld_partial(rp);
                    for (int q = 1; q < CL; q++) {
                        const Partial pq = ld_partial(rp + q);
                        better_first(c.first_v, c.first_d, pq.first_v, pq.first_d);
                        better_best(c.best_v, c.best_d, pq.best_v, pq.best_d);
                        c.npos += pq.npos;
                    }
                    a.res[r] = row_result(u, c);
                }
            } else {
                *cluster.map_shared_rank(parts + crank, 0) = t;
            }
        }
    }
    cluster.sync();
    if (a.res && !idle && sc == 1 && crank == 0 && tid == 0) {
        Partial t = parts[0];
        for (int q = 1; q < CL; q++) {
            better_first(t.first_v, t.first_d, parts[q].first_v, parts[q].first_d);
            better_best(t.best_v, t.best_d, parts[q].best_v, parts[q].best_d);
            t.npos += parts[q].npos;
        }
        const bm_row_result o = row_result(u, t);
        if (a.host_res) {
            bm_row_result* d = a.res + r;
            d->first_pos = o.first_pos;
            d->first_delta = o.first_delta;
            d->best = o.best;
            d->best_delta = o.best_delta;
            d->npos = o.npos;
            __threadfence_system();
            *reinterpret_cast<volatile int32_t*>(&d->row) = o.row;
        } else {
            a.res[r] = o;
        }
    }
}

// Work estimate of every row u (what the split plan weighs): the 2-hop
// entries T1..T4 of u plus kItemCost per first-hop item.  One warp per row.
constexpr int kWorkThreads = 256;
__global__ void __launch_bounds__(kWorkThreads) row_work_kernel(RowArgs a, int32_t* __restrict__ work) {
    const int32_t u = (int32_t)((blockIdx.x * (size_t)kWorkThreads + threadIdx.x) >> 5) + 1;
    const int lane = threadIdx.x & 31;
    if (u > a.n) return;
    const int32_t fu = __ldg(a.pi + u);
    long long s = 0;
    auto walk = [&](const int32_t* ptr, const uint32_t* ent, int32_t i, bool map, const int32_t* ptr2) {
        const int32_t o = __ldg(ptr + i), e = __ldg(ptr + i + 1);
        for (int32_t j = o + lane; j < e; j += 32) {
            const uint32_t x = __ldg(ent + j);
            if (!x) continue;
            const int32_t y = map ? __ldg(a.pi + bm_eid(x)) : bm_eid(x);
            s += kItemCost + (__ldg(ptr2 + y + 1) - __ldg(ptr2 + y));
        }
    };
    walk(a.Aout_ptr, a.Aout_ent, u, true, a.Bin_ptr);   // T1: B-in lists of pi x
    walk(a.Ain_ptr, a.Ain_ent, u, true, a.Bout_ptr);    // T2: B-out lists of pi x
    walk(a.Bout_ptr, a.Bout_ent, fu, false, a.Ain_ptr); // T3: A-in lists of y
    walk(a.Bin_ptr, a.Bin_ent, fu, false, a.Aout_ptr);  // T4: A-out lists of y
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) work[u] = (int32_t)min(s, (long long)INT_MAX);
}

template <int THREADS, bool REFCPU>
bm_status launch_rows_t(bm_ctx* ctx, const RowArgs& args, int cl, size_t smem, cudaStream_t stream) {
    static bool configured[64] = {false};
    auto kern = rows_kernel<THREADS, REFCPU>;
    if (!configured[ctx->device & 63]) {
        BM_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->smem_optin));
        configured[ctx->device & 63] = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(args.nslots * cl), 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    // clusters placed for load balance rather than spread: with the two
    // cluster sizes of a tiered launch resident together, spreading left
    // clusters for a second wave well below the resident-cluster count
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeClusterSchedulingPolicyPreference;
    attr[1].val.clusterSchedulingPolicyPreference = cudaClusterSchedulingPolicyLoadBalancing;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    BM_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, args));
    BM_LAUNCH_CHECK(ctx, "rows_kernel");
    return BM_OK;
}

template <int THREADS>
bm_status max_clusters_t(bm_ctx* ctx, int cl, size_t smem, int* out) {
    auto kern = rows_kernel<THREADS, false>;
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

bm_status bm_rows_prepare(bm_ctx* ctx) {
    // split-row buffers, sized for n and at most split_slots_max slots
    const int32_t smax = 2 * ctx->num_sms;
    if (ctx->split_n != ctx->n || ctx->split_slots_max != smax) {
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        bm_cuda_free(ctx->rwork); bm_cuda_free(ctx->spart); bm_cuda_free(ctx->scnt); bm_cuda_free(ctx->rpart); bm_cuda_free(ctx->slots);
        ctx->rwork = nullptr; ctx->spart = nullptr; ctx->scnt = nullptr; ctx->rpart = nullptr; ctx->rcnt = nullptr;
        ctx->slots = nullptr;
        ctx->split_n = 0;
        BM_CUDA(ctx, bm_cuda_malloc(&ctx->rwork, sizeof(int32_t) * (size_t)ctx->nvec));
        BM_CUDA(ctx, bm_cuda_malloc(&ctx->spart, sizeof(int32_t) * (size_t)ctx->nvec * (size_t)smax));
        const size_t cnt_bytes = sizeof(unsigned) * (size_t)smax * (kMaxCluster + 1);
        BM_CUDA(ctx, bm_cuda_malloc(&ctx->scnt, cnt_bytes));
        ctx->rcnt = ctx->scnt + (size_t)smax * kMaxCluster;
        BM_CUDA(ctx, bm_cuda_malloc(&ctx->rpart, sizeof(Partial) * (size_t)smax * kMaxCluster));
        BM_CUDA(ctx, bm_cuda_malloc(&ctx->slots, sizeof(int4) * (size_t)smax));
        if (!ctx->h_slots) BM_CUDA(ctx, bm_cuda_host_alloc((void**)&ctx->h_slots, sizeof(int4) * (size_t)2 * ctx->num_sms,
                                                      cudaHostAllocDefault));
        if (!ctx->slots_ev) BM_CUDA(ctx, cudaEventCreateWithFlags(&ctx->slots_ev, cudaEventDisableTiming));
        BM_CUDA(ctx, cudaMemsetAsync(ctx->scnt, 0, cnt_bytes, ctx->stream));
        ctx->split_n = ctx->n;
        ctx->split_slots_max = smax;
        for (int& c : ctx->split_active) c = 0;
    }
    return bm_rows_refresh_work(ctx);
}

bm_status bm_rows_refresh_work(bm_ctx* ctx) {
    if (!ctx->rwork || !ctx->pi || ctx->n <= 0) return BM_OK;
    const DevGraph& A = ctx->g[0];
    const DevGraph& B = ctx->g[1];
    RowArgs args = {};
    args.Aout_ptr = A.out_ptr;
    args.Ain_ptr = A.in_ptr;
    args.Aout_ent = A.out_ent;
    args.Ain_ent = A.in_ent;
    args.Bout_ptr = B.out_ptr;
    args.Bin_ptr = B.in_ptr;
    args.Bout_ent = B.out_ent;
    args.Bin_ent = B.in_ent;
    args.pi = ctx->pi;
    args.ximg = ctx->ximg;
    args.n = ctx->n;
    const size_t threads = (size_t)ctx->n * 32;
    const unsigned blocks = (unsigned)((threads + kWorkThreads - 1) / kWorkThreads);
    row_work_kernel<<<blocks, kWorkThreads, 0, ctx->stream>>>(args, ctx->rwork);
    BM_LAUNCH_CHECK(ctx, "row_work_kernel");
    // the plan is made on the host, from rows the host holds
    ctx->h_rwork.resize((size_t)ctx->n + 1);
    BM_CUDA(ctx, cudaMemcpyAsync(ctx->h_rwork.data(), ctx->rwork, sizeof(int32_t) * ((size_t)ctx->n + 1),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

namespace {

// Split plan for host-held rows: row i weighs w_i = max(1, rwork[rows[i]]);
// with L the smallest integer (at least min_work) such that sum_i c_i <= S,
// c_i = min(kMaxParts, ceil(w_i / L)), row i gets c_i consecutive slots
// {i, j, c_i}.  Returns the slots used (sum_i c_i).  kMinSlotWork (the
// automatic setting's min_work) keeps rows whose scatter would take less than
// the global-memory merge unsplit.
constexpr int kMaxParts = 16;
constexpr int64_t kMinSlotWork = 300000;

int32_t host_split_plan(const bm_ctx* ctx, const int32_t* h_rows, int32_t nrows, int32_t S, int64_t min_work,
                        std::vector<int4>& out) {
    std::vector<int64_t> w((size_t)nrows);
    int64_t wmax = 1;
    for (int32_t i = 0; i < nrows; i++) {
        const int32_t u = h_rows[i];
        w[(size_t)i] = (u >= 1 && u <= ctx->n) ? std::max<int64_t>(1, ctx->h_rwork[(size_t)u]) : 1;
        wmax = std::max(wmax, w[(size_t)i]);
    }
    auto parts = [&](int64_t wi, int64_t L) { return (int32_t)std::min<int64_t>(kMaxParts, (wi + L - 1) / L); };
    auto f = [&](int64_t L) {
        int64_t s = 0;
        for (int64_t wi : w) s += parts(wi, L);
        return s;
    };
    int64_t lo = 1, hi = wmax;  // f(wmax) = nrows <= S
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (f(mid) <= S) hi = mid; else lo = mid + 1;
    }
    lo = std::max(lo, min_work);
    out.clear();
    for (int32_t i = 0; i < nrows; i++) {
        const int32_t c = parts(w[(size_t)i], lo);
        for (int32_t j = 0; j < c; j++) out.push_back(make_int4(i, j, c, 0));
    }
    return (int32_t)out.size();
}

// Resident clusters of cl CTAs for the current n (occupancy query, cached
// per thread count and cluster size).
bm_status resident_clusters(bm_ctx* ctx, int cl, size_t smem, int* out) {
    int& v = ctx->split_active[(ctx->row_threads == 256 ? 0 : 1) * (kMaxCluster + 1) + cl];
    if (v == 0) {
        const bm_status st = (ctx->row_threads == 256) ? max_clusters_t<256>(ctx, cl, smem, &v)
                                                      : max_clusters_t<512>(ctx, cl, smem, &v);
        if (st != BM_OK) return st;
        if (v <= 0) v = -1;
    }
    *out = v;
    return BM_OK;
}

// Rows of a launch of nrows rows in cl-CTA clusters that go to the 2 cl tier.
// A 2 cl cluster takes the room of two cl clusters in a GPC, so the H rows
// and the other nrows - H fit at once while nrows + H stays below the
// resident cl clusters (one cluster of margin) and H within the resident
// 2 cl clusters; capped by the caller's setting.  Measured at 57 rows in 4-CTA
// clusters (71 resident, so H = 13): H = 6 +8 %, H = 13-15 +12 % over one
// launch; H = 17 puts clusters in a second wave.
int32_t tier_rows(bm_ctx* ctx, int32_t nrows, int cl, size_t smem, bm_status* st) {
    int m1 = 0, m2 = 0;
    if ((*st = resident_clusters(ctx, cl, smem, &m1)) != BM_OK) return 0;
    if ((*st = resident_clusters(ctx, 2 * cl, smem, &m2)) != BM_OK) return 0;
    if (m1 <= 0 || m2 <= 0) return 0;
    int64_t h = std::min<int64_t>({(int64_t)nrows, (int64_t)m1 - nrows - 1, (int64_t)m2});
    if (ctx->row_tiers > 0) h = std::min<int64_t>(h, ctx->row_tiers);
    return (int32_t)std::max<int64_t>(h, 0);
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
                         bm_row_result* d_res, const int32_t* h_rows) {
    return bm_launch_rows_ex(ctx, d_rows, d_col_lo, nrows, d_full, d_res, nullptr, 0, 0, h_rows);
}

bm_status bm_launch_rows_ex(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                            int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym,
                            const int32_t* h_rows) {
    return bm_launch_rows_gen(ctx, d_rows, d_col_lo, nrows, d_full, d_res, d_tab, tab_ld, tab_sym, nullptr, 0, nullptr,
                              h_rows);
}

bm_status bm_launch_rows_gen(bm_ctx* ctx, const int32_t* d_rows, const int32_t* d_col_lo, int32_t nrows,
                             int64_t* d_full, bm_row_result* d_res, int32_t* d_tab, int64_t tab_ld, int32_t tab_sym,
                             const int32_t* d_cols, int32_t ncols, int32_t* d_colout, const int32_t* h_rows) {
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
    // one-sided gains (d_cols) are not swaps: they keep the exact rule
    args.refcpu = (ctx->semantics == BM_SEMANTICS_REF_CPU && !d_cols) ? 1 : 0;
    args.has_self = args.refcpu ? A.has_self : (A.has_self && B.has_self);
    args.hb = hview(B);
    args.pi = ctx->pi;
    args.ximg = ctx->ximg;
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
    args.nslots = nrows;
    args.slots = nullptr;
    args.spart = (int4*)ctx->spart;
    args.scnt = ctx->scnt;
    args.rcnt = ctx->rcnt;
    args.rpart = (Partial*)ctx->rpart;
    if (h_rows && ctx->row_split >= 0 && !d_cols && ctx->slots && nrows < ctx->split_slots_max &&
        ctx->h_rwork.size() == (size_t)ctx->n + 1) {
        // slots: the resident clusters of this shape when they are at least
        // four times the rows (automatic: launches of a few rows, where most
        // of the GPU would wait on the heaviest row), or the set count
        int32_t S = ctx->row_split;
        if (S == 0) {
            int& cached = ctx->split_active[(ctx->row_threads == 256 ? 0 : 1) * (kMaxCluster + 1) + cl];
            if (cached == 0) {
                const size_t sm = rows_smem_bytes(ctx->n);
                st = (ctx->row_threads == 256) ? max_clusters_t<256>(ctx, cl, sm, &cached)
                                               : max_clusters_t<512>(ctx, cl, sm, &cached);
                if (st != BM_OK) return st;
                if (cached <= 0) cached = -1;
            }
            S = (cached >= 4 * nrows) ? cached : 0;
        }
        S = min(S, ctx->split_slots_max);
        if (S > nrows) {
            std::vector<int4> plan;
            // a set slot count splits whatever it can (min_work 1); the
            // automatic one only rows worth a global-memory merge
            const int32_t used = host_split_plan(ctx, h_rows, nrows, S, ctx->row_split ? 1 : kMinSlotWork, plan);
            if (used > nrows) {
                // the pinned table is rewritten only after the previous upload ran
                BM_CUDA(ctx, cudaEventSynchronize(ctx->slots_ev));
                std::copy(plan.begin(), plan.end(), ctx->h_slots);
                BM_CUDA(ctx, cudaMemcpyAsync(ctx->slots, ctx->h_slots, sizeof(int4) * (size_t)used,
                                             cudaMemcpyHostToDevice, ctx->stream));
                BM_CUDA(ctx, cudaEventRecord(ctx->slots_ev, ctx->stream));
                args.slots = ctx->slots;
                args.nslots = used;
            }
        }
    }
    auto launch = [&](const RowArgs& x, int c, cudaStream_t strm) -> bm_status {
        if (x.refcpu)
            return (ctx->row_threads == 256) ? launch_rows_t<256, true>(ctx, x, c, smem, strm)
                                             : launch_rows_t<512, true>(ctx, x, c, smem, strm);
        return (ctx->row_threads == 256) ? launch_rows_t<256, false>(ctx, x, c, smem, strm)
                                         : launch_rows_t<512, false>(ctx, x, c, smem, strm);
    };
    args.host_res = ctx->row_host_res ? 1 : 0;
    args.rank_work = nullptr;
    args.rank_lo = 0;
    // Tiers: when the launch leaves resident CTA slots free, the H rows with
    // the largest work estimate (ranked on the device) get clusters of 2 cl
    // in a launch on a second stream, concurrent with the cl-CTA launch of
    // the others.  A launch waits on its heaviest row, and a row's scatter
    // rate grows with its CTAs.  The two launches together must stay
    // resident (tier_rows): a cluster left for a second wave costs more than
    // the tier saves.
    const int32_t H = (args.slots || ctx->row_ctas != 0 || ctx->row_tiers < 0 || cl >= kMaxCluster || !ctx->rwork ||
                       nrows > kItemChunk)
                          ? 0 : tier_rows(ctx, nrows, cl, smem, &st);
    if (st != BM_OK) return st;
    if (H > 0) {
        if (!ctx->row_side) {
            BM_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->row_side, cudaStreamNonBlocking));
            BM_CUDA(ctx, cudaEventCreateWithFlags(&ctx->row_fork, cudaEventDisableTiming));
            BM_CUDA(ctx, cudaEventCreateWithFlags(&ctx->row_join, cudaEventDisableTiming));
        }
        RowArgs hv = args, lt = args;
        hv.nrows = lt.nrows = nrows;
        hv.rank_work = lt.rank_work = ctx->rwork;
        hv.rank_lo = 0;
        hv.nslots = H;
        lt.rank_lo = H;
        lt.nslots = nrows - H;
        BM_CUDA(ctx, cudaEventRecord(ctx->row_fork, ctx->stream));
        BM_CUDA(ctx, cudaStreamWaitEvent(ctx->row_side, ctx->row_fork, 0));
        if ((st = launch(hv, 2 * cl, ctx->row_side)) != BM_OK) return st;
        BM_CUDA(ctx, cudaEventRecord(ctx->row_join, ctx->row_side));
        if (H < nrows && (st = launch(lt, cl, ctx->stream)) != BM_OK) return st;
        BM_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->row_join, 0));
        return BM_OK;
    }
    // grid.x is limited to 2^31-1; chunk very long row lists
    const int32_t max_rows_per_launch = 1 << 20;
    for (int32_t r0 = 0; r0 < nrows; r0 += max_rows_per_launch) {
        RowArgs ar = args;
        ar.nrows = min(max_rows_per_launch, nrows - r0);
        if (!args.slots) ar.nslots = ar.nrows;  // one slot per row (a split launch is never chunked)
        ar.rows = d_rows + r0;
        ar.col_lo = d_col_lo ? d_col_lo + r0 : nullptr;
        ar.full = d_full ? d_full + (size_t)r0 * ((size_t)ctx->n + 1) : nullptr;
        ar.res = d_res ? d_res + r0 : nullptr;
        ar.colout = d_colout ? d_colout + (size_t)r0 * (size_t)ncols : nullptr;
        if ((st = launch(ar, cl, ctx->stream)) != BM_OK) return st;
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
    if ((s = bm_launch_rows(ctx, d_rows, nullptr, nrows, d_out, nullptr, rows)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(deltas, d_out, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

namespace {

// Whether a host-row launch of nrows rows would take a split plan (then the
// plan, made per call from the rows, keeps it off the graph path).  An
// unqueried occupancy counts as yes: the plain path queries it.
bool split_would_apply(const bm_ctx* ctx, int32_t nrows) {
    if (ctx->row_split < 0 || !ctx->slots || nrows >= ctx->split_slots_max || ctx->h_rwork.size() != (size_t)ctx->n + 1)
        return false;
    if (ctx->row_split > 0) return true;
    int cl = ctx->row_ctas;
    if (cl == 0) {
        cl = 1;
        while (cl < kMaxCluster && (int64_t)nrows * cl * 2 <= (int64_t)ctx->num_sms * 2) cl *= 2;
    }
    const int cached = ctx->split_active[(ctx->row_threads == 256 ? 0 : 1) * (kMaxCluster + 1) + cl];
    return cached == 0 || cached >= 4 * nrows;
}

constexpr int32_t kRowGraphMaxRows = 4096;
constexpr int64_t kRowPollMax = 20000000;  // result polls before waiting on the stream (about a second)

// bm_rows_best without column bounds as a replayed CUDA graph: the rows are
// copied (CPU) into pinned staging, the graph copies them in and runs the row
// launches (tiers included), which write the row results straight into pinned
// staging (zero copy: 32 bytes a row over the host link, no copy-out step),
// from which they are copied (CPU) to the caller.  Each result's row id
// (1..n, every row having been checked) is written last, after a
// system-scope fence, so the call polls the ids (reset to 0 before the
// launch) and returns once all have arrived, without waiting for the stream
// to drain; the graph's last steps complete in stream order before any later
// work of the context.  The polling is bounded, then the stream is waited
// for (a failed launch reports its error there).  The first call of a row
// count runs plainly and then captures the graph; a change of row count,
// staging buffers, graphs, semantics or row settings captures it again.
bm_status rows_best_graph(bm_ctx* ctx, const int32_t* rows, int32_t nrows, bm_row_result* out) {
    const size_t rb = (sizeof(int32_t) * (size_t)nrows + 255) & ~(size_t)255;
    const size_t ob = sizeof(bm_row_result) * (size_t)nrows;
    bm_status s = bm_stage(ctx, rb + ob);
    if (s != BM_OK) return s;
    if ((s = bm_hstage(ctx, rb + ob)) != BM_OK) return s;
    bm_ctx::RowGraph& G = ctx->row_graph;
    const bool hit = G.exec && G.nrows == nrows && G.n == ctx->n && G.semantics == ctx->semantics &&
                     G.row_tiers == ctx->row_tiers && G.row_ctas == ctx->row_ctas && G.row_threads == ctx->row_threads &&
                     G.stage == ctx->stage && G.hstage == ctx->hstage && G.pi == ctx->pi && G.ov == ctx->ov &&
                     G.ximg == ctx->ximg &&
                     G.a == ctx->g[0].out_ptr && G.b == ctx->g[1].out_ptr;
    int32_t* d_rows = (int32_t*)ctx->stage;
    bm_row_result* d_out = (bm_row_result*)((char*)ctx->stage + rb);
    int32_t* h_in = (int32_t*)ctx->hstage;
    bm_row_result* h_out = (bm_row_result*)((char*)ctx->hstage + rb);
    if (hit) {
        std::memcpy(h_in, rows, sizeof(int32_t) * (size_t)nrows);
        for (int32_t r = 0; r < nrows; r++) h_out[r].row = 0;
        BM_CUDA(ctx, cudaGraphLaunch(G.exec, ctx->stream));
        auto arrived = [&]() {
            for (int32_t r = 0; r < nrows; r++)
                if (*reinterpret_cast<volatile int32_t*>(&h_out[r].row) == 0) return false;
            return true;
        };
        bool done = false;
        for (int64_t it = 0; !done; it++) {
            done = arrived();
            // every 1024 polls: stop polling once the stream has finished or
            // failed, or after about a second
            if (!done && (it & 1023) == 1023 &&
                (cudaStreamQuery(ctx->stream) != cudaErrorNotReady || it > (int64_t)kRowPollMax))
                break;
        }
        if (!done) {
            BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (!arrived()) return bm_fail(ctx, BM_CUDA_ERROR, "row results missing after the row graph finished");
        }
        ctx->launches += G.launches;
        std::memcpy(out, h_out, ob);
        return BM_OK;
    }
    if (G.exec) {
        cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
    }
    // this call runs plainly (it also sets the kernel attributes and the
    // occupancy figures the launches read), then the graph is captured
    BM_CUDA(ctx, cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_rows(ctx, d_rows, nullptr, nrows, nullptr, d_out, nullptr)) != BM_OK) return s;
    BM_CUDA(ctx, cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const int64_t l0 = ctx->launches;
    cudaGraph_t graph = nullptr;
    BM_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t c1 = cudaMemcpyAsync(d_rows, h_in, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream);
    ctx->row_host_res = true;
    const bm_status ls = c1 == cudaSuccess ? bm_launch_rows(ctx, d_rows, nullptr, nrows, nullptr, h_out, nullptr) : BM_OK;
    ctx->row_host_res = false;
    const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    const int64_t captured = ctx->launches - l0;
    ctx->launches = l0;
    if (ls != BM_OK || c1 != cudaSuccess || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (ls != BM_OK) return ls;
        return bm_cuda_fail(ctx, c1 != cudaSuccess ? c1 : ce, "row graph capture");
    }
    const cudaError_t ie = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        G.exec = nullptr;
        return bm_cuda_fail(ctx, ie, "row graph instantiation");
    }
    G.launches = captured;
    G.nrows = nrows;
    G.n = ctx->n;
    G.semantics = ctx->semantics;
    G.row_tiers = ctx->row_tiers;
    G.row_ctas = ctx->row_ctas;
    G.row_threads = ctx->row_threads;
    G.stage = ctx->stage;
    G.hstage = ctx->hstage;
    G.pi = ctx->pi;
    G.ov = ctx->ov;
    G.ximg = ctx->ximg;
    G.a = ctx->g[0].out_ptr;
    G.b = ctx->g[1].out_ptr;
    return BM_OK;
}

}  // namespace

extern "C" bm_status bm_rows_best(bm_ctx* ctx, const int32_t* rows, const int32_t* col_lo, int32_t nrows,
                                  bm_row_result* out) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if (nrows < 0 || (nrows > 0 && (!rows || !out))) return bm_fail(ctx, BM_INVALID_ARG, "bad row buffers");
    if (nrows == 0) return BM_OK;
    if ((s = check_rows(ctx, rows, nrows)) != BM_OK) return s;
    if (!col_lo && nrows <= kRowGraphMaxRows && !split_would_apply(ctx, nrows)) return rows_best_graph(ctx, rows, nrows, out);
    const size_t rb = (sizeof(int32_t) * (size_t)nrows + 255) & ~(size_t)255;
    const size_t ob = sizeof(bm_row_result) * (size_t)nrows;
    if ((s = bm_stage(ctx, 2 * rb + ob)) != BM_OK) return s;
    int32_t* d_rows = (int32_t*)ctx->stage;
    int32_t* d_col = (int32_t*)((char*)ctx->stage + rb);
    bm_row_result* d_out = (bm_row_result*)((char*)ctx->stage + 2 * rb);
    BM_CUDA(ctx, cudaMemcpyAsync(d_rows, rows, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if (col_lo)
        BM_CUDA(ctx, cudaMemcpyAsync(d_col, col_lo, sizeof(int32_t) * (size_t)nrows, cudaMemcpyHostToDevice, ctx->stream));
    if ((s = bm_launch_rows(ctx, d_rows, col_lo ? d_col : nullptr, nrows, nullptr, d_out, rows)) != BM_OK) return s;
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
