// bm_api.cu — context lifecycle, graph upload, mapping state and device
// utilities of the C ABI declared in include/bm_cuda.h.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bm_internal.cuh"

// ------------------------------------------------------------------ errors

bm_status bm_fail(bm_ctx* ctx, bm_status s, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return s;
}

bm_status bm_cuda_fail(bm_ctx* ctx, cudaError_t e, const char* what) {
    bm_status s = (e == cudaErrorMemoryAllocation) ? BM_OOM : BM_CUDA_ERROR;
    return bm_fail(ctx, s, "%s: %s", what, cudaGetErrorString(e));
}

extern "C" const char* bm_status_str(bm_status s) {
    switch (s) {
    case BM_OK: return "ok";
    case BM_INVALID_ARG: return "invalid argument";
    case BM_OOM: return "out of memory";
    case BM_CUDA_ERROR: return "CUDA error";
    case BM_TIMEOUT: return "budget exhausted";
    case BM_PARITY_FAIL: return "self-check failed";
    case BM_UNSUPPORTED: return "unsupported by this kernel";
    case BM_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char* bm_ctx_last_error(const bm_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

// --------------------------------------------------------------- lifecycle

static void free_graph(DevGraph& g) {
    cudaFree(g.out_ptr); cudaFree(g.in_ptr);
    cudaFree(g.out_ent); cudaFree(g.in_ent);
    cudaFree(g.self_w);
    cudaFree(g.out_twin); cudaFree(g.in_twin);
    cudaFree(g.out_ent0); cudaFree(g.in_ent0);
    cudaFree(g.hash);
    g = DevGraph();
}

extern "C" bm_status bm_ctx_create(int device, bm_ctx** out) {
    if (!out) return BM_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return BM_NO_DEVICE;
    }
    if (device < 0 || device >= count) return BM_NO_DEVICE;
    bm_ctx* ctx = new (std::nothrow) bm_ctx();
    if (!ctx) return BM_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return BM_CUDA_ERROR; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete ctx; return BM_CUDA_ERROR; }
    if (prop.major < 10) {
        delete ctx;
        return BM_UNSUPPORTED;  // built for sm_100a only
    }
    ctx->num_sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return BM_CUDA_ERROR;
    }
    if (cudaMalloc(&ctx->d_score, 64) != cudaSuccess) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return BM_OOM;
    }
    *out = ctx;
    return BM_OK;
}

extern "C" void bm_ctx_destroy(bm_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_graph(ctx->g[0]);
    free_graph(ctx->g[1]);
    cudaFree(ctx->pi); cudaFree(ctx->pinv); cudaFree(ctx->ov);
    cudaFree(ctx->d_score);
    cudaFree(ctx->stage);
    cudaFree(ctx->flush_buf);
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" void* bm_ctx_stream(bm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

extern "C" bm_status bm_sync(bm_ctx* ctx) {
    if (!ctx) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BM_OK;
}

extern "C" int64_t bm_launch_count(const bm_ctx* ctx) { return ctx ? ctx->launches : 0; }

bm_status bm_stage(bm_ctx* ctx, size_t bytes) {
    if (ctx->stage_bytes >= bytes) return BM_OK;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    size_t sz = bytes < (1u << 20) ? (1u << 20) : bytes;
    BM_CUDA(ctx, cudaMalloc(&ctx->stage, sz));
    ctx->stage_bytes = sz;
    return BM_OK;
}

bm_status bm_hstage(bm_ctx* ctx, size_t bytes) {
    if (ctx->hstage_bytes >= bytes) return BM_OK;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    ctx->hstage = nullptr;
    ctx->hstage_bytes = 0;
    size_t sz = bytes < (1u << 20) ? (1u << 20) : bytes;
    BM_CUDA(ctx, cudaMallocHost(&ctx->hstage, sz));
    ctx->hstage_bytes = sz;
    return BM_OK;
}

bm_status bm_require_mapped(bm_ctx* ctx) {
    if (!ctx) return BM_INVALID_ARG;
    if (!ctx->g[0].loaded || !ctx->g[1].loaded)
        return bm_fail(ctx, BM_INVALID_ARG, "both graphs must be set first");
    if (!ctx->mapped) return bm_fail(ctx, BM_INVALID_ARG, "mapping not set");
    return BM_OK;
}

// ------------------------------------------------------------ graph upload

template <typename T>
static bm_status upload(bm_ctx* ctx, T** d, const T* h, size_t count) {
    size_t bytes = sizeof(T) * (count > 0 ? count : 1);
    BM_CUDA(ctx, cudaMalloc((void**)d, bytes));
    if (count > 0) BM_CUDA(ctx, cudaMemcpy(*d, h, sizeof(T) * count, cudaMemcpyHostToDevice));
    return BM_OK;
}

#define BM_TRY(x)                          \
    do {                                   \
        bm_status _s = (x);                \
        if (_s != BM_OK) return _s;        \
    } while (0)

extern "C" bm_status bm_set_graph(bm_ctx* ctx, int side, int32_t n, int64_t m, const int32_t* src,
                                  const int32_t* dst, const int32_t* w) {
    if (!ctx) return BM_INVALID_ARG;
    if (side != BM_SIDE_A && side != BM_SIDE_B) return bm_fail(ctx, BM_INVALID_ARG, "side must be 0 (A) or 1 (B)");
    if (n < 1 || n > BM_MAX_N) return bm_fail(ctx, BM_INVALID_ARG, "n=%d outside 1..%d", n, BM_MAX_N);
    if (m < 0 || m >= (int64_t)0x7fffffff) return bm_fail(ctx, BM_INVALID_ARG, "edge count %lld out of range", (long long)m);
    if (m > 0 && (!src || !dst || !w)) return bm_fail(ctx, BM_INVALID_ARG, "null edge arrays");
    int other = 1 - side;
    if (ctx->g[other].loaded && ctx->g[other].n != n)
        return bm_fail(ctx, BM_INVALID_ARG, "n=%d differs from the other graph's n=%d", n, ctx->g[other].n);
    for (int64_t e = 0; e < m; e++) {
        if (src[e] < 1 || src[e] > n || dst[e] < 1 || dst[e] > n)
            return bm_fail(ctx, BM_INVALID_ARG, "edge %lld: id outside 1..%d", (long long)e, n);
        if (w[e] < 0 || w[e] > BM_MAX_W)
            return bm_fail(ctx, BM_INVALID_ARG, "edge %lld: weight %d outside 0..%d", (long long)e, w[e], BM_MAX_W);
    }
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

    // Which entries survive: B keeps the last weight of a duplicated edge
    // (the matrix store of add_edge); A keeps every entry.  Zero weights
    // never contribute to min(w, .) and are dropped.
    std::vector<int32_t> self((size_t)n + 1, 0);
    std::vector<char> keep((size_t)m, 1);
    int has_self = 0;
    std::vector<unsigned long long> htab;
    int hlog2 = 0;
    if (side == BM_SIDE_B) {
        int64_t cap = 1024;
        hlog2 = 10;
        while (cap * 3 < (m + 1) * 4) { cap <<= 1; hlog2++; }
        // map key -> last edge index, in a temporary table
        std::vector<unsigned long long> kk((size_t)cap, BM_HASH_EMPTY);
        std::vector<int64_t> vi((size_t)cap, -1);
        unsigned long long np1 = (unsigned long long)n + 1;
        for (int64_t e = 0; e < m; e++) {
            unsigned long long key = (unsigned long long)src[e] * np1 + (unsigned long long)dst[e];
            unsigned long long s = bm_hash_slot0(key, hlog2);
            while (kk[s] != BM_HASH_EMPTY && kk[s] != key) s = (s + 1) & (unsigned long long)(cap - 1);
            if (kk[s] == key) keep[(size_t)vi[s]] = 0;
            kk[s] = key;
            vi[s] = e;
        }
        htab.assign((size_t)cap, BM_HASH_EMPTY);
        for (int64_t e = 0; e < m; e++) {
            if (!keep[e]) continue;
            if (w[e] == 0) { keep[e] = 0; continue; }
            if (src[e] == dst[e]) { self[src[e]] = w[e]; has_self = 1; keep[e] = 0; continue; }
            unsigned long long key = (unsigned long long)src[e] * np1 + (unsigned long long)dst[e];
            unsigned long long s = bm_hash_slot0(key, hlog2);
            while (htab[s] != BM_HASH_EMPTY) s = (s + 1) & (unsigned long long)(cap - 1);
            htab[s] = (key << 16) | (unsigned long long)w[e];
        }
    } else {
        for (int64_t e = 0; e < m; e++) {
            if (w[e] == 0) { keep[e] = 0; continue; }
            if (src[e] == dst[e]) {
                if (self[src[e]] != 0)
                    return bm_fail(ctx, BM_INVALID_ARG, "vertex %d has more than one self-loop in graph A", src[e]);
                self[src[e]] = w[e];
                has_self = 1;
                keep[e] = 0;
            }
        }
    }

    // CSR (out) sorted by (src, dst) and CSC (in) sorted by (dst, src), by
    // two stable counting sorts each.
    std::vector<int32_t> optr((size_t)n + 2, 0), iptr((size_t)n + 2, 0);
    int64_t mk = 0;
    for (int64_t e = 0; e < m; e++)
        if (keep[e]) { optr[(size_t)src[e] + 1]++; iptr[(size_t)dst[e] + 1]++; mk++; }
    for (int32_t i = 1; i <= n + 1; i++) { optr[i] += optr[i - 1]; iptr[i] += iptr[i - 1]; }
    std::vector<int64_t> by_dst((size_t)mk), by_src((size_t)mk);
    {
        std::vector<int32_t> f(iptr.begin(), iptr.end() - 1);
        for (int64_t e = 0; e < m; e++) if (keep[e]) by_dst[(size_t)f[dst[e]]++] = e;
        std::vector<int32_t> g(optr.begin(), optr.end() - 1);
        for (int64_t e = 0; e < m; e++) if (keep[e]) by_src[(size_t)g[src[e]]++] = e;
    }
    std::vector<uint32_t> oent((size_t)mk), ient((size_t)mk);
    std::vector<int32_t> opos_of((size_t)(side == BM_SIDE_B ? m : 0));
    std::vector<int32_t> ipos_of((size_t)(side == BM_SIDE_B ? m : 0));
    {
        // out: iterate edges in dst order, place by src (stable) -> rows sorted by dst
        std::vector<int32_t> f(optr.begin(), optr.end() - 1);
        for (int64_t k = 0; k < mk; k++) {
            int64_t e = by_dst[(size_t)k];
            int32_t p = f[src[e]]++;
            oent[(size_t)p] = bm_pack((uint32_t)dst[e], (uint32_t)w[e]);
            if (side == BM_SIDE_B) opos_of[(size_t)e] = p;
        }
        std::vector<int32_t> g(iptr.begin(), iptr.end() - 1);
        for (int64_t k = 0; k < mk; k++) {
            int64_t e = by_src[(size_t)k];
            int32_t p = g[dst[e]]++;
            ient[(size_t)p] = bm_pack((uint32_t)src[e], (uint32_t)w[e]);
            if (side == BM_SIDE_B) ipos_of[(size_t)e] = p;
        }
    }
    int32_t max_deg = 0;
    int64_t max_wdeg = 0;
    {
        std::vector<int64_t> wd((size_t)n + 1, 0);
        for (int64_t e = 0; e < m; e++)
            if (keep[e]) { wd[src[e]] += w[e]; wd[dst[e]] += w[e]; }
        for (int32_t v = 1; v <= n; v++) {
            int32_t d = (optr[v + 1] - optr[v]) + (iptr[v + 1] - iptr[v]);
            if (d > max_deg) max_deg = d;
            if (wd[v] + self[v] > max_wdeg) max_wdeg = wd[v] + self[v];
        }
    }

    if (side == BM_SIDE_A && max_wdeg >= ((int64_t)1 << 29))
        return bm_fail(ctx, BM_INVALID_ARG, "weighted degree %lld of graph A is 2^29 or more", (long long)max_wdeg);

    // Replacing a graph drops the mapping state.
    ctx->mapped = false;
    free_graph(ctx->g[side]);
    DevGraph& G = ctx->g[side];
    G.n = n;
    G.m = mk;
    BM_TRY(upload(ctx, &G.out_ptr, optr.data(), optr.size()));
    BM_TRY(upload(ctx, &G.in_ptr, iptr.data(), iptr.size()));
    BM_TRY(upload(ctx, &G.out_ent, oent.data(), oent.size()));
    BM_TRY(upload(ctx, &G.in_ent, ient.data(), ient.size()));
    BM_TRY(upload(ctx, &G.self_w, self.data(), self.size()));
    if (side == BM_SIDE_B) {
        std::vector<int32_t> otw((size_t)mk), itw((size_t)mk);
        for (int64_t e = 0; e < m; e++)
            if (keep[e]) { otw[(size_t)opos_of[e]] = ipos_of[e]; itw[(size_t)ipos_of[e]] = opos_of[e]; }
        BM_TRY(upload(ctx, &G.out_twin, otw.data(), otw.size()));
        BM_TRY(upload(ctx, &G.in_twin, itw.data(), itw.size()));
        BM_TRY(upload(ctx, &G.out_ent0, oent.data(), oent.size()));
        BM_TRY(upload(ctx, &G.in_ent0, ient.data(), ient.size()));
        BM_TRY(upload(ctx, &G.hash, htab.data(), htab.size()));
        G.hash_log2 = hlog2;
    }
    if (side == BM_SIDE_A) {
        ctx->hA_optr = optr;
        ctx->hA_iptr = iptr;
        ctx->hA_oent = oent;
        ctx->hA_ient = ient;
    }
    G.max_deg = max_deg;
    G.max_wdeg = max_wdeg;
    G.has_self = has_self;
    G.loaded = true;
    ctx->n = n;
    return BM_OK;
}

extern "C" bm_status bm_graph_info(bm_ctx* ctx, int side, int32_t* n, int64_t* m_nonself, int32_t* max_degree,
                                   int64_t* max_weighted_degree) {
    if (!ctx || (side != 0 && side != 1)) return BM_INVALID_ARG;
    const DevGraph& G = ctx->g[side];
    if (!G.loaded) return bm_fail(ctx, BM_INVALID_ARG, "graph %d not set", side);
    if (n) *n = G.n;
    if (m_nonself) *m_nonself = G.m;
    if (max_degree) *max_degree = G.max_deg;
    if (max_weighted_degree) *max_weighted_degree = G.max_wdeg;
    return BM_OK;
}

// ----------------------------------------------------------------- mapping

extern "C" bm_status bm_set_mapping(bm_ctx* ctx, const int32_t* pi) {
    if (!ctx || !pi) return BM_INVALID_ARG;
    if (!ctx->g[0].loaded || !ctx->g[1].loaded) return bm_fail(ctx, BM_INVALID_ARG, "both graphs must be set first");
    int32_t n = ctx->n;
    std::vector<int32_t> h((size_t)n + 1), hinv((size_t)n + 1, 0);
    h[0] = 0;
    for (int32_t i = 1; i <= n; i++) {
        int32_t f = pi[i];
        if (f < 1 || f > n) return bm_fail(ctx, BM_INVALID_ARG, "pi(%d)=%d outside 1..%d", i, f, n);
        if (hinv[f] != 0) return bm_fail(ctx, BM_INVALID_ARG, "pi is not a bijection: image %d used twice", f);
        h[i] = f;
        hinv[f] = i;
    }
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!ctx->pi) {
        BM_CUDA(ctx, cudaMalloc(&ctx->pi, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->pinv, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->ov, sizeof(int32_t) * ((size_t)n + 1)));
    } else {
        // sizes may have changed with a new graph
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->pi); cudaFree(ctx->pinv); cudaFree(ctx->ov);
        ctx->pi = ctx->pinv = ctx->ov = nullptr;
        BM_CUDA(ctx, cudaMalloc(&ctx->pi, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->pinv, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->ov, sizeof(int32_t) * ((size_t)n + 1)));
    }
    BM_CUDA(ctx, cudaMemcpyAsync(ctx->pi, h.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(ctx->pinv, hinv.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
    BM_TRY(bm_launch_relabel(ctx));
    int64_t s = 0;
    BM_TRY(bm_launch_score(ctx, &s));
    ctx->score = s;
    ctx->mapped = true;
    return BM_OK;
}

extern "C" bm_status bm_get_mapping(bm_ctx* ctx, int32_t* pi) {
    BM_TRY(bm_require_mapped(ctx));
    if (!pi) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaMemcpyAsync(pi, ctx->pi, sizeof(int32_t) * ((size_t)ctx->n + 1), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    pi[0] = 0;
    return BM_OK;
}

extern "C" bm_status bm_score(bm_ctx* ctx, int64_t* score) {
    BM_TRY(bm_require_mapped(ctx));
    if (!score) return BM_INVALID_ARG;
    return bm_launch_score(ctx, score);
}

extern "C" bm_status bm_tracked_score(bm_ctx* ctx, int64_t* score) {
    BM_TRY(bm_require_mapped(ctx));
    if (!score) return BM_INVALID_ARG;
    *score = ctx->score;
    return BM_OK;
}

extern "C" bm_status bm_get_overlap(bm_ctx* ctx, int32_t* ov) {
    BM_TRY(bm_require_mapped(ctx));
    if (!ov) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaMemcpyAsync(ov, ctx->ov, sizeof(int32_t) * ((size_t)ctx->n + 1), cudaMemcpyDeviceToHost, ctx->stream));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ov[0] = 0;
    return BM_OK;
}

// ------------------------------------------------------- device utilities

extern "C" bm_status bm_dev_alloc(bm_ctx* ctx, int64_t bytes, void** d_ptr) {
    if (!ctx || !d_ptr || bytes < 0) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    BM_CUDA(ctx, cudaMalloc(d_ptr, (size_t)(bytes > 0 ? bytes : 1)));
    return BM_OK;
}

extern "C" bm_status bm_dev_free(bm_ctx* ctx, void* d_ptr) {
    if (!ctx) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    BM_CUDA(ctx, cudaFree(d_ptr));
    return BM_OK;
}

extern "C" bm_status bm_memcpy_h2d(bm_ctx* ctx, void* d_dst, const void* h_src, int64_t bytes) {
    if (!ctx || bytes < 0) return BM_INVALID_ARG;
    if (bytes == 0) return BM_OK;
    BM_CUDA(ctx, cudaMemcpyAsync(d_dst, h_src, (size_t)bytes, cudaMemcpyHostToDevice, ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_memcpy_d2h(bm_ctx* ctx, void* h_dst, const void* d_src, int64_t bytes) {
    if (!ctx || bytes < 0) return BM_INVALID_ARG;
    if (bytes == 0) return BM_OK;
    BM_CUDA(ctx, cudaMemcpyAsync(h_dst, d_src, (size_t)bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_host_alloc_pinned(int64_t bytes, void** h_ptr) {
    if (!h_ptr || bytes < 0) return BM_INVALID_ARG;
    cudaError_t e = cudaMallocHost(h_ptr, (size_t)(bytes > 0 ? bytes : 1));
    if (e != cudaSuccess) { cudaGetLastError(); return e == cudaErrorMemoryAllocation ? BM_OOM : BM_CUDA_ERROR; }
    return BM_OK;
}

extern "C" bm_status bm_host_free_pinned(void* h_ptr) {
    if (cudaFreeHost(h_ptr) != cudaSuccess) { cudaGetLastError(); return BM_CUDA_ERROR; }
    return BM_OK;
}

extern "C" bm_status bm_l2_flush(bm_ctx* ctx) {
    if (!ctx) return BM_INVALID_ARG;
    if (!ctx->flush_buf) {
        int l2 = 0;
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->device);
        size_t bytes = (size_t)(l2 > 0 ? l2 : (128 << 20)) * 2;
        BM_CUDA(ctx, cudaMalloc(&ctx->flush_buf, bytes));
        ctx->flush_bytes = bytes;
    }
    BM_CUDA(ctx, cudaMemsetAsync(ctx->flush_buf, ctx->launches & 0xff, ctx->flush_bytes, ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_event_create(bm_ctx* ctx, void** ev) {
    if (!ctx || !ev) return BM_INVALID_ARG;
    cudaEvent_t e;
    BM_CUDA(ctx, cudaEventCreate(&e));
    *ev = (void*)e;
    return BM_OK;
}

extern "C" bm_status bm_event_destroy(bm_ctx* ctx, void* ev) {
    if (!ctx) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaEventDestroy((cudaEvent_t)ev));
    return BM_OK;
}

extern "C" bm_status bm_event_record(bm_ctx* ctx, void* ev) {
    if (!ctx) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaEventRecord((cudaEvent_t)ev, ctx->stream));
    return BM_OK;
}

extern "C" bm_status bm_event_elapsed_ms(bm_ctx* ctx, void* a, void* b, float* ms) {
    if (!ctx || !ms) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaEventSynchronize((cudaEvent_t)b));
    BM_CUDA(ctx, cudaEventElapsedTime(ms, (cudaEvent_t)a, (cudaEvent_t)b));
    return BM_OK;
}

extern "C" bm_status bm_set_row_tiling(bm_ctx* ctx, int32_t ctas_per_row, int32_t threads) {
    if (!ctx) return BM_INVALID_ARG;
    if (ctas_per_row != 0 && ctas_per_row != 1 && ctas_per_row != 2 && ctas_per_row != 4 && ctas_per_row != 8)
        return bm_fail(ctx, BM_INVALID_ARG, "ctas_per_row must be 1, 2, 4 or 8");
    if (threads != 0 && threads != 256 && threads != 512)
        return bm_fail(ctx, BM_INVALID_ARG, "threads must be 256 or 512");
    if (ctas_per_row) ctx->row_ctas = ctas_per_row;
    if (threads) ctx->row_threads = threads;
    return BM_OK;
}

extern "C" bm_status bm_get_row_tiling(bm_ctx* ctx, int32_t* ctas_per_row, int32_t* threads) {
    if (!ctx) return BM_INVALID_ARG;
    if (ctas_per_row) *ctas_per_row = ctx->row_ctas;
    if (threads) *threads = ctx->row_threads;
    return BM_OK;
}
