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
    cudaFree(ctx->tscr);
    cudaFree(ctx->rwork); cudaFree(ctx->spart); cudaFree(ctx->scnt); cudaFree(ctx->rpart); cudaFree(ctx->slots);
    if (ctx->hstage) cudaFreeHost(ctx->hstage);
    if (ctx->h_slots) cudaFreeHost(ctx->h_slots);
    if (ctx->slots_ev) cudaEventDestroy(ctx->slots_ev);
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

extern "C" bm_status bm_device_pci_bus_id(bm_ctx* ctx, char* buf, int32_t len) {
    if (!ctx || !buf || len < 13) return BM_INVALID_ARG;
    BM_CUDA(ctx, cudaDeviceGetPCIBusId(buf, len, ctx->device));
    return BM_OK;
}

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
    int other = 1 - side;
    if (ctx->g[other].loaded && ctx->g[other].n != n)
        return bm_fail(ctx, BM_INVALID_ARG, "n=%d differs from the other graph's n=%d", n, ctx->g[other].n);
    HostCsr H;
    std::string err;
    if (bm_build_host_csr(side == BM_SIDE_B, n, m, src, dst, w, H, err) != 0)
        return bm_fail(ctx, BM_INVALID_ARG, "%s", err.c_str());
    BM_CUDA(ctx, cudaSetDevice(ctx->device));
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));

    // Replacing a graph drops the mapping state.
    ctx->mapped = false;
    free_graph(ctx->g[side]);
    DevGraph& G = ctx->g[side];
    G.n = n;
    G.m_out = H.m_out();
    G.m_in = H.m_in();
    G.m_real = H.m_real;
    BM_TRY(upload(ctx, &G.out_ptr, H.optr.data(), H.optr.size()));
    BM_TRY(upload(ctx, &G.in_ptr, H.iptr.data(), H.iptr.size()));
    BM_TRY(upload(ctx, &G.out_ent, H.oent.data(), H.oent.size()));
    BM_TRY(upload(ctx, &G.in_ent, H.ient.data(), H.ient.size()));
    BM_TRY(upload(ctx, &G.self_w, H.self.data(), H.self.size()));
    if (side == BM_SIDE_B) {
        BM_TRY(upload(ctx, &G.out_twin, H.otw.data(), H.otw.size()));
        BM_TRY(upload(ctx, &G.in_twin, H.itw.data(), H.itw.size()));
        BM_TRY(upload(ctx, &G.out_ent0, H.oent.data(), H.oent.size()));
        BM_TRY(upload(ctx, &G.in_ent0, H.ient.data(), H.ient.size()));
        BM_TRY(upload(ctx, &G.hash, H.htab.data(), H.htab.size()));
        G.hash_log2 = H.hlog2;
    } else {
        ctx->hA_optr = H.optr;
        ctx->hA_iptr = H.iptr;
        ctx->hA_oent = H.oent;
        ctx->hA_ient = H.ient;
    }
    G.max_deg = H.max_deg;
    G.max_wdeg = H.max_wdeg;
    G.has_self = H.has_self;
    G.loaded = true;
    ctx->n = n;
    ctx->nvec = (n + 1 + 3) & ~3;
    return BM_OK;
}

extern "C" bm_status bm_graph_info(bm_ctx* ctx, int side, int32_t* n, int64_t* m_nonself, int32_t* max_degree,
                                   int64_t* max_weighted_degree) {
    if (!ctx || (side != 0 && side != 1)) return BM_INVALID_ARG;
    const DevGraph& G = ctx->g[side];
    if (!G.loaded) return bm_fail(ctx, BM_INVALID_ARG, "graph %d not set", side);
    if (n) *n = G.n;
    if (m_nonself) *m_nonself = G.m_real;
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
        BM_CUDA(ctx, cudaMalloc(&ctx->ov, sizeof(int32_t) * (size_t)ctx->nvec));
    } else {
        // sizes may have changed with a new graph
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->pi); cudaFree(ctx->pinv); cudaFree(ctx->ov);
        ctx->pi = ctx->pinv = ctx->ov = nullptr;
        BM_CUDA(ctx, cudaMalloc(&ctx->pi, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->pinv, sizeof(int32_t) * ((size_t)n + 1)));
        BM_CUDA(ctx, cudaMalloc(&ctx->ov, sizeof(int32_t) * (size_t)ctx->nvec));
    }
    BM_CUDA(ctx, cudaMemcpyAsync(ctx->pi, h.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
    BM_CUDA(ctx, cudaMemcpyAsync(ctx->pinv, hinv.data(), sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, ctx->stream));
    BM_TRY(bm_launch_relabel(ctx));
    int64_t s = 0;
    BM_TRY(bm_launch_score(ctx, &s));
    BM_TRY(bm_rows_prepare(ctx));
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
    if (ctas_per_row < 0 || ctas_per_row > 8)
        return bm_fail(ctx, BM_INVALID_ARG, "ctas_per_row must be 0 (automatic) or 1..8");
    if (threads != 0 && threads != 256 && threads != 512)
        return bm_fail(ctx, BM_INVALID_ARG, "threads must be 256 or 512");
    if (ctas_per_row) ctx->row_ctas = ctas_per_row;
    if (threads) ctx->row_threads = threads;
    return BM_OK;
}

extern "C" bm_status bm_set_semantics(bm_ctx* ctx, int32_t mode) {
    if (!ctx) return BM_INVALID_ARG;
    if (mode != BM_SEMANTICS_EXACT && mode != BM_SEMANTICS_REF_CPU)
        return bm_fail(ctx, BM_INVALID_ARG, "semantics must be BM_SEMANTICS_EXACT (0) or BM_SEMANTICS_REF_CPU (1)");
    ctx->semantics = mode;
    return BM_OK;
}

extern "C" bm_status bm_get_semantics(bm_ctx* ctx, int32_t* mode) {
    if (!ctx || !mode) return BM_INVALID_ARG;
    *mode = ctx->semantics;
    return BM_OK;
}

extern "C" bm_status bm_set_row_split(bm_ctx* ctx, int32_t slots) {
    if (!ctx) return BM_INVALID_ARG;
    if (slots < -1) return bm_fail(ctx, BM_INVALID_ARG, "slots must be -1 (off), 0 (automatic) or a slot count");
    ctx->row_split = slots;
    return BM_OK;
}

extern "C" bm_status bm_get_row_split(bm_ctx* ctx, int32_t* slots) {
    if (!ctx || !slots) return BM_INVALID_ARG;
    *slots = ctx->row_split;
    return BM_OK;
}

extern "C" bm_status bm_get_row_tiling(bm_ctx* ctx, int32_t* ctas_per_row, int32_t* threads) {
    if (!ctx) return BM_INVALID_ARG;
    if (ctas_per_row) *ctas_per_row = ctx->row_ctas;
    if (threads) *threads = ctx->row_threads;
    return BM_OK;
}
