// bm_comm.cu — ranks of a sharded search (one process per GPU) and their
// exchange, in place of the reference's MPI drivers
// (src/graph-re-alignment-mpi-omp.c:76-123, src/graph-re-alignment-mpi-gpu.cu:
// 349-396).
//
// Two transports behind one interface:
//   TCP   host sockets in a star around rank 0 (rank 0 listens on addr, the
//         others connect).  Every collective gathers the ranks' buffers at
//         rank 0 and sends the rank-ordered result back.  It needs no GPU: the
//         protocol's CPU tests run on it, and it serves ranks that share a GPU.
//   NCCL  libnccl (loaded with dlopen when asked for) over NVLink / NVSwitch,
//         collectives on device buffers on the context's stream; rank 0's
//         socket carries only the ncclUniqueId.  NVLS (in-switch reduction) is
//         left off unless NCCL_NVLS_ENABLE is set: the payloads are a few KB.
// Every wait is bounded by the communicator's timeout: a socket that stays
// silent, a peer that closes, or an NCCL collective that does not finish in
// time makes the call return BM_TIMEOUT (the NCCL communicator is then
// aborted).  Every rank must make the same collective calls in the same order.
//
// The sharded search keeps one mapping replicated on every rank: each round
// every rank evaluates its share of the round's rows on its own GPU (best
// improving partner per row), the candidates are all-gathered in rank order,
// and every rank runs the same deterministic independent-subset selection
// (bm_select_independent's rule) on the same list, so all ranks apply the same
// swaps with no broadcast of the mapping.  Island synchronisation is one
// all-reduce of a packed (score, rank) key and one broadcast of the winner's
// mapping (sync_best_solutions, src/graph-re-alignment-mpi-omp.c:76-123).
#include <arpa/inet.h>
#include <dlfcn.h>
#include <errno.h>
#include <netdb.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <poll.h>
#include <sys/socket.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <nccl.h>

#include "bm_internal.cuh"

namespace {

using clk = std::chrono::steady_clock;
double secs_since(clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); }

// The NCCL entry points used here, resolved from libnccl.so.2 at run time.
struct NcclApi {
    void* lib = nullptr;
    ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
    ncclResult_t (*AllGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*Broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

template <class F>
bool sym(void* lib, const char* name, F& f) {
    f = reinterpret_cast<F>(dlsym(lib, name));
    return f != nullptr;
}

}  // namespace

struct bm_comm {
    int32_t kind = BM_COMM_TCP;
    int32_t rank = 0, world = 1;
    double timeout_s = 60.0;
    bm_ctx* ctx = nullptr;
    int listen_fd = -1;
    std::vector<int> fd;  // rank 0: socket of each rank (fd[0] unused); others: fd[0] = rank 0
    // NCCL
    NcclApi api;
    ncclComm_t nc = nullptr;
    bool aborted = false;
    void* d_buf = nullptr;  // device staging of the collectives
    size_t d_bytes = 0;
    std::string err;
};

namespace {

bm_status comm_fail(bm_comm* c, bm_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
    if (c->ctx) c->ctx->err = buf;
    return s;
}

// ------------------------------------------------------------------- TCP

// Wait until fd is readable (or writable); false when the deadline passes.
bool wait_fd(int fd, bool write, clk::time_point deadline) {
    for (;;) {
        const double left = std::chrono::duration<double>(deadline - clk::now()).count();
        if (left <= 0) return false;
        pollfd p{fd, (short)(write ? POLLOUT : POLLIN), 0};
        const int ms = (int)std::min(1000.0, left * 1000.0) + 1;
        const int r = poll(&p, 1, ms);
        if (r > 0) return true;
        if (r < 0 && errno != EINTR) return false;
    }
}

bm_status send_all(bm_comm* c, int fd, const void* buf, size_t len, int peer) {
    const auto deadline = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(c->timeout_s));
    const char* p = static_cast<const char*>(buf);
    while (len > 0) {
        if (!wait_fd(fd, true, deadline)) return comm_fail(c, BM_TIMEOUT, "rank %d: sending to rank %d timed out", c->rank, peer);
        const ssize_t k = send(fd, p, len, MSG_NOSIGNAL);
        if (k < 0) {
            if (errno == EINTR || errno == EAGAIN) continue;
            return comm_fail(c, BM_TIMEOUT, "rank %d: rank %d is gone (send: %s)", c->rank, peer, strerror(errno));
        }
        p += k;
        len -= (size_t)k;
    }
    return BM_OK;
}

bm_status recv_all(bm_comm* c, int fd, void* buf, size_t len, int peer) {
    const auto deadline = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(c->timeout_s));
    char* p = static_cast<char*>(buf);
    while (len > 0) {
        if (!wait_fd(fd, false, deadline))
            return comm_fail(c, BM_TIMEOUT, "rank %d: waiting for rank %d timed out", c->rank, peer);
        const ssize_t k = recv(fd, p, len, 0);
        if (k == 0) return comm_fail(c, BM_TIMEOUT, "rank %d: rank %d closed its connection", c->rank, peer);
        if (k < 0) {
            if (errno == EINTR || errno == EAGAIN) continue;
            return comm_fail(c, BM_TIMEOUT, "rank %d: rank %d is gone (recv: %s)", c->rank, peer, strerror(errno));
        }
        p += k;
        len -= (size_t)k;
    }
    return BM_OK;
}

bool parse_addr(const char* addr, std::string& host, int& port) {
    if (!addr) return false;
    const char* colon = strrchr(addr, ':');
    if (!colon) return false;
    host.assign(addr, colon - addr);
    port = atoi(colon + 1);
    return port > 0 && port < 65536 && !host.empty();
}

bm_status tcp_connect(bm_comm* c, const char* addr) {
    std::string host;
    int port = 0;
    if (!parse_addr(addr, host, port)) return comm_fail(c, BM_INVALID_ARG, "address must be host:port, got %s", addr ? addr : "(null)");
    sockaddr_in sa{};
    sa.sin_family = AF_INET;
    sa.sin_port = htons((uint16_t)port);
    if (inet_pton(AF_INET, host.c_str(), &sa.sin_addr) != 1) {
        addrinfo hints{}, *res = nullptr;
        hints.ai_family = AF_INET;
        if (getaddrinfo(host.c_str(), nullptr, &hints, &res) != 0 || !res)
            return comm_fail(c, BM_INVALID_ARG, "cannot resolve %s", host.c_str());
        sa.sin_addr = reinterpret_cast<sockaddr_in*>(res->ai_addr)->sin_addr;
        freeaddrinfo(res);
    }
    const auto t0 = clk::now();
    const int one = 1;
    if (c->rank == 0) {
        c->listen_fd = socket(AF_INET, SOCK_STREAM, 0);
        if (c->listen_fd < 0) return comm_fail(c, BM_CUDA_ERROR, "socket: %s", strerror(errno));
        setsockopt(c->listen_fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof one);
        if (bind(c->listen_fd, reinterpret_cast<sockaddr*>(&sa), sizeof sa) != 0 || listen(c->listen_fd, c->world) != 0)
            return comm_fail(c, BM_INVALID_ARG, "rank 0 cannot listen on %s: %s", addr, strerror(errno));
        c->fd.assign((size_t)c->world, -1);
        for (int k = 1; k < c->world; k++) {
            const auto deadline = t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(c->timeout_s));
            if (!wait_fd(c->listen_fd, false, deadline))
                return comm_fail(c, BM_TIMEOUT, "rank 0: only %d of %d ranks connected in time", k, c->world);
            const int f = accept(c->listen_fd, nullptr, nullptr);
            if (f < 0) return comm_fail(c, BM_CUDA_ERROR, "accept: %s", strerror(errno));
            setsockopt(f, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
            int32_t r = -1;
            c->fd.push_back(f);  // kept for closing if the rank id is bad
            bm_status s = recv_all(c, f, &r, sizeof r, -1);
            if (s != BM_OK) return s;
            if (r < 1 || r >= c->world || c->fd[(size_t)r] >= 0)
                return comm_fail(c, BM_INVALID_ARG, "rank 0: a peer announced rank %d", r);
            c->fd.pop_back();
            c->fd[(size_t)r] = f;
        }
        const int32_t go = c->world;
        for (int r = 1; r < c->world; r++) {
            bm_status s = send_all(c, c->fd[(size_t)r], &go, sizeof go, r);
            if (s != BM_OK) return s;
        }
        return BM_OK;
    }
    // other ranks: connect to rank 0, retrying while it starts
    for (;;) {
        const int f = socket(AF_INET, SOCK_STREAM, 0);
        if (f < 0) return comm_fail(c, BM_CUDA_ERROR, "socket: %s", strerror(errno));
        if (connect(f, reinterpret_cast<sockaddr*>(&sa), sizeof sa) == 0) {
            setsockopt(f, IPPROTO_TCP, TCP_NODELAY, &one, sizeof one);
            c->fd.assign(1, f);
            break;
        }
        close(f);
        if (secs_since(t0) >= c->timeout_s) return comm_fail(c, BM_TIMEOUT, "rank %d: rank 0 did not answer at %s", c->rank, addr);
        std::this_thread::sleep_for(std::chrono::milliseconds(50));
    }
    const int32_t me = c->rank;
    bm_status s = send_all(c, c->fd[0], &me, sizeof me, 0);
    if (s != BM_OK) return s;
    int32_t go = 0;
    if ((s = recv_all(c, c->fd[0], &go, sizeof go, 0)) != BM_OK) return s;
    if (go != c->world) return comm_fail(c, BM_INVALID_ARG, "rank %d: rank 0 runs a world of %d, not %d", c->rank, go, c->world);
    return BM_OK;
}

// Gather every rank's bytes at rank 0 and send the rank-ordered concatenation
// back: out = [len_0 .. len_{W-1} (int64 each)] then the payloads in rank order.
bm_status tcp_allgatherv(bm_comm* c, const void* mine, int64_t len, std::vector<char>& out) {
    const int W = c->world;
    if (c->rank == 0) {
        std::vector<int64_t> lens((size_t)W);
        std::vector<std::vector<char>> parts((size_t)W);
        lens[0] = len;
        parts[0].assign(static_cast<const char*>(mine), static_cast<const char*>(mine) + len);
        for (int r = 1; r < W; r++) {
            bm_status s = recv_all(c, c->fd[(size_t)r], &lens[(size_t)r], sizeof(int64_t), r);
            if (s != BM_OK) return s;
            if (lens[(size_t)r] < 0 || lens[(size_t)r] > (int64_t)1 << 34) return comm_fail(c, BM_INVALID_ARG, "rank %d sent a bad length", r);
            parts[(size_t)r].resize((size_t)lens[(size_t)r]);
            if ((s = recv_all(c, c->fd[(size_t)r], parts[(size_t)r].data(), (size_t)lens[(size_t)r], r)) != BM_OK) return s;
        }
        out.assign(sizeof(int64_t) * (size_t)W, 0);
        memcpy(out.data(), lens.data(), sizeof(int64_t) * (size_t)W);
        for (int r = 0; r < W; r++) out.insert(out.end(), parts[(size_t)r].begin(), parts[(size_t)r].end());
        const int64_t total = (int64_t)out.size();
        for (int r = 1; r < W; r++) {
            bm_status s = send_all(c, c->fd[(size_t)r], &total, sizeof total, r);
            if (s != BM_OK) return s;
            if ((s = send_all(c, c->fd[(size_t)r], out.data(), out.size(), r)) != BM_OK) return s;
        }
        return BM_OK;
    }
    bm_status s = send_all(c, c->fd[0], &len, sizeof len, 0);
    if (s != BM_OK) return s;
    if (len > 0 && (s = send_all(c, c->fd[0], mine, (size_t)len, 0)) != BM_OK) return s;
    int64_t total = 0;
    if ((s = recv_all(c, c->fd[0], &total, sizeof total, 0)) != BM_OK) return s;
    if (total < (int64_t)sizeof(int64_t) * W || total > (int64_t)1 << 36) return comm_fail(c, BM_INVALID_ARG, "rank 0 sent a bad length");
    out.resize((size_t)total);
    return recv_all(c, c->fd[0], out.data(), out.size(), 0);
}

// ------------------------------------------------------------------ NCCL

bm_status nccl_load(bm_comm* c) {
    void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
    if (!lib) return comm_fail(c, BM_UNSUPPORTED, "NCCL transport: cannot load libnccl.so.2 (%s)", dlerror());
    NcclApi& a = c->api;
    a.lib = lib;
    if (!sym(lib, "ncclGetUniqueId", a.GetUniqueId) || !sym(lib, "ncclCommInitRank", a.CommInitRank) ||
        !sym(lib, "ncclCommDestroy", a.CommDestroy) || !sym(lib, "ncclCommAbort", a.CommAbort) ||
        !sym(lib, "ncclAllGather", a.AllGather) || !sym(lib, "ncclAllReduce", a.AllReduce) ||
        !sym(lib, "ncclBroadcast", a.Broadcast) || !sym(lib, "ncclGetErrorString", a.GetErrorString))
        return comm_fail(c, BM_UNSUPPORTED, "NCCL transport: libnccl lacks an entry point");
    return BM_OK;
}

bm_status nccl_check(bm_comm* c, ncclResult_t r, const char* what) {
    if (r == ncclSuccess) return BM_OK;
    return comm_fail(c, BM_CUDA_ERROR, "%s: %s", what, c->api.GetErrorString(r));
}

// Wait for the collectives queued on the context's stream, within the
// timeout; on expiry the communicator is aborted (its kernels end).
bm_status nccl_wait(bm_comm* c, const char* what) {
    const auto t0 = clk::now();
    for (;;) {
        const cudaError_t e = cudaStreamQuery(c->ctx->stream);
        if (e == cudaSuccess) return BM_OK;
        if (e != cudaErrorNotReady) return bm_cuda_fail(c->ctx, e, what);
        if (secs_since(t0) >= c->timeout_s) {
            c->api.CommAbort(c->nc);
            c->nc = nullptr;
            c->aborted = true;
            return comm_fail(c, BM_TIMEOUT, "rank %d: %s did not complete in %.1f s; communicator aborted", c->rank, what,
                             c->timeout_s);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

bm_status nccl_buf(bm_comm* c, size_t bytes) {
    if (c->d_bytes >= bytes) return BM_OK;
    BM_CUDA(c->ctx, cudaStreamSynchronize(c->ctx->stream));
    bm_cuda_free(c->d_buf);
    c->d_buf = nullptr;
    c->d_bytes = 0;
    const size_t sz = std::max<size_t>(bytes, 1 << 16);
    BM_CUDA(c->ctx, bm_cuda_malloc(&c->d_buf, sz));
    c->d_bytes = sz;
    return BM_OK;
}

// All-gather of equal-sized blocks (bytes each) through the device buffer.
bm_status nccl_allgather(bm_comm* c, const void* mine, size_t bytes, void* all) {
    bm_status s = nccl_buf(c, bytes * (size_t)(c->world + 1));
    if (s != BM_OK) return s;
    char* d_in = static_cast<char*>(c->d_buf);
    char* d_out = d_in + bytes;
    BM_CUDA(c->ctx, cudaMemcpyAsync(d_in, mine, bytes, cudaMemcpyHostToDevice, c->ctx->stream));
    if ((s = nccl_check(c, c->api.AllGather(d_in, d_out, bytes, ncclChar, c->nc, c->ctx->stream), "ncclAllGather")) !=
        BM_OK)
        return s;
    BM_CUDA(c->ctx, cudaMemcpyAsync(all, d_out, bytes * (size_t)c->world, cudaMemcpyDeviceToHost, c->ctx->stream));
    return nccl_wait(c, "ncclAllGather");
}

bm_status comm_ready(bm_comm* c) {
    if (!c) return BM_INVALID_ARG;
    if (c->aborted) return comm_fail(c, BM_TIMEOUT, "the communicator was aborted after a timeout");
    if (c->kind == BM_COMM_NCCL) BM_CUDA(c->ctx, cudaSetDevice(c->ctx->device));
    return BM_OK;
}

// Rank-ordered variable-length all-gather on either transport.
bm_status allgatherv(bm_comm* c, const void* mine, int64_t len, std::vector<int64_t>& lens, std::vector<char>& data) {
    const int W = c->world;
    lens.assign((size_t)W, 0);
    data.clear();
    if (c->kind == BM_COMM_TCP) {
        std::vector<char> out;
        bm_status s = W == 1 ? BM_OK : tcp_allgatherv(c, mine, len, out);
        if (s != BM_OK) return s;
        if (W == 1) {
            lens[0] = len;
            data.assign(static_cast<const char*>(mine), static_cast<const char*>(mine) + len);
            return BM_OK;
        }
        memcpy(lens.data(), out.data(), sizeof(int64_t) * (size_t)W);
        data.assign(out.begin() + (ptrdiff_t)(sizeof(int64_t) * (size_t)W), out.end());
        return BM_OK;
    }
    // NCCL: lengths first, then blocks padded to the longest
    bm_status s = nccl_allgather(c, &len, sizeof len, lens.data());
    if (s != BM_OK) return s;
    int64_t mx = 0;
    for (int64_t l : lens) mx = std::max(mx, l);
    const size_t blk = ((size_t)mx + 15) & ~(size_t)15;
    if (blk == 0) return BM_OK;
    std::vector<char> pad(blk, 0), all(blk * (size_t)W);
    if (len > 0) memcpy(pad.data(), mine, (size_t)len);
    if ((s = nccl_allgather(c, pad.data(), blk, all.data())) != BM_OK) return s;
    for (int r = 0; r < W; r++) data.insert(data.end(), all.begin() + (ptrdiff_t)(blk * r), all.begin() + (ptrdiff_t)(blk * r + lens[(size_t)r]));
    return BM_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI

extern "C" bm_status bm_comm_create(int32_t kind, int32_t rank, int32_t world, const char* addr, double timeout_s,
                                    bm_ctx* ctx, bm_comm** out) {
    if (!out) return BM_INVALID_ARG;
    *out = nullptr;
    if (world < 1 || rank < 0 || rank >= world || !(timeout_s > 0)) return BM_INVALID_ARG;
    if (kind != BM_COMM_TCP && kind != BM_COMM_NCCL) return BM_INVALID_ARG;
    if (kind == BM_COMM_NCCL && !ctx) return BM_INVALID_ARG;
    bm_comm* c = new (std::nothrow) bm_comm();
    if (!c) return BM_OOM;
    c->kind = kind;
    c->rank = rank;
    c->world = world;
    c->timeout_s = timeout_s;
    c->ctx = ctx;
    bm_status s = BM_OK;
    if (world > 1) s = tcp_connect(c, addr);
    if (s == BM_OK && kind == BM_COMM_NCCL) {
        if ((s = nccl_load(c)) == BM_OK) {
            setenv("NCCL_NVLS_ENABLE", "0", 0);  // small payloads; no multicast objects
            ncclUniqueId id;
            memset(&id, 0, sizeof id);
            if (rank == 0) s = nccl_check(c, c->api.GetUniqueId(&id), "ncclGetUniqueId");
            if (s == BM_OK && world > 1) {
                std::vector<char> all;
                s = tcp_allgatherv(c, &id, rank == 0 ? (int64_t)sizeof id : 0, all);
                if (s == BM_OK) memcpy(&id, all.data() + sizeof(int64_t) * (size_t)world, sizeof id);
            }
            if (s == BM_OK) {
                cudaSetDevice(ctx->device);
                s = nccl_check(c, c->api.CommInitRank(&c->nc, world, id, rank), "ncclCommInitRank");
            }
        }
    }
    if (s != BM_OK) {
        if (ctx) ctx->err = c->err;
        bm_comm_destroy(c);
        return s;
    }
    *out = c;
    return BM_OK;
}

extern "C" void bm_comm_destroy(bm_comm* c) {
    if (!c) return;
    if (c->nc && c->api.CommDestroy) {
        if (c->ctx) cudaStreamSynchronize(c->ctx->stream);
        c->api.CommDestroy(c->nc);
    }
    if (c->d_buf) bm_cuda_free(c->d_buf);
    for (int f : c->fd)
        if (f >= 0) close(f);
    if (c->listen_fd >= 0) close(c->listen_fd);
    if (c->api.lib) dlclose(c->api.lib);
    delete c;
}

extern "C" const char* bm_comm_last_error(const bm_comm* c) { return c ? c->err.c_str() : ""; }

extern "C" bm_status bm_comm_barrier(bm_comm* c) {
    bm_status s = comm_ready(c);
    if (s != BM_OK) return s;
    std::vector<int64_t> lens;
    std::vector<char> data;
    const int32_t z = 0;
    return allgatherv(c, &z, sizeof z, lens, data);
}

extern "C" bm_status bm_comm_allreduce_sum(bm_comm* c, int64_t value, int64_t* total) {
    bm_status s = comm_ready(c);
    if (s != BM_OK) return s;
    if (!total) return comm_fail(c, BM_INVALID_ARG, "output required");
    std::vector<int64_t> lens;
    std::vector<char> data;
    if ((s = allgatherv(c, &value, sizeof value, lens, data)) != BM_OK) return s;
    int64_t t = 0;
    for (int r = 0; r < c->world; r++) {
        int64_t v;
        memcpy(&v, data.data() + sizeof(int64_t) * (size_t)r, sizeof v);
        t += v;
    }
    *total = t;
    return BM_OK;
}

extern "C" bm_status bm_comm_allgather_swaps(bm_comm* c, const int32_t* pairs, const int64_t* deltas, int32_t count,
                                             int32_t cap, int32_t* all_pairs, int64_t* all_deltas, int32_t* total) {
    bm_status s = comm_ready(c);
    if (s != BM_OK) return s;
    if (count < 0 || cap < 0 || !total || (count > 0 && (!pairs || !deltas)) || (cap > 0 && (!all_pairs || !all_deltas)))
        return comm_fail(c, BM_INVALID_ARG, "bad candidate buffers");
    // records of 16 bytes: u, v, delta
    std::vector<int32_t> rec((size_t)count * 4);
    for (int32_t i = 0; i < count; i++) {
        rec[(size_t)4 * i] = pairs[2 * i];
        rec[(size_t)4 * i + 1] = pairs[2 * i + 1];
        memcpy(&rec[(size_t)4 * i + 2], &deltas[i], sizeof(int64_t));
    }
    std::vector<int64_t> lens;
    std::vector<char> data;
    if ((s = allgatherv(c, rec.data(), (int64_t)rec.size() * 4, lens, data)) != BM_OK) return s;
    const int64_t n = (int64_t)data.size() / 16;
    *total = (int32_t)n;
    if (n > cap) return comm_fail(c, BM_INVALID_ARG, "%lld gathered candidates exceed the capacity %d", (long long)n, cap);
    for (int64_t i = 0; i < n; i++) {
        int32_t r4[4];
        memcpy(r4, data.data() + 16 * i, 16);
        all_pairs[2 * i] = r4[0];
        all_pairs[2 * i + 1] = r4[1];
        memcpy(&all_deltas[i], &r4[2], sizeof(int64_t));
    }
    return BM_OK;
}

extern "C" bm_status bm_comm_island_best(bm_comm* c, int64_t score, int32_t* pi, int32_t n, int64_t* best_score,
                                         int32_t* best_rank) {
    bm_status s = comm_ready(c);
    if (s != BM_OK) return s;
    if (!pi || n < 1) return comm_fail(c, BM_INVALID_ARG, "mapping required");
    if (score < 0 || score >= ((int64_t)1 << 47)) return comm_fail(c, BM_INVALID_ARG, "score outside 0..2^47");
    // packed key: the best score wins, the lowest rank on ties
    const int64_t key = (score << 16) | (int64_t)(0xFFFF - c->rank);
    int64_t best = key;
    if (c->kind == BM_COMM_NCCL) {
        if ((s = nccl_buf(c, 16)) != BM_OK) return s;
        int64_t* d = static_cast<int64_t*>(c->d_buf);
        BM_CUDA(c->ctx, cudaMemcpyAsync(d, &key, sizeof key, cudaMemcpyHostToDevice, c->ctx->stream));
        if ((s = nccl_check(c, c->api.AllReduce(d, d + 1, 1, ncclInt64, ncclMax, c->nc, c->ctx->stream), "ncclAllReduce")) != BM_OK)
            return s;
        BM_CUDA(c->ctx, cudaMemcpyAsync(&best, d + 1, sizeof best, cudaMemcpyDeviceToHost, c->ctx->stream));
        if ((s = nccl_wait(c, "ncclAllReduce")) != BM_OK) return s;
    } else {
        std::vector<int64_t> lens;
        std::vector<char> data;
        if ((s = allgatherv(c, &key, sizeof key, lens, data)) != BM_OK) return s;
        for (int r = 0; r < c->world; r++) {
            int64_t v;
            memcpy(&v, data.data() + sizeof(int64_t) * (size_t)r, sizeof v);
            best = std::max(best, v);
        }
    }
    const int32_t br = 0xFFFF - (int32_t)(best & 0xFFFF);
    const size_t bytes = sizeof(int32_t) * ((size_t)n + 1);
    if (c->kind == BM_COMM_NCCL) {
        if ((s = nccl_buf(c, bytes)) != BM_OK) return s;
        BM_CUDA(c->ctx, cudaMemcpyAsync(c->d_buf, pi, bytes, cudaMemcpyHostToDevice, c->ctx->stream));
        if ((s = nccl_check(c, c->api.Broadcast(c->d_buf, c->d_buf, bytes, ncclChar, br, c->nc, c->ctx->stream), "ncclBroadcast")) != BM_OK)
            return s;
        BM_CUDA(c->ctx, cudaMemcpyAsync(pi, c->d_buf, bytes, cudaMemcpyDeviceToHost, c->ctx->stream));
        if ((s = nccl_wait(c, "ncclBroadcast")) != BM_OK) return s;
    } else if (c->world > 1) {
        // the winner's mapping, through the all-gather (only the winner sends it)
        std::vector<int64_t> lens;
        std::vector<char> data;
        if ((s = allgatherv(c, pi, c->rank == br ? (int64_t)bytes : 0, lens, data)) != BM_OK) return s;
        if (data.size() != bytes) return comm_fail(c, BM_INVALID_ARG, "mapping sizes differ between ranks");
        memcpy(pi, data.data(), bytes);
    }
    if (best_score) *best_score = best >> 16;
    if (best_rank) *best_rank = br;
    return BM_OK;
}

// ---------------------------------------------------------- sharded search

extern "C" bm_status bm_search_sharded(bm_ctx* ctx, bm_comm* c, const int32_t* row_order, int32_t nrows,
                                       int32_t rows_per_rank, int64_t max_rounds, double time_budget_s,
                                       bm_progress* prog) {
    bm_status s = bm_require_mapped(ctx);
    if (s != BM_OK) return s;
    if ((s = comm_ready(c)) != BM_OK) return s;
    if (!prog) return bm_fail(ctx, BM_INVALID_ARG, "progress struct required");
    if (c->ctx && c->ctx != ctx) return bm_fail(ctx, BM_INVALID_ARG, "the communicator belongs to another context");
    if ((s = bm_rows_smem_check(ctx)) != BM_OK) return s;
    const int32_t n = ctx->n;
    std::vector<int32_t> order;
    if (row_order) {
        if (nrows <= 0) return bm_fail(ctx, BM_INVALID_ARG, "empty row order");
        order.assign(row_order, row_order + nrows);
        for (int32_t i = 0; i < nrows; i++)
            if (order[(size_t)i] < 1 || order[(size_t)i] > n)
                return bm_fail(ctx, BM_INVALID_ARG, "row_order[%d] = %d outside 1..%d", i, order[(size_t)i], n);
    } else {
        order.resize((size_t)n);
        for (int32_t i = 0; i < n; i++) order[(size_t)i] = i + 1;
    }
    const int32_t nr = (int32_t)order.size();
    const int32_t W = c->world, me = c->rank;
    const int32_t R = std::max(1, rows_per_rank > 0 ? rows_per_rank : 2 * ctx->num_sms);
    const int64_t per_round = (int64_t)W * R;
    const int64_t rounds_per_pass = (nr + per_round - 1) / per_round;
    // staging: this rank's rows, results, gathered candidates, chosen swaps
    const size_t rb = ((size_t)R * sizeof(int32_t) + 255) & ~(size_t)255;
    const size_t resb = ((size_t)R * sizeof(bm_row_result) + 255) & ~(size_t)255;
    const size_t pb = ((size_t)per_round * 2 * sizeof(int32_t) + 255) & ~(size_t)255;
    if ((s = bm_stage(ctx, rb + resb + pb)) != BM_OK) return s;
    if ((s = bm_hstage(ctx, rb + resb + pb)) != BM_OK) return s;
    int32_t* d_rows = static_cast<int32_t*>(ctx->stage);
    bm_row_result* d_res = reinterpret_cast<bm_row_result*>(static_cast<char*>(ctx->stage) + rb);
    int32_t* d_pairs = reinterpret_cast<int32_t*>(static_cast<char*>(ctx->stage) + rb + resb);
    int32_t* h_rows = static_cast<int32_t*>(ctx->hstage);
    bm_row_result* h_res = reinterpret_cast<bm_row_result*>(static_cast<char*>(ctx->hstage) + rb);
    int32_t* h_pairs = reinterpret_cast<int32_t*>(static_cast<char*>(ctx->hstage) + rb + resb);
    if ((s = bm_rows_refresh_work(ctx)) != BM_OK) return s;
    // gathered: at most one candidate per row of the round, plus one stop
    // record per rank
    const size_t gcap = (size_t)per_round + (size_t)W;
    std::vector<int32_t> cand_pairs, all_pairs(gcap * 2), chosen(gcap);
    std::vector<int64_t> cand_deltas, all_deltas(gcap);
    const auto t0 = clk::now();
    int64_t rnd = 0, pass_accepts = 0, rnd_in_pass = 0;
    prog->converged = 0;
    bm_status ret = BM_OK;
    for (;;) {
        if (max_rounds >= 0 && rnd >= max_rounds) break;
        // this rank's rows of the round: every W-th of the round's rows
        int32_t k = 0;
        for (int64_t i = me; i < per_round; i += W) h_rows[k++] = order[(size_t)((rnd * per_round + i) % nr)];
        BM_CUDA(ctx, cudaMemcpyAsync(d_rows, h_rows, sizeof(int32_t) * (size_t)k, cudaMemcpyHostToDevice, ctx->stream));
        if ((s = bm_launch_rows(ctx, d_rows, nullptr, k, nullptr, d_res, h_rows)) != BM_OK) return s;
        BM_CUDA(ctx, cudaMemcpyAsync(h_res, d_res, sizeof(bm_row_result) * (size_t)k, cudaMemcpyDeviceToHost, ctx->stream));
        BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        prog->launches++;
        prog->evaluated += (int64_t)k * (n - 1);
        prog->rows_done += k;
        // candidates, then a stop flag from this rank's budget as one more
        // record (u = v = 0), so every rank stops after the same round
        cand_pairs.clear();
        cand_deltas.clear();
        for (int32_t i = 0; i < k; i++)
            if (h_res[i].best_delta > 0) {
                cand_pairs.push_back(h_res[i].row);
                cand_pairs.push_back(h_res[i].best);
                cand_deltas.push_back(h_res[i].best_delta);
            }
        const bool want_stop = time_budget_s > 0 && secs_since(t0) >= time_budget_s;
        if (want_stop) {
            cand_pairs.push_back(0);
            cand_pairs.push_back(0);
            cand_deltas.push_back(0);
        }
        int32_t total = 0;
        s = bm_comm_allgather_swaps(c, cand_pairs.data(), cand_deltas.data(), (int32_t)cand_deltas.size(),
                                    (int32_t)all_deltas.size(), all_pairs.data(), all_deltas.data(), &total);
        if (s != BM_OK) return s;
        bool stop = false;
        int32_t m = 0;  // drop the stop records, keep the rank order of the rest
        for (int32_t i = 0; i < total; i++) {
            if (all_pairs[(size_t)2 * i] == 0) { stop = true; continue; }
            all_pairs[(size_t)2 * m] = all_pairs[(size_t)2 * i];
            all_pairs[(size_t)2 * m + 1] = all_pairs[(size_t)2 * i + 1];
            all_deltas[(size_t)m] = all_deltas[(size_t)i];
            m++;
        }
        int32_t nch = 0;
        if ((s = bm_select_independent(ctx, all_pairs.data(), all_deltas.data(), m, chosen.data(), &nch)) != BM_OK)
            return s;
        if (nch > 0) {
            int64_t gain = 0;
            for (int32_t j = 0; j < nch; j++) {
                const int32_t i = chosen[(size_t)j];
                h_pairs[2 * j] = all_pairs[(size_t)2 * i];
                h_pairs[2 * j + 1] = all_pairs[(size_t)2 * i + 1];
                gain += all_deltas[(size_t)i];
            }
            BM_CUDA(ctx, cudaMemcpyAsync(d_pairs, h_pairs, sizeof(int32_t) * 2 * (size_t)nch, cudaMemcpyHostToDevice,
                                         ctx->stream));
            if ((s = bm_launch_apply(ctx, d_pairs, nch)) != BM_OK) return s;
            ctx->score += gain;
            prog->accepts += nch;
            pass_accepts += nch;
        }
        rnd++;
        if (++rnd_in_pass == rounds_per_pass) {
            prog->sweeps++;
            if (pass_accepts == 0) { prog->converged = 1; break; }
            pass_accepts = 0;
            rnd_in_pass = 0;
        }
        if (stop) { ret = BM_TIMEOUT; break; }
    }
    BM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    prog->seconds += secs_since(t0);
    s = bm_check_score(ctx);
    prog->score = ctx->score;
    if (s != BM_OK) return s;
    // the ranks must hold one mapping: compare a checksum of it across ranks
    std::vector<int32_t> pi((size_t)n + 1);
    BM_CUDA(ctx, cudaMemcpy(pi.data(), ctx->pi, sizeof(int32_t) * pi.size(), cudaMemcpyDeviceToHost));
    uint64_t h = 1469598103934665603ull;
    for (int32_t v : pi) h = (h ^ (uint32_t)v) * 1099511628211ull;
    std::vector<int64_t> lens;
    std::vector<char> data;
    if ((s = allgatherv(c, &h, sizeof h, lens, data)) != BM_OK) return s;
    for (int r = 0; r < W; r++)
        if (memcmp(data.data() + sizeof h * (size_t)r, &h, sizeof h) != 0)
            return bm_fail(ctx, BM_PARITY_FAIL, "rank %d's mapping differs from rank %d's after the sharded search", r, me);
    return ret;
}
