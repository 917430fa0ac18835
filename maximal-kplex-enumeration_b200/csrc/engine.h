// Host engine internals shared by the C ABI (engine.cu) and the request
// server (server.cu): device buffers, per-stream workspaces and the prepared
// graph sets they search.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "device.cuh"

namespace kplex {

void set_last_error(const std::string& msg);


#define CK(call)                                                                    \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            ::kplex::set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
            return KPLEX_ERR_CUDA;                                                  \
        }                                                                           \
    } while (0)

// ------------------------------------------------------------------ device buffer cache
// Grown on demand with the stream-ordered allocator, so that a workspace that
// grows does not wait for kernels running on other workspaces' streams.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    uint32_t allocs = 0;   // bumped on every (re)allocation: captured launches hold the old address
    int ensure(size_t want) {
        if (want <= bytes && p) return KPLEX_OK;
        if (p) { cudaFreeAsync(p, stream); p = nullptr; bytes = 0; }
        if (want == 0) want = 16;
        ++allocs;
        cudaError_t e = cudaMallocAsync(&p, want, stream);
        if (e != cudaSuccess) { cudaGetLastError(); p = nullptr; set_last_error(std::string("cudaMallocAsync ") + std::to_string(want) + ": " + cudaGetErrorString(e)); return KPLEX_ERR_NOMEM; }
        bytes = want;
        return KPLEX_OK;
    }
    void release() { if (p) cudaFreeAsync(p, stream); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Mapped pinned host memory (cudaHostAllocMapped), grown on demand.
struct HostMappedBuf {
    void* h = nullptr;
    void* d = nullptr;
    size_t bytes = 0;
    uint32_t allocs = 0;
    int ensure(size_t want) {
        if (want <= bytes && h) return KPLEX_OK;
        release();
        ++allocs;
        cudaError_t e = cudaHostAlloc(&h, want, cudaHostAllocMapped | cudaHostAllocPortable);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(&d, h, 0);
        if (e != cudaSuccess) { cudaGetLastError(); h = d = nullptr; set_last_error(std::string("pinned host spill buffer: ") + cudaGetErrorString(e)); return KPLEX_ERR_NOMEM; }
        bytes = want;
        return KPLEX_OK;
    }
    void release() { if (h) cudaFreeHost(h); h = d = nullptr; bytes = 0; }
};

// Everything one search needs besides the prepared graphs: a stream, the
// decomposition arena, the task pool, branch stacks and the spill ring.  The
// library keeps one per device for the plain calls; a server owns one per slot.
struct Workspace {
    Workspace() = default;
    Workspace(const Workspace&) = delete;   // bufs[] points into this object
    Workspace& operator=(const Workspace&) = delete;
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;
    DevBuf roots, ctr, scratch, arena, pool_seq, pool_data, pool, ks, stacks, jobs, spill_ctl, spill_seq;
    HostMappedBuf spill_data;
    Counters* h_ctr = nullptr;   // pinned
    Pool* h_pool = nullptr;      // pinned
    DevBuf* bufs[12] = {&roots, &ctr, &scratch, &arena, &pool_seq, &pool_data, &pool, &ks, &stacks, &jobs, &spill_ctl, &spill_seq};

    uint64_t generation() const {
        uint64_t g = spill_data.allocs;
        for (const DevBuf* x : bufs) g += x->allocs;
        return g;
    }
    size_t device_bytes() const {
        size_t b = 0;
        for (const DevBuf* x : bufs) b += x->bytes;
        return b;
    }
    void destroy() {
        if (!stream) return;
        cudaSetDevice(device);
        for (DevBuf* x : bufs) x->release();
        cudaStreamSynchronize(stream);
        spill_data.release();
        if (h_ctr) cudaFreeHost(h_ctr);
        if (h_pool) cudaFreeHost(h_pool);
        h_ctr = nullptr;
        h_pool = nullptr;
        cudaStreamDestroy(stream);
        stream = nullptr;
    }
};

int workspace_init(Workspace& w, int device, int sms);
struct Replay;   // a search captured as a CUDA graph (engine.cu)

struct DeviceState {
    bool init = false;
    int sms = 0;
    Workspace ws;
};

int device_state(int device, DeviceState** out);

}  // namespace kplex

// A set of preprocessed graphs resident on one device (one graph for
// kplex_prepare, many for kplex_prepare_batch).  Graph g's pruned vertices are
// [vbase, vbase + pn) of the concatenated CSR and its roots [root_base,
// root_base + nroots) of the concatenated root order.
struct kplex_prepared {
    int device = 0;
    int clock_khz = 0;               // the device's rated SM clock (cycle counters -> ms)
    cudaStream_t stream = nullptr;   // the workspace stream its buffers are ordered on
    kplex_params p{};
    uint32_t ngraphs = 0;
    uint32_t pn = 0, pm = 0, pn_max = 0, nroots = 0;
    double ms_pre = 0;
    std::vector<kplex::GraphInfo> ginfo;
    std::vector<uint32_t> gpm;
    uint32_t* d_off = nullptr;
    uint32_t* d_adj = nullptr;
    int32_t* d_dpos = nullptr;
    int32_t* d_dseq = nullptr;
    uint32_t* d_orig = nullptr;
    kplex::GraphInfo* d_graphs = nullptr;
    unsigned long long* d_gcount = nullptr;
    unsigned long long* d_ghash = nullptr;
    unsigned int* d_gvalid = nullptr;
    uint8_t* d_owner = nullptr;      // cost-weighted shard of each root (KPLEX_FLAG_SHARD_WEIGHTED)
    kplex::Replay* replay = nullptr;  // the captured form of this set's search, once it has run
};

namespace kplex {

struct HostJob {
    const uint32_t* off;
    const uint32_t* adj;
    uint32_t n;
    uint64_t m;
    int k, q, truss;
};

int check_kq(int k, int q);
void free_prepared(kplex_prepared* h);
// Validates, preprocesses and uploads a set of graphs on workspace d's stream.
int prepare_set(const std::vector<HostJob>& jobs, const kplex_params* p, Workspace* d, kplex_prepared** out_h,
                kplex_result* out);
// One search of a prepared set on workspace d; grid_div > 1 gives the persistent
// kernel 1/grid_div of the device so that concurrent workspaces share the SMs.
int search_impl(kplex_prepared* h, Workspace* d, kplex_result* out, kplex_result* per_graph = nullptr,
                uint32_t grid_div = 1);
double ms_since(std::chrono::steady_clock::time_point t0);

}  // namespace kplex
