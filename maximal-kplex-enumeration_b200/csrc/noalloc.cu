// kplex_search_noalloc: the device search with no device-memory allocation.
//
// Who needs it: callers that may not call cudaMalloc at all, or not after
// start-up. Three examples:
//  * a process whose device memory is already fully reserved by another
//    framework's caching allocator;
//  * a service with a fixed memory plan that forbids allocation on its
//    request path;
//  * code that must not trigger the implicit device synchronisation a
//    cudaMalloc/cudaFree can cause.
// kplex_enumerate_csr and kplex_search grow cached device buffers on demand.
// This entry point instead carves every scratch buffer from one file-scope
// __device__ array of NOALLOC_BYTES (64 MiB): counters, root descriptors,
// root arena, decomposition scratch, task pool and branch stacks.  The caller
// passes the inputs, i.e. the pruned graph from kplex_preprocess_csr in its
// own device buffers, and a host struct for the result.
//
// Host code must not hand the array's name to a kernel: on the host it is
// only a stand-in symbol.  The device address is fetched once per device with
// cudaGetSymbolAddress, on the first call made with that device current, and
// cached.  That first call should therefore happen before any stream capture.
// Every call reuses the same array, which keeps the previous call's
// contents; everything that must start at zero is cleared on each call.
// Two calls whose work overlaps on one GPU race on the array.
//
// The call works on cudaStreamPerThread, so the input buffers must be
// complete before it starts (written on that stream or on the legacy default
// stream, or synchronised); it returns after the search has finished.  It
// makes p->device current while it runs and restores the caller's device.
// ms_device is not measured (0); ms_total is the call's host wall time.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "device.cuh"

namespace kplex {

constexpr size_t NOALLOC_BYTES = 64ull << 20;
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_BYTES / 4];

__global__ void decompose_kernel(SearchParams sp);
__global__ void init_decomp_scratch(uint32_t* scratch, uint64_t words_per_warp, uint32_t pn, uint32_t nwarps);
__global__ void init_pool(uint32_t* seq, unsigned long long cap, Pool* pool);
__global__ void job_prefix_kernel(const RootDesc* roots, uint32_t nroots, uint32_t* job_base, unsigned int* work);
uint64_t decomp_scratch_words_host(uint32_t pn);
void set_last_error(const std::string& msg);

namespace {
std::mutex g_na_mu;
uint32_t* g_na_ptr[64] = {};   // device address of g_noalloc_scratch, per device
int g_na_sms[64] = {};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
}  // namespace

}  // namespace kplex

using namespace kplex;

#define NA_CK(call)                                                                 \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));     \
            if (out) out->status = KPLEX_ERR_CUDA;                                  \
            return KPLEX_ERR_CUDA;                                                  \
        }                                                                           \
    } while (0)

extern "C" int kplex_search_noalloc(const uint32_t* d_off, const uint32_t* d_adj, const int32_t* d_dpos,
                                    const int32_t* d_dseq, const uint32_t* d_orig, uint32_t pn,
                                    const kplex_params* p, kplex_result* out) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    const auto t0 = std::chrono::steady_clock::now();
    if (out) memset(out, 0, sizeof(*out));
    if (!p || !out || (pn && (!d_off || !d_dpos || !d_dseq || !d_orig))) { set_last_error("null argument"); return KPLEX_ERR_PARAM; }
    if (p->k < 2 || p->k > MAX_K - 1 || p->q < 2 * p->k - 1 || !(p->thres > 0.0f) || p->thres > 1.0f) {
        set_last_error("unsupported k/q/thres");
        return out->status = KPLEX_ERR_PARAM;
    }
    if (p->device < 0 || p->device >= 64) { set_last_error("bad device"); return out->status = KPLEX_ERR_PARAM; }
    // the caller's current device is restored on every return after this point
    int prev_device = -1;
    if (cudaGetDevice(&prev_device) != cudaSuccess) { cudaGetLastError(); prev_device = -1; }
    struct RestoreDevice {
        int d;
        ~RestoreDevice() { if (d >= 0) cudaSetDevice(d); }
    } restore{prev_device};
    auto finish = [&](int st) { out->status = st; return st; };
    NA_CK(cudaSetDevice(p->device));
    if (!g_na_ptr[p->device]) {   // set-up, once per device, with that device current
        void* ptr = nullptr;
        NA_CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        cudaDeviceProp prop;
        NA_CK(cudaGetDeviceProperties(&prop, p->device));
        if (prop.major != 10) { set_last_error("kernels are built for sm_100a only"); return finish(KPLEX_ERR_NO_DEVICE); }
        g_na_sms[p->device] = prop.multiProcessorCount;
        g_na_ptr[p->device] = static_cast<uint32_t*>(ptr);
    }
    uint8_t* base = reinterpret_cast<uint8_t*>(g_na_ptr[p->device]);
    const int sms = g_na_sms[p->device];
    cudaStream_t st = cudaStreamPerThread;

    const long long lim = (long long)pn - (long long)p->q + 2;   // src:44-45
    const uint32_t nroots = lim > 0 ? (uint32_t)std::min<long long>(lim, pn) : 0u;
    // ---- layout, phase 1: counters | pool header | roots | job prefix | arena ... | decomposition scratch (at the end)
    const uint64_t scratch_words = decomp_scratch_words_host(pn);
    // decomposition warps: two per SM, fewer when their scratch would take over half the array
    uint32_t dec_warps = std::max<uint32_t>(8, std::min<uint32_t>((uint32_t)sms * 2 / 8 * 8, ((nroots + 7) / 8) * 8));
    while (dec_warps > 8 && (size_t)dec_warps * scratch_words * 4 > NOALLOC_BYTES / 2) dec_warps = std::max<uint32_t>(8, dec_warps / 16 * 8);
    size_t off = 0;
    Counters* ctr = reinterpret_cast<Counters*>(base + off); off = align_up(off + sizeof(Counters), 256);
    Pool* pool = reinterpret_cast<Pool*>(base + off); off = align_up(off + sizeof(Pool), 256);
    RootDesc* roots = reinterpret_cast<RootDesc*>(base + off); off = align_up(off + (size_t)std::max<uint32_t>(nroots, 1) * sizeof(RootDesc), 256);
    uint32_t* job_base = reinterpret_cast<uint32_t*>(base + off); off = align_up(off + ((size_t)nroots + 1) * 4, 256);
    GraphInfo* graph = reinterpret_cast<GraphInfo*>(base + off); off = align_up(off + sizeof(GraphInfo), 256);
    unsigned long long* gres = reinterpret_cast<unsigned long long*>(base + off); off = align_up(off + 3 * 8, 256);
    const size_t dec_bytes = (size_t)dec_warps * scratch_words * 4;
    if (off + dec_bytes + (1u << 20) > NOALLOC_BYTES) {
        set_last_error("graph too large for the 64 MiB no-allocation scratch (pn = " + std::to_string(pn) + ")");
        return finish(KPLEX_ERR_NOMEM);
    }
    const size_t arena_off = off;
    const size_t dec_off = align_up(NOALLOC_BYTES - dec_bytes - 256, 256);

    SearchParams sp{};
    sp.nroots = nroots; sp.pn = pn;
    sp.graphs = graph; sp.ngraphs = 1;
    sp.gcount = gres; sp.ghash = gres + 1; sp.gvalid = reinterpret_cast<unsigned int*>(gres + 2);
    const GraphInfo gi{0u, pn, 0u, nroots, p->k, p->q, {0u, 0u}};
    sp.off = d_off; sp.adj = d_adj; sp.dpos = d_dpos; sp.dseq = d_dseq; sp.orig = d_orig;
    sp.roots = roots;
    sp.ctr = ctr;
    sp.arena = reinterpret_cast<uint32_t*>(base + arena_off);
    sp.arena_cap = (dec_off - arena_off) / 4;
    sp.warp_scratch = reinterpret_cast<uint32_t*>(base + dec_off);
    sp.scratch_words = scratch_words;
    sp.hash_on = (p->flags & KPLEX_FLAG_NO_HASH) ? 0u : 1u;
    sp.shard_index = p->shard_count > 1 ? p->shard_index : 0u;
    sp.shard_count = p->shard_count > 1 ? p->shard_count : 1u;
    sp.root_begin = p->root_end ? p->root_begin : 0u;
    sp.root_end = p->root_end ? p->root_end : 0xffffffffu;
    sp.spin_limit = 1ull << 24;
    if (p->flags & KPLEX_FLAG_TEST_NO_WAIT) {   // failure-detection test hook, as in kplex_enumerate_csr
        sp.test_stuck = 1;
        sp.spin_limit = 1u << 14;
    }
    uint32_t launches = 0;

    NA_CK(cudaMemsetAsync(ctr, 0, sizeof(Counters), st));
    NA_CK(cudaMemsetAsync(gres, 0, 3 * 8, st));
    NA_CK(cudaMemcpyAsync(graph, &gi, sizeof(GraphInfo), cudaMemcpyHostToDevice, st));
    Counters hc;
    memset(&hc, 0, sizeof hc);
    if (nroots) {
        init_decomp_scratch<<<sms * 4, 256, 0, st>>>(sp.warp_scratch, scratch_words, pn, dec_warps);
        decompose_kernel<<<dec_warps / 8, 256, 0, st>>>(sp);
        launches += 2;
        NA_CK(cudaGetLastError());
        NA_CK(cudaMemcpyAsync(&hc, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        NA_CK(cudaStreamSynchronize(st));
        if (hc.error) {
            set_last_error(hc.error == KPLEX_ERR_NOMEM      ? "root arena exceeds the 64 MiB no-allocation scratch"
                           : hc.error == KPLEX_ERR_CAPACITY ? "a root's 2-hop subgraph exceeds 2048 vertices or its left set 8192"
                                                            : "device error in decomposition");
            return finish((int)hc.error);
        }
        job_prefix_kernel<<<1, 1024, 0, st>>>(roots, nroots, job_base, &ctr->work);
        ++launches;
        uint32_t njobs = 0;
        NA_CK(cudaMemcpyAsync(&njobs, job_base + nroots, 4, cudaMemcpyDeviceToHost, st));
        NA_CK(cudaStreamSynchronize(st));
        sp.njobs = njobs;
    }
    sp.job_base = job_base;
    // ---- phase 2: the decomposition scratch is dead; pool and stacks follow the used arena
    const uint32_t nmax = std::max<uint32_t>(hc.max_n, 1);
    const uint32_t Wt = std::max<uint32_t>(hc.max_w, 4);
    sp.Wt = Wt;
    sp.slot_words = 4 + 3 * Wt;
    size_t o2 = align_up(arena_off + (size_t)hc.arena_top * 4, 256);
    const int warps_per_block = SEARCH_WARPS;
    sp.a_words = 0;
    const uint32_t nw = search_words_per_lane(Wt);
    const SearchKernel kfn = search_kernel_for(nw, 3);
    const size_t smem_bytes = (size_t)(ks_slot_words_host(nmax, sp.slot_words, nw) +
                                       warps_per_block * bnb_smem_words_host(nmax, sp.slot_words, 0, nw)) * 4;
    NA_CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    int per_sm = 0;
    NA_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, warps_per_block * 32, smem_bytes));
    uint32_t blocks = (uint32_t)sms * (uint32_t)std::max(per_sm, 1);
    sp.stack_depth = 4;   // a power of two of at least nmax + 2
    while (sp.stack_depth < nmax + 2) sp.stack_depth *= 2;
    const size_t stack_per_warp = (size_t)sp.stack_depth * sp.slot_words * 4;
    const size_t rec_bytes = (size_t)sp.slot_words * 4 + 4;
    const size_t min_slots = 4096;
    while (blocks > 1 && o2 + (size_t)blocks * warps_per_block * stack_per_warp + min_slots * rec_bytes > NOALLOC_BYTES) blocks /= 2;
    const size_t stacks_bytes = (size_t)blocks * warps_per_block * stack_per_warp;
    if (o2 + stacks_bytes + min_slots * rec_bytes + 512 > NOALLOC_BYTES) {
        set_last_error("task pool and stacks do not fit the 64 MiB no-allocation scratch");
        return finish(KPLEX_ERR_NOMEM);
    }
    sp.stacks = reinterpret_cast<uint32_t*>(base + o2);
    o2 = align_up(o2 + stacks_bytes, 256);
    const unsigned long long fit = std::min<unsigned long long>((NOALLOC_BYTES - o2 - 512) / rec_bytes, 1ull << 20);
    unsigned long long cap = 1;   // a ring's capacity is a power of two
    while (cap * 2 <= fit) cap *= 2;
    sp.pool = pool;
    sp.pool_seq = reinterpret_cast<uint32_t*>(base + o2);
    o2 = align_up(o2 + (size_t)cap * 4, 256);
    sp.pool_data = reinterpret_cast<uint32_t*>(base + o2);
    sp.nwarps = blocks * warps_per_block;
    sp.low_water = 2 * sp.nwarps;
    const long long pause = (long long)std::floor((double)cap * (double)p->thres) - (long long)blocks;
    sp.pause_at = (unsigned long long)std::max<long long>(pause, 1);
    init_pool<<<sms * 4, 256, 0, st>>>(sp.pool_seq, cap, sp.pool);
    ++launches;
    if (nroots) {
        kfn<<<blocks, warps_per_block * 32, smem_bytes, st>>>(sp, nmax);
        ++launches;
        NA_CK(cudaGetLastError());
    }
    Pool hp;
    NA_CK(cudaMemcpyAsync(&hc, ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&hp, pool, sizeof(Pool), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    int status = (int)hc.error;
    // a bounded wait that gave up may leave work in k-search jobs, block queues or warp
    // stacks while the pool itself is empty: the work counter covers all of them
    if (!status && nroots && (hp.head != hp.tail || hc.work != 0 || hc.timeouts != 0)) {
        status = KPLEX_ERR_TIMEOUT;
        set_last_error("branch warps gave up with work left");
    }
    out->count = hc.count;
    out->hash = hc.hash;
    out->valid_roots = hc.valid_roots;
    out->tasks = hc.tasks;
    out->nodes = hc.nodes;
    out->pn = pn;
    out->max_local_n = hc.max_n;
    out->max_left = hc.max_left;
    out->pauses = hc.ks_paused;
    out->gpu_launches = launches;
    out->bnb_bytes = hc.bnb_bytes;
    out->roots_bytes = hc.roots_bytes;
    out->ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out->ms_device = 0;   // not measured here (ms_total is the host wall time of the call)
    return finish(status);
}
