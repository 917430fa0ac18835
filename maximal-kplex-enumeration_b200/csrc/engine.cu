// Host engine: the C ABI of include/kplex.h.
//
// Replaces decomposableSearch (inc/host_funcs.h:722-1161).  The reference
// allocates ~40 GB of fixed per-warp slabs (inc/gpu_memory_allocation.h:10-63,
// host:916-1011), launches five kernels per wave of 4,544 roots and reads a
// flag back after every BNB wave (host:253-335).  Here one search is:
//   decompose_kernel  all roots at once into a bump-allocated arena
//   search_kernel     persistent: producer warps run k-search into the task pool
//                     (pausing on the device at thres * capacity records), consumer
//                     warps drain it depth-first (pause-and-resume, host:1094-1122,
//                     without a host round trip)
// with two 128-byte counter reads in total.  Device buffers are cached
// per device and grown on demand.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "graph_io.h"
#include "preprocess.h"

namespace kplex {

__global__ void decompose_kernel(SearchParams sp);
__global__ void job_prefix_kernel(const RootDesc* roots, uint32_t nroots, uint32_t* job_base, unsigned int* work);
uint64_t decomp_scratch_words_host(uint32_t pn);

// ------------------------------------------------------------------ small kernels
__global__ void init_decomp_scratch(uint32_t* scratch, uint64_t words_per_warp, uint32_t pn, uint32_t nwarps) {
    const uint64_t total = (uint64_t)nwarps * 2 * pn;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t w = i / (2ull * pn), o = i % (2ull * pn);
        scratch[w * words_per_warp + o] = (o < pn) ? 0xffffffffu : 0u;
    }
}
__global__ void init_pool(uint32_t* seq, unsigned long long cap, Pool* pool) {
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < cap; i += (unsigned long long)gridDim.x * blockDim.x)
        seq[i] = (uint32_t)i;
    if (blockIdx.x == 0 && threadIdx.x == 0) { pool->head = 0; pool->tail = 0; pool->cap = cap; pool->pad = 0; }
}
__global__ void init_ks_slots(uint32_t* slots, uint32_t nwarps, uint32_t words) {
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nwarps; w += gridDim.x * blockDim.x) slots[(uint64_t)w * words] = 0xffffffffu;
}

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

int workspace_init(Workspace& w, int device, int sms) {
    w.device = device;
    w.sms = sms;
    CK(cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking));
    CK(cudaMallocHost(&w.h_ctr, sizeof(Counters)));
    CK(cudaMallocHost(&w.h_pool, sizeof(Pool)));
    for (DevBuf* x : w.bufs) x->stream = w.stream;
    return KPLEX_OK;
}

static std::mutex g_mu;
static DeviceState g_dev[64];

int device_state(int device, DeviceState** out) {
    if (device < 0 || device >= 64) return KPLEX_ERR_PARAM;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device >= n) { cudaGetLastError(); g_last_error = "no CUDA device"; return KPLEX_ERR_NO_DEVICE; }
    CK(cudaSetDevice(device));
    DeviceState& d = g_dev[device];
    if (!d.init) {
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10) { g_last_error = "kernels are built for sm_100a only"; return KPLEX_ERR_NO_DEVICE; }
        d.sms = prop.multiProcessorCount;
        // the dynamic shared-memory cap is raised once to the per-block maximum, so
        // that concurrent searches never race on a per-function attribute
        for (uint32_t nw : {1u, 2u})
            for (int minb : {2, 3})
                CK(cudaFuncSetAttribute(search_kernel_for(nw, minb), cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
        int rc = workspace_init(d.ws, device, d.sms);
        if (rc) return rc;
        d.init = true;
    }
    *out = &d;
    return KPLEX_OK;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace kplex

using namespace kplex;

namespace kplex {

// A prepared set's search captured as one CUDA graph (memsets, decomposition,
// job prefix, pool init, the persistent search kernel and the result copies),
// built on the second search of the set once the first has fixed every size
// (arena, pool, stacks, shared memory, grid) and replayed with one launch and
// one synchronisation from then on.  Valid while the workspace keeps its
// buffers (generation) and the set keeps its parameters.
struct Replay {
    Workspace* ws = nullptr;
    uint64_t gen = 0;
    kplex_params p{};
    uint32_t grid_div = 1;
    SearchParams sp{};
    uint32_t dec_warps = 0, blocks = 0, nmax = 0, launches = 0;
    size_t smem = 0;
    SearchKernel kfn = nullptr;
    unsigned long long cap = 0, scap = 0;
    cudaGraphExec_t exec = nullptr;
    bool exec_per_graph = false;
    cudaEvent_t ev[6] = {};
    unsigned long long* h_gc = nullptr;   // pinned per-graph results
    unsigned long long* h_gh = nullptr;
    unsigned int* h_gv = nullptr;
    ~Replay() {
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : ev) if (e) cudaEventDestroy(e);
        if (h_gc) cudaFreeHost(h_gc);
        if (h_gh) cudaFreeHost(h_gh);
        if (h_gv) cudaFreeHost(h_gv);
    }
};

int check_kq(int k, int q) {
    if (k < 2 || k > MAX_K - 1) { g_last_error = "k must be in [2, 31]"; return KPLEX_ERR_PARAM; }
    if (q < 2 * k - 1) { g_last_error = "q must be >= 2k-1"; return KPLEX_ERR_PARAM; }
    return KPLEX_OK;
}

static int check_params(const kplex_params* p) {
    if (!p) { g_last_error = "null params"; return KPLEX_ERR_PARAM; }
    int rc = check_kq(p->k, p->q);
    if (rc) return rc;
    if (!(p->thres > 0.0f) || p->thres > 1.0f) { g_last_error = "thres must be in (0, 1]"; return KPLEX_ERR_PARAM; }
    return KPLEX_OK;
}

void free_prepared(kplex_prepared* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    delete h->replay;
    void* ps[10] = {h->d_off, h->d_adj, h->d_dpos, h->d_dseq, h->d_orig, h->d_graphs, h->d_gcount, h->d_ghash, h->d_gvalid,
                    h->d_owner};
    for (void* x : ps) if (x) cudaFreeAsync(x, h->stream);
    delete h;
}

// Validates, preprocesses (one host thread per graph when there are several)
// and uploads a set of graphs.
int prepare_set(const std::vector<HostJob>& jobs, const kplex_params* p, Workspace* d, kplex_prepared** out_h,
                       kplex_result* out) {
    if (!p || !(p->thres > 0.0f) || p->thres > 1.0f) { g_last_error = "thres must be in (0, 1]"; return KPLEX_ERR_PARAM; }
    const size_t G = jobs.size();
    for (const HostJob& j : jobs) {
        int rc = check_kq(j.k, j.q);
        if (rc) return rc;
        if (!j.off || (!j.adj && j.m) || (j.n && j.off[j.n] != j.m) || j.m > 0xffffffffull) { g_last_error = "inconsistent CSR"; return KPLEX_ERR_FORMAT; }
    }
    CK(cudaSetDevice(d->device));
    auto t0 = std::chrono::steady_clock::now();
    std::vector<Prepped> pres(G);
    std::vector<int> status(G, KPLEX_OK);
    std::vector<std::string> errs(G);
    auto one = [&](size_t g, int threads) {
        const HostJob& j = jobs[g];
        Csr c;
        c.n = j.n;
        c.off.assign(j.off, j.off + j.n + 1);
        c.adj.assign(j.adj, j.adj + j.m);
        status[g] = validate_csr(c, &errs[g]);
        if (status[g] == KPLEX_OK) preprocess(c, j.k, j.q, j.truss, threads, pres[g]);
    };
    if (G == 1) one(0, (int)p->omp_threads);
    else {
#pragma omp parallel for schedule(dynamic, 1)
        for (long long g = 0; g < (long long)G; ++g) one((size_t)g, 1);
    }
    for (size_t g = 0; g < G; ++g) if (status[g]) { g_last_error = errs[g]; return status[g]; }
    const double ms_pre = ms_since(t0);
    if (G == 1 && !(p->flags & KPLEX_FLAG_QUIET)) printf("\npn = %u\n", pres[0].g.n);

    kplex_prepared* h = new kplex_prepared();
    h->device = d->device;
    h->stream = d->stream;
    if (cudaDeviceGetAttribute(&h->clock_khz, cudaDevAttrClockRate, d->device) != cudaSuccess) { cudaGetLastError(); h->clock_khz = 0; }
    h->p = *p;
    h->ngraphs = (uint32_t)G;
    h->ms_pre = ms_pre;
    h->ginfo.resize(G);
    h->gpm.resize(G);
    uint64_t PN = 0, PM = 0, R = 0;
    for (size_t g = 0; g < G; ++g) {
        const Prepped& pr = pres[g];
        const uint32_t pn = pr.g.n, pm = pn ? pr.g.off[pn] : 0;
        const long long lim = (long long)pn - (long long)jobs[g].q + 2;   // src:44-45
        const uint32_t nr = lim > 0 ? (uint32_t)std::min<long long>(lim, pn) : 0u;
        h->ginfo[g] = GraphInfo{(uint32_t)PN, pn, (uint32_t)R, nr, jobs[g].k, jobs[g].q, {0, 0}};
        h->gpm[g] = pm;
        h->pn_max = std::max(h->pn_max, pn);
        PN += pn; PM += pm; R += nr;
    }
    if (PN > 0x7fffffffull || PM > 0xffffffffull || R > 0x7fffffffull) { delete h; g_last_error = "batch too large"; return KPLEX_ERR_PARAM; }
    h->pn = (uint32_t)PN; h->pm = (uint32_t)PM; h->nroots = (uint32_t)R;
    std::vector<uint32_t> off(PN + 1), adj(std::max<uint64_t>(PM, 1)), orig(std::max<uint64_t>(PN, 1));
    std::vector<int32_t> dpos(std::max<uint64_t>(PN, 1)), dseq(std::max<uint64_t>(R, 1));
    uint64_t eb = 0;
    for (size_t g = 0; g < G; ++g) {
        const Prepped& pr = pres[g];
        const GraphInfo& gi = h->ginfo[g];
        for (uint32_t i = 0; i < gi.pn; ++i) {
            off[gi.vbase + i] = (uint32_t)(eb + pr.g.off[i]);
            dpos[gi.vbase + i] = pr.dpos[i];
            orig[gi.vbase + i] = pr.orig[i];
        }
        for (uint32_t e = 0; e < h->gpm[g]; ++e) adj[eb + e] = gi.vbase + pr.g.adj[e];
        for (uint32_t r = 0; r < gi.nroots; ++r) dseq[gi.root_base + r] = (int32_t)(gi.vbase + (uint32_t)pr.dseq[r]);
        eb += h->gpm[g];
    }
    off[PN] = (uint32_t)PM;
    auto fail = [&](int code) { free_prepared(h); return code; };
    auto dm = [&](auto** ptr, size_t bytes) { return cudaMallocAsync((void**)ptr, bytes, d->stream) == cudaSuccess; };
    if (!dm(&h->d_off, (PN + 1) * 4) || !dm(&h->d_adj, adj.size() * 4) || !dm(&h->d_dpos, dpos.size() * 4) ||
        !dm(&h->d_dseq, dseq.size() * 4) || !dm(&h->d_orig, orig.size() * 4) || !dm(&h->d_graphs, G * sizeof(GraphInfo)) ||
        !dm(&h->d_gcount, G * 8) || !dm(&h->d_ghash, G * 8) || !dm(&h->d_gvalid, G * 4)) {
        cudaGetLastError(); g_last_error = "cudaMalloc for the pruned graphs failed"; return fail(KPLEX_ERR_NOMEM);
    }
    CK(cudaMemcpyAsync(h->d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(h->d_adj, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(h->d_dpos, dpos.data(), dpos.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(h->d_dseq, dseq.data(), dseq.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(h->d_orig, orig.data(), orig.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CK(cudaMemcpyAsync(h->d_graphs, h->ginfo.data(), G * sizeof(GraphInfo), cudaMemcpyHostToDevice, d->stream));
    std::vector<uint8_t> owner;
    if ((p->flags & KPLEX_FLAG_SHARD_WEIGHTED) && p->shard_count > 1) {
        // cost-weighted shards: every graph's roots, each graph partitioned on its own
        if (p->shard_count > 255) { g_last_error = "at most 255 weighted shards"; return fail(KPLEX_ERR_PARAM); }
        owner.assign(std::max<uint64_t>(R, 1), 0);
        for (size_t g = 0; g < G; ++g)
            weighted_root_owners(pres[g].g, pres[g].dpos, pres[g].dseq, h->ginfo[g].nroots, p->shard_count,
                                 owner.data() + h->ginfo[g].root_base);
        if (!dm(&h->d_owner, owner.size())) { cudaGetLastError(); g_last_error = "cudaMalloc for the root owners failed"; return fail(KPLEX_ERR_NOMEM); }
        CK(cudaMemcpyAsync(h->d_owner, owner.data(), owner.size(), cudaMemcpyHostToDevice, d->stream));
    }
    CK(cudaStreamSynchronize(d->stream));
    if (out) { out->pn = h->pn; out->pm = h->pm; out->ms_preprocess = ms_pre; }
    *out_h = h;
    return KPLEX_OK;
}

static int prepare_impl(const uint32_t* off, const uint32_t* adj, uint32_t n, uint64_t m, const kplex_params* p,
                        kplex_prepared** out_h, kplex_result* out) {
    int rc = check_params(p);
    if (rc) return rc;
    DeviceState* dev = nullptr;
    if ((rc = device_state(p->device, &dev))) return rc;
    return prepare_set({HostJob{off, adj, n, m, p->k, p->q, p->truss}}, p, &dev->ws, out_h, out);
}

static bool same_params(const kplex_params& a, const kplex_params& b) {
    return a.k == b.k && a.q == b.q && a.thres == b.thres && a.truss == b.truss && a.flags == b.flags &&
           a.device == b.device && a.pool_slots == b.pool_slots && a.shard_index == b.shard_index &&
           a.shard_count == b.shard_count && a.blocks_per_sm == b.blocks_per_sm && a.stage_after == b.stage_after &&
           a.root_begin == b.root_begin && a.root_end == b.root_end;
}

static void fill_result(const kplex_prepared* h, const Counters& hc, float ms, double ms_dec, double ms_bnb,
                        uint32_t launches, uint32_t search_warps, kplex_result* out) {
    if (!out) return;
    out->count = hc.count;
    out->hash = hc.hash;
    out->valid_roots = hc.valid_roots;
    out->tasks = hc.tasks;
    out->nodes = hc.nodes;
    out->pn = h->pn;
    out->pm = h->pm;
    out->max_local_n = hc.max_n;
    out->max_left = hc.max_left;
    out->pauses = hc.ks_paused;
    out->spilled = (uint32_t)std::min<unsigned long long>(hc.spilled, 0xffffffffull);
    out->ms_preprocess = h->ms_pre;
    out->ms_device = ms;
    out->ms_ref_region = h->ms_pre + ms;
    out->gpu_launches = launches;
    out->ms_decompose = ms_dec;
    out->ms_ksearch = 0;
    out->ms_bnb = ms_bnb;
    out->bnb_bytes = hc.bnb_bytes;
    out->roots_bytes = hc.roots_bytes;
    out->ks_tasks = hc.ks_tasks;
    out->stage_copies = hc.stage_copies;
    // SM cycles converted at the device's rated clock; their ratios (the shares of warp
    // time) do not depend on the clock the run actually saw
    const double khz = h->clock_khz > 0 ? (double)h->clock_khz : 1.965e6;
    out->ks_warp_ms = (double)hc.ks_cycles / khz;
    out->bnb_warp_ms = (double)hc.bnb_cycles / khz;
    out->idle_warp_ms = (double)hc.idle_cycles / khz;
    out->search_warps = search_warps;
    out->status = (int)hc.error;
}

static int replay_capture(kplex_prepared* h, Replay& r, Workspace* d, bool per_graph) {
    cudaStream_t st = d->stream;
    const SearchParams& sp = r.sp;
    const size_t G = h->ngraphs;
    if (r.exec) { cudaGraphExecDestroy(r.exec); r.exec = nullptr; }
    for (cudaEvent_t& e : r.ev) if (!e) CK(cudaEventCreate(&e));
    if (per_graph && !r.h_gc) {
        CK(cudaMallocHost(&r.h_gc, G * 8));
        CK(cudaMallocHost(&r.h_gh, G * 8));
        CK(cudaMallocHost(&r.h_gv, G * 4));
    }
    const SearchKernel kfn = r.kfn;
    // events become event-record nodes of the graph (external records), so that the
    // host can wait on the last one and time the phases after a replay
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaEventRecordWithFlags(r.ev[0], st, cudaEventRecordExternal);
    cudaMemsetAsync(sp.ctr, 0, sizeof(Counters), st);
    cudaMemsetAsync(sp.gcount, 0, G * 8, st);
    cudaMemsetAsync(sp.ghash, 0, G * 8, st);
    cudaMemsetAsync(sp.gvalid, 0, G * 4, st);
    if (h->nroots) {
        init_decomp_scratch<<<d->sms * 4, 256, 0, st>>>(sp.warp_scratch, sp.scratch_words, h->pn_max, r.dec_warps);
        cudaEventRecordWithFlags(r.ev[1], st, cudaEventRecordExternal);
        decompose_kernel<<<r.dec_warps / 8, 256, 0, st>>>(sp);
        cudaEventRecordWithFlags(r.ev[2], st, cudaEventRecordExternal);
    }
    job_prefix_kernel<<<1, 1024, 0, st>>>(sp.roots, h->nroots, d->jobs.as<uint32_t>(), &sp.ctr->work);
    init_pool<<<d->sms * 4, 256, 0, st>>>(sp.pool_seq, r.cap, sp.pool);
    if (sp.spill_on) init_pool<<<d->sms * 4, 256, 0, st>>>(sp.spill_seq, r.scap, sp.spill_pool);
    cudaEventRecordWithFlags(r.ev[3], st, cudaEventRecordExternal);
    if (h->nroots) kfn<<<r.blocks, SEARCH_WARPS * 32, r.smem, st>>>(sp, r.nmax);
    cudaEventRecordWithFlags(r.ev[4], st, cudaEventRecordExternal);
    cudaMemcpyAsync(d->h_ctr, sp.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(d->h_pool, sp.pool, sizeof(Pool), cudaMemcpyDeviceToHost, st);
    if (per_graph) {
        cudaMemcpyAsync(r.h_gc, sp.gcount, G * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(r.h_gh, sp.ghash, G * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(r.h_gv, sp.gvalid, G * 4, cudaMemcpyDeviceToHost, st);
    }
    cudaEventRecordWithFlags(r.ev[5], st, cudaEventRecordExternal);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (ce != cudaSuccess || !g) {
        cudaGetLastError();
        g_last_error = std::string("stream capture of the search: ") + cudaGetErrorString(ce);
        return KPLEX_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&r.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) { cudaGetLastError(); r.exec = nullptr; g_last_error = std::string("graph instantiate: ") + cudaGetErrorString(ie); return KPLEX_ERR_CUDA; }
    r.exec_per_graph = per_graph;
    return KPLEX_OK;
}

static int replay_search(kplex_prepared* h, Replay& r, Workspace* d, kplex_result* out, kplex_result* per_graph) {
    int rc = KPLEX_OK;
    if (!r.exec || (per_graph && !r.exec_per_graph))
        if ((rc = replay_capture(h, r, d, per_graph != nullptr))) return rc;
    CK(cudaGraphLaunch(r.exec, d->stream));
    CK(cudaEventSynchronize(r.ev[5]));
    Counters& hc = *d->h_ctr;
    const Pool& hp = *d->h_pool;
    float ms = 0, t_dec = 0, t_bnb = 0;
    CK(cudaEventElapsedTime(&ms, r.ev[0], r.ev[5]));
    if (h->nroots) CK(cudaEventElapsedTime(&t_dec, r.ev[1], r.ev[2]));
    CK(cudaEventElapsedTime(&t_bnb, r.ev[3], r.ev[4]));
    if (!hc.error && (hp.head != hp.tail || hc.work != 0)) { hc.error = KPLEX_ERR_TIMEOUT; g_last_error = "branch warps gave up with work left"; }
    if (hc.error && g_last_error.empty()) g_last_error = "device error in a replayed search";
    if (per_graph) {
        for (size_t g = 0; g < h->ngraphs; ++g) {
            kplex_result& x = per_graph[g];
            memset(&x, 0, sizeof x);
            x.count = r.h_gc[g]; x.hash = r.h_gh[g]; x.valid_roots = r.h_gv[g];
            x.pn = h->ginfo[g].pn; x.pm = h->gpm[g];
            x.status = (int)hc.error;
        }
    }
    fill_result(h, hc, ms, t_dec, t_bnb, r.launches, r.blocks * SEARCH_WARPS, out);
    return (int)hc.error;
}

int search_impl(kplex_prepared* h, Workspace* d, kplex_result* out, kplex_result* per_graph, uint32_t grid_div) {
    int rc = KPLEX_OK;
    if (h->replay) {
        Replay& r = *h->replay;
        if (r.ws == d && r.gen == d->generation() && r.grid_div == grid_div && same_params(r.p, h->p)) {
            CK(cudaSetDevice(d->device));
            rc = replay_search(h, r, d, out, per_graph);
            if (rc) { delete h->replay; h->replay = nullptr; }
            return rc;
        }
        delete h->replay;
        h->replay = nullptr;
    }
    CK(cudaSetDevice(d->device));
    const kplex_params& P = h->p;
    cudaStream_t st = d->stream;
    const uint32_t nroots = h->nroots;
    uint32_t launches = 0;
    struct Events {   // destroyed on every return path
        cudaEvent_t e[4] = {};
        ~Events() { for (cudaEvent_t x : e) if (x) cudaEventDestroy(x); }
    } evs;
    for (cudaEvent_t& x : evs.e) CK(cudaEventCreate(&x));
    cudaEvent_t e0 = evs.e[0], e1 = evs.e[1], ka = evs.e[2], kb = evs.e[3];
    CK(cudaEventRecord(e0, st));
    double ms_dec = 0, ms_bnb = 0;
    auto timed = [&](auto&& launch, double& acc) -> int {
        CK(cudaEventRecord(ka, st));
        launch();
        CK(cudaGetLastError());
        CK(cudaEventRecord(kb, st));
        CK(cudaEventSynchronize(kb));
        float t = 0;
        CK(cudaEventElapsedTime(&t, ka, kb));
        acc += t;
        return KPLEX_OK;
    };

    SearchParams sp{};
    sp.nroots = nroots; sp.pn = h->pn_max;
    sp.off = h->d_off; sp.adj = h->d_adj; sp.dpos = h->d_dpos; sp.dseq = h->d_dseq; sp.orig = h->d_orig;
    sp.graphs = h->d_graphs; sp.ngraphs = h->ngraphs;
    sp.gcount = h->d_gcount; sp.ghash = h->d_ghash; sp.gvalid = h->d_gvalid;
    sp.hash_on = (P.flags & KPLEX_FLAG_NO_HASH) ? 0u : 1u;
    sp.shard_index = P.shard_count > 1 ? P.shard_index : 0u;
    sp.shard_count = P.shard_count > 1 ? P.shard_count : 1u;
    sp.root_begin = P.root_end ? P.root_begin : 0u;
    sp.root_end = P.root_end ? P.root_end : 0xffffffffu;
    sp.root_owner = h->d_owner;
    sp.spin_limit = 1ull << 24;

    if ((rc = d->ctr.ensure(sizeof(Counters)))) return rc;
    if ((rc = d->roots.ensure(std::max<size_t>(nroots, 1) * sizeof(RootDesc)))) return rc;
    sp.ctr = d->ctr.as<Counters>();
    sp.roots = d->roots.as<RootDesc>();

    // ---------------- decomposition (with arena growth on overflow)
    const uint32_t dec_warps = std::max<uint32_t>(8, std::min<uint32_t>((uint32_t)d->sms * 16, ((nroots + 7) / 8) * 8));
    sp.scratch_words = decomp_scratch_words_host(h->pn_max);
    if ((rc = d->scratch.ensure((size_t)dec_warps * sp.scratch_words * 4))) return rc;
    sp.warp_scratch = d->scratch.as<uint32_t>();
    size_t arena_words = std::max<size_t>(d->arena.bytes / 4, (size_t)1 << 22);
    Counters& hc = *d->h_ctr;
    for (int attempt = 0;; ++attempt) {
        if ((rc = d->arena.ensure(arena_words * 4))) return rc;
        sp.arena = d->arena.as<uint32_t>();
        sp.arena_cap = arena_words;
        CK(cudaMemsetAsync(sp.ctr, 0, sizeof(Counters), st));
        CK(cudaMemsetAsync(sp.gcount, 0, (size_t)h->ngraphs * 8, st));
        CK(cudaMemsetAsync(sp.ghash, 0, (size_t)h->ngraphs * 8, st));
        CK(cudaMemsetAsync(sp.gvalid, 0, (size_t)h->ngraphs * 4, st));
        if (nroots) {
            init_decomp_scratch<<<d->sms * 4, 256, 0, st>>>(sp.warp_scratch, sp.scratch_words, h->pn_max, dec_warps);
            if ((rc = timed([&] { decompose_kernel<<<dec_warps / 8, 256, 0, st>>>(sp); }, ms_dec))) return rc;
            launches += 2;
        }
        CK(cudaMemcpyAsync(&hc, sp.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (hc.error == KPLEX_ERR_NOMEM && attempt < 6) {
            arena_words = std::max<size_t>(arena_words * 2, (size_t)(hc.arena_top * 5 / 4 + 1024));
            continue;
        }
        break;
    }
    if (hc.error) {
        g_last_error = hc.error == KPLEX_ERR_CAPACITY ? "a root's 2-hop subgraph exceeds 2048 vertices or its left set 8192"
                                                      : "device error in decomposition";
        if (out) {   // the sizes that failed, for the caller's message
            out->max_local_n = hc.max_n;
            out->max_left = hc.max_left;
            out->valid_roots = hc.valid_roots;
        }
        return (int)hc.error;
    }
    // k-search jobs: a valid root with |C2| = n - hop owns |C2| + 1 independent jobs
    if ((rc = d->jobs.ensure(((size_t)nroots + 1) * 4))) return rc;
    sp.job_base = d->jobs.as<uint32_t>();
    job_prefix_kernel<<<1, 1024, 0, st>>>(sp.roots, nroots, d->jobs.as<uint32_t>(), &sp.ctr->work);
    ++launches;
    uint32_t njobs = 0;
    CK(cudaMemcpyAsync(&njobs, d->jobs.as<uint32_t>() + nroots, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    sp.njobs = njobs;
    const uint32_t nmax = std::max<uint32_t>(hc.max_n, 1);
    const uint32_t Wt = std::max<uint32_t>(hc.max_w, 4);
    sp.Wt = Wt;
    sp.slot_words = 4 + 3 * Wt;

    // ---------------- pool, k-search slots, branch stacks
    // MAX_CAP (inc/common.h:10) by default; a ring's capacity is a power of two
    unsigned long long cap = 4;
    while (cap < (P.pool_slots ? P.pool_slots : 4194304ull)) cap *= 2;
    if ((rc = d->pool.ensure(sizeof(Pool)))) return rc;
    if ((rc = d->pool_seq.ensure((size_t)cap * 4))) return rc;
    if ((rc = d->pool_data.ensure((size_t)cap * sp.slot_words * 4))) return rc;
    sp.pool = d->pool.as<Pool>();
    sp.pool_seq = d->pool_seq.as<uint32_t>();
    sp.pool_data = d->pool_data.as<uint32_t>();
    init_pool<<<d->sms * 4, 256, 0, st>>>(sp.pool_seq, cap, sp.pool);
    ++launches;
    const int warps_per_block = SEARCH_WARPS;
    // schedule knobs, from kplex_params only: blocks per SM the kernel is compiled for
    // (2 or 3) and how many nodes a warp processes on one root before copying its A to
    // shared memory
    const int minb = P.blocks_per_sm == 3 ? 3 : 2;   // measured: 2 blocks x 128 registers beats 3 x 80 + spills
    const int stage_after = P.stage_after ? P.stage_after : 8;
    sp.stage_after = stage_after > 0 ? (uint32_t)stage_after : 0u;
    // one bitset word per lane while every root fits 1024 vertices, two beyond
    const uint32_t nw = search_words_per_lane(hc.max_w);
    const SearchKernel kfn = search_kernel_for(nw, minb);
    // stage adjacency matrices in shared memory when minb blocks still fit on an SM
    int per_sm = 0;
    size_t smem_bytes = 0;
    for (int stage = sp.stage_after ? 1 : 0; stage >= 0; --stage) {
        sp.a_words = stage ? ((hc.max_nw + 3u) & ~3u) : 0u;
        smem_bytes = (size_t)(ks_slot_words_host(nmax, sp.slot_words, nw) +
                              warps_per_block * bnb_smem_words_host(nmax, sp.slot_words, sp.a_words, nw)) * 4;
        if (smem_bytes > 227 * 1024) continue;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, warps_per_block * 32, smem_bytes));
        if (per_sm >= minb || !stage) break;
    }
    per_sm = std::max(per_sm, 1);
    const uint32_t blocks = std::max<uint32_t>(1u, (uint32_t)d->sms * (uint32_t)per_sm / std::max<uint32_t>(grid_div, 1u));
    const uint32_t nwarps = blocks * warps_per_block;
    sp.nwarps = nwarps;
    sp.stack_depth = 4;   // a power of two of at least nmax + 2 (DFS depth is bounded by |C| <= n)
    while (sp.stack_depth < nmax + 2) sp.stack_depth *= 2;
    sp.low_water = nwarps;
    // the reference pauses at MAX_CAP * thres - WARPS (src:2083, 2384): one record of slack per producer
    const long long pause = (long long)std::floor((double)cap * (double)P.thres) - (long long)blocks;
    sp.pause_at = (unsigned long long)std::max<long long>(pause, 1);
    if ((rc = d->stacks.ensure((size_t)nwarps * sp.stack_depth * sp.slot_words * 4))) return rc;
    sp.stacks = d->stacks.as<uint32_t>();
    unsigned long long scap_used = 0;
    if (P.flags & KPLEX_FLAG_SPILL_HOST) {
        // spill ring: control and sequence words in HBM, records in mapped pinned host memory
        const unsigned long long scap = std::min<unsigned long long>(4 * cap, 1ull << 24);
        scap_used = scap;
        if ((rc = d->spill_ctl.ensure(sizeof(Pool)))) return rc;
        if ((rc = d->spill_seq.ensure((size_t)scap * 4))) return rc;
        if ((rc = d->spill_data.ensure((size_t)scap * sp.slot_words * 4))) return rc;
        sp.spill_pool = d->spill_ctl.as<Pool>();
        sp.spill_seq = d->spill_seq.as<uint32_t>();
        sp.spill_data = static_cast<uint32_t*>(d->spill_data.d);
        sp.spill_on = 1;
        sp.spill_pause_at = scap > blocks ? scap - blocks : 1;
        init_pool<<<d->sms * 4, 256, 0, st>>>(sp.spill_seq, scap, sp.spill_pool);
        ++launches;
    }
    if (P.flags & KPLEX_FLAG_TEST_NO_WAIT) {   // failure-detection test hook
        sp.test_stuck = 1;
        sp.spin_limit = 1u << 14;
    }

    // ---------------- k-search + branch-and-bound, one persistent launch
    if (nroots) {
        if ((rc = timed([&] { kfn<<<blocks, warps_per_block * 32, smem_bytes, st>>>(sp, nmax); }, ms_bnb))) return rc;
        ++launches;
    }
    CK(cudaMemcpyAsync(&hc, sp.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    Pool hp;
    CK(cudaMemcpyAsync(&hp, sp.pool, sizeof(Pool), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (!hc.error && (hp.head != hp.tail || hc.work != 0)) { hc.error = KPLEX_ERR_TIMEOUT; g_last_error = "branch warps gave up with work left"; }
    if (per_graph) {
        const size_t G = h->ngraphs;
        std::vector<unsigned long long> gc(G), gh(G);
        std::vector<unsigned int> gv(G);
        CK(cudaMemcpyAsync(gc.data(), sp.gcount, G * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(gh.data(), sp.ghash, G * 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(gv.data(), sp.gvalid, G * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t g = 0; g < G; ++g) {
            kplex_result& r = per_graph[g];
            memset(&r, 0, sizeof r);
            r.count = gc[g]; r.hash = gh[g]; r.valid_roots = gv[g];
            r.pn = h->ginfo[g].pn; r.pm = h->gpm[g];
            r.status = (int)hc.error;
        }
    }
    fill_result(h, hc, ms, ms_dec, ms_bnb, launches, nroots ? nwarps : 0u, out);
    if (!hc.error && !(P.flags & KPLEX_FLAG_TEST_NO_WAIT)) {   // sizes are now known: later searches replay a graph
        Replay* r = new Replay();
        r->ws = d;
        r->gen = d->generation();
        r->p = h->p;
        r->grid_div = grid_div;
        r->sp = sp;
        r->dec_warps = dec_warps;
        r->blocks = blocks;
        r->nmax = nmax;
        r->smem = smem_bytes;
        r->kfn = kfn;
        r->cap = cap;
        r->scap = sp.spill_on ? scap_used : 0;
        r->launches = launches;
        h->replay = r;
    }
    return (int)hc.error;
}

}  // namespace kplex

// ------------------------------------------------------------------ C ABI
extern "C" {

int kplex_version(void) { return 1; }

long long kplex_preprocess_csr(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n, uint64_t m_directed,
                               int k, int q, int truss, uint32_t omp_threads,
                               uint32_t* out_off, uint32_t* out_adj, int32_t* out_dpos, int32_t* out_dseq,
                               uint32_t* out_orig, uint64_t* out_m) {
    if (!offsets || (!neighbors && m_directed) || !out_off || !out_m) return -KPLEX_ERR_PARAM;
    if (offsets[n] != m_directed || m_directed > 0xffffffffull) return -KPLEX_ERR_FORMAT;
    Csr g;
    g.n = n;
    g.off.assign(offsets, offsets + n + 1);
    g.adj.assign(neighbors, neighbors + m_directed);
    std::string err;
    int rc = validate_csr(g, &err);
    if (rc) { g_last_error = err; return -rc; }
    Prepped pre;
    preprocess(g, k, q, truss, (int)omp_threads, pre);
    const uint32_t pn = pre.g.n;
    memcpy(out_off, pre.g.off.data(), ((size_t)pn + 1) * 4);
    if (!pre.g.adj.empty()) memcpy(out_adj, pre.g.adj.data(), pre.g.adj.size() * 4);
    if (pn) {
        memcpy(out_dpos, pre.dpos.data(), (size_t)pn * 4);
        memcpy(out_dseq, pre.dseq.data(), (size_t)pn * 4);
        memcpy(out_orig, pre.orig.data(), (size_t)pn * 4);
    }
    *out_m = pre.g.adj.size();
    return pn;
}

long long kplex_partition_roots(const uint32_t* offsets, const uint32_t* neighbors, const int32_t* dpos,
                                const int32_t* dseq, uint32_t pn, int q, uint32_t shards, uint8_t* owner_out) {
    if (!offsets || (!neighbors && offsets[pn]) || (pn && (!dpos || !dseq)) || !owner_out || shards == 0 || shards > 255)
        return -KPLEX_ERR_PARAM;
    Csr g;
    g.n = pn;
    g.off.assign(offsets, offsets + pn + 1);
    g.adj.assign(neighbors, neighbors + offsets[pn]);
    std::vector<int32_t> dp(dpos, dpos + pn), ds(dseq, dseq + pn);
    const long long lim = (long long)pn - (long long)q + 2;   // src:44-45
    const uint32_t nroots = lim > 0 ? (uint32_t)std::min<long long>(lim, pn) : 0u;
    weighted_root_owners(g, dp, ds, nroots, shards, owner_out);
    return nroots;
}

const char* kplex_status_string(int s) {
    switch (s) {
        case KPLEX_OK: return "ok";
        case KPLEX_ERR_PARAM: return "unsupported parameter";
        case KPLEX_ERR_IO: return "io error";
        case KPLEX_ERR_FORMAT: return "malformed graph";
        case KPLEX_ERR_CUDA: return "cuda error";
        case KPLEX_ERR_NOMEM: return "out of memory";
        case KPLEX_ERR_CAPACITY: return "root subgraph exceeds 2048 vertices (or its left set 8192)";
        case KPLEX_ERR_TIMEOUT: return "bounded device wait gave up";
        case KPLEX_ERR_NO_DEVICE: return "no usable CUDA device";
        case KPLEX_ERR_INTERNAL: return "internal device check failed";
        default: return "unknown status";
    }
}

const char* kplex_last_error(void) { return g_last_error.c_str(); }

int kplex_device_ok(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceState* d = nullptr;
    return device_state(device, &d) == KPLEX_OK ? 1 : 0;
}

int kplex_load_bin(const char* path, kplex_graph* out) {
    if (!path || !out) return KPLEX_ERR_PARAM;
    Csr g;
    std::string err;
    int rc = load_bin(path, g, &err);
    if (rc) { g_last_error = err; return rc; }
    out->n = g.n;
    out->m_directed = g.m_directed();
    out->offsets = (uint32_t*)malloc(((size_t)g.n + 1) * 4);
    out->neighbors = (uint32_t*)malloc(std::max<size_t>(g.adj.size(), 1) * 4);
    if (!out->offsets || !out->neighbors) { free(out->offsets); free(out->neighbors); return KPLEX_ERR_NOMEM; }
    memcpy(out->offsets, g.off.data(), ((size_t)g.n + 1) * 4);
    if (!g.adj.empty()) memcpy(out->neighbors, g.adj.data(), g.adj.size() * 4);
    return KPLEX_OK;
}

int kplex_save_bin(const char* path, const kplex_graph* g) {
    if (!path || !g) return KPLEX_ERR_PARAM;
    Csr c;
    c.n = g->n;
    c.off.assign(g->offsets, g->offsets + g->n + 1);
    c.adj.assign(g->neighbors, g->neighbors + g->m_directed);
    std::string err;
    int rc = save_bin(path, c, &err);
    if (rc) g_last_error = err;
    return rc;
}

void kplex_free_graph(kplex_graph* g) {
    if (!g) return;
    free(g->offsets); free(g->neighbors);
    g->offsets = g->neighbors = nullptr;
    g->n = 0; g->m_directed = 0;
}

int kplex_generate(const kplex_gen_spec* s, kplex_graph* out) {
    if (!s || !out) return KPLEX_ERR_PARAM;
    GenSpec gs;
    gs.seed = s->seed; gs.n = s->n; gs.base_edges = s->base_edges; gs.exponent = s->exponent; gs.max_degree = s->max_degree;
    gs.groups = s->groups; gs.group_min = s->group_min; gs.group_max = s->group_max;
    gs.density_min = s->density_min; gs.density_max = s->density_max;
    Csr g;
    std::string err;
    int rc = generate(gs, g, &err);
    if (rc) { g_last_error = err; return rc; }
    out->n = g.n;
    out->m_directed = g.m_directed();
    out->offsets = (uint32_t*)malloc(((size_t)g.n + 1) * 4);
    out->neighbors = (uint32_t*)malloc(std::max<size_t>(g.adj.size(), 1) * 4);
    if (!out->offsets || !out->neighbors) { free(out->offsets); free(out->neighbors); return KPLEX_ERR_NOMEM; }
    memcpy(out->offsets, g.off.data(), ((size_t)g.n + 1) * 4);
    if (!g.adj.empty()) memcpy(out->neighbors, g.adj.data(), g.adj.size() * 4);
    return KPLEX_OK;
}

int kplex_prepare(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n, uint64_t m_directed,
                  const kplex_params* p, kplex_prepared** h, kplex_result* out) {
    if (!h) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(g_mu);
    if (out) memset(out, 0, sizeof(*out));
    int rc = prepare_impl(offsets, neighbors, n, m_directed, p, h, out);
    if (out) out->status = rc;
    return rc;
}

int kplex_search(kplex_prepared* h, kplex_result* out) {
    if (!h) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(g_mu);
    auto t0 = std::chrono::steady_clock::now();
    DeviceState* dev = nullptr;
    int rc = device_state(h->device, &dev);
    if (rc == KPLEX_OK) rc = search_impl(h, &dev->ws, out);
    if (out) { out->status = rc; out->ms_total = ms_since(t0); }
    return rc;
}

void kplex_release(kplex_prepared* h) {
    std::lock_guard<std::mutex> lk(g_mu);
    free_prepared(h);
}

int kplex_enumerate_csr(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n, uint64_t m_directed,
                        const kplex_params* p, kplex_result* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto t0 = std::chrono::steady_clock::now();
    kplex_result tmp;
    kplex_result* r = out ? out : &tmp;
    memset(r, 0, sizeof(*r));
    kplex_prepared* h = nullptr;
    const bool verbose = p && !(p->flags & KPLEX_FLAG_QUIET);
    int rc = prepare_impl(offsets, neighbors, n, m_directed, p, &h, r);
    if (rc == KPLEX_OK) {
        if (verbose) { printf("Start copying graph to GPU....\n"); printf("Done copying graph to GPU....\n"); }
        DeviceState* dev = nullptr;
        rc = device_state(h->device, &dev);
        if (rc == KPLEX_OK) rc = search_impl(h, &dev->ws, r);
        free_prepared(h);
    }
    r->status = rc;
    r->ms_total = ms_since(t0);
    if (verbose && rc == KPLEX_OK) {
        printf("Total Time Elapsed: %f ms\n", r->ms_ref_region);
        printf("Total Valid Blocks: %d, Maximal k-Plexes: %u\n", (int)r->valid_roots, (unsigned)(r->count & 0xffffffffu));
        printf("Total tasks generated: %u\n", (unsigned)(r->tasks & 0xffffffffu));
        printf("\nKernel Launch Successfully\n");
    }
    return rc;
}

int kplex_prepare_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common, kplex_prepared** h,
                        kplex_result* total) {
    if (!h || !common || (!jobs && njobs)) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(g_mu);
    if (total) memset(total, 0, sizeof(*total));
    if (njobs == 0) { g_last_error = "empty batch"; return KPLEX_ERR_PARAM; }
    std::vector<HostJob> hj(njobs);
    for (uint32_t i = 0; i < njobs; ++i)
        hj[i] = HostJob{jobs[i].offsets, jobs[i].neighbors, jobs[i].n, jobs[i].m_directed, jobs[i].k, jobs[i].q, jobs[i].truss};
    kplex_params p = *common;
    p.flags |= KPLEX_FLAG_QUIET;
    DeviceState* dev = nullptr;
    int rc = device_state(p.device, &dev);
    if (rc == KPLEX_OK) rc = prepare_set(hj, &p, &dev->ws, h, total);
    if (total) total->status = rc;
    return rc;
}

int kplex_search_batch(kplex_prepared* h, kplex_result* per_job, kplex_result* total) {
    if (!h) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(g_mu);
    auto t0 = std::chrono::steady_clock::now();
    kplex_result tmp;
    kplex_result* r = total ? total : &tmp;
    memset(r, 0, sizeof(*r));
    DeviceState* dev = nullptr;
    int rc = device_state(h->device, &dev);
    if (rc == KPLEX_OK) rc = search_impl(h, &dev->ws, r, per_job);
    r->status = rc;
    r->ms_total = ms_since(t0);
    return rc;
}

int kplex_enumerate_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common, kplex_result* per_job,
                          kplex_result* total) {
    auto t0 = std::chrono::steady_clock::now();
    kplex_prepared* h = nullptr;
    kplex_result tmp;
    kplex_result* r = total ? total : &tmp;
    int rc = kplex_prepare_batch(jobs, njobs, common, &h, r);
    if (rc) return rc;
    const double ms_pre = r->ms_preprocess;
    rc = kplex_search_batch(h, per_job, r);
    r->ms_preprocess = ms_pre;
    r->ms_ref_region = ms_pre + r->ms_device;
    kplex_release(h);
    r->ms_total = ms_since(t0);
    return rc;
}

int kplex_autotune_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common, uint32_t sample,
                         kplex_params* best, double* best_ms) {
    if (!jobs || !njobs || !common || !best) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(g_mu);
    sample = std::max<uint32_t>(1u, std::min(sample, njobs));
    std::vector<HostJob> hj;
    for (uint32_t i = 0; i < sample; ++i) {
        const kplex_job& j = jobs[(uint64_t)i * njobs / sample];
        hj.push_back(HostJob{j.offsets, j.neighbors, j.n, j.m_directed, j.k, j.q, j.truss});
    }
    DeviceState* dev = nullptr;
    int rc = device_state(common->device, &dev);
    if (rc) return rc;
    kplex_params p = *common;
    p.flags |= KPLEX_FLAG_QUIET;
    kplex_prepared* h = nullptr;
    kplex_result tot{};
    if ((rc = prepare_set(hj, &p, &dev->ws, &h, &tot))) return rc;
    struct Cand { uint32_t bps; int32_t stage; uint64_t pool; float thres; };
    std::vector<Cand> cands;
    for (uint32_t bps : {2u, 3u})
        for (int32_t stage : {8, 32, -1})
            for (uint64_t pool : {1ull << 20, 1ull << 22})
                for (float th : {0.25f, 0.5f}) cands.push_back(Cand{bps, stage, pool, th});
    double best_t = 1e300;
    uint64_t ref_count = 0, ref_hash = 0;
    bool have_ref = false;
    for (const Cand& c : cands) {
        h->p.blocks_per_sm = c.bps;
        h->p.stage_after = c.stage;
        h->p.pool_slots = c.pool;
        h->p.thres = c.thres;
        double t = 1e300;
        for (int rep = 0; rep < 2; ++rep) {   // the first run grows the workspace for this shape
            kplex_result r{};
            if ((rc = search_impl(h, &dev->ws, &r))) { free_prepared(h); return rc; }
            if (!have_ref) { ref_count = r.count; ref_hash = r.hash; have_ref = true; }
            if (r.count != ref_count || r.hash != ref_hash) {
                free_prepared(h);
                g_last_error = "autotune candidates disagree on the sample's result";
                return KPLEX_ERR_INTERNAL;
            }
            if (rep == 1) t = r.ms_device;
        }
        if (t < best_t) {
            best_t = t;
            *best = *common;
            best->blocks_per_sm = c.bps;
            best->stage_after = c.stage;
            best->pool_slots = c.pool;
            best->thres = c.thres;
        }
    }
    free_prepared(h);
    if (best_ms) *best_ms = best_t;
    return KPLEX_OK;
}

int kplex_enumerate_file(const char* path, const kplex_params* p, kplex_result* out) {
    kplex_graph g{};
    int rc = kplex_load_bin(path, &g);
    if (rc) { if (out) { memset(out, 0, sizeof(*out)); out->status = rc; } return rc; }
    if (p && !(p->flags & KPLEX_FLAG_QUIET)) printf("n=%u, m=%u (undirected)\n", g.n, (unsigned)g.m_directed);
    rc = kplex_enumerate_csr(g.offsets, g.neighbors, g.n, g.m_directed, p, out);
    kplex_free_graph(&g);
    return rc;
}

}  // extern "C"
