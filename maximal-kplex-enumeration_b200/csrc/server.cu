// Request server: continuous batching of enumeration requests on one GPU.
//
// No reference counterpart (CudaPlex enumerates one graph per process,
// main.cu:56-61).  Requests are queued by kplex_server_submit as they arrive.
// Each of `slots` worker threads owns a Workspace (its own CUDA stream, arena,
// task pool, branch stacks and spill ring).  A worker that is free admits, in
// arrival order, every waiting request that fits the device-memory budget (up
// to max_batch; a request estimated at large_bytes or more goes alone),
// preprocesses them on the host, uploads them and enumerates them as one batched launch (prepare_set + search_impl, the path of
// kplex_enumerate_batch).  Requests that arrive meanwhile wait for the next free
// worker, so while one launch searches, the next batch is preprocessed, uploaded
// and decomposed on another stream.  With split_grid each launch's persistent
// kernel takes 1/slots of the SMs so that the launches also run side by side.
//
// Memory admission: the budget covers every worker's workspace buffers (device
// bytes plus the pinned spill ring) and each admitted request's estimated
// footprint until its launch completes.  A request whose estimate alone exceeds
// the budget is refused at submit; one that does not fit next to the requests
// in flight waits; a request is always admitted when nothing else is in flight.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace kplex {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t tag = 0;
    int k = 0, q = 0, truss = 0;
    uint32_t n = 0;
    std::vector<uint32_t> off, adj;
    Clock::time_point t_submit;
    uint64_t est_bytes = 0;
};

// Device bytes a request adds while in flight: its pruned CSR and vertex maps
// (bounded by the input's), its result slots, and the decomposition arena of
// its roots, bounded per root by a local subgraph of min(degree + 1, MAX_LOCAL)
// vertices holding three adjacency-sized bit matrices and the id tables.
static uint64_t estimate_request_bytes(const Request& r) {
    const uint64_t m = r.adj.size();
    uint64_t b = 4ull * (r.n + 1) + 4ull * m + 12ull * r.n + 64;
    for (uint32_t v = 0; v < r.n; ++v) {
        const uint64_t d = std::min<uint64_t>(r.off[v + 1] - r.off[v] + 1, MAX_LOCAL);
        if ((int64_t)d < r.q) continue;   // cannot hold a plex of q vertices
        const uint64_t w = ((d + 31) / 32 + 3) & ~3ull;
        b += 4ull * (3 * d * w + 2 * d);
    }
    return b;
}

}  // namespace kplex

using namespace kplex;

struct kplex_server {
    kplex_server_config cfg{};
    int device = 0;
    std::vector<std::unique_ptr<Workspace>> ws;
    std::vector<uint64_t> ws_bytes;
    std::vector<std::thread> workers;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::unique_ptr<Request>> pending;
    std::deque<kplex_completion> done;
    uint64_t inflight_bytes = 0;
    uint64_t submitted = 0, completed = 0, rejected = 0, launches = 0, peak = 0;
    uint32_t active = 0, max_active = 0, max_batch_seen = 0;
    bool stop = false;

    uint64_t resident_locked() const {
        uint64_t b = inflight_bytes;
        for (uint64_t x : ws_bytes) b += x;
        return b;
    }
    void worker(uint32_t slot);
    void run_batch(uint32_t slot, std::vector<std::unique_ptr<Request>>& batch, Clock::time_point t_start);
};

// Runs one launch for `batch` on the slot's workspace; a failed launch of several
// requests is retried request by request so that only the failing one reports it.
void kplex_server::run_batch(uint32_t slot, std::vector<std::unique_ptr<Request>>& batch, Clock::time_point t_start) {
    Workspace* w = ws[slot].get();
    const size_t G = batch.size();
    std::vector<HostJob> jobs(G);
    for (size_t i = 0; i < G; ++i) {
        const Request& r = *batch[i];
        jobs[i] = HostJob{r.off.data(), r.adj.data(), r.n, (uint64_t)r.adj.size(), r.k, r.q, r.truss};
    }
    kplex_params p{};
    p.k = 2; p.q = 3;
    p.thres = cfg.thres;
    p.flags = cfg.flags | KPLEX_FLAG_QUIET;
    p.device = device;
    p.pool_slots = cfg.pool_slots;
    const uint32_t div = cfg.split_grid ? std::max<uint32_t>(cfg.slots, 1u) : 1u;

    std::vector<kplex_result> per(G);
    kplex_result tot{};
    kplex_prepared* h = nullptr;
    int rc = prepare_set(jobs, &p, w, &h, &tot);
    if (rc == KPLEX_OK) {
        rc = search_impl(h, w, &tot, per.data(), div);
        free_prepared(h);
    }
    cudaStreamSynchronize(w->stream);
    if (rc != KPLEX_OK && G > 1) {
        for (size_t i = 0; i < G; ++i) {
            kplex_prepared* h1 = nullptr;
            kplex_result t1{};
            memset(&per[i], 0, sizeof(kplex_result));
            int r1 = prepare_set({jobs[i]}, &p, w, &h1, &t1);
            if (r1 == KPLEX_OK) {
                r1 = search_impl(h1, w, &t1, &per[i], div);
                free_prepared(h1);
            }
            per[i].status = r1;
        }
        cudaStreamSynchronize(w->stream);
    } else if (rc != KPLEX_OK) {
        per[0].status = rc;
    }
    const Clock::time_point t_end = Clock::now();
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < G; ++i) {
        const Request& r = *batch[i];
        kplex_completion c{};
        c.tag = r.tag;
        c.status = per[i].status;
        c.batch_size = (uint32_t)G;
        c.count = per[i].count;
        c.hash = per[i].hash;
        c.valid_roots = per[i].valid_roots;
        c.pn = per[i].pn;
        c.slot = slot;
        c.ms_queue = std::chrono::duration<double, std::milli>(t_start - r.t_submit).count();
        c.ms_service = std::chrono::duration<double, std::milli>(t_end - t_start).count();
        c.ms_latency = std::chrono::duration<double, std::milli>(t_end - r.t_submit).count();
        done.push_back(c);
        inflight_bytes -= r.est_bytes;
    }
    completed += G;
    ws_bytes[slot] = w->device_bytes() + w->spill_data.bytes;
    peak = std::max(peak, resident_locked());
    --active;
    cv_done.notify_all();
    cv_work.notify_all();
}

void kplex_server::worker(uint32_t slot) {
    cudaSetDevice(device);
    const uint32_t max_batch = cfg.max_batch ? cfg.max_batch : 1024u;
    for (;;) {
        std::vector<std::unique_ptr<Request>> batch;
        Clock::time_point t_start;
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (!pending.empty()) {
                    uint64_t add = 0;
                    const uint64_t base = resident_locked();
                    while (!pending.empty() && batch.size() < max_batch) {
                        const uint64_t e = pending.front()->est_bytes;
                        const bool large = e >= cfg.large_bytes;
                        if (large && !batch.empty()) break;   // a large request gets a launch of its own
                        const bool alone = batch.empty() && inflight_bytes == 0;
                        if (!alone && base + add + e > cfg.mem_budget) break;   // arrival order: no overtaking
                        add += e;
                        batch.push_back(std::move(pending.front()));
                        pending.pop_front();
                        if (large) break;
                    }
                    if (!batch.empty()) {
                        inflight_bytes += add;
                        peak = std::max(peak, resident_locked());
                        ++active;
                        ++launches;
                        max_active = std::max(max_active, active);
                        max_batch_seen = std::max<uint32_t>(max_batch_seen, (uint32_t)batch.size());
                        break;
                    }
                }
                if (stop && pending.empty()) return;
                cv_work.wait(lk);
            }
            t_start = Clock::now();
        }
        run_batch(slot, batch, t_start);
    }
}

extern "C" {

int kplex_server_create(const kplex_server_config* cfg, kplex_server** out) {
    if (!cfg || !out) return KPLEX_ERR_PARAM;
    *out = nullptr;
    if (cfg->thres < 0.0f || cfg->thres > 1.0f) { set_last_error("thres must be in (0, 1]"); return KPLEX_ERR_PARAM; }
    DeviceState* dev = nullptr;
    int rc = device_state(cfg->device, &dev);   // device checks and one-time kernel attributes
    if (rc) return rc;
    auto* s = new kplex_server();
    s->cfg = *cfg;
    if (!s->cfg.slots) s->cfg.slots = 2;
    if (s->cfg.slots > 16) s->cfg.slots = 16;
    if (!s->cfg.max_batch) s->cfg.max_batch = 1024;
    if (!s->cfg.mem_budget) s->cfg.mem_budget = 16ull << 30;
    if (!(s->cfg.thres > 0.0f)) s->cfg.thres = 0.25f;
    if (!s->cfg.large_bytes) s->cfg.large_bytes = 32ull << 20;
    s->device = cfg->device;
    for (uint32_t i = 0; i < s->cfg.slots; ++i) {
        s->ws.emplace_back(new Workspace());
        if ((rc = workspace_init(*s->ws.back(), s->device, dev->sms))) {
            for (auto& w : s->ws) w->destroy();
            delete s;
            return rc;
        }
    }
    s->ws_bytes.assign(s->cfg.slots, 0);
    for (uint32_t i = 0; i < s->cfg.slots; ++i) s->workers.emplace_back([s, i] { s->worker(i); });
    *out = s;
    return KPLEX_OK;
}

int kplex_server_submit(kplex_server* s, const kplex_job* job, uint64_t tag) {
    if (!s || !job) return KPLEX_ERR_PARAM;
    int rc = check_kq(job->k, job->q);
    if (rc) return rc;
    if (!job->offsets || (!job->neighbors && job->m_directed) || job->offsets[job->n] != job->m_directed ||
        job->m_directed > 0xffffffffull) {
        set_last_error("inconsistent CSR");
        return KPLEX_ERR_FORMAT;
    }
    auto r = std::make_unique<Request>();
    r->tag = tag;
    r->k = job->k; r->q = job->q; r->truss = job->truss;
    r->n = job->n;
    r->off.assign(job->offsets, job->offsets + job->n + 1);
    r->adj.assign(job->neighbors, job->neighbors + job->m_directed);
    r->est_bytes = estimate_request_bytes(*r);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) { set_last_error("server is shutting down"); return KPLEX_ERR_PARAM; }
    if (r->est_bytes > s->cfg.mem_budget) {
        ++s->rejected;
        set_last_error("request needs about " + std::to_string(r->est_bytes) + " device bytes, over the server budget");
        return KPLEX_ERR_NOMEM;
    }
    r->t_submit = Clock::now();
    s->pending.push_back(std::move(r));
    ++s->submitted;
    s->cv_work.notify_one();
    return KPLEX_OK;
}

int kplex_server_poll(kplex_server* s, kplex_completion* out, uint32_t max, int timeout_ms) {
    if (!s || (!out && max)) return -KPLEX_ERR_PARAM;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [s] { return !s->done.empty() || s->completed == s->submitted; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (timeout_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    uint32_t n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    return (int)n;
}

int kplex_server_drain(kplex_server* s, int timeout_ms) {
    if (!s) return KPLEX_ERR_PARAM;
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [s] { return s->completed == s->submitted; };
    if (timeout_ms < 0) { s->cv_done.wait(lk, idle); return KPLEX_OK; }
    return s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle) ? KPLEX_OK : KPLEX_ERR_TIMEOUT;
}

int kplex_server_stats_get(kplex_server* s, kplex_server_stats* out) {
    if (!s || !out) return KPLEX_ERR_PARAM;
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->launches = s->launches;
    out->device_bytes = s->resident_locked();
    out->peak_device_bytes = s->peak;
    out->max_concurrent = s->max_active;
    out->max_batch_seen = s->max_batch_seen;
    return KPLEX_OK;
}

void kplex_server_destroy(kplex_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& w : s->ws) w->destroy();
    delete s;
}

}  // extern "C"
