// Host preprocessing: (q-k)-core, optional (q-2k)-truss, degeneracy order.
//
// Each step reproduces the reference's result bit for bit, because the search
// that follows depends on the exact peeled numbering and order:
//  * core_peel       inc/host_funcs.h:16-122 — the (q-k)-core is unique, so a
//                    parallel frontier peel gives the same survivors; ids are
//                    renumbered in ascending order and each neighbour list
//                    keeps its order (sequence::pack, inc/sequence.h:474-491).
//  * truss_prune     inc/host_funcs.h:761-823 and fast_truss_peeling :463-559.
//                    The peel is order dependent (each directed entry keeps its
//                    own support counter), so it stays serial and LIFO exactly
//                    as there; only the initial triangle count is parallel.
//  * degeneracy      inc/degeneracy.h ListLinearHeap + inc/host_funcs.h:829-851:
//                    bucket lists with head insertion (LIFO ties) and a minimum
//                    pointer that only moves up when a bucket empties.
#include "preprocess.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <omp.h>

namespace kplex {

// (q-k)-core with order-preserving renumbering.  orig_of_new is composed with
// the incoming map (empty = identity).
static Csr core_peel(const Csr& g, int bd, std::vector<uint32_t>& orig_of_new) {
    const uint32_t n = g.n;
    std::vector<uint8_t> alive(n, 1);
    std::vector<std::atomic<int>> res(n);
    std::vector<uint32_t> frontier, next;
    for (uint32_t i = 0; i < n; ++i) {
        res[i].store((int)g.deg(i), std::memory_order_relaxed);
        if ((int)g.deg(i) < bd) { alive[i] = 0; frontier.push_back(i); }
    }
    while (!frontier.empty()) {
        next.clear();
#pragma omp parallel
        {
            std::vector<uint32_t> local;
#pragma omp for schedule(dynamic, 256) nowait
            for (long long f = 0; f < (long long)frontier.size(); ++f) {
                const uint32_t v = frontier[f];
                for (uint32_t j = g.off[v]; j < g.off[v + 1]; ++j) {
                    const uint32_t w = g.adj[j];
                    if (!__atomic_load_n(&alive[w], __ATOMIC_RELAXED)) continue;
                    const int old = res[w].fetch_sub(1, std::memory_order_relaxed);
                    if (old == bd) { __atomic_store_n(&alive[w], 0, __ATOMIC_RELAXED); local.push_back(w); }
                }
            }
#pragma omp critical
            next.insert(next.end(), local.begin(), local.end());
        }
        frontier.swap(next);
    }
    std::vector<uint32_t> newid(n, 0), keep;
    keep.reserve(n);
    for (uint32_t i = 0; i < n; ++i) if (alive[i]) { newid[i] = (uint32_t)keep.size(); keep.push_back(i); }
    Csr r;
    r.n = (uint32_t)keep.size();
    r.off.assign((size_t)r.n + 1, 0);
    std::vector<uint32_t> d(r.n);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)r.n; ++i) {
        uint32_t c = 0;
        for (uint32_t j = g.off[keep[i]]; j < g.off[keep[i] + 1]; ++j) c += alive[g.adj[j]];
        d[i] = c;
    }
    for (uint32_t i = 0; i < r.n; ++i) r.off[i + 1] = r.off[i] + d[i];
    r.adj.resize(r.off[r.n]);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)r.n; ++i) {
        uint32_t cur = r.off[i];
        for (uint32_t j = g.off[keep[i]]; j < g.off[keep[i] + 1]; ++j)
            if (alive[g.adj[j]]) r.adj[cur++] = newid[g.adj[j]];
    }
    std::vector<uint32_t> composed(r.n);
    for (uint32_t i = 0; i < r.n; ++i) composed[i] = orig_of_new.empty() ? keep[i] : orig_of_new[keep[i]];
    orig_of_new.swap(composed);
    return r;
}

static inline int64_t find_pos(const Csr& g, uint32_t u, uint32_t v) {
    const uint32_t* b = g.adj.data() + g.off[u];
    const uint32_t* e = g.adj.data() + g.off[u + 1];
    const uint32_t* it = std::lower_bound(b, e, v);
    if (it == e || *it != v) return -1;
    return it - g.adj.data();
}

// Directed-entry support counters, initial edge queue (u < v, ascending), and
// the serial LIFO peel.  Mutates g (compacted in place).
static void truss_prune(Csr& g, int thr) {
    const uint32_t n = g.n;
    const uint32_t m = g.off[n];
    std::vector<int> tri(m, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const uint32_t i = (uint32_t)ii;
        for (uint32_t p = g.off[i]; p < g.off[i + 1]; ++p) {
            const uint32_t v = g.adj[p];
            uint32_t a = g.off[i], ea = g.off[i + 1], b = g.off[v], eb = g.off[v + 1];
            int c = 0;
            while (a < ea && b < eb) {
                const uint32_t x = g.adj[a], y = g.adj[b];
                if (x == y) { ++c; ++a; ++b; } else if (x < y) ++a; else ++b;
            }
            tri[p] = c;
        }
    }
    std::vector<std::pair<uint32_t, uint32_t>> Q;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t p = g.off[i]; p < g.off[i + 1]; ++p)
            if (i < g.adj[p] && tri[p] < thr) Q.emplace_back(i, g.adj[p]);
    std::vector<uint8_t> dead(m, 0);
    while (!Q.empty()) {
        const uint32_t u = Q.back().first, v = Q.back().second;
        Q.pop_back();
        const int64_t puv = find_pos(g, u, v), pvu = find_pos(g, v, u);
        if (puv >= 0) dead[puv] = 1;
        if (pvu >= 0) dead[pvu] = 1;
        uint32_t a = g.off[u], ea = g.off[u + 1], b = g.off[v], eb = g.off[v + 1];
        while (a < ea && b < eb) {
            while (a < ea && dead[a]) ++a;
            while (b < eb && dead[b]) ++b;
            if (a >= ea || b >= eb) break;
            const uint32_t x = g.adj[a], y = g.adj[b];
            if (x == y) {
                int prev = tri[a];
                if (prev > 0) { tri[a] = prev - 1; if (prev == thr) Q.emplace_back(u, x); }
                prev = tri[b];
                if (prev > 0) { tri[b] = prev - 1; if (prev == thr) Q.emplace_back(v, x); }
                ++a; ++b;
            } else if (x < y) ++a; else ++b;
        }
    }
    uint32_t w = 0;
    for (uint32_t u = 0; u < n; ++u) {
        const uint32_t b = g.off[u], e = g.off[u + 1];
        g.off[u] = w;
        for (uint32_t i = b; i < e; ++i) if (!dead[i]) g.adj[w++] = g.adj[i];
    }
    g.off[n] = w;
    g.adj.resize(w);
}

static void degeneracy_order(const Csr& g, std::vector<int32_t>& dpos, std::vector<int32_t>& dseq) {
    const int n = (int)g.n;
    dpos.assign(n, INT_MAX);
    dseq.assign(n, 0);
    if (n == 0) return;
    const int NIL = n;
    std::vector<int> key(n), prv(n), nxt(n), head(n, NIL);
    int min_key = n - 1;
    auto insert = [&](int id, int k) {
        key[id] = k; prv[id] = NIL; nxt[id] = head[k];
        if (head[k] != NIL) prv[head[k]] = id;
        head[k] = id;
        if (k < min_key) min_key = k;
    };
    auto unlink = [&](int id) {
        if (prv[id] == NIL) { head[key[id]] = nxt[id]; if (nxt[id] != NIL) prv[nxt[id]] = NIL; }
        else { nxt[prv[id]] = nxt[id]; if (nxt[id] != NIL) prv[nxt[id]] = prv[id]; }
    };
    for (int i = 0; i < n; ++i) insert(i, (int)g.deg(i));
    for (int i = 0; i < n; ++i) {
        while (head[min_key] == NIL) ++min_key;
        const int u = head[min_key];
        head[min_key] = nxt[u];
        if (head[min_key] != NIL) prv[head[min_key]] = NIL;
        dpos[u] = i;
        dseq[i] = u;
        for (uint32_t j = g.off[u]; j < g.off[u + 1]; ++j) {
            const int w = (int)g.adj[j];
            if (dpos[w] == INT_MAX) { const int nk = key[w] - 1; unlink(w); insert(w, nk); }
        }
    }
}

int preprocess(const Csr& in, int k, int q, int truss, int threads, Prepped& out) {
    if (threads > 0) omp_set_num_threads(threads);
    out.orig.clear();
    out.g = core_peel(in, q - k, out.orig);
    if (truss) {
        truss_prune(out.g, q - 2 * k);
        out.g = core_peel(out.g, q - k, out.orig);
    }
    degeneracy_order(out.g, out.dpos, out.dseq);
    return 0;
}

}  // namespace kplex

namespace kplex {

// Cost-weighted partition of the root ranks [0, nroots) over `shards` owners, for
// multi-GPU runs.  A root's work grows with its local subgraph, whose first layer
// is the root's later neighbours (C1 is drawn from them, at most 1023 of them are
// kept, src:87-131); the cost estimate is (later + 1)^2.  Roots are handed out
// largest first to the least loaded owner (longest-processing-time rule), ties to
// the smaller rank and the smaller owner, so every process computes the same
// assignment from the same pruned graph.
void weighted_root_owners(const Csr& g, const std::vector<int32_t>& dpos, const std::vector<int32_t>& dseq,
                          uint32_t nroots, uint32_t shards, uint8_t* owner) {
    std::vector<std::pair<uint64_t, uint32_t>> cost(nroots);
    for (uint32_t r = 0; r < nroots; ++r) {
        const uint32_t v = (uint32_t)dseq[r];
        uint64_t later = 0;
        for (uint32_t e = g.off[v]; e < g.off[v + 1]; ++e) later += dpos[g.adj[e]] > dpos[v];
        later = std::min<uint64_t>(later, 1023);
        cost[r] = {(later + 1) * (later + 1), r};
    }
    std::stable_sort(cost.begin(), cost.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::vector<uint64_t> load(shards, 0);
    for (const auto& c : cost) {
        uint32_t best = 0;
        for (uint32_t s = 1; s < shards; ++s) if (load[s] < load[best]) best = s;
        load[best] += c.first;
        owner[c.second] = (uint8_t)best;
    }
}

}  // namespace kplex
