// Seeded synthetic graph generator (project-defined; the reference ships only
// two real .bin files, dataset/*.bin).
//
// Base graph: Chung-Lu with expected degree w_i = min(cap, c * (r_i+1)^(-1/(gamma-1)))
// over a random rank permutation r, c chosen so that sum(w) = 2 * base_edges.
// Edges are drawn by picking both endpoints proportionally to w (Walker alias
// table) and rejecting self loops, duplicates and endpoints already at the
// hard degree cap, until exactly base_edges distinct edges exist.
// Planted groups: disjoint vertex sets chosen uniformly; each group's internal
// pairs are set to a clique minus exactly round((1-d) * C(s,2)) pairs chosen
// uniformly (pairs removed here also remove a base edge if there was one).
#include "graph_io.h"

#include <algorithm>
#include <cmath>
#include <unordered_set>

namespace kplex {

namespace {
struct Alias {
    std::vector<double> prob;
    std::vector<uint32_t> alias;
    explicit Alias(const std::vector<double>& w) {
        const size_t n = w.size();
        prob.resize(n); alias.resize(n);
        double sum = 0; for (double x : w) sum += x;
        std::vector<double> sc(n);
        std::vector<uint32_t> small, large;
        for (size_t i = 0; i < n; ++i) { sc[i] = w[i] * n / sum; (sc[i] < 1.0 ? small : large).push_back((uint32_t)i); }
        while (!small.empty() && !large.empty()) {
            uint32_t s = small.back(); small.pop_back();
            uint32_t l = large.back(); large.pop_back();
            prob[s] = sc[s]; alias[s] = l;
            sc[l] = (sc[l] + sc[s]) - 1.0;
            (sc[l] < 1.0 ? small : large).push_back(l);
        }
        for (uint32_t i : large) { prob[i] = 1.0; alias[i] = i; }
        for (uint32_t i : small) { prob[i] = 1.0; alias[i] = i; }
    }
    uint32_t sample(Xoshiro256& rng) const {
        uint32_t i = (uint32_t)rng.below(prob.size());
        return rng.uniform() < prob[i] ? i : alias[i];
    }
};
inline uint64_t ekey(uint32_t a, uint32_t b) { if (a > b) std::swap(a, b); return ((uint64_t)a << 32) | b; }
}  // namespace

int generate(const GenSpec& s, Csr& out, std::string* err) {
    if (s.n < 2) { if (err) *err = "n < 2"; return KPLEX_ERR_PARAM; }
    const uint64_t max_pairs = (uint64_t)s.n * (s.n - 1) / 2;
    const uint32_t cap = (s.max_degree == 0 || s.max_degree > s.n - 1) ? s.n - 1 : s.max_degree;
    if (s.base_edges > max_pairs || s.base_edges > (uint64_t)cap * s.n / 2) { if (err) *err = "too many base edges"; return KPLEX_ERR_PARAM; }
    if (s.exponent <= 1.0) { if (err) *err = "exponent must be > 1"; return KPLEX_ERR_PARAM; }
    uint64_t group_total = 0;
    Xoshiro256 rng(s.seed);

    // group sizes first so that the stream layout is fixed
    std::vector<uint32_t> gsize(s.groups);
    for (uint32_t g = 0; g < s.groups; ++g) {
        if (s.group_min < 2 || s.group_max < s.group_min) { if (err) *err = "bad group size range"; return KPLEX_ERR_PARAM; }
        gsize[g] = s.group_min + (uint32_t)rng.below(s.group_max - s.group_min + 1);
        group_total += gsize[g];
    }
    if (group_total > s.n) { if (err) *err = "groups larger than n"; return KPLEX_ERR_PARAM; }

    // expected degrees over a random rank permutation
    std::vector<uint32_t> rank(s.n);
    for (uint32_t i = 0; i < s.n; ++i) rank[i] = i;
    for (uint32_t i = s.n - 1; i > 0; --i) std::swap(rank[i], rank[rng.below(i + 1)]);
    const double alpha = 1.0 / (s.exponent - 1.0);
    std::vector<double> base(s.n);
    for (uint32_t i = 0; i < s.n; ++i) base[i] = std::pow((double)rank[i] + 1.0, -alpha);
    const double target = 2.0 * (double)s.base_edges;
    auto total = [&](double c) { double t = 0; for (double b : base) t += std::min((double)cap, c * b); return t; };
    double lo = 0, hi = 1;
    while (total(hi) < target && hi < 1e30) hi *= 2;
    for (int it = 0; it < 200; ++it) { double mid = 0.5 * (lo + hi); (total(mid) < target ? lo : hi) = mid; }
    std::vector<double> w(s.n);
    for (uint32_t i = 0; i < s.n; ++i) w[i] = std::max(1e-12, std::min((double)cap, hi * base[i]));
    Alias table(w);

    std::unordered_set<uint64_t> edges;
    edges.reserve(s.base_edges * 2 + 16);
    std::vector<uint32_t> deg(s.n, 0);
    uint64_t attempts = 0;
    const uint64_t max_attempts = 200 * s.base_edges + 1000;
    while (edges.size() < s.base_edges) {
        uint32_t a, b;
        if (attempts++ < max_attempts) { a = table.sample(rng); b = table.sample(rng); }
        else { a = (uint32_t)rng.below(s.n); b = (uint32_t)rng.below(s.n); }
        if (a == b || deg[a] >= cap || deg[b] >= cap) continue;
        if (!edges.insert(ekey(a, b)).second) continue;
        ++deg[a]; ++deg[b];
    }

    // planted groups: disjoint uniform vertex sets
    std::vector<uint32_t> perm(s.n);
    for (uint32_t i = 0; i < s.n; ++i) perm[i] = i;
    uint64_t pos = 0;
    for (uint32_t g = 0; g < s.groups; ++g) {
        const uint32_t sz = gsize[g];
        for (uint32_t j = 0; j < sz; ++j) {
            uint64_t r = pos + j + rng.below(s.n - pos - j);
            std::swap(perm[pos + j], perm[r]);
        }
        std::vector<uint32_t> mem(perm.begin() + pos, perm.begin() + pos + sz);
        pos += sz;
        const double d = s.density_min + (s.density_max - s.density_min) * rng.uniform();
        const uint64_t npairs = (uint64_t)sz * (sz - 1) / 2;
        const uint64_t ndel = (uint64_t)std::llround((1.0 - d) * (double)npairs);
        std::vector<uint64_t> pairs;
        pairs.reserve(npairs);
        for (uint32_t a = 0; a < sz; ++a)
            for (uint32_t b = a + 1; b < sz; ++b) pairs.push_back(((uint64_t)a << 32) | b);
        for (uint64_t j = 0; j < ndel; ++j) std::swap(pairs[j], pairs[j + rng.below(npairs - j)]);
        for (uint64_t j = 0; j < npairs; ++j) {
            const uint32_t a = mem[pairs[j] >> 32], b = mem[pairs[j] & 0xffffffffu];
            if (j < ndel) edges.erase(ekey(a, b));
            else edges.insert(ekey(a, b));
        }
    }

    // CSR
    std::vector<uint32_t> d2(s.n, 0);
    for (uint64_t e : edges) { ++d2[e >> 32]; ++d2[e & 0xffffffffu]; }
    out.n = s.n;
    out.off.assign((size_t)s.n + 1, 0);
    for (uint32_t v = 0; v < s.n; ++v) out.off[v + 1] = out.off[v] + d2[v];
    out.adj.assign(out.off[s.n], 0);
    std::vector<uint32_t> cur(out.off.begin(), out.off.end() - 1);
    for (uint64_t e : edges) {
        const uint32_t a = (uint32_t)(e >> 32), b = (uint32_t)(e & 0xffffffffu);
        out.adj[cur[a]++] = b; out.adj[cur[b]++] = a;
    }
    for (uint32_t v = 0; v < s.n; ++v) std::sort(out.adj.begin() + out.off[v], out.adj.begin() + out.off[v + 1]);
    return KPLEX_OK;
}

}  // namespace kplex
