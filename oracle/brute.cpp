// CPU ORACLE (second, independent check) — test infrastructure only.
//
// Exhaustive maximal k-plex enumeration that uses none of the reference's
// pruning rules (no pair classes, no upper bounds, no C1/C2 split): for each
// vertex v of the (q-k)-core, in index order, enumerate every k-plex whose
// smallest vertex is v by include/exclude branching over the vertices within
// two hops of v, keeping C (later) and X (earlier or excluded) equal to the
// set of vertices that extend the current P.  A leaf with C = X = {} and
// |P| >= q is a maximal k-plex.  Valid for q >= 2k-1 (a k-plex with at least
// 2k-1 vertices has diameter <= 2, so every extender lies within two hops).
// Vertices outside the (q-k)-core cannot extend a k-plex of size >= q, so
// maximality inside the core equals maximality in the input graph.
#include <cstdint>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace brute {
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static const uint64_t HASH_SEED = 0x6b706c6578b200ULL;

struct Local {
    int n, k, q;
    std::vector<std::vector<uint64_t>> A;   // adjacency bit rows
    int W;
    std::vector<uint32_t> ids;              // original ids
    uint64_t count = 0, hsum = 0;
    bool adj(int a, int b) const { return (A[a][b >> 6] >> (b & 63)) & 1; }
};

static int popc_and(const std::vector<uint64_t>& a, const std::vector<uint64_t>& b) {
    int c = 0; for (size_t i = 0; i < a.size(); ++i) c += __builtin_popcountll(a[i] & b[i]); return c;
}

// P, C, X as bitsets; deg[u] = |N(u) ∩ P| tracked implicitly by popcount.
static void rec(Local& L, std::vector<uint64_t>& P, int np, std::vector<int> C, std::vector<int> X) {
    if (np + (int)C.size() < L.q) return;
    if (C.empty()) {
        if (X.empty() && np >= L.q) {
            std::vector<uint32_t> ids;
            for (int i = 0; i < L.n; ++i) if ((P[i >> 6] >> (i & 63)) & 1) ids.push_back(L.ids[i]);
            std::sort(ids.begin(), ids.end());
            uint64_t x = splitmix64(HASH_SEED ^ (uint64_t)ids.size());
            for (uint32_t v : ids) x = splitmix64(x ^ (uint64_t)v);
            L.count++; L.hsum += x;
        }
        return;
    }
    const int c = C[0];
    std::vector<int> Crest(C.begin() + 1, C.end());
    // include c
    P[c >> 6] |= 1ull << (c & 63);
    const int np2 = np + 1;
    // members' degrees inside P'
    std::vector<int> members;
    for (int i = 0; i < L.n; ++i) if ((P[i >> 6] >> (i & 63)) & 1) members.push_back(i);
    std::vector<int> dP(L.n, 0);
    for (int u : members) dP[u] = popc_and(L.A[u], P);
    auto extends = [&](int u) {   // P' + u is a k-plex
        if (popc_and(L.A[u], P) + L.k < np2 + 1) return false;
        for (int w : members) if (dP[w] + L.k == np2 && !L.adj(w, u)) return false;
        return true;
    };
    std::vector<int> C2, X2;
    for (int u : Crest) if (extends(u)) C2.push_back(u);
    for (int u : X) if (extends(u)) X2.push_back(u);
    rec(L, P, np2, C2, X2);
    P[c >> 6] &= ~(1ull << (c & 63));
    // exclude c
    std::vector<int> X3 = X; X3.push_back(c);
    rec(L, P, np, Crest, X3);
}
}  // namespace brute

extern "C" int oracle_bruteforce_csr(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q,
                                     int threads, uint64_t* out_count, uint64_t* out_hash) {
    using namespace brute;
    if (k < 1 || q < 2 * k - 1) return 1;
    // (q-k)-core
    std::vector<int> deg(n); std::vector<char> alive(n, 1); std::vector<uint32_t> st;
    for (uint32_t v = 0; v < n; ++v) { deg[v] = off[v + 1] - off[v]; if (deg[v] < q - k) { alive[v] = 0; st.push_back(v); } }
    while (!st.empty()) { uint32_t v = st.back(); st.pop_back(); for (uint32_t j = off[v]; j < off[v + 1]; ++j) { uint32_t w = adj[j]; if (alive[w] && --deg[w] < q - k) { alive[w] = 0; st.push_back(w); } } }
    uint64_t tc = 0, th = 0;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : tc, th)
    for (long long vv = 0; vv < (long long)n; ++vv) {
        const uint32_t v = (uint32_t)vv;
        if (!alive[v]) continue;
        std::vector<uint32_t> loc{v};
        std::vector<char> mark(n, 0); mark[v] = 1;
        for (uint32_t j = off[v]; j < off[v + 1]; ++j) { uint32_t w = adj[j]; if (alive[w] && !mark[w]) { mark[w] = 1; loc.push_back(w); } }
        const size_t h1 = loc.size();
        for (size_t i = 1; i < h1; ++i) for (uint32_t j = off[loc[i]]; j < off[loc[i] + 1]; ++j) { uint32_t w = adj[j]; if (alive[w] && !mark[w]) { mark[w] = 1; loc.push_back(w); } }
        Local L; L.n = (int)loc.size(); L.k = k; L.q = q; L.W = (L.n + 63) / 64; L.ids = loc;
        L.A.assign(L.n, std::vector<uint64_t>(L.W, 0));
        for (int i = 0; i < L.n; ++i) for (int j = 0; j < L.n; ++j)
            if (i != j && std::binary_search(adj + off[loc[i]], adj + off[loc[i] + 1], loc[j])) L.A[i][j >> 6] |= 1ull << (j & 63);
        std::vector<uint64_t> P(L.W, 0); P[0] = 1;  // local 0 = v
        std::vector<int> C, X;
        for (int i = 1; i < L.n; ++i) (loc[i] > v ? C : X).push_back(i);
        rec(L, P, 1, C, X);
        tc += L.count; th += L.hsum;
    }
    *out_count = tc; *out_hash = th;
    return 0;
}
#ifdef BRUTE_MAIN
#include <cstdlib>
#include <cstring>
int main(int argc, char** argv) {
    FILE* f = fopen(argv[1], "rb"); uint32_t h[2]; if (!f || fread(h, 4, 2, f) != 2) return 2;
    std::vector<uint32_t> deg(h[0]), off(h[0] + 1, 0), adj(h[1]);
    if (fread(deg.data(), 4, h[0], f) != h[0]) return 2;
    for (uint32_t i = 0; i < h[0]; ++i) off[i + 1] = off[i] + deg[i];
    if (fread(adj.data(), 4, h[1], f) != h[1]) return 2;
    int k = atoi(argv[2]), q = atoi(argv[3]);
    uint64_t c, hs; int rc = oracle_bruteforce_csr(off.data(), adj.data(), h[0], k, q, 0, &c, &hs);
    printf("rc=%d count=%llu hash=0x%016llx\n", rc, (unsigned long long)c, (unsigned long long)hs);
}
#endif
