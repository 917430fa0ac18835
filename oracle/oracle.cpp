// CPU ORACLE — test infrastructure only.
//
// A plain C++/OpenMP restatement of the reference CudaPlex algorithm
// (MuhammadShaheer1/Maximal-kPlex-Enumeration), used to check the B200 build.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// arm may load it; the product (libkplex.so) never links or calls it.
//
// What it restates, function by function (reference paths are relative to the
// reference project root; "src" = src/device_funcs.cu, "host" = inc/host_funcs.h):
//   peel_core        host:16-122       (q-k)-core + order-preserving renumber (sequence::pack)
//   truss_prune      host:761-823 + fast_truss_peeling host:463-559 + find_pos_sorted host:405-415
//   degeneracy       inc/degeneracy.h:6-204 (ListLinearHeap) + host:829-851
//   decompose_root   src:28-298 (decompose), src:300-351 (calculateDegrees),
//                    src:353-460 (fillNeighbors), src:1727-1853 (commonEle/buildCommonMtx)
//   ksearch          src:1855-2444 (kSearch state machine, states 0..5) with
//                    updateCand13/23 src:1042-1122, recoverCand12/23 src:1124-1195,
//                    upperBoundK2 src:1002-1020, isKplex2 src:568-584, addG/subG src:624-641
//   bnb_node         src:1516-1724 (BNB) with initializePCX src:1474-1513,
//                    enqueue_exclude_child src:1197-1270, enqueue_include_child src:1273-1465,
//                    isKplex3 src:586-599, isKplexPC2 src:601-622, upperBound2 src:1022-1040
//   is_maximal       src:703-841 (isMaximal_opt), src:843-1000 (isMaximalPC_opt),
//                    canGlobalAdd(2) src:643-679, intersection src:680-702
//
// Deliberate differences, none of which changes the enumerated sets:
//  * Local vertex order.  The reference assigns local slots with shared-memory
//    atomics (src:87-131, 255-261), so its order is nondeterministic.  Here the
//    order is fixed: root, then C1 in CSR order (ascending peeled id), then C2
//    ascending; left ascending.  The B200 kernels use the same order, so the
//    two produce the same search tree and the same task counts.
//  * kSearch recovery tags are depth+1 instead of depth (src:1078, 1117 use
//    sz-1), so tag 0 means "not dropped".  In the reference a drop at depth 0
//    writes the already-zero tag; the only observable difference is the final
//    recovery of the depth-0 frame, which runs after the last emission.
//  * Counts are 64-bit (the reference's plex_count is u32, src:1585).
//  * k-search runs each root as |C2|+1 independent jobs, as the device does:
//    job d is the frame at depth d of the root's initial exclude chain,
//    started from C2 = its first |C2|-d vertices in ascending order.  The
//    reference's single state machine reaches that frame with C2 permuted
//    (finished frames re-append included and recovered vertices at the end,
//    src:2405-2441), so it lists some subsets under different branches; every
//    subset S of C2 with |S| <= k-1 is still enumerated exactly once, so the
//    k-plexes found are the same.  oracle_enumerate_sequential (CLI -seq)
//    keeps the reference's order.
// Parity anchors: README.md:142 (soc-epinions k=4 q=30 -> 13,172,906) and
// README.md:144 (email-euall k=3 q=12 -> 32,639,016), checked by tests/.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>
#include <vector>
#include <string>
#include <algorithm>
#include <atomic>
#include <memory>
#include <chrono>
#include <omp.h>

namespace oracle {

static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static const uint64_t HASH_SEED = 0x6b706c6578b200ULL;

struct Graph {
    uint32_t n = 0;
    std::vector<uint32_t> off, adj, deg;
};

enum : uint8_t { LP = 0, LC = 1, LX = 2, LU = 3, LH = 5 };                 // common.h:27-34
enum : uint8_t { UNLINK2LESS = 0, LINK2LESS = 1, UNLINK2EQUAL = 2, LINK2EQUAL = 3, UNLINK2MORE = 4, LINK2MORE = 5 };  // common.h:37-44

// The reference keeps at most MAX_BLK_SIZE = 1024 one-hop neighbours of a root
// (common.h:8): 1023 later ones and 1024 earlier ones in CSR order (src:87-131);
// the rest are dropped.  That truncation is part of its semantics and is kept.
static const int REF_BLK = 1024;
// Capacity of a root's local subgraph (root, C1, C2).  The reference overruns
// its 1024-entry buffers beyond REF_BLK (src:255); this restatement and the
// device build accept up to 2048 local vertices and left sets up to 8192.
static const int MAX_LOCAL = 2048;
static const int MAX_LEFT = 8192;
// The reference's k-search stack holds MAX_DEPTH = 1000 frames (common.h:15) and
// abandons the rest of a root when it would go deeper (src:1987-1991), which
// loses results on roots with about 1000 or more C2 vertices.  A path pushes at
// most one frame per C2 vertex plus a leaf frame, so a stack of MAX_LOCAL + 8
// frames never fills here and no root is abandoned; where the reference's
// stack does not fill, the two enumerate the same sets.
static const int MAX_DEPTH = MAX_LOCAL + 8;

struct Params { int k, q, truss; };

// ---------------------------------------------------------------- preprocessing
// host:16-122.  Survivors are the (q-k)-core; ids are renumbered in ascending
// order and each kept neighbour list keeps its order.  `orig` maps new -> old.
static Graph peel_core(const Graph& g, int bd, std::vector<uint32_t>& orig_of_new) {
    const uint32_t n = g.n;
    std::vector<char> alive(n, 1);
    std::vector<int> res(n);
    std::vector<uint32_t> q;
    for (uint32_t i = 0; i < n; ++i) { res[i] = (int)g.deg[i]; if ((int)g.deg[i] < bd) { alive[i] = 0; q.push_back(i); } }
    for (size_t h = 0; h < q.size(); ++h) {
        uint32_t v = q[h];
        for (uint32_t j = g.off[v]; j < g.off[v + 1]; ++j) {
            uint32_t w = g.adj[j];
            if (alive[w]) { if (res[w]-- == bd) { alive[w] = 0; q.push_back(w); } }
        }
    }
    std::vector<int64_t> mp(n, -1);
    std::vector<uint32_t> keep;
    for (uint32_t i = 0; i < n; ++i) if (alive[i]) { mp[i] = keep.size(); keep.push_back(i); }
    Graph r;
    r.n = keep.size();
    r.off.assign(r.n + 1, 0);
    r.deg.assign(r.n, 0);
    for (uint32_t i = 0; i < r.n; ++i) {
        uint32_t o = keep[i], c = 0;
        for (uint32_t j = g.off[o]; j < g.off[o + 1]; ++j) if (alive[g.adj[j]]) ++c;
        r.deg[i] = c; r.off[i + 1] = r.off[i] + c;
    }
    r.adj.resize(r.off[r.n]);
    for (uint32_t i = 0; i < r.n; ++i) {
        uint32_t o = keep[i], cur = r.off[i];
        for (uint32_t j = g.off[o]; j < g.off[o + 1]; ++j) if (alive[g.adj[j]]) r.adj[cur++] = (uint32_t)mp[g.adj[j]];
    }
    std::vector<uint32_t> composed(r.n);
    for (uint32_t i = 0; i < r.n; ++i) composed[i] = orig_of_new.empty() ? keep[i] : orig_of_new[keep[i]];
    orig_of_new.swap(composed);
    return r;
}

static int find_pos_sorted(const Graph& g, uint32_t u, uint32_t v) {   // host:405-415
    auto b = g.adj.begin() + g.off[u], e = g.adj.begin() + g.off[u + 1];
    auto it = std::lower_bound(b, e, v);
    if (it == e || *it != v) return -1;
    return (int)(it - g.adj.begin());
}

// host:761-822 (triangle count + initial edge queue) and host:463-559
// (serial LIFO edge peel with per-direction support counters).  Mutates g.
static void truss_prune(Graph& g, int thr /* = q - 2k */) {
    const uint32_t pn = g.n;
    const uint32_t m = g.off[pn];
    std::vector<int> tri(m, 0);
    std::vector<std::pair<uint32_t, uint32_t>> Qe;
    for (uint32_t i = 0; i < pn; ++i) {
        for (uint32_t p = g.off[i]; p < g.off[i + 1]; ++p) {
            uint32_t v = g.adj[p];
            uint32_t iu = g.off[i], eu = g.off[i + 1], iv = g.off[v], ev = g.off[v + 1];
            int common = 0;
            while (iu < eu && iv < ev) {
                uint32_t a = g.adj[iu], b = g.adj[iv];
                if (a == b) { ++common; ++iu; ++iv; } else if (a < b) ++iu; else ++iv;
            }
            tri[p] = common;
        }
    }
    for (uint32_t i = 0; i < pn; ++i)
        for (uint32_t p = g.off[i]; p < g.off[i + 1]; ++p)
            if (i < g.adj[p] && tri[p] < thr) Qe.push_back({i, g.adj[p]});
    std::vector<uint8_t> dead(m, 0);
    while (!Qe.empty()) {
        auto uv = Qe.back(); Qe.pop_back();
        uint32_t u = uv.first, v = uv.second;
        int puv = find_pos_sorted(g, u, v), pvu = find_pos_sorted(g, v, u);
        if (puv >= 0 && !dead[puv]) { dead[puv] = 1; g.deg[u]--; }
        if (pvu >= 0 && !dead[pvu]) { dead[pvu] = 1; g.deg[v]--; }
        uint32_t iu = g.off[u], eu = g.off[u + 1], iv = g.off[v], ev = g.off[v + 1];
        while (iu < eu && iv < ev) {
            while (iu < eu && dead[iu]) ++iu;
            while (iv < ev && dead[iv]) ++iv;
            if (iu >= eu || iv >= ev) break;
            uint32_t a = g.adj[iu], b = g.adj[iv];
            if (a == b) {
                if (!dead[iu]) { int prev = tri[iu]; if (prev > 0) { tri[iu] = prev - 1; if (prev == thr) Qe.push_back({u, a}); } }
                if (!dead[iv]) { int prev = tri[iv]; if (prev > 0) { tri[iv] = prev - 1; if (prev == thr) Qe.push_back({v, a}); } }
                ++iu; ++iv;
            } else if (a < b) ++iu; else ++iv;
        }
    }
    uint32_t w = 0;
    for (uint32_t u = 0; u < pn; ++u) {
        uint32_t b = g.off[u], e = g.off[u + 1];
        g.off[u] = w;
        for (uint32_t i = b; i < e; ++i) if (!dead[i]) g.adj[w++] = g.adj[i];
    }
    g.off[pn] = w;
    g.adj.resize(w);
}

// inc/degeneracy.h ListLinearHeap restated (LIFO bucket lists, min pointer
// that only rises in tighten()) and the pop loop of host:829-851.
static void degeneracy(const Graph& g, std::vector<int>& dpos, std::vector<int>& dseq) {
    const int n = (int)g.n;
    dpos.assign(n, INT_MAX); dseq.assign(n, 0);
    if (n == 0) return;
    const int NIL = n;
    std::vector<int> keys(n), pres(n), nexts(n), heads(n, NIL);
    int min_key = n - 1;
    auto insert = [&](int id, int key) {
        keys[id] = key; pres[id] = NIL; nexts[id] = heads[key];
        if (heads[key] != NIL) pres[heads[key]] = id;
        heads[key] = id;
        if (key < min_key) min_key = key;
    };
    auto remove = [&](int id) {
        if (pres[id] == NIL) { heads[keys[id]] = nexts[id]; if (nexts[id] != NIL) pres[nexts[id]] = NIL; }
        else { int pid = pres[id]; nexts[pid] = nexts[id]; if (nexts[id] != NIL) pres[nexts[id]] = pid; }
    };
    for (int i = 0; i < n; ++i) insert(i, (int)g.deg[i]);
    for (int i = 0; i < n; ++i) {
        while (heads[min_key] == NIL) ++min_key;
        int u = heads[min_key];
        heads[min_key] = nexts[u];
        if (heads[min_key] != NIL) pres[heads[min_key]] = NIL;
        dpos[u] = i; dseq[i] = u;
        for (uint32_t j = 0; j < g.deg[u]; ++j) {
            int w = (int)g.adj[g.off[u] + j];
            if (dpos[w] == INT_MAX) { int nk = keys[w] - 1; remove(w); insert(w, nk); }
        }
    }
}

// ---------------------------------------------------------------- per-root subgraph
struct Sub {
    int n = 0, hop = 0, nleft = 0;
    uint32_t root_rank = 0;
    std::vector<uint32_t> gid, lgid;        // peeled ids of blk / left
    std::vector<std::vector<int>> nb;       // local adjacency, ascending local index
    std::vector<std::vector<int>> lnb;      // left adjacency (left indices), ascending
    std::vector<int> degHop;
    std::vector<uint8_t> cls;               // n*n pair class
    std::vector<uint64_t> bits;             // n*n adjacency bits
    bool adj(int u, int v) const { size_t c = (size_t)u * n + v; return (bits[c >> 6] >> (c & 63)) & 1; }
};

struct Stats {
    std::atomic<uint64_t> count{0}, hash{0}, tasks{0}, valid{0}, truncated{0}, depth_cap{0}, too_big{0};
    std::atomic<uint32_t> max_n{0}, max_left{0};
};

static bool in_sorted(const Graph& g, uint32_t v, uint32_t x) {   // binary_search src:14-26
    return std::binary_search(g.adj.begin() + g.off[v], g.adj.begin() + g.off[v + 1], x);
}

// Returns false if the root is skipped (src:148, 279-283).
static bool decompose_root(const Graph& g, const std::vector<int>& dpos, const std::vector<int>& dseq,
                           uint32_t ri, const Params& P, Sub& s, Stats& st) {
    const int k = P.k, q = P.q, lb2k = q - 2 * k, bd = q - k;
    const uint32_t r = dseq[ri];
    const int pos = dpos[r];
    std::vector<uint32_t> later, earlier;
    for (uint32_t j = g.off[r]; j < g.off[r + 1]; ++j) {
        uint32_t w = g.adj[j];
        if (pos < dpos[w]) later.push_back(w); else earlier.push_back(w);
    }
    if (later.size() + 1 > (size_t)REF_BLK || earlier.size() > (size_t)REF_BLK) st.truncated++;
    if (later.size() + 1 > (size_t)REF_BLK) later.resize(REF_BLK - 1);
    if (earlier.size() > (size_t)REF_BLK) earlier.resize(REF_BLK);
    // C1 peel, src:142-180: synchronous rounds until nothing is removed
    std::vector<uint32_t> c1 = later;
    for (;;) {
        if ((int)c1.size() < bd) return false;
        std::vector<uint32_t> nxt;
        for (uint32_t u : c1) {
            int cnt = 0;
            for (uint32_t v : c1) if (in_sorted(g, u, v)) ++cnt;
            if (cnt >= lb2k) nxt.push_back(u);
        }
        if (nxt.size() == c1.size()) break;
        c1.swap(nxt);
    }
    const int hop = 1 + (int)c1.size();
    // left filter, src:188-213
    std::vector<uint32_t> left;
    for (uint32_t u : earlier) {
        int cnt = 0;
        for (uint32_t v : c1) if (in_sorted(g, u, v)) ++cnt;
        if (cnt >= lb2k + 1) left.push_back(u);
    }
    // 2-hop scan, src:217-273 (visited = root, kept C1, kept left, scanned).
    // Membership marks live in a per-thread array indexed by peeled id and are
    // cleared before returning.
    thread_local std::vector<uint8_t> mark;
    if (mark.size() < g.n) mark.assign(g.n, 0);
    std::vector<uint32_t> touched;
    auto put = [&](uint32_t v) { if (!mark[v]) touched.push_back(v); mark[v] = 1; };
    put(r);
    for (uint32_t v : c1) put(v);
    for (uint32_t v : left) put(v);
    std::vector<uint32_t> c2, left2;
    for (uint32_t nei : later) {
        for (uint32_t j = g.off[nei]; j < g.off[nei + 1]; ++j) {
            uint32_t w = g.adj[j];
            if (mark[w]) continue;   // visited, or already scanned
            const bool lat = pos < dpos[w];
            const int thr = lb2k + (lat ? 2 : 3);
            if (std::min<int>((int)g.deg[w], hop - 1) < thr) continue;
            int cnt = 0;
            for (uint32_t v : c1) if (in_sorted(g, w, v)) ++cnt;
            put(w);
            if (lat) { if (cnt >= lb2k + 2) c2.push_back(w); }
            else { if (cnt >= lb2k + 3) left2.push_back(w); }
        }
    }
    for (uint32_t v : touched) mark[v] = 0;
    std::sort(c2.begin(), c2.end());
    left.insert(left.end(), left2.begin(), left2.end());
    std::sort(left.begin(), left.end());
    const int n = hop + (int)c2.size();
    s.n = n; s.nleft = (int)left.size();
    if (n < q) return false;
    st.valid++;
    if (n > MAX_LOCAL || (int)left.size() > MAX_LEFT) { st.too_big++; return false; }
    {
        uint32_t cur = st.max_n.load(); while ((uint32_t)n > cur && !st.max_n.compare_exchange_weak(cur, n)) {}
        cur = st.max_left.load(); while ((uint32_t)left.size() > cur && !st.max_left.compare_exchange_weak(cur, (uint32_t)left.size())) {}
    }
    s.n = n; s.hop = hop; s.nleft = (int)left.size(); s.root_rank = ri;
    s.gid.clear(); s.gid.push_back(r); s.gid.insert(s.gid.end(), c1.begin(), c1.end()); s.gid.insert(s.gid.end(), c2.begin(), c2.end());
    s.lgid = left;
    // fillNeighbors src:405-443: local and left adjacency lists in ascending
    // local (left) index, found through per-thread id -> index maps
    thread_local std::vector<int32_t> lidx, leftidx;
    if (lidx.size() < g.n) { lidx.assign(g.n, -1); leftidx.assign(g.n, -1); }
    for (int i = 0; i < n; ++i) lidx[s.gid[i]] = i;
    for (int j = 0; j < s.nleft; ++j) leftidx[left[j]] = j;
    s.nb.assign(n, {}); s.lnb.assign(n, {}); s.degHop.assign(n, 0);
    s.bits.assign(((size_t)n * n + 63) / 64, 0);
    s.cls.assign((size_t)n * n, 0);
    for (int i = 0; i < n; ++i) {
        const uint32_t o = s.gid[i];
        for (uint32_t e = g.off[o]; e < g.off[o + 1]; ++e) {
            const int j = lidx[g.adj[e]], jl = leftidx[g.adj[e]];
            if (j >= 0) s.nb[i].push_back(j);
            if (jl >= 0) s.lnb[i].push_back(jl);
        }
        std::sort(s.nb[i].begin(), s.nb[i].end());
        std::sort(s.lnb[i].begin(), s.lnb[i].end());
        int cnt = 0;
        for (int j : s.nb[i]) {
            size_t c = (size_t)i * n + j; s.bits[c >> 6] |= 1ull << (c & 63);
            s.cls[(size_t)i * n + j] = 1;
            if (j < hop) ++cnt;
        }
        s.degHop[i] = cnt;
    }
    for (int i = 0; i < n; ++i) lidx[s.gid[i]] = -1;
    for (int j = 0; j < s.nleft; ++j) leftidx[left[j]] = -1;
    // buildCommonMtx src:1751-1853
    const int tPP1 = q - k - 2 * std::max(k - 2, 0), tPP2 = q - k - 2 * std::max(k - 3, 0);
    const int tPC1 = q - 2 * k - std::max(k - 2, 0), tPC2 = q - k - 1 - std::max(k - 2, 0) - std::max(k - 3, 0);
    const int tCC1 = q - 2 * k - (k - 1), tCC2 = q - 2 * k + 2 - (k - 1);
    // commonEle src:1727-1749: common neighbours of i and j among local ids [0, hop),
    // counted as the popcount of their adjacency rows restricted to [0, hop)
    const int hw = (hop + 63) / 64;
    std::vector<uint64_t> hb((size_t)n * hw, 0);
    for (int i = 0; i < n; ++i)
        for (int j : s.nb[i]) { if (j >= hop) break; hb[(size_t)i * hw + (j >> 6)] |= 1ull << (j & 63); }
    auto common = [&](int i, int j) {
        int c = 0;
        for (int w = 0; w < hw; ++w) c += __builtin_popcountll(hb[(size_t)i * hw + w] & hb[(size_t)j * hw + w]);
        return c;
    };
    auto classify = [&](int i, int j, int t1, int t2) {
        const int c = common(i, j);
        uint8_t& cell = s.cls[(size_t)i * n + j];
        if (cell) cell = c > t1 ? LINK2MORE : (c == t1 ? LINK2EQUAL : LINK2LESS);
        else cell = c > t2 ? UNLINK2MORE : (c == t2 ? UNLINK2EQUAL : UNLINK2LESS);
        s.cls[(size_t)j * n + i] = cell;
    };
    for (int i = 0; i < hop; ++i) for (int j = 0; j < i; ++j) classify(i, j, tCC1, tCC2);
    for (int i = hop; i < n; ++i) {
        for (int j = 0; j < hop; ++j) classify(i, j, tPC1, tPC2);
        if (k == 2) continue;   // src:1822: C2 x C2 keep raw 0/1 when k == 2
        for (int j = hop; j < i; ++j) classify(i, j, tPP1, tPP2);
    }
    return true;
}

// ---------------------------------------------------------------- search state
struct Task {
    std::vector<uint8_t> lab;
    std::vector<uint16_t> g, p;
    int np = 0, nc = 0, nx = 0;
};

struct Ctx {
    const Sub& s;
    const Params& P;
    const std::vector<uint32_t>& orig;  // peeled id -> original id
    Stats& st;
    uint64_t cnt = 0, hsum = 0, tasks = 0;
    std::vector<uint16_t> sat, commons;
    std::vector<uint32_t> uni;
    Ctx(const Sub& s_, const Params& p_, const std::vector<uint32_t>& o, Stats& st_) : s(s_), P(p_), orig(o), st(st_) {
        sat.resize(MAX_LOCAL); commons.resize(MAX_LEFT); uni.assign(MAX_LEFT / 32, 0);
    }
};

static void emit_plex(Ctx& c, const std::vector<int>& a, const std::vector<int>& b) {
    std::vector<uint32_t> ids;
    ids.reserve(a.size() + b.size());
    for (int v : a) ids.push_back(c.orig[c.s.gid[v]]);
    for (int v : b) ids.push_back(c.orig[c.s.gid[v]]);
    std::sort(ids.begin(), ids.end());
    uint64_t x = splitmix64(HASH_SEED ^ (uint64_t)ids.size());
    for (uint32_t v : ids) x = splitmix64(x ^ (uint64_t)v);
    c.cnt++; c.hsum += x;
}

static bool lbin(const std::vector<int>& l, int x) { return std::binary_search(l.begin(), l.end(), x); }

// isMaximal_opt / isMaximalPC_opt, src:703-1000.  S = plex (+ cand for the PC
// form); nn[] is neiInP (resp. neiInG).  True if no left vertex u makes S+u a k-plex.
static bool is_maximal(Ctx& c, const std::vector<int>& plex, const std::vector<int>* cand, const uint16_t* nn) {
    const Sub& s = c.s;
    const int k = c.P.k;
    const int PlexSz = (int)plex.size(), CandSz = cand ? (int)cand->size() : 0, tot = PlexSz + CandSz;
    auto at = [&](int i) { return i < PlexSz ? plex[i] : (*cand)[i - PlexSz]; };
    int nsat = 0;
    for (int i = 0; i < tot; ++i) { int v = at(i); if (nn[v] + k < tot + 1) c.sat[nsat++] = (uint16_t)v; }
    auto can_add = [&](int u) {   // canGlobalAdd(2) src:643-679
        int cnt = 0;
        for (int i = 0; i < tot; ++i) if (lbin(s.lnb[at(i)], u)) ++cnt;
        return cnt + k >= tot + 1;
    };
    bool maximal = true;
    if (nsat) {
        const auto& l0 = s.lnb[c.sat[0]];
        int szcom = (int)l0.size();
        for (int i = 0; i < szcom; ++i) c.commons[i] = (uint16_t)l0[i];
        for (int i = 1; i < nsat; ++i) {
            const auto& l = s.lnb[c.sat[i]];
            int a = 0, b = 0, w = 0;
            while (a < szcom && b < (int)l.size()) {
                if (c.commons[a] == l[b]) { c.commons[w++] = c.commons[a]; ++a; ++b; }
                else if (c.commons[a] < l[b]) ++a; else ++b;
            }
            szcom = w;
        }
        if (nsat == 1) {
            for (int t = 0; t < k; ++t) for (int v : s.lnb[at(t)]) c.uni[v >> 5] |= 1u << (v & 31);
            int w = 0;
            for (int i = 0; i < szcom; ++i) { int v = c.commons[i]; if ((c.uni[v >> 5] >> (v & 31)) & 1u) c.commons[w++] = (uint16_t)v; }
            szcom = w;
        }
        for (int i = 0; i < szcom && maximal; ++i) if (can_add(c.commons[i])) maximal = false;
        std::fill(c.uni.begin(), c.uni.end(), 0u);
    } else {
        int szcom = 0;
        for (int t = 0; t < k; ++t)
            for (int v : s.lnb[at(t)]) {
                if ((c.uni[v >> 5] >> (v & 31)) & 1u) continue;
                c.commons[szcom++] = (uint16_t)v;
                c.uni[v >> 5] |= 1u << (v & 31);
            }
        for (int i = 0; i < szcom && maximal; ++i) if (can_add(c.commons[i])) maximal = false;
        std::fill(c.uni.begin(), c.uni.end(), 0u);
    }
    return maximal;
}

// isKplex3 src:586-599 (isKplex2 src:568-584 is the same predicate evaluated by a warp)
static bool is_kplex3(const Sub& s, int v, int k, int PlexSz, const uint16_t* nP, const std::vector<int>& plex) {
    if (nP[v] + k < PlexSz + 1) return false;
    for (int i = 0; i < PlexSz; ++i) { int u = plex[i]; if (nP[u] + k == PlexSz && !s.adj(u, v)) return false; }
    return true;
}

static void subG(const Sub& s, int j, uint16_t* g) { for (int w : s.nb[j]) g[w]--; }   // src:624-631
static void addG(const Sub& s, int j, uint16_t* g) { for (int w : s.nb[j]) g[w]++; }   // src:633-641

// The warp reduction of the candidate pivot (src:1628-1663, 1669-1697): lane L
// scans cand[i] for i = L, L+32, ...; then a shfl_down tree with offsets
// 16..1 keeps the current value unless the other is strictly smaller in
// neiInG, or equal with a strictly smaller neiInP.
template <typename F>
static void lane_select(const std::vector<int>& cand, F consider, int init_min, int init_piv,
                        const uint16_t* g, const uint16_t* p, int& out_min, int& out_piv) {
    int lm[32], li[32];
    for (int L = 0; L < 32; ++L) { lm[L] = init_min; li[L] = init_piv; }
    for (size_t i = 0; i < cand.size(); ++i) {
        const int L = (int)(i & 31), v = cand[i];
        if (!consider(v)) continue;
        if ((int)g[v] < lm[L]) { lm[L] = g[v]; li[L] = v; }
        else if ((int)g[v] == lm[L] && p[li[L]] > p[v]) li[L] = v;
    }
    for (int off = 16; off > 0; off >>= 1) {
        int nm[32], ni[32];
        for (int L = 0; L < 32; ++L) {
            int om = (L + off < 32) ? lm[L + off] : lm[L];
            int oi = (L + off < 32) ? li[L + off] : li[L];
            nm[L] = lm[L]; ni[L] = li[L];
            if (om < lm[L] || (om == lm[L] && oi != -1 && p[li[L]] > p[oi])) { nm[L] = om; ni[L] = oi; }
        }
        memcpy(lm, nm, sizeof lm); memcpy(li, ni, sizeof li);
    }
    out_min = lm[0]; out_piv = li[0];
}

static void bnb(Ctx& c, Task& t);

// enqueue_exclude_child + enqueue_include_child (src:1197-1465), children run depth-first.
static void branch(Ctx& c, Task& t, std::vector<int>& plex, std::vector<int>& cand, std::vector<int>& excl, int v) {
    const Sub& s = c.s;
    const int k = c.P.k, q = c.P.q, n = s.n;
    {   // exclude child
        Task e;
        e.lab.assign(n, LU);
        for (int u : plex) e.lab[u] = LP;
        for (int u : cand) e.lab[u] = LC;
        for (int u : excl) e.lab[u] = LX;
        e.lab[v] = LX;
        e.g = t.g; e.p = t.p;
        subG(s, v, e.g.data());
        e.np = (int)plex.size(); e.nc = (int)cand.size() - 1; e.nx = (int)excl.size() + 1;
        c.tasks++;
        bnb(c, e);
    }
    // include child: works on t's arrays in place (the reference does too)
    plex.push_back(v);
    for (size_t i = 0; i < cand.size(); ++i) if (cand[i] == v) { std::swap(cand[i], cand.back()); cand.pop_back(); break; }
    for (int w : s.nb[v]) t.p[w]++;
    const int PlexSz = (int)plex.size();
    const uint8_t* row = &s.cls[(size_t)v * n];
    std::vector<int> keep;
    for (int u : cand) {
        if (!(row[u] < UNLINK2EQUAL) && is_kplex3(s, u, k, PlexSz, t.p.data(), plex)) keep.push_back(u);
        else subG(s, u, t.g.data());
    }
    cand.swap(keep);
    for (int u : plex) if (t.g[u] + k < q) return;   // upperBound2 src:1022-1040
    std::vector<int> kx;
    for (int u : excl) if (!(row[u] < UNLINK2MORE) && is_kplex3(s, u, k, PlexSz, t.p.data(), plex)) kx.push_back(u);
    Task ic;
    ic.lab.assign(n, LU);
    for (int u : plex) ic.lab[u] = LP;
    for (int u : cand) ic.lab[u] = LC;
    for (int u : kx) ic.lab[u] = LX;
    ic.g.swap(t.g); ic.p.swap(t.p);
    ic.np = PlexSz; ic.nc = (int)cand.size(); ic.nx = (int)kx.size();
    c.tasks++;
    bnb(c, ic);
}

// BNB kernel body, src:1516-1724, for one task.
static void bnb(Ctx& c, Task& t) {
    const Sub& s = c.s;
    const int k = c.P.k, q = c.P.q, n = s.n;
    std::vector<int> plex, cand, excl;   // initializePCX: ascending local index
    for (int i = 0; i < n; ++i) { if (t.lab[i] == LP) plex.push_back(i); else if (t.lab[i] == LC) cand.push_back(i); else if (t.lab[i] == LX) excl.push_back(i); }
    const int PlexSz = (int)plex.size(), CandSz = (int)cand.size(), ExclSz = (int)excl.size();
    if (PlexSz + CandSz < q) return;
    if (CandSz == 0) {
        if (ExclSz == 0 && PlexSz >= q && is_maximal(c, plex, nullptr, t.p.data())) emit_plex(c, plex, {});
        return;
    }
    const uint16_t* g = t.g.data();
    const uint16_t* p = t.p.data();
    int minP = INT_MAX, pp = -1;
    for (int v : plex) if ((int)g[v] < minP || ((int)g[v] == minP && v < pp)) { minP = g[v]; pp = v; }
    if (minP + k < std::max(q, PlexSz)) return;
    if (minP + k < PlexSz + CandSz) {
        int mn, piv;
        lane_select(cand, [&](int v) { return !s.adj(v, pp); }, INT_MAX, -1, g, p, mn, piv);
        branch(c, t, plex, cand, excl, piv);
        return;
    }
    int mn, piv;
    lane_select(cand, [](int) { return true; }, minP, pp, g, p, mn, piv);
    if (mn >= PlexSz + CandSz - k) {
        if (PlexSz + CandSz < q) return;
        const int tot = PlexSz + CandSz;
        for (int v : excl) {   // isKplexPC2 src:601-622
            if (g[v] + k < tot + 1) continue;
            bool ok = true;
            for (int u : plex) if (g[u] + k == tot && !s.adj(u, v)) { ok = false; break; }
            if (ok) for (int u : cand) if (g[u] + k == tot && !s.adj(u, v)) { ok = false; break; }
            if (ok) return;
        }
        if (is_maximal(c, plex, &cand, g)) emit_plex(c, plex, cand);
        return;
    }
    branch(c, t, plex, cand, excl, piv);
}

// ---------------------------------------------------------------- kSearch
// src:1855-2444, state machine restated for one root; each emitted task is
// handed to `sink` (which runs branch-and-bound on it).
template <typename Sink>
static void ksearch(const Sub& s, const Params& P, Stats& st, uint64_t& tasks, Sink sink, int job_d = -1) {
    const int n = s.n, k = P.k, q = P.q, hop = s.hop;
    std::vector<uint16_t> G(n), Pn(n, 0);
    for (int i = 0; i < n; ++i) G[i] = (uint16_t)s.degHop[i];
    for (int w : s.nb[0]) Pn[w]++;
    std::vector<int> plex{0}, cand1, cand2, excl;
    for (int i = 1; i < hop; ++i) cand1.push_back(i);
    for (int i = hop; i < n; ++i) cand2.push_back(i);
    std::vector<int> rec1(n, 0), rec2(n, 0);
    std::vector<int> res(MAX_DEPTH + 2), br(MAX_DEPTH + 2), state(MAX_DEPTH + 2), v2d(MAX_DEPTH + 2);
    auto UB = [&]() { for (int u : plex) if (G[u] + k < q) return false; return true; };   // upperBoundK2
    auto include = [&](int u) {
        plex.push_back(u);
        for (int w : s.nb[u]) Pn[w]++;
        addG(s, u, G.data());
    };
    auto update13 = [&](int node, int tag) {   // updateCand13 src:1042-1097
        const uint8_t* row = &s.cls[(size_t)node * n];
        std::vector<int> keep;
        for (int v : cand1) { if (!(row[v] < UNLINK2EQUAL)) keep.push_back(v); else { rec1[v] = tag; subG(s, v, G.data()); } }
        cand1.swap(keep);
    };
    auto update23 = [&](int node, int tag) {   // updateCand23 src:1099-1122
        const uint8_t* row = &s.cls[(size_t)node * n];
        std::vector<int> keep;
        for (int v : cand2) { if (!(row[v] < UNLINK2EQUAL)) keep.push_back(v); else rec2[v] = tag; }
        cand2.swap(keep);
    };
    auto remove_excl = [&](int u) {
        for (size_t i = 0; i < excl.size(); ++i) if (excl[i] == u) { excl[i] = excl.back(); excl.pop_back(); return; }
    };
    auto emit = [&]() {
        Task t;
        t.lab.assign(n, LU);
        for (int v : plex) t.lab[v] = LP;
        for (int v : cand1) t.lab[v] = LC;
        for (int v : cand2) t.lab[v] = LH;
        for (int v : excl) t.lab[v] = LX;
        t.g = G; t.p = Pn;
        t.np = (int)plex.size(); t.nc = (int)cand1.size(); t.nx = (int)excl.size();
        tasks++;
        sink(t);
    };
    int sz = 0;
    res[0] = k - 1; br[0] = 1; state[0] = 0; sz = 1;
    if (job_d >= 0) {
        // job d of the root (see ks_start in the device code): the exclude-chain frame at
        // depth d, from state 2 (d < |C2|) or the chain's bottom leaf (d == |C2|)
        const int m = n - hop;
        for (int i = 0; i < job_d; ++i) { excl.push_back(cand2.back()); cand2.pop_back(); }
        state[0] = job_d < m ? 2 : 0;
    }
    while (sz) {
        if (sz >= MAX_DEPTH) { st.depth_cap++; break; }   // cannot happen (see MAX_DEPTH)
        const int f = sz - 1;
        const int tag = f + 1;
        switch (state[f]) {
        case 0:
            if (cand2.empty()) {
                if ((int)(plex.size() + cand1.size()) < q) { sz--; continue; }
                if (plex.size() > 1 && !UB()) { sz--; continue; }
                emit();
                sz--; continue;
            } else {
                int u = cand2.back(); cand2.pop_back(); excl.push_back(u); v2d[f] = u;
                res[sz] = res[f]; br[sz] = 1; state[sz] = 0; state[f] = 1; sz++;
                continue;
            }
        case 1: {
            state[f] = 2; int u = v2d[f]; cand2.push_back(u); remove_excl(u);
            continue;
        }
        case 2:
            if (br[f] < res[f]) {
                int u = cand2.back(); cand2.pop_back();
                include(u);
                update13(u, tag);
                update23(u, tag);
                if (!cand2.empty()) {
                    int w = cand2.back(); cand2.pop_back(); excl.push_back(w); v2d[f] = w;
                    state[f] = 3; res[sz] = res[f] - br[f]; br[sz] = 1; state[sz] = 0; sz++;
                } else {
                    state[f] = 4; res[sz] = res[f] - br[f]; br[sz] = 1; state[sz] = 0; sz++;
                }
                continue;
            }
            state[f] = 4;
            continue;
        case 3: {
            br[f]++; state[f] = 2; int u = v2d[f]; cand2.push_back(u); remove_excl(u);
            continue;
        }
        case 4:
            if (br[f] == res[f]) {
                int u = cand2.back(); cand2.pop_back();
                include(u);
                update13(u, tag);
                if ((int)(plex.size() + cand1.size()) < q) { state[f] = 5; continue; }
                if (plex.size() > 1 && !UB()) { state[f] = 5; continue; }
                // isKplex2 filter, src:2296-2313: failing C1 vertices are swapped to
                // the tail (Cand1Sz shrinks) and restored after the emission (src:2397-2403)
                const int PlexSz = (int)plex.size();
                std::vector<int> removed;
                for (int i = 0; i < (int)cand1.size(); ++i) {
                    int v = cand1[i];
                    if (!is_kplex3(s, v, k, PlexSz, Pn.data(), plex)) {
                        std::swap(cand1[i], cand1.back());
                        cand1.pop_back();
                        removed.push_back(v);
                        subG(s, v, G.data());
                        --i;
                    }
                }
                emit();
                for (size_t i = removed.size(); i-- > 0;) { cand1.push_back(removed[i]); addG(s, removed[i], G.data()); }
                state[f] = 5;
                continue;
            }
            state[f] = 5;
            continue;
        case 5:
            for (int i = br[f]; i >= 1; --i) {
                int node = plex.back(); plex.pop_back(); cand2.push_back(node);
                for (int w : s.nb[node]) Pn[w]--;
                subG(s, node, G.data());
            }
            for (int i = 0; i < n; ++i) if (rec1[i] == tag) { cand1.push_back(i); rec1[i] = 0; addG(s, i, G.data()); }
            for (int i = 0; i < n; ++i) if (rec2[i] == tag) { cand2.push_back(i); rec2[i] = 0; }
            sz--;
            continue;
        }
    }
}

// ---------------------------------------------------------------- driver
struct Result {
    uint64_t count = 0, hash = 0, tasks = 0, valid = 0, truncated = 0, depth_cap = 0, too_big = 0;
    uint32_t pn = 0, pm = 0, max_n = 0, max_left = 0;
    double ms_pre = 0, ms_search = 0;
};

static void preprocess(const Graph& g0, const Params& P, Graph& pg, std::vector<int>& dpos, std::vector<int>& dseq,
                       std::vector<uint32_t>& orig) {
    orig.clear();
    pg = peel_core(g0, P.q - P.k, orig);
    if (P.truss) {
        truss_prune(pg, P.q - 2 * P.k);
        pg = peel_core(pg, P.q - P.k, orig);
    }
    degeneracy(pg, dpos, dseq);
}

static Result run(const Graph& g0, const Params& P, int threads, uint64_t root_begin, uint64_t root_end,
                  uint32_t shard_index = 0, uint32_t shard_count = 1, bool sequential_ksearch = false,
                  const uint8_t* owner = nullptr, uint64_t nowner = 0) {
    Result R;
    auto t0 = std::chrono::steady_clock::now();
    Graph pg; std::vector<int> dpos, dseq; std::vector<uint32_t> orig;
    preprocess(g0, P, pg, dpos, dseq, orig);
    auto t1 = std::chrono::steady_clock::now();
    R.pn = pg.n; R.pm = pg.off.empty() ? 0 : pg.off[pg.n];
    Stats st;
    const long long lim = (long long)pg.n - (long long)P.q + 2;   // src:44-45
    const uint64_t nroots = lim > 0 ? (uint64_t)lim : 0;
    const uint64_t rb = std::min(root_begin, nroots), re = std::min(root_end, nroots);
    std::atomic<uint64_t> tot_cnt{0}, tot_hash{0}, tot_tasks{0};
    if (threads > 0) omp_set_num_threads(threads);
    // plain pointers so that nested tasks never reference a finished task's frame
    const Graph* PG = &pg; const std::vector<int>* DP = &dpos; const std::vector<int>* DS = &dseq;
    const std::vector<uint32_t>* OR = &orig; Stats* ST = &st; const Params* PP = &P;
    std::atomic<uint64_t>* TC = &tot_cnt; std::atomic<uint64_t>* TH = &tot_hash; std::atomic<uint64_t>* TT = &tot_tasks;
    const bool seq = sequential_ksearch;
    // Branch-and-bound tasks are deferred while fewer than `max_out` wait to run
    // and run inline in the producing k-search otherwise, so memory stays bounded
    // on roots that produce millions of tasks.
    std::atomic<int> outstanding{0};
    std::atomic<int>* OUT = &outstanding;
    const int max_out = 8 * std::max(1, omp_get_max_threads());
#pragma omp parallel
#pragma omp single
    {
        for (uint64_t ri = rb; ri < re; ++ri) {
            if (owner ? (ri >= nowner || owner[ri] != shard_index) : (shard_count > 1 && ri % shard_count != shard_index)) continue;
#pragma omp task firstprivate(ri, PG, DP, DS, OR, ST, PP, TC, TH, TT, OUT, seq, max_out)
            {
                std::shared_ptr<Sub> sub = std::make_shared<Sub>();
                if (decompose_root(*PG, *DP, *DS, (uint32_t)ri, *PP, *sub, *ST)) {
                    const int njobs = seq ? 1 : sub->n - sub->hop + 1;
                    for (int d = 0; d < njobs; ++d) {
#pragma omp task firstprivate(d, sub, OR, ST, PP, TC, TH, TT, OUT, seq, max_out)
                        {
                            uint64_t kt = 0;
                            Ctx inl(*sub, *PP, *OR, *ST);
                            auto sink = [&](Task& t) {
                                if (OUT->load(std::memory_order_relaxed) < max_out) {
                                    OUT->fetch_add(1);
                                    std::shared_ptr<Task> tp = std::make_shared<Task>(std::move(t));
#pragma omp task firstprivate(tp, sub, OR, ST, PP, TC, TH, TT, OUT)
                                    {
                                        Ctx c(*sub, *PP, *OR, *ST);
                                        bnb(c, *tp);
                                        *TC += c.cnt; *TH += c.hsum; *TT += c.tasks;
                                        OUT->fetch_sub(1);
                                    }
                                } else {
                                    bnb(inl, t);
                                }
                            };
                            if (seq) ksearch(*sub, *PP, *ST, kt, sink);
                            else ksearch(*sub, *PP, *ST, kt, sink, d);
                            *TC += inl.cnt; *TH += inl.hsum; *TT += inl.tasks + kt;
                        }
                    }
                }
            }
        }
    }
    auto t2 = std::chrono::steady_clock::now();
    R.count = tot_cnt; R.hash = tot_hash; R.tasks = tot_tasks;
    R.valid = st.valid; R.truncated = st.truncated; R.depth_cap = st.depth_cap; R.too_big = st.too_big;
    R.max_n = st.max_n; R.max_left = st.max_left;
    R.ms_pre = std::chrono::duration<double, std::milli>(t1 - t0).count();
    R.ms_search = std::chrono::duration<double, std::milli>(t2 - t1).count();
    return R;
}

static int load_bin(const char* path, Graph& g) {
    FILE* f = fopen(path, "rb");
    if (!f) return 2;
    uint32_t h[2];
    if (fread(h, 4, 2, f) != 2) { fclose(f); return 3; }
    g.n = h[0];
    g.deg.resize(g.n);
    if (g.n && fread(g.deg.data(), 4, g.n, f) != g.n) { fclose(f); return 3; }
    g.off.assign(g.n + 1, 0);
    for (uint32_t i = 0; i < g.n; ++i) g.off[i + 1] = g.off[i] + g.deg[i];
    if (g.off[g.n] != h[1]) { fclose(f); return 3; }
    g.adj.resize(h[1]);
    if (h[1] && fread(g.adj.data(), 4, h[1], f) != h[1]) { fclose(f); return 3; }
    fclose(f);
    return 0;
}

static Graph from_csr(const uint32_t* off, const uint32_t* adj, uint32_t n) {
    Graph g;
    g.n = n;
    g.off.assign(off, off + n + 1);
    g.adj.assign(adj, adj + off[n]);
    g.deg.resize(n);
    for (uint32_t i = 0; i < n; ++i) g.deg[i] = off[i + 1] - off[i];
    return g;
}

}  // namespace oracle

// ---------------------------------------------------------------- C ABI for tests
extern "C" {

struct oracle_result {
    uint64_t count, hash, tasks, valid_roots, truncated_roots, depth_capped_roots, oversized_roots;
    uint32_t pn, pm, max_n, max_left;
    double ms_preprocess, ms_search;
};

int oracle_enumerate_csr(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                         int threads, uint64_t root_begin, uint64_t root_end, oracle_result* out) {
    if (k < 2 || q < 1) return 1;
    oracle::Graph g = oracle::from_csr(off, adj, n);
    oracle::Params P{k, q, truss};
    oracle::Result R = oracle::run(g, P, threads, root_begin, root_end);
    *out = oracle_result{R.count, R.hash, R.tasks, R.valid, R.truncated, R.depth_cap, R.too_big,
                         R.pn, R.pm, R.max_n, R.max_left, R.ms_pre, R.ms_search};
    return 0;
}

int oracle_enumerate_shard(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                           int threads, uint32_t shard_index, uint32_t shard_count, oracle_result* out) {
    if (k < 2 || q < 1 || shard_count == 0 || shard_index >= shard_count) return 1;
    oracle::Graph g = oracle::from_csr(off, adj, n);
    oracle::Params P{k, q, truss};
    oracle::Result R = oracle::run(g, P, threads, 0, UINT64_MAX, shard_index, shard_count);
    *out = oracle_result{R.count, R.hash, R.tasks, R.valid, R.truncated, R.depth_cap, R.too_big,
                         R.pn, R.pm, R.max_n, R.max_left, R.ms_pre, R.ms_search};
    return 0;
}

// The roots r (degeneracy rank) with owner[r] == me, for an explicit partition of
// the roots (the device's cost-weighted shards).
int oracle_enumerate_owned(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                           int threads, const uint8_t* owner, uint64_t nowner, uint32_t me, oracle_result* out) {
    if (k < 2 || q < 1 || !owner) return 1;
    oracle::Graph g = oracle::from_csr(off, adj, n);
    oracle::Params P{k, q, truss};
    oracle::Result R = oracle::run(g, P, threads, 0, UINT64_MAX, me, 2, false, owner, nowner);
    *out = oracle_result{R.count, R.hash, R.tasks, R.valid, R.truncated, R.depth_cap, R.too_big,
                         R.pn, R.pm, R.max_n, R.max_left, R.ms_pre, R.ms_search};
    return 0;
}

// Checks that the |C2|+1 k-search jobs of every root emit exactly the tasks of
// the sequential k-search (as multisets of label arrays).  Returns the number
// of roots that differ.
long long oracle_check_ksearch_jobs(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss) {
    oracle::Graph g = oracle::from_csr(off, adj, n), pg;
    oracle::Params P{k, q, truss};
    std::vector<int> dpos, dseq; std::vector<uint32_t> orig;
    oracle::preprocess(g, P, pg, dpos, dseq, orig);
    const long long lim = (long long)pg.n - q + 2;
    const uint64_t nroots = lim > 0 ? (uint64_t)lim : 0;
    oracle::Stats st;
    std::atomic<long long> bad{0};
#pragma omp parallel for schedule(dynamic, 1)
    for (long long ri = 0; ri < (long long)nroots; ++ri) {
        oracle::Sub s;
        if (!oracle::decompose_root(pg, dpos, dseq, (uint32_t)ri, P, s, st)) continue;
        auto sig = [](const oracle::Task& t) {
            std::string x(t.lab.begin(), t.lab.end());
            for (size_t i = 0; i < x.size(); ++i) if (x[i] == 5) x[i] = 3;   // H and U both mean "not in P, C, X"
            return x;
        };
        std::vector<std::string> a, b;
        uint64_t ta = 0, tb = 0;
        oracle::ksearch(s, P, st, ta, [&](oracle::Task& t) { a.push_back(sig(t)); });
        for (int d = 0; d <= s.n - s.hop; ++d)
            oracle::ksearch(s, P, st, tb, [&](oracle::Task& t) { b.push_back(sig(t)); }, d);
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        if (a != b) bad++;
    }
    return bad;
}

// Decomposition only: per root rank, the local size n (0 if skipped/invalid) and |left|.
long long oracle_root_sizes(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                            uint32_t* out_n, uint32_t* out_left, uint64_t cap) {
    oracle::Graph g = oracle::from_csr(off, adj, n), pg;
    oracle::Params P{k, q, truss};
    std::vector<int> dpos, dseq; std::vector<uint32_t> orig;
    oracle::preprocess(g, P, pg, dpos, dseq, orig);
    const long long lim = (long long)pg.n - q + 2;
    const uint64_t nroots = lim > 0 ? (uint64_t)lim : 0;
    oracle::Stats st;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long ri = 0; ri < (long long)std::min<uint64_t>(nroots, cap); ++ri) {
        oracle::Sub s;
        // size-only pass: decompose_root rejects n > 1024 before building matrices
        s.n = 0; s.nleft = 0;
        oracle::decompose_root(pg, dpos, dseq, (uint32_t)ri, P, s, st);
        out_n[ri] = (uint32_t)s.n;
        out_left[ri] = (uint32_t)s.nleft;
    }
    return (long long)nroots;
}

// The reference's own k-search order: one sequential state machine per root.
int oracle_enumerate_sequential(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                                int threads, oracle_result* out) {
    if (k < 2 || q < 1) return 1;
    oracle::Graph g = oracle::from_csr(off, adj, n);
    oracle::Params P{k, q, truss};
    oracle::Result R = oracle::run(g, P, threads, 0, UINT64_MAX, 0, 1, true);
    *out = oracle_result{R.count, R.hash, R.tasks, R.valid, R.truncated, R.depth_cap, R.too_big,
                         R.pn, R.pm, R.max_n, R.max_left, R.ms_pre, R.ms_search};
    return 0;
}

int oracle_enumerate_file(const char* path, int k, int q, int truss, int threads, oracle_result* out) {
    oracle::Graph g;
    int rc = oracle::load_bin(path, g);
    if (rc) return rc;
    oracle::Params P{k, q, truss};
    oracle::Result R = oracle::run(g, P, threads, 0, UINT64_MAX);
    *out = oracle_result{R.count, R.hash, R.tasks, R.valid, R.truncated, R.depth_cap, R.too_big,
                         R.pn, R.pm, R.max_n, R.max_left, R.ms_pre, R.ms_search};
    return 0;
}

// Preprocessing only: writes the peeled CSR, dpos/dseq and the peeled->original map
// into caller buffers sized n (+1 / m).  Returns pn, or -1.
long long oracle_preprocess(const uint32_t* off, const uint32_t* adj, uint32_t n, int k, int q, int truss,
                            uint32_t* out_off, uint32_t* out_adj, int32_t* out_dpos, int32_t* out_dseq,
                            uint32_t* out_orig, uint64_t* out_m) {
    oracle::Graph g = oracle::from_csr(off, adj, n), pg;
    oracle::Params P{k, q, truss};
    std::vector<int> dpos, dseq; std::vector<uint32_t> orig;
    oracle::preprocess(g, P, pg, dpos, dseq, orig);
    for (uint32_t i = 0; i <= pg.n; ++i) out_off[i] = pg.off[i];
    for (uint32_t i = 0; i < pg.off[pg.n]; ++i) out_adj[i] = pg.adj[i];
    for (uint32_t i = 0; i < pg.n; ++i) { out_dpos[i] = dpos[i]; out_dseq[i] = dseq[i]; out_orig[i] = orig[i]; }
    *out_m = pg.off[pg.n];
    return pg.n;
}

}  // extern "C"

#ifdef ORACLE_MAIN
int main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s <graph.bin> -k K -q Q [-tr 0|1] [-threads N] [-roots B E] [-shard I S] [-seq]\n", argv[0]); return 1; }
    int k = 2, q = 8, tr = 0, th = 0;
    bool seq = false;
    uint64_t rb = 0, re = UINT64_MAX;
    uint32_t si = 0, sc = 1;
    for (int i = 2; i < argc; ++i) {
        if (!strcmp(argv[i], "-k") && i + 1 < argc) k = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-q") && i + 1 < argc) q = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-tr") && i + 1 < argc) tr = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-threads") && i + 1 < argc) th = atoi(argv[++i]);
        else if (!strcmp(argv[i], "-roots") && i + 2 < argc) { rb = strtoull(argv[++i], 0, 10); re = strtoull(argv[++i], 0, 10); }
        else if (!strcmp(argv[i], "-seq")) seq = true;
        else if (!strcmp(argv[i], "-shard") && i + 2 < argc) { si = (uint32_t)atoi(argv[++i]); sc = (uint32_t)atoi(argv[++i]); }
    }
    oracle::Graph g;
    if (oracle::load_bin(argv[1], g)) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
    oracle::Params P{k, q, tr};
    oracle::Result R = oracle::run(g, P, th, rb, re, si, sc, seq);
    printf("pn=%u pm=%u valid_roots=%llu max_n=%u max_left=%u truncated=%llu depth_capped=%llu oversized=%llu\n",
           R.pn, R.pm, (unsigned long long)R.valid, R.max_n, R.max_left, (unsigned long long)R.truncated,
           (unsigned long long)R.depth_cap, (unsigned long long)R.too_big);
    printf("count=%llu hash=0x%016llx tasks=%llu\n", (unsigned long long)R.count, (unsigned long long)R.hash, (unsigned long long)R.tasks);
    printf("ms_preprocess=%.1f ms_search=%.1f threads=%d\n", R.ms_pre, R.ms_search, omp_get_max_threads());
    return 0;
}
#endif
