// .bin graph reader/writer.
//
// Layout (inc/graph.h:45-62, writer description inc/graphIO.h:13-27):
//   u32 n, u32 m (number of DIRECTED adjacency entries = 2|E|),
//   u32 degree[n], then for each vertex in order its neighbour list (u32 ids).
// The reference reader (inc/graph.h:37-65) trusts the file; this one checks
// the header against the file size, the degree sum against m and every id
// against n, and reports a status instead of exiting.
#include "graph_io.h"

#include <cstdio>
#include <cstring>
#include <algorithm>

namespace kplex {

static int read_all(FILE* f, void* dst, size_t bytes) {
    uint8_t* p = static_cast<uint8_t*>(dst);
    size_t got = 0;
    while (got < bytes) {
        size_t r = fread(p + got, 1, bytes - got, f);
        if (r == 0) return -1;
        got += r;
    }
    return 0;
}

int load_bin(const char* path, Csr& g, std::string* err) {
    FILE* f = fopen(path, "rb");
    if (!f) { if (err) *err = std::string("cannot open ") + path; return KPLEX_ERR_IO; }
    fseek(f, 0, SEEK_END);
    long long fsize = ftell(f);
    fseek(f, 0, SEEK_SET);
    uint32_t hdr[2];
    if (fsize < 8 || read_all(f, hdr, 8)) { fclose(f); if (err) *err = "truncated header"; return KPLEX_ERR_FORMAT; }
    const uint32_t n = hdr[0];
    const uint64_t m = hdr[1];
    const long long want = 8LL + 4LL * (long long)n + 4LL * (long long)m;
    if (fsize != want) {
        fclose(f);
        if (err) *err = "file size " + std::to_string(fsize) + " != header-implied " + std::to_string(want);
        return KPLEX_ERR_FORMAT;
    }
    std::vector<uint32_t> deg(n);
    if (n && read_all(f, deg.data(), 4ull * n)) { fclose(f); if (err) *err = "truncated degrees"; return KPLEX_ERR_FORMAT; }
    g.n = n;
    g.off.assign((size_t)n + 1, 0);
    uint64_t s = 0;
    for (uint32_t v = 0; v < n; ++v) { g.off[v] = (uint32_t)s; s += deg[v]; if (s > 0xFFFFFFFFull) break; }
    if (s != m) { fclose(f); if (err) *err = "degree sum != m"; return KPLEX_ERR_FORMAT; }
    g.off[n] = (uint32_t)s;
    g.adj.resize(m);
    if (m && read_all(f, g.adj.data(), 4ull * m)) { fclose(f); if (err) *err = "truncated adjacency"; return KPLEX_ERR_FORMAT; }
    fclose(f);
    return validate_csr(g, err);
}

int validate_csr(const Csr& g, std::string* err) {
    for (uint32_t v = 0; v < g.n; ++v) {
        const uint32_t b = g.off[v], e = g.off[v + 1];
        if (e < b) { if (err) *err = "offsets not monotone"; return KPLEX_ERR_FORMAT; }
        for (uint32_t i = b; i < e; ++i) {
            const uint32_t w = g.adj[i];
            if (w >= g.n) { if (err) *err = "neighbour id out of range at vertex " + std::to_string(v); return KPLEX_ERR_FORMAT; }
            if (w == v) { if (err) *err = "self loop at vertex " + std::to_string(v); return KPLEX_ERR_FORMAT; }
            if (i > b && g.adj[i - 1] >= w) { if (err) *err = "neighbour list not strictly ascending at vertex " + std::to_string(v); return KPLEX_ERR_FORMAT; }
        }
    }
    return KPLEX_OK;
}

int save_bin(const char* path, const Csr& g, std::string* err) {
    FILE* f = fopen(path, "wb");
    if (!f) { if (err) *err = std::string("cannot create ") + path; return KPLEX_ERR_IO; }
    const uint32_t hdr[2] = {g.n, (uint32_t)g.m_directed()};
    bool ok = fwrite(hdr, 4, 2, f) == 2;
    std::vector<uint32_t> deg(g.n);
    for (uint32_t v = 0; v < g.n; ++v) deg[v] = g.deg(v);
    if (g.n) ok = ok && fwrite(deg.data(), 4, g.n, f) == g.n;
    if (g.m_directed()) ok = ok && fwrite(g.adj.data(), 4, g.m_directed(), f) == g.m_directed();
    ok = (fclose(f) == 0) && ok;
    if (!ok) { if (err) *err = "short write"; return KPLEX_ERR_IO; }
    return KPLEX_OK;
}

}  // namespace kplex
