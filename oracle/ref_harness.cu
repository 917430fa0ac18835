// CHECKER — test infrastructure only (built into oracle/_ref/, never shipped).
//
// Runs the reference's own host preprocessing, compiled from its sources where
// they lie: graph<intT>(path) (inc/graph.h:37-65), peelGraph (inc/host_funcs.h:16-122),
// fast_truss_peeling (inc/host_funcs.h:463-559) and ListLinearHeap
// (inc/degeneracy.h).  The triangle count and the initial edge queue that
// decomposableSearch builds inline (inc/host_funcs.h:761-819) are restated
// here.  Writes: u32 pn, u32 m, u32 off[pn+1], u32 adj[m], i32 dpos[pn], i32 dseq[pn].
// Usage: ref_preprocess <graph.bin> <k> <q> <truss> <out.bin>
#include <atomic>
#include <cmath>
#include <queue>
#include <cassert>
#include <functional>
#include <chrono>
#include "inc/host_funcs.h"
#include <climits>

int main(int argc, char** argv) {
    if (argc < 6) { fprintf(stderr, "usage: %s graph.bin k q truss out.bin\n", argv[0]); return 1; }
    k = atoi(argv[2]); lb = atoi(argv[3]); truss = atoi(argv[4]); bd = lb - k;
    graph<intT> g(argv[1]);
    bool* mark = new bool[g.n];
    int* resNei = new int[g.n];
    graph<intT> pg = peelGraph(g, mark, resNei);
    int pn = pg.n;
    if (truss) {
        std::vector<int> tri(pg.m, 0);
        std::vector<std::pair<int, int>> Qe;
        for (int i = 0; i < pn; ++i)
            for (unsigned p = pg.offsets[i]; p < pg.offsets[i + 1]; ++p) {
                const unsigned v = pg.neighbors[p];
                unsigned a = pg.offsets[i], ea = pg.offsets[i + 1], b = pg.offsets[v], eb = pg.offsets[v + 1];
                int c = 0;
                while (a < ea && b < eb) {
                    if (pg.neighbors[a] == pg.neighbors[b]) { ++c; ++a; ++b; }
                    else if (pg.neighbors[a] < pg.neighbors[b]) ++a; else ++b;
                }
                tri[p] = c;
            }
        for (int i = 0; i < pn; ++i)
            for (unsigned p = pg.offsets[i]; p < pg.offsets[i + 1]; ++p)
                if ((unsigned)i < pg.neighbors[p] && tri[p] < lb - 2 * k) Qe.push_back({i, (int)pg.neighbors[p]});
        fast_truss_peeling(pg.neighbors, pg.offsets, pg.degree, Qe, pn, &pg.m, tri);
        pg = peelGraph(pg, mark, resNei);
        pn = pg.n;
    }
    std::vector<int> dpos(pn > 0 ? pn : 1, INT_MAX), dseq(pn > 0 ? pn : 1, 0);
    if (pn > 0) {
        ListLinearHeap<int>* heap = new ListLinearHeap<int>(pn, pn - 1);
        heap->init(pn, pn - 1);
        for (int i = 0; i < pn; ++i) heap->insert(i, pg.degree[i]);
        for (int i = 0; i < pn; ++i) {
            int u, key;
            heap->pop_min(u, key);
            dpos[u] = i; dseq[i] = u;
            for (unsigned j = 0; j < pg.degree[u]; ++j) {
                const int w = pg.neighbors[pg.offsets[u] + j];
                if (dpos[w] == INT_MAX) heap->decrement(w);
            }
        }
        delete heap;
    }
    FILE* f = fopen(argv[5], "wb");
    if (!f) return 2;
    const unsigned hdr[2] = {(unsigned)pn, (unsigned)pg.m};
    fwrite(hdr, 4, 2, f);
    fwrite(pg.offsets, 4, pn + 1, f);
    if (pg.m) fwrite(pg.neighbors, 4, pg.m, f);
    if (pn) { fwrite(dpos.data(), 4, pn, f); fwrite(dseq.data(), 4, pn, f); }
    fclose(f);
    return 0;
}
