// Root decomposition: one warp builds one root's 2-hop subgraph as bitsets.
//
// Restates, for root rank r (root = dseq[r]):
//   decompose        src/device_funcs.cu:28-298   later/earlier split, C1 peel to
//                    (q-2k) support inside C1, left filter (q-2k+1), 2-hop scan
//                    (q-2k+2 later -> C2, q-2k+3 earlier -> left), valid if |blk| >= q
//   calculateDegrees src:300-351, computeOffsets inc/host_funcs.h:124-156 and
//   fillNeighbors    src:353-460   -> here the adjacency bit matrix A, the left
//                    adjacency LA and its transpose LT replace the local CSRs
//   buildCommonMtx   src:1727-1853 -> the 6-way pair class collapses to the two
//                    predicates the search reads: class >= UNLINK2EQUAL (M2) and
//                    class >= UNLINK2MORE (M4)
// Local order is fixed (root, C1 ascending, C2 ascending); the reference's is
// set by shared-memory atomics and is not reproducible.  2-hop candidates are
// counted from C1's adjacency (every accepted vertex has >= q-2k+2 >= 1
// neighbours in C1 because q >= 2k-1 is required by the host).
//
// Per-warp scratch (global, L2 resident): loc[pn] maps a pruned id to its
// local id (< MAX_LOCAL), to LOC_LEFT + left index, to EXCL, or NONE; cnt[pn]
// counts C1 neighbours of 2-hop candidates.  Both are restored before the warp
// moves to its next root.
#include "warp.cuh"

namespace kplex {

constexpr uint32_t LOC_NONE = 0xffffffffu;
constexpr uint32_t LOC_EXCL = 0xfffffffeu;
constexpr uint32_t LOC_LEFT = MAX_LOCAL;   // loc of left vertex i: LOC_LEFT + i
constexpr int LATER_WORDS = REF_BLK / 32;  // bitset over the (at most 1023) later neighbours

struct DecompScratch {
    uint32_t* loc;      // pn
    uint32_t* cnt;      // pn
    uint32_t* later;    // REF_BLK
    uint32_t* earlier;  // REF_BLK
    uint32_t* blk;      // MAX_LOCAL + 32 (root, C1, C2)
    uint32_t* left;     // MAX_LEFT + 32
    uint32_t* tmp;      // MAX_LEFT + 32
};

__host__ __device__ inline uint64_t decomp_scratch_words(uint32_t pn) {
    return 2ull * pn + 2 * REF_BLK + (MAX_LOCAL + 32) + 2 * (MAX_LEFT + 32) + 64;
}

__device__ inline DecompScratch decomp_scratch(const SearchParams& sp, unsigned warp) {
    uint32_t* b = sp.warp_scratch + (uint64_t)warp * sp.scratch_words;
    DecompScratch s;
    s.loc = b; b += sp.pn;
    s.cnt = b; b += sp.pn;
    s.later = b; b += REF_BLK;
    s.earlier = b; b += REF_BLK;
    s.blk = b; b += MAX_LOCAL + 32;
    s.left = b; b += MAX_LEFT + 32;
    s.tmp = b;
    return s;
}

// |N(u) ∩ {local ids in [lo, hi)}| counted through loc[]
__device__ __forceinline__ int count_local_nbrs(const SearchParams& sp, const uint32_t* loc, uint32_t u, uint32_t lo, uint32_t hi) {
    const unsigned l = lane_id();
    int c = 0;
    for (uint32_t j = sp.off[u] + l; j < sp.off[u + 1]; j += 32) {
        const uint32_t x = loc[sp.adj[j]];
        c += (x >= lo && x < hi);
    }
    return warp_sum(c);
}

// Rank sort of m distinct values (m <= MAX_LEFT) from src into dst.
__device__ void rank_sort(const uint32_t* src, uint32_t* dst, int m) {
    const unsigned l = lane_id();
    __syncwarp();
    for (int i = l; i < m; i += 32) {
        const uint32_t v = src[i];
        int r = 0;
        for (int j = 0; j < m; ++j) r += src[j] < v;
        dst[r] = v;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(256) decompose_kernel(SearchParams sp) {
    const unsigned l = lane_id();
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    DecompScratch S = decomp_scratch(sp, warp);
    __shared__ uint32_t s_alive_all[8][LATER_WORDS];
    __shared__ uint32_t s_row_all[8][MAX_WORDS + MAX_LEFT_WORDS];
    uint32_t* s_alive = s_alive_all[threadIdx.x >> 5];
    uint32_t* s_row = s_row_all[threadIdx.x >> 5];

    for (;;) {
        uint32_t r = 0;
        if (l == 0) r = atomicAdd(&sp.ctr->decomp_next, 1u);
        r = __shfl_sync(FULL, r, 0);
        if (r >= sp.nroots) break;
        // the root's graph: the last g with root_base <= r
        uint32_t g = 0;
        {
            uint32_t lo = 0, hi = sp.ngraphs;
            while (hi - lo > 1) { const uint32_t mid = (lo + hi) >> 1; if (sp.graphs[mid].root_base <= r) lo = mid; else hi = mid; }
            g = lo;
        }
        const GraphInfo gi = sp.graphs[g];
        const int k = gi.k, q = gi.q;
        const int lb2k = q - 2 * k, bd = q - k;
        RootDesc desc{};
        desc.graph = g;
        desc.k = k;
        desc.q = q;
        const bool other = sp.root_owner ? sp.root_owner[r] != sp.shard_index
                                         : (sp.shard_count > 1 && r % sp.shard_count != sp.shard_index);
        if (other ||   // another GPU's root
            r - gi.root_base < sp.root_begin || r - gi.root_base >= sp.root_end) {   // outside the stated range
            if (l == 0) sp.roots[r] = desc;
            __syncwarp();
            continue;
        }
        // loc/cnt are indexed by the graph's own vertex ids (vertex - vbase)
        uint32_t* const loc = S.loc - gi.vbase;
        uint32_t* const cnt = S.cnt - gi.vbase;
        const uint32_t root = (uint32_t)sp.dseq[r];
        const int pos = sp.dpos[root];
        desc.gid = root;

        // ---- later / earlier split in CSR order (src:87-131)
        int nlater = 0, nearlier = 0;
        bool truncated = false;
        for (uint32_t b = sp.off[root]; b < sp.off[root + 1]; b += 32) {
            const uint32_t j = b + l;
            uint32_t w = 0;
            bool valid = j < sp.off[root + 1];
            bool lat = false;
            if (valid) { w = sp.adj[j]; lat = pos < sp.dpos[w]; }
            const unsigned ml = __ballot_sync(FULL, valid && lat);
            const unsigned me = __ballot_sync(FULL, valid && !lat);
            const unsigned below = (1u << l) - 1;
            if (valid && lat) {
                const int idx = nlater + __popc(ml & below);
                if (idx < REF_BLK - 1) S.later[idx] = w;
            }
            if (valid && !lat) {
                const int idx = nearlier + __popc(me & below);
                if (idx < REF_BLK) S.earlier[idx] = w;
            }
            nlater += __popc(ml);
            nearlier += __popc(me);
        }
        if (nlater > REF_BLK - 1) { nlater = REF_BLK - 1; truncated = true; }
        if (nearlier > REF_BLK) { nearlier = REF_BLK; truncated = true; }
        __syncwarp();
        // loc: later j -> j (temporary), earlier -> EXCL until the left filter
        for (int i = l; i < nlater; i += 32) loc[S.later[i]] = (uint32_t)i;
        for (int i = l; i < nearlier; i += 32) loc[S.earlier[i]] = LOC_EXCL;
        if (l == 0) loc[root] = LOC_EXCL;
        __syncwarp();

        // ---- C1 peel (src:142-180): synchronous rounds to the (q-2k) core of C1
        {
            const int lo = (int)l * 32;
            s_alive[l] = nlater >= lo + 32 ? FULL : (nlater > lo ? ((1u << (nlater - lo)) - 1) : 0u);
            s_row[l] = 0u;
            s_row[MAX_WORDS + l] = 0u;
        }
        __syncwarp();
        int alive = nlater;
        bool skip = false;
        for (;;) {
            if (alive < bd) { skip = true; break; }
            // count every alive later vertex's alive-later neighbours
            int removed = 0;
            for (int i = 0; i < nlater; ++i) {
                if (!test_bit(s_alive, i)) continue;
                int c = 0;
                const uint32_t u = S.later[i];
                for (uint32_t j = sp.off[u] + l; j < sp.off[u + 1]; j += 32) {
                    const uint32_t x = loc[sp.adj[j]];
                    c += (x < (uint32_t)nlater) && test_bit(s_alive, x);
                }
                c = warp_sum(c);
                // synchronous round: record removals in s_row, apply after the pass
                if (c < lb2k) {
                    if (l == 0) s_row[MAX_WORDS + (i >> 5)] |= 1u << (i & 31);
                    ++removed;
                }
            }
            __syncwarp();
            if (removed == 0) break;
            if (l < LATER_WORDS) { s_alive[l] &= ~s_row[MAX_WORDS + l]; s_row[MAX_WORDS + l] = 0; }
            __syncwarp();
            alive -= removed;
        }
        if (l < LATER_WORDS) s_row[MAX_WORDS + l] = 0;
        __syncwarp();

        int hop = 0, n = 0, nleft = 0;
        bool oversized = false;
        if (!skip) {
            // ---- C1 list in CSR order, local ids 1..hop-1 (src:167-178)
            int cntc = 0;
            for (int b = 0; b < nlater; b += 32) {
                const int i = b + l;
                const bool a = i < nlater && test_bit(s_alive, i);
                const unsigned m = __ballot_sync(FULL, a);
                if (a) S.blk[1 + cntc + __popc(m & ((1u << l) - 1))] = S.later[i];
                cntc += __popc(m);
            }
            __syncwarp();
            hop = 1 + cntc;
            if (l == 0) S.blk[0] = root;
            // later vertices: C1 members get local ids, peeled ones are excluded
            for (int i = l; i < nlater; i += 32) loc[S.later[i]] = LOC_EXCL;
            __syncwarp();
            for (int i = 1 + l; i < hop; i += 32) loc[S.blk[i]] = (uint32_t)i;
            if (l == 0) loc[root] = 0;
            __syncwarp();

            // ---- left filter (src:188-213): >= q-2k+1 neighbours in C1
            int nl1 = 0;
            for (int i = 0; i < nearlier; ++i) {
                const uint32_t u = S.earlier[i];
                const int c = count_local_nbrs(sp, loc, u, 1, (uint32_t)hop);
                if (c >= lb2k + 1) { if (l == 0) S.left[nl1] = u; ++nl1; }
            }
            __syncwarp();
            for (int i = l; i < nl1; i += 32) loc[S.left[i]] = LOC_LEFT + (uint32_t)i;  // marks membership
            __syncwarp();

            // ---- 2-hop scan (src:217-273): count C1 neighbours of unvisited vertices
            for (int i = 1; i < hop; ++i) {
                const uint32_t c1v = S.blk[i];
                for (uint32_t j = sp.off[c1v] + l; j < sp.off[c1v + 1]; j += 32) {
                    const uint32_t w = sp.adj[j];
                    if (loc[w] == LOC_NONE) atomicAdd(&cnt[w], 1u);
                }
            }
            __syncwarp();
            int nc2 = 0, nl2 = 0;
            const int cap2 = MAX_LOCAL - hop + 1;    // one past the limit to detect overflow
            const int capl = MAX_LEFT + 1 - nl1;   // one past the limit to detect overflow
            for (int i = 1; i < hop; ++i) {
                const uint32_t c1v = S.blk[i];
                for (uint32_t b = sp.off[c1v]; b < sp.off[c1v + 1]; b += 32) {
                    const uint32_t j = b + l;
                    bool takeC2 = false, takeL = false;
                    uint32_t w = 0;
                    if (j < sp.off[c1v + 1]) {
                        w = sp.adj[j];
                        if (loc[w] == LOC_NONE) {
                            const uint32_t c = atomicExch(&cnt[w], 0u);
                            if (c) {
                                if (pos < sp.dpos[w]) takeC2 = (int)c >= lb2k + 2;
                                else takeL = (int)c >= lb2k + 3;
                            }
                        }
                    }
                    const unsigned m2 = __ballot_sync(FULL, takeC2);
                    const unsigned ml = __ballot_sync(FULL, takeL);
                    if (takeC2) { const int idx = nc2 + __popc(m2 & ((1u << l) - 1)); if (idx < cap2) S.tmp[idx] = w; }
                    if (takeL) { const int idx = nl2 + __popc(ml & ((1u << l) - 1)); if (idx < capl) S.left[nl1 + idx] = w; }
                    nc2 += __popc(m2);
                    nl2 += __popc(ml);
                }
            }
            __syncwarp();
            n = hop + nc2;
            nleft = nl1 + nl2;
            if (n > MAX_LOCAL || nleft > MAX_LEFT) oversized = true;
            if (!oversized) {
                rank_sort(S.tmp, S.blk + hop, nc2);                 // C2 ascending
                for (int i = l; i < nleft; i += 32) S.tmp[i] = S.left[i];
                rank_sort(S.tmp, S.left, nleft);                    // left ascending
            }
        }

        const bool valid = !skip && n >= q;
        if (valid && !oversized) {
            // final loc: blk -> local id, left -> LOC_LEFT + index
            for (int i = l; i < n; i += 32) loc[S.blk[i]] = (uint32_t)i;
            for (int i = l; i < nleft; i += 32) loc[S.left[i]] = LOC_LEFT + (uint32_t)i;
            __syncwarp();
            const uint32_t W = ((uint32_t)((n + 31) >> 5) + 3u) & ~3u;
            const uint32_t WL = nleft ? ((uint32_t)((nleft + 31) >> 5) + 3u) & ~3u : 0u;
            const uint64_t words = ((3ull * n * W + (uint64_t)n * WL + (uint64_t)nleft * W + 2ull * n) + 3ull) & ~3ull;
            unsigned long long base = 0;
            if (l == 0) base = atomicAdd(&sp.ctr->arena_top, (unsigned long long)words);
            base = __shfl_sync(FULL, base, 0);
            if (base + words > sp.arena_cap) {
                if (l == 0) raise_error(sp.ctr, KPLEX_ERR_NOMEM);
            } else {
                uint32_t* A = sp.arena + base;
                uint32_t* M2 = A + (uint64_t)n * W;
                uint32_t* M4 = M2 + (uint64_t)n * W;
                uint32_t* LA = M4 + (uint64_t)n * W;
                uint32_t* LT = LA + (uint64_t)n * WL;
                uint32_t* sorig = LT + (uint64_t)nleft * W;
                uint32_t* srank = sorig + n;
                for (uint64_t i = l; i < words; i += 32) A[i] = 0u;
                __syncwarp();
                __threadfence_block();
                // A, LA, LT rows (src:405-443)
                for (int i = 0; i < n; ++i) {
                    for (uint32_t w = l; w < MAX_WORDS + WL; w += 32) s_row[w] = 0u;
                    __syncwarp();
                    const uint32_t u = S.blk[i];
                    for (uint32_t j = sp.off[u] + l; j < sp.off[u + 1]; j += 32) {
                        const uint32_t x = loc[sp.adj[j]];
                        if (x < (uint32_t)n) atomicOr(&s_row[x >> 5], 1u << (x & 31));
                        else if (x >= LOC_LEFT && x < LOC_LEFT + (uint32_t)nleft) {
                            const uint32_t jl = x - LOC_LEFT;
                            atomicOr(&s_row[MAX_WORDS + (jl >> 5)], 1u << (jl & 31));
                            atomicOr(&LT[(uint64_t)jl * W + (i >> 5)], 1u << (i & 31));
                        }
                    }
                    __syncwarp();
                    for (uint32_t w = l; w < W; w += 32) A[(uint64_t)i * W + w] = s_row[w];
                    for (uint32_t w = l; w < WL; w += 32) LA[(uint64_t)i * WL + w] = s_row[MAX_WORDS + w];
                    __syncwarp();
                }
                __threadfence_block();
                __syncwarp();
                // pair classes (src:1751-1853) -> M2 (class >= 2), M4 (class >= 4)
                const int tCC1 = q - 2 * k - (k - 1), tCC2 = q - 2 * k + 2 - (k - 1);
                const int tPC1 = q - 2 * k - max(k - 2, 0), tPC2 = q - k - 1 - max(k - 2, 0) - max(k - 3, 0);
                const int tPP1 = q - k - 2 * max(k - 2, 0), tPP2 = q - k - 2 * max(k - 3, 0);
                const int hw = (hop + 31) >> 5;   // words covering [0, hop)
                for (int i = 0; i < n; ++i) {
                    const uint32_t* Ai = A + (uint64_t)i * W;
                    for (int jb = 0; jb < n; jb += 32) {
                        const int j = jb + l;
                        bool m2 = false, m4 = false;
                        if (j < n && j != i) {
                            const uint32_t* Aj = A + (uint64_t)j * W;
                            int c = 0;
                            for (int w = 0; w < hw; ++w) {
                                uint32_t mk = FULL;
                                if (w == hw - 1 && (hop & 31)) mk = (1u << (hop & 31)) - 1;
                                c += __popc(Ai[w] & Aj[w] & mk);
                            }
                            const bool adj = (Ai[j >> 5] >> (j & 31)) & 1u;
                            const bool ih = i < hop, jh = j < hop;
                            int t1, t2;
                            bool raw = false;
                            if (ih && jh) { t1 = tCC1; t2 = tCC2; }
                            else if (ih != jh) { t1 = tPC1; t2 = tPC2; }
                            else { t1 = tPP1; t2 = tPP2; raw = (k == 2); }
                            if (!raw) {
                                if (adj) { m2 = c >= t1; m4 = c > t1; }
                                else { m2 = c >= t2; m4 = c > t2; }
                            }
                        }
                        const unsigned b2 = __ballot_sync(FULL, m2), b4 = __ballot_sync(FULL, m4);
                        if (l == 0) { M2[(uint64_t)i * W + (jb >> 5)] = b2; M4[(uint64_t)i * W + (jb >> 5)] = b4; }
                    }
                }
                // sorted original ids and ranks (for the output hash)
                for (int i = l; i < n; i += 32) {
                    const uint32_t g = S.blk[i];
                    int rk = 0;
                    for (int j = 0; j < n; ++j) rk += S.blk[j] < g;
                    sorig[rk] = sp.orig[g];
                    srank[i] = (uint32_t)rk;
                }
                desc.n = (uint32_t)n; desc.hop = (uint32_t)hop; desc.nleft = (uint32_t)nleft;
                desc.W = W; desc.WL = WL; desc.base = base;
                desc.flags = ROOT_VALID;
                if (l == 0) {
                    atomicAdd(&sp.ctr->valid_roots, 1u);
                    atomicAdd(&sp.gvalid[g], 1u);
                    atomicMax(&sp.ctr->max_n, (unsigned)n);
                    atomicMax(&sp.ctr->max_left, (unsigned)nleft);
                    atomicMax(&sp.ctr->max_w, W);
                    atomicMax(&sp.ctr->max_nw, (unsigned)n * W);
                    // CSR words of every local vertex read once + the root block written once
                    unsigned long long csr = 0;
                    for (int i = 0; i < n; ++i) csr += sp.off[S.blk[i] + 1] - sp.off[S.blk[i]];
                    atomicAdd(&sp.ctr->roots_bytes, 4ull * csr + 4ull * words);
                }
            }
        } else if (valid && oversized) {
            desc.flags = ROOT_VALID | ROOT_OVERSIZED;
            if (l == 0) {
                atomicAdd(&sp.ctr->valid_roots, 1u);
                atomicAdd(&sp.gvalid[g], 1u);
                atomicAdd(&sp.ctr->oversized, 1u);
                atomicMax(&sp.ctr->max_n, (unsigned)n);
                atomicMax(&sp.ctr->max_left, (unsigned)nleft);
                raise_error(sp.ctr, KPLEX_ERR_CAPACITY);
            }
        } else if (skip) {
            desc.flags = ROOT_SKIPPED;
        }
        if (truncated) {
            desc.flags |= ROOT_TRUNCATED;
            if (l == 0) atomicAdd(&sp.ctr->truncated, 1u);
        }
        __syncwarp();
        // ---- restore scratch: loc for every id written, cnt already zeroed by exchange
        for (int i = l; i < nlater; i += 32) loc[S.later[i]] = LOC_NONE;
        for (int i = l; i < nearlier; i += 32) loc[S.earlier[i]] = LOC_NONE;
        if (!skip && !oversized) {
            for (int i = l; i < n; i += 32) loc[S.blk[i]] = LOC_NONE;
            for (int i = l; i < nleft; i += 32) loc[S.left[i]] = LOC_NONE;
        }
        if (l == 0) loc[root] = LOC_NONE;
        __syncwarp();
        if (l == 0) sp.roots[r] = desc;
        __syncwarp();
    }
}

uint64_t decomp_scratch_words_host(uint32_t pn) { return decomp_scratch_words(pn); }

// k-search job prefix: a valid root with |C2| = n - hop owns |C2| + 1 jobs;
// job_base[r] = jobs of roots < r, job_base[nroots] = total.  One block.
__global__ void __launch_bounds__(1024) job_prefix_kernel(const RootDesc* roots, uint32_t nroots, uint32_t* job_base,
                                                                unsigned int* work) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x, T = blockDim.x;
    const uint32_t per = (nroots + T - 1) / T;
    const uint32_t b = t * per, e = min(nroots, b + per);
    uint32_t sum = 0;
    for (uint32_t r = b; r < e; ++r) {
        const RootDesc& rd = roots[r];
        sum += ((rd.flags & ROOT_VALID) && rd.n) ? rd.n - rd.hop + 1 : 0u;
    }
    part[t] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < T; o <<= 1) {   // inclusive Hillis-Steele scan
        const uint32_t v = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = t ? part[t - 1] : 0u;
    for (uint32_t r = b; r < e; ++r) {
        job_base[r] = run;
        const RootDesc& rd = roots[r];
        run += ((rd.flags & ROOT_VALID) && rd.n) ? rd.n - rd.hop + 1 : 0u;
    }
    if (t == T - 1) {
        job_base[nroots] = part[T - 1];
        if (work) *work = part[T - 1];   // every job is one outstanding unit of work
    }
}

}  // namespace kplex
