// k-search over C2 and task-based branch-and-bound in one persistent kernel.
//
// Reference structure (src/device_funcs.cu, inc/host_funcs.h): kSearch
// (src:1855-2444) fills queue A with tasks, pausing when A holds
// thres * MAX_CAP - WARPS records; the host then drains A with waves of the
// BNB kernel (src:1516-1724) through auxiliary queues B and C (host:253-335),
// reading a flag back after every wave, and relaunches kSearch (host:1094-1122).
//
// Here both run inside search_kernel:
//  * warp 0 of every block is a producer: it claims roots and runs the k-search
//    state machine with its whole state in shared memory.  Each leaf is one
//    task (P, C, X bitsets) pushed into the pool, a bounded lock-free ring in
//    HBM (the reference's queue A).  When the pool holds pause_at records the
//    producer pauses and works as a consumer until the pool drains below
//    half of that, then resumes (pause-and-resume without a host round trip).
//    A push that finds the ring full is kept and processed by the producer.
//  * the other warps are consumers: each pops a record and runs the branch
//    and bound on it depth-first, continuing with the include child and
//    stacking the exclude child in its own stack, and gives its oldest stacked
//    record back to the pool when the pool runs low (load balancing that the
//    reference gets from its queues B and C).
// neiInG / neiInP, which the reference stores per task (u16 arrays, common.h:144-170),
// are recomputed from the bitsets: neiInG[v] = |N(v) ∩ (P ∪ C)|, neiInP[v] = |N(v) ∩ P|.
//
// A bitset over a root's local vertices is held by the warp in registers, NW
// words per lane: lane l holds words l, l + 32, ... (NW = 1 covers 1024
// vertices, NW = 2 covers MAX_LOCAL = 2048).  The kernel is compiled for both;
// a search uses NW = 2 only when one of its roots has more than 1024 vertices.
#include "warp.cuh"
#include <climits>

namespace kplex {

// ============================================================== root view
// The root's block in the arena: A, M2, M4 ([n][W] each), LA ([n][WL]),
// LT ([nleft][W]), sorig, srank ([n]).  Only A's address is kept; the others
// are derived on use, which keeps a warp's registers for its search state.
struct RootView {
    uint32_t n, hop, nleft, W, WL, graph;
    int k, q;
    const uint32_t* A;
    __device__ __forceinline__ const uint32_t* M2() const { return A + (uint64_t)n * W; }
    __device__ __forceinline__ const uint32_t* M4() const { return A + 2ull * n * W; }
    __device__ __forceinline__ const uint32_t* LA() const { return A + 3ull * n * W; }
    __device__ __forceinline__ const uint32_t* LT() const { return LA() + (uint64_t)n * WL; }
    __device__ __forceinline__ const uint32_t* sorig() const { return LT() + (uint64_t)nleft * W; }
    __device__ __forceinline__ const uint32_t* srank() const { return sorig() + n; }
};

__device__ __forceinline__ RootView root_view(const SearchParams& sp, uint32_t r) {
    const RootDesc d = sp.roots[r];
    RootView v;
    v.n = d.n; v.hop = d.hop; v.nleft = d.nleft; v.W = d.W; v.WL = d.WL;
    v.graph = d.graph; v.k = d.k; v.q = d.q;
    v.A = sp.arena + d.base;
    return v;
}

// ============================================================== per-lane bitset words
// Bits<NW>: this lane's NW words of a bitset of 32 * NW words (word l + 32 j in
// w[j]).  Every index into w[] is a compile-time constant after unrolling, so
// the words stay in registers.
template <int NW>
struct Bits {
    uint32_t w[NW];
};

template <int NW>
__device__ __forceinline__ Bits<NW> bits_zero() {
    Bits<NW> b;
#pragma unroll
    for (int j = 0; j < NW; ++j) b.w[j] = 0u;
    return b;
}
// words l + 32 j of p, 0 at and beyond word `nwords`
template <int NW>
__device__ __forceinline__ Bits<NW> bits_load(const uint32_t* p, uint32_t nwords) {
    Bits<NW> b;
    const unsigned l = lane_id();
#pragma unroll
    for (int j = 0; j < NW; ++j) b.w[j] = (l + 32u * j < nwords) ? p[l + 32u * j] : 0u;
    return b;
}
template <int NW>
__device__ __forceinline__ Bits<NW> bits_ldg(const uint32_t* p, uint32_t nwords) {
    Bits<NW> b;
    const unsigned l = lane_id();
#pragma unroll
    for (int j = 0; j < NW; ++j) b.w[j] = (l + 32u * j < nwords) ? __ldg(p + l + 32u * j) : 0u;
    return b;
}
// all 32 * NW words to a shared-memory array
template <int NW>
__device__ __forceinline__ void bits_store(uint32_t* p, const Bits<NW>& b) {
    const unsigned l = lane_id();
#pragma unroll
    for (int j = 0; j < NW; ++j) p[l + 32u * j] = b.w[j];
}
template <int NW>
__device__ __forceinline__ void bits_fill(uint32_t* p, uint32_t v) {
    const unsigned l = lane_id();
#pragma unroll
    for (int j = 0; j < NW; ++j) p[l + 32u * j] = v;
}
template <int NW>
__device__ __forceinline__ int bits_count(const Bits<NW>& b) {
    int c = 0;
#pragma unroll
    for (int j = 0; j < NW; ++j) c += __popc(b.w[j]);
    return warp_sum(c);
}
// OR `m` into word `wi` (held by lane wi % 32, slot wi / 32)
template <int NW>
__device__ __forceinline__ void bits_or_word(Bits<NW>& b, uint32_t wi, uint32_t m) {
    if ((wi & 31u) != lane_id()) return;
#pragma unroll
    for (int j = 0; j < NW; ++j) if ((wi >> 5) == (uint32_t)j) b.w[j] |= m;
}
template <int NW>
__device__ __forceinline__ void bits_set(Bits<NW>& b, uint32_t v) { bits_or_word(b, v >> 5, 1u << (v & 31)); }
template <int NW>
__device__ __forceinline__ void bits_clear(Bits<NW>& b, uint32_t v) {
    if (((v >> 5) & 31u) != lane_id()) return;
#pragma unroll
    for (int j = 0; j < NW; ++j) if ((v >> 10) == (uint32_t)j) b.w[j] &= ~(1u << (v & 31));
}
template <int NW>
__device__ __forceinline__ Bits<NW> bits_or(const Bits<NW>& a, const Bits<NW>& b) {
    Bits<NW> r;
#pragma unroll
    for (int j = 0; j < NW; ++j) r.w[j] = a.w[j] | b.w[j];
    return r;
}
// ascending list of the set bits' indices; returns their count
template <int NW>
__device__ __forceinline__ int bits_list(const Bits<NW>& b, uint16_t* list) {
    int off = 0;
#pragma unroll
    for (int j = 0; j < NW; ++j) off += bits_to_list(b.w[j], list + off, 1024u * j);
    return off;
}
// the lists of two disjoint bitsets in one pass over their non-zero words: a's
// members to la, b's to lb (both ascending)
template <int NW>
__device__ __forceinline__ void bits_list2(const Bits<NW>& a, const Bits<NW>& b, uint16_t* la, uint16_t* lb) {
    const unsigned l = lane_id();
    const unsigned below = (1u << l) - 1u;
    int oa = 0, ob = 0;
#pragma unroll
    for (int j = 0; j < NW; ++j) {
        unsigned nz = __ballot_sync(FULL, (a.w[j] | b.w[j]) != 0u);
        while (nz) {
            const int i = __ffs(nz) - 1;
            nz &= nz - 1;
            const unsigned wa = __shfl_sync(FULL, a.w[j], i), wb = __shfl_sync(FULL, b.w[j], i);
            const uint16_t x = (uint16_t)(1024u * j + i * 32 + l);
            if ((wa >> l) & 1u) la[oa + __popc(wa & below)] = x;
            if ((wb >> l) & 1u) lb[ob + __popc(wb & below)] = x;
            oa += __popc(wa);
            ob += __popc(wb);
        }
    }
    __syncwarp();
}

// ============================================================== k-search state (shared memory)
// Layout in words, sized by the largest root n_max of the search:
//   hdr (root, sz, np, nc2) | P stack [MAX_K] | frames | C2 list | C1 tags | C2 tags |
//   C1 member list | C1, X, P bitsets [3 x BW] | scratch masks [3 x BW]
// with BW = 32 * NW.  Along any stack path every pushed frame moves one C2
// vertex to X or P (the last push may add one leaf frame), so n_max + 8
// frames suffice.
struct KsLayout { uint32_t fr, c2, t1, t2, lst, bits, aux, total, bw; };

__host__ __device__ inline KsLayout ks_layout(uint32_t nmax, uint32_t nw) {
    KsLayout L;
    L.bw = 32 * nw;
    uint32_t o = 8 + MAX_K;
    const uint32_t frames = ((nmax + 8 < (uint32_t)KS_MAX_DEPTH ? nmax + 8 : (uint32_t)KS_MAX_DEPTH) + 3u) & ~3u;
    const uint32_t half = (((nmax + 1) / 2) + 3u) & ~3u;
    L.fr = o; o += frames;
    L.c2 = o; o += half;
    L.t1 = o; o += half;
    L.t2 = o; o += half;
    L.lst = o; o += half;
    L.bits = o; o += 3 * L.bw;
    L.aux = o; o += 3 * L.bw;
    L.total = o;
    return L;
}

// frame: res (8) | br (8) | state (4) | v2delete (12)
__device__ __forceinline__ uint32_t fr_pack(uint32_t res, uint32_t br, uint32_t st, uint32_t v) {
    return res | (br << 8) | (st << 16) | (v << 20);
}
__device__ __forceinline__ uint32_t fr_res(uint32_t f) { return f & 0xff; }
__device__ __forceinline__ uint32_t fr_br(uint32_t f) { return (f >> 8) & 0xff; }
__device__ __forceinline__ uint32_t fr_st(uint32_t f) { return (f >> 16) & 0xf; }
__device__ __forceinline__ uint32_t fr_v(uint32_t f) { return f >> 20; }

template <int NW>
struct KsSlot {
    static constexpr uint32_t BW = 32 * NW;
    uint32_t* w;
    KsLayout L;
    __device__ uint32_t& root() const { return w[0]; }
    __device__ uint32_t& sz() const { return w[1]; }
    __device__ uint32_t& np() const { return w[2]; }
    __device__ uint32_t& nc2() const { return w[3]; }
    __device__ uint32_t* P() const { return w + 8; }
    __device__ uint32_t* fr() const { return w + L.fr; }
    __device__ uint16_t* c2() const { return reinterpret_cast<uint16_t*>(w + L.c2); }
    __device__ uint16_t* t1() const { return reinterpret_cast<uint16_t*>(w + L.t1); }
    __device__ uint16_t* t2() const { return reinterpret_cast<uint16_t*>(w + L.t2); }
    __device__ uint16_t* lst() const { return reinterpret_cast<uint16_t*>(w + L.lst); }
    __device__ uint32_t* c1bits() const { return w + L.bits; }
    __device__ uint32_t* xbits() const { return w + L.bits + BW; }
    __device__ uint32_t* pbits() const { return w + L.bits + 2 * BW; }
    __device__ uint32_t* mask() const { return w + L.aux; }
    __device__ uint32_t* aux() const { return w + L.aux + BW; }
    __device__ uint32_t* keep() const { return w + L.aux + 2 * BW; }
};

// Initial state of k-search job (r, d).  The reference's k-search for a root
// (src:1993-2442, from the initial sets of src:447-460 and 1953-1975:
// P = {0}, C1 = [1,hop), C2 = [hop,n) in ascending order) starts with an
// exclude chain: state 0 moves the last C2 vertex to X and pushes a child, m
// times for |C2| = m, with no inclusion in between.  The frame at chain depth
// d therefore sees P = {0}, C1 = [1,hop), C2 = the first m-d vertices and
// X = the last d.  When its exclude child returns (state 1) it puts its vertex
// back and runs its include branches (state 2, br = 1).  Job d < m is exactly
// that frame from state 2 on; job m is the chain's bottom (C2 empty, state 0).
// The jobs are independent, so one root's k-search spreads over many warps,
// and their emissions are the reference's emissions for the root.
template <int NW>
__device__ void ks_start(const SearchParams& sp, const KsSlot<NW>& S, uint32_t r, uint32_t d, const RootDesc& rd) {
    const unsigned l = lane_id();
    const uint32_t n = rd.n, hop = rd.hop, m = n - hop;
    const uint32_t keep = m - d;   // C2 list = [hop, hop + keep), X = [hop + keep, n)
#pragma unroll
    for (int j = 0; j < NW; ++j) {
        const uint32_t wi = l + 32u * j, lo = wi * 32;
        uint32_t c1 = 0, x = 0;
        #pragma unroll 1
        for (uint32_t b = 0; b < 32; ++b) {
            const uint32_t v = lo + b;
            if (v >= 1 && v < hop) c1 |= 1u << b;
            if (v >= hop + keep && v < n) x |= 1u << b;
        }
        S.c1bits()[wi] = c1;
        S.xbits()[wi] = x;
        S.pbits()[wi] = (wi == 0) ? 1u : 0u;
    }
    #pragma unroll 1
    for (uint32_t i = l; i < n; i += 32) {
        if (i >= hop && i < hop + keep) S.c2()[i - hop] = (uint16_t)i;
        S.t1()[i] = 0;
        S.t2()[i] = 0;
    }
    if (l == 0) {
        S.P()[0] = 0;
        S.np() = 1;
        S.nc2() = keep;
        S.sz() = 1;
        S.w[4] = d;   // chain depth: the frame's depth in the reference's stack
        S.fr()[0] = fr_pack((uint32_t)(rd.k - 1), 1, d < m ? 2u : 0u, 0);
        S.root() = r;
    }
    __syncwarp();
}

// upperBoundK2 (src:1002-1020): every P member keeps neiInG + k >= q, neiInG over P ∪ C1.
template <int NW>
__device__ bool ks_upper_bound(const SearchParams& sp, const RootView& R, const KsSlot<NW>& S, uint32_t np,
                               const Bits<NW>& PC1) {
    const unsigned l = lane_id();
    bits_store(S.mask(), PC1);
    __syncwarp();
    bool ok = true;
    #pragma unroll 1
    for (uint32_t i = l; i < np; i += 32) {
        const uint32_t u = S.P()[i];
        if (row_and_popc(R.A + (uint64_t)u * R.W, S.mask(), R.W) + R.k < R.q) ok = false;
    }
    ok = __all_sync(FULL, ok);
    __syncwarp();
    return ok;
}

template <int NW>
struct Emitted {
    uint32_t np, nc, nx;
    Bits<NW> P, C, X;   // this lane's words
};

// Runs the k-search state machine (src:1993-2442) of the root held in S until
// it emits one task (returns 1, task in *e) or the root is finished (returns 0).
// The frame bookkeeping after an emission is done before returning, so the
// saved state resumes exactly where the reference resumes after its pause.
template <int NW>
__device__ int ks_advance(const SearchParams& sp, const KsSlot<NW>& S, Emitted<NW>* e) {
    const unsigned l = lane_id();
    const uint32_t r = S.root();
    const RootView R = root_view(sp, r);
    const int k = R.k, q = R.q;
    const uint32_t n = R.n, W = R.W;
    Bits<NW> C1 = bits_load<NW>(S.c1bits(), S.BW), X = bits_load<NW>(S.xbits(), S.BW), P = bits_load<NW>(S.pbits(), S.BW);
    uint32_t sz = S.sz(), np = S.np(), nc2 = S.nc2();
    int emitted = 0;
    Bits<NW> emitC = bits_zero<NW>();

    auto update13 = [&](uint32_t node, uint16_t tag) {   // updateCand13, src:1042-1097
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            const uint32_t wi = l + 32u * j;
            const uint32_t m2 = (wi < W) ? __ldg(R.M2() + (uint64_t)node * W + wi) : 0u;
            uint32_t drop = C1.w[j] & ~m2;
            C1.w[j] &= m2;
            while (drop) { const int b = __ffs(drop) - 1; S.t1()[wi * 32 + b] = tag; drop &= drop - 1; }
        }
    };
    auto update23 = [&](uint32_t node, uint16_t tag) {   // updateCand23, src:1099-1122 (order preserving)
        const uint32_t* m2row = R.M2() + (uint64_t)node * W;
        uint32_t write = 0;
        #pragma unroll 1
        for (uint32_t b = 0; b < nc2; b += 32) {
            const uint32_t i = b + l;
            uint16_t v = 0;
            bool keep = false;
            if (i < nc2) { v = S.c2()[i]; keep = (__ldg(m2row + (v >> 5)) >> (v & 31)) & 1u; }
            const unsigned km = __ballot_sync(FULL, keep);
            __syncwarp();
            if (i < nc2) {
                if (keep) S.c2()[write + __popc(km & ((1u << l) - 1))] = v;
                else S.t2()[v] = tag;
            }
            write += __popc(km);
            __syncwarp();
        }
        nc2 = write;
    };
    auto include = [&](uint32_t u) {
        if (l == 0) S.P()[np] = u;
        ++np;
        bits_set(P, u);
        __syncwarp();
    };
    auto c2_pop = [&]() -> uint32_t { --nc2; return S.c2()[nc2]; };
    auto c2_push = [&](uint32_t u) { __syncwarp(); if (l == 0) S.c2()[nc2] = (uint16_t)u; ++nc2; __syncwarp(); };
    auto setfr = [&](uint32_t f, uint32_t val) { __syncwarp(); if (l == 0) S.fr()[f] = val; __syncwarp(); };

    while (sz && !emitted) {
        if (sz + 1 >= S.L.c2 - S.L.fr) {
            // a frame stack sized n_max + 8 cannot fill (see KS_MAX_DEPTH); guard the
            // shared-memory layout all the same
            if (l == 0) { atomicAdd(&sp.ctr->depth_capped, 1u); raise_error(sp.ctr, KPLEX_ERR_INTERNAL); }
            sz = 0;
            break;
        }
        const uint32_t f = sz - 1;
        const uint16_t tag = (uint16_t)(f + 1);
        const uint32_t F = S.fr()[f];
        const uint32_t res = fr_res(F), br = fr_br(F), st = fr_st(F);
        if (st == 0) {
            if (nc2 == 0) {   // leaf: emit (P, C1, X) (src:2005-2092)
                const int nc1 = bits_count(C1);
                bool ok = (int)np + nc1 >= q;
                if (ok && np > 1) ok = ks_upper_bound(sp, R, S, np, bits_or(P, C1));
                --sz;
                if (ok) { emitted = 1; emitC = C1; }
                continue;
            }
            const uint32_t u = c2_pop();   // exclude the last C2 vertex first
            bits_set(X, u);
            setfr(f, fr_pack(res, br, 1, u));
            setfr(sz, fr_pack(res, 1, 0, 0));
            ++sz;
            continue;
        }
        if (st == 1 || st == 3) {   // child returned: the excluded vertex goes back to C2's end
            const uint32_t u = fr_v(F);
            c2_push(u);
            bits_clear(X, u);
            setfr(f, fr_pack(res, st == 3 ? br + 1 : br, 2, u));
            continue;
        }
        if (st == 2) {
            if (br < res) {   // include one more C2 vertex, exclude the next, recurse with res - br
                const uint32_t u = c2_pop();
                include(u);
                update13(u, tag);
                update23(u, tag);
                if (nc2) {
                    const uint32_t w = c2_pop();
                    bits_set(X, w);
                    setfr(f, fr_pack(res, br, 3, w));
                } else {
                    setfr(f, fr_pack(res, br, 4, 0));
                }
                setfr(sz, fr_pack(res - br, 1, 0, 0));
                ++sz;
                continue;
            }
            setfr(f, fr_pack(res, br, 4, 0));
            continue;
        }
        if (st == 4) {
            setfr(f, fr_pack(res, br, 5, 0));
            if (br == res) {   // budget used: include the last one and emit with C1 filtered (src:2259-2403)
                const uint32_t u = c2_pop();
                include(u);
                update13(u, tag);
                const int nc1 = bits_count(C1);
                if ((int)np + nc1 < q) continue;
                if (np > 1 && !ks_upper_bound(sp, R, S, np, bits_or(P, C1))) continue;
                // isKplex2 (src:568-584): c stays if P + c is a k-plex
                bits_store(S.mask(), P);
                bits_fill<NW>(S.aux(), 0u);
                bits_fill<NW>(S.keep(), 0u);
                __syncwarp();
                #pragma unroll 1
                for (uint32_t i = l; i < np; i += 32) {
                    const uint32_t v = S.P()[i];
                    if (row_and_popc(R.A + (uint64_t)v * W, S.mask(), W) + k == (int)np) atomicOr(&S.aux()[v >> 5], 1u << (v & 31));
                }
                const int m1 = bits_list(C1, S.lst());
                #pragma unroll 1
                for (int i = l; i < m1; i += 32) {
                    const uint32_t v = S.lst()[i];
                    const uint32_t* row = R.A + (uint64_t)v * W;
                    bool ok = row_and_popc(row, S.mask(), W) + k >= (int)np + 1;
                    #pragma unroll 1
                    for (uint32_t w = 0; ok && w < W; ++w) if (S.aux()[w] & ~__ldg(row + w)) ok = false;
                    if (ok) atomicOr(&S.keep()[v >> 5], 1u << (v & 31));
                }
                __syncwarp();
                emitted = 1;
                emitC = bits_load<NW>(S.keep(), S.BW);
                continue;
            }
            continue;
        }
        // st == 5: undo this frame (src:2405-2441)
        #pragma unroll 1
        for (uint32_t i = 0; i < br; ++i) {
            const uint32_t node = S.P()[np - 1];
            --np;
            bits_clear(P, node);
            c2_push(node);
        }
        #pragma unroll 1
        for (uint32_t b = 0; b < n; b += 32) {
            const uint32_t i = b + l;
            bool h1 = false, h2 = false;
            if (i < n) { h1 = S.t1()[i] == tag; h2 = S.t2()[i] == tag; }
            const unsigned m1 = __ballot_sync(FULL, h1), m2 = __ballot_sync(FULL, h2);
            if (h1) S.t1()[i] = 0;
            if (h2) { S.t2()[i] = 0; S.c2()[nc2 + __popc(m2 & ((1u << l) - 1))] = (uint16_t)i; }
            bits_or_word(C1, b >> 5, m1);
            nc2 += __popc(m2);
            __syncwarp();
        }
        --sz;
    }
    if (emitted) {
        e->np = np;
        e->nc = (uint32_t)bits_count(emitC);
        e->nx = (uint32_t)bits_count(X);
        e->P = P; e->C = emitC; e->X = X;
    }
    __syncwarp();
    bits_store(S.c1bits(), C1);
    bits_store(S.xbits(), X);
    bits_store(S.pbits(), P);
    if (l == 0) { S.sz() = sz; S.np() = np; S.nc2() = nc2; }
    __syncwarp();
    return emitted;
}

// ============================================================== branch-and-bound
// Adjacency rows are read through a generic pointer: the warp's copy of the
// root's A in shared memory when it fits, else the arena in global memory.
// W is a multiple of 4 and at least 4: the first 16-byte chunk is outside the
// loop (rows of up to 256 vertices take one or two chunks).
__device__ __forceinline__ int rowg_popc(const uint32_t* row, const uint32_t* mask, unsigned W) {
    const uint4* r4 = reinterpret_cast<const uint4*>(row);
    const uint4* m4 = reinterpret_cast<const uint4*>(mask);
    const uint4 a0 = r4[0], m0 = m4[0];
    int c = __popc(a0.x & m0.x) + __popc(a0.y & m0.y) + __popc(a0.z & m0.z) + __popc(a0.w & m0.w);
#pragma unroll 1
    for (unsigned w = 1; w < W / 4; ++w) {
        const uint4 a = r4[w], m = m4[w];
        c += __popc(a.x & m.x) + __popc(a.y & m.y) + __popc(a.z & m.z) + __popc(a.w & m.w);
    }
    return c;
}
// popcount of row & mask, and whether every bit of sat is in row
__device__ __forceinline__ int rowg_popc_covers(const uint32_t* row, const uint32_t* mask, const uint32_t* sat,
                                                unsigned W, bool* covers) {
    const uint4* r4 = reinterpret_cast<const uint4*>(row);
    const uint4* m4 = reinterpret_cast<const uint4*>(mask);
    const uint4* s4 = reinterpret_cast<const uint4*>(sat);
    const uint4 a0 = r4[0], m0 = m4[0], t0 = s4[0];
    int c = __popc(a0.x & m0.x) + __popc(a0.y & m0.y) + __popc(a0.z & m0.z) + __popc(a0.w & m0.w);
    uint32_t miss = (t0.x & ~a0.x) | (t0.y & ~a0.y) | (t0.z & ~a0.z) | (t0.w & ~a0.w);
#pragma unroll 1
    for (unsigned w = 1; w < W / 4; ++w) {
        const uint4 a = r4[w], m = m4[w], t = s4[w];
        c += __popc(a.x & m.x) + __popc(a.y & m.y) + __popc(a.z & m.z) + __popc(a.w & m.w);
        miss |= (t.x & ~a.x) | (t.y & ~a.y) | (t.z & ~a.z) | (t.w & ~a.w);
    }
    *covers = (miss == 0);
    return c;
}

// whether every bit of sat is in row
__device__ __forceinline__ bool rowg_covers(const uint32_t* row, const uint32_t* sat, unsigned W) {
    const uint4* r4 = reinterpret_cast<const uint4*>(row);
    const uint4* s4 = reinterpret_cast<const uint4*>(sat);
    const uint4 a0 = r4[0], t0 = s4[0];
    uint32_t miss = (t0.x & ~a0.x) | (t0.y & ~a0.y) | (t0.z & ~a0.z) | (t0.w & ~a0.w);
#pragma unroll 1
    for (unsigned w = 1; w < W / 4; ++w) {
        const uint4 a = r4[w], t = s4[w];
        miss |= (t.x & ~a.x) | (t.y & ~a.y) | (t.z & ~a.z) | (t.w & ~a.w);
    }
    return miss == 0;
}

// popcounts of row & m1 and row & m2 in one pass over the row
__device__ __forceinline__ void rowg_popc2(const uint32_t* row, const uint32_t* m1, const uint32_t* m2, unsigned W,
                                           int& c1, int& c2) {
    const uint4* r4 = reinterpret_cast<const uint4*>(row);
    const uint4* x4 = reinterpret_cast<const uint4*>(m1);
    const uint4* y4 = reinterpret_cast<const uint4*>(m2);
    const uint4 a0 = r4[0], x0 = x4[0], y0 = y4[0];
    int a1 = __popc(a0.x & x0.x) + __popc(a0.y & x0.y) + __popc(a0.z & x0.z) + __popc(a0.w & x0.w);
    int a2 = __popc(a0.x & y0.x) + __popc(a0.y & y0.y) + __popc(a0.z & y0.z) + __popc(a0.w & y0.w);
#pragma unroll 1
    for (unsigned w = 1; w < W / 4; ++w) {
        const uint4 a = r4[w], x = x4[w], y = y4[w];
        a1 += __popc(a.x & x.x) + __popc(a.y & x.y) + __popc(a.z & x.z) + __popc(a.w & x.w);
        a2 += __popc(a.x & y.x) + __popc(a.y & y.y) + __popc(a.z & y.z) + __popc(a.w & y.w);
    }
    c1 = a1;
    c2 = a2;
}

// The newest STACK_CACHE records a warp pushes on its depth-first stack are
// also kept in its shared memory (tagged with their stack index), so that the
// usual pop, of the record pushed last, does not wait for an L2 round trip.
constexpr uint32_t STACK_CACHE = 4;

__host__ __device__ inline uint32_t stack_cache_words(uint32_t slot_words) {
    return (STACK_CACHE * slot_words + STACK_CACHE + 3u) & ~3u;
}

__host__ __device__ inline uint32_t bnb_fixed_words(uint32_t nmax, uint32_t slot_words, uint32_t bw) {
    return ((slot_words + 9 * bw + 3 * ((nmax + 1) / 2)) + 3u) & ~3u;
}

__host__ __device__ inline uint32_t bnb_smem_words(uint32_t nmax, uint32_t slot_words, uint32_t a_words, uint32_t bw) {
    return bnb_fixed_words(nmax, slot_words, bw) + 32u + stack_cache_words(slot_words) + a_words;
}

// Per-warp shared memory of the branch-and-bound.  In words from the warp's base:
//   rec [slot_words] | P, PC, SAT, ROW, M2, M4, NC, NX, SB [BW each] |
//   list, gv, pv [nmax u16 each] | 16 counters (u64) | STACK_CACHE tags + records | A [a_words]
// with BW = 32 * NW.  Only the base address and two sizes are kept; every region's
// address is derived on use, which keeps a warp's registers for its search state.
struct BnbSmem {
    uint32_t* base;
    uint32_t sw;     // slot_words
    uint32_t half;   // words of one u16 list of nmax entries
    uint32_t bw;     // bitset words
    __device__ __forceinline__ uint32_t* rec() const { return base; }
    __device__ __forceinline__ uint32_t* P() const { return base + sw; }
    __device__ __forceinline__ uint32_t* PC() const { return base + sw + bw; }
    __device__ __forceinline__ uint32_t* SAT() const { return base + sw + 2 * bw; }
    __device__ __forceinline__ uint32_t* ROW() const { return base + sw + 3 * bw; }
    __device__ __forceinline__ uint32_t* M2() const { return base + sw + 4 * bw; }
    __device__ __forceinline__ uint32_t* M4() const { return base + sw + 5 * bw; }
    __device__ __forceinline__ uint32_t* NC() const { return base + sw + 6 * bw; }
    __device__ __forceinline__ uint32_t* NX() const { return base + sw + 7 * bw; }
    __device__ __forceinline__ uint32_t* SB() const { return base + sw + 8 * bw; }
    __device__ __forceinline__ uint16_t* list() const { return reinterpret_cast<uint16_t*>(base + sw + 9 * bw); }
    __device__ __forceinline__ uint16_t* gv() const { return reinterpret_cast<uint16_t*>(base + sw + 9 * bw + half); }
    __device__ __forceinline__ uint16_t* pv() const { return reinterpret_cast<uint16_t*>(base + sw + 9 * bw + 2 * half); }
    __device__ __forceinline__ uint32_t fixed() const { return (sw + 9 * bw + 3 * half + 3u) & ~3u; }
    __device__ __forceinline__ unsigned long long* CT() const { return reinterpret_cast<unsigned long long*>(base + fixed()); }
    __device__ __forceinline__ uint32_t* SCT() const { return base + fixed() + 32; }
    __device__ __forceinline__ uint32_t* SC() const { return SCT() + STACK_CACHE; }
    __device__ __forceinline__ uint32_t* A() const { return SCT() + stack_cache_words(sw); }
};

__device__ __forceinline__ BnbSmem bnb_smem(uint32_t* base, uint32_t nmax, uint32_t slot_words, uint32_t bw) {
    return BnbSmem{base, slot_words, (nmax + 1) / 2, bw};
}

// The reference's warp pivot rule (src:1628-1663, 1669-1697): the shfl_down
// tree keeps the current pivot unless the other lane's is strictly smaller in
// neiInG, or equal with a strictly smaller neiInP.
// Each step keeps the lower lane's pivot on a tie, so among lanes holding the
// smallest (neiInG, neiInP) the tree returns the one whose lane index, read
// with its 5 bits reversed, is smallest (lane 0 before 16 before 8 before 24
// ...), and lane 0's empty state when no lane has a candidate.  That order is
// folded into one key for a hardware min-reduction and a ballot.
__device__ __forceinline__ void pivot_tree(int& m, int& v, int& p, int& idx) {
    const unsigned rank = __brev(lane_id()) >> 27;
    const unsigned key = (v != -1) ? (((unsigned)m << 21) | ((unsigned)p << 5) | rank) : 0xffffffffu;
    const unsigned best = __reduce_min_sync(FULL, key);
    const int src = __ffs(__ballot_sync(FULL, key == best)) - 1;
    m = __shfl_sync(FULL, m, src); v = __shfl_sync(FULL, v, src);
    p = __shfl_sync(FULL, p, src); idx = __shfl_sync(FULL, idx, src);
}

// isMaximal_opt / isMaximalPC_opt (src:703-1000): true when no vertex of the
// root's left set extends S (list[0..s), degrees deg[], bitset sS) to a k-plex.
// Candidates must be adjacent to every saturated member of S and to one of any
// k members; each candidate's count is its popcount against S.
// Out of line (with its arguments by value): it runs only at the leaves, and
// keeping it out of the node loop keeps that loop's code small.
__device__ __noinline__ bool left_maximal(const RootView R, const BnbSmem m, int s, const uint16_t* deg,
                                          const uint32_t* sS, unsigned long long* bb) {
    const unsigned l = lane_id();
    const int k = R.k;
    if (R.nleft == 0) return true;
    const uint32_t WL = R.WL, W = R.W;
    int nrows = 0;
    bool found = false;
    // the left set's words in chunks of 32, one word per lane
    #pragma unroll 1
    for (uint32_t base = 0; base < WL && !found; base += 32) {
        const uint32_t w = base + l;
        uint32_t lc = 0;
        if (w < WL) {
            const int lo = (int)w * 32, nl = (int)R.nleft;
            lc = nl >= lo + 32 ? FULL : (nl > lo ? ((1u << (nl - lo)) - 1) : 0u);
        }
        #pragma unroll 1
        for (int b = 0; b < s; b += 32) {   // adjacent to every saturated member
            const int i = b + (int)l;
            const bool sat = i < s && (int)deg[i] + k <= s;
            unsigned msk = __ballot_sync(FULL, sat);
            while (msk) {
                const int j = __ffs(msk) - 1;
                msk &= msk - 1;
                const uint32_t u = m.list()[b + j];
                if (w < WL) lc &= __ldg(R.LA() + (uint64_t)u * WL + w);
            }
        }
        uint32_t un = 0;   // and to one of any k members
        #pragma unroll 1
        for (int t = 0; t < k && t < s; ++t) {
            const uint32_t u = m.list()[t];
            if (w < WL) un |= __ldg(R.LA() + (uint64_t)u * WL + w);
        }
        lc &= un;
        bool f = false;
        uint32_t c = lc;
        while (c && !f) {
            const int bit = __ffs(c) - 1;
            c &= c - 1;
            const uint32_t j = w * 32 + bit;
            const int cnt = row_and_popc(R.LT() + (uint64_t)j * W, sS, W);
            ++nrows;
            if (cnt + k >= s + 1) f = true;
        }
        found = __any_sync(FULL, f);
    }
    nrows = warp_sum(nrows);
    if (l == 0) *bb += (unsigned long long)nrows * 4ull * W + (unsigned long long)(k + 1) * 4ull * WL;
    return !found;
}

// Adds one maximal k-plex (list[0..s)) to the count and hash.
template <int NW>
__device__ __noinline__ void emit_plex(const RootView R, const BnbSmem m, int s, uint32_t hash_on,
                                       unsigned long long* cnt, unsigned long long* hsum) {
    const unsigned l = lane_id();
    if (l == 0) ++*cnt;
    if (!hash_on) return;
    bits_fill<NW>(m.SB(), 0u);
    __syncwarp();
    #pragma unroll 1
    for (int i = l; i < s; i += 32) {
        const uint32_t rk = __ldg(R.srank() + m.list()[i]);
        atomicOr(&m.SB()[rk >> 5], 1u << (rk & 31));
    }
    __syncwarp();
    // the sorted original ids, word by word in ascending order: lane L walks word
    // 32 j + L and passes the running hash on to lane L + 1
    uint64_t x = plex_hash_begin((uint32_t)s);
#pragma unroll
    for (int j = 0; j < NW; ++j) {
        uint32_t w = m.SB()[32 * j + l];
        for (int L = 0; L < 32; ++L) {
            if ((int)l == L) {
                while (w) {
                    const int b = __ffs(w) - 1;
                    w &= w - 1;
                    x = plex_hash_step(x, __ldg(R.sorig() + (32 * j + L) * 32 + b));
                }
            }
            x = __shfl_sync(FULL, x, L);
        }
    }
    if (l == 0) *hsum += x;
}

template <int NW>
struct Node {
    uint32_t root, np, nc, nx;
    Bits<NW> P, C, X;   // this lane's words of each bitset
};

// Counters live in the warp's shared memory (m.CT()) and are updated by lane 0.
enum : int { CT_CNT, CT_HSUM, CT_TASKS, CT_NODES, CT_BB, CT_TOT_CNT, CT_TOT_HSUM, CT_STAGE, CT_KS_CYC, CT_SPILL,
             CT_REFILL, CT_BNB_CYC, CT_IDLE_CYC, CT_KS_TASKS };
// A warp's depth-first stack (records [sbot, stop) of `stack`, a ring of
// stack_depth records, a power of two, so a record's slot is its index masked)
// and its counters in shared memory.  The indices are 32-bit: the stack empties
// (both reset) long before they could wrap.
struct WarpWork {
    uint32_t* stack;
    uint32_t sbot, stop;
    unsigned long long* ct;
    __device__ __forceinline__ unsigned long long& cnt() const { return ct[CT_CNT]; }
    __device__ __forceinline__ unsigned long long& hsum() const { return ct[CT_HSUM]; }
    __device__ __forceinline__ unsigned long long& tasks() const { return ct[CT_TASKS]; }
    __device__ __forceinline__ unsigned long long& nodes() const { return ct[CT_NODES]; }
    __device__ __forceinline__ unsigned long long& bb() const { return ct[CT_BB]; }
};

// One branch-and-bound node (BNB, src:1516-1724).  Returns true when the node
// produced an include child, which is left in *t; the exclude child is pushed
// on the warp's stack.
template <int NW>
__device__ bool bnb_node(const SearchParams& sp, const BnbSmem& m, const RootView& R, const uint32_t* A, Node<NW>* t,
                         WarpWork& ww) {
    const unsigned l = lane_id();
    const int k = R.k, q = R.q;
    const uint32_t W = R.W, Wt = sp.Wt, SW = sp.slot_words;
    const uint32_t np = t->np, nc = t->nc, nx = t->nx;
    const Bits<NW> P = t->P, C = t->C, X = t->X;
    if ((int)(np + nc) < q) return false;
    bits_store(m.P(), P);
    bits_store(m.PC(), bits_or(P, C));
    __syncwarp();
    bits_list2(P, C, m.list(), m.list() + np);
    const int tot = (int)(np + nc);
    #pragma unroll 1
    for (int i = l; i < tot; i += 32) {
        int g, p;
        rowg_popc2(A + (uint32_t)m.list()[i] * W, m.PC(), m.P(), W, g, p);
        m.gv()[i] = (uint16_t)g;
        m.pv()[i] = (uint16_t)p;
    }
    if (l == 0) ww.bb() += (unsigned long long)(tot + 3) * 4ull * W;   // rows + the record's P, C, X
    __syncwarp();
    if (nc == 0) {   // src:1579-1588
        if (nx == 0 && (int)np >= q && left_maximal(R, m, (int)np, m.pv(), m.P(), &ww.bb()))
            emit_plex<NW>(R, m, (int)np, sp.hash_on, &ww.cnt(), &ww.hsum());
        return false;
    }
    // pivot in P: minimum neiInG, ties to the smaller index (src:1592-1620)
    unsigned long long key = ~0ull;   // (neiInG, vertex, neiInP) of this lane's best P member
    #pragma unroll 1
    for (int i = l; i < (int)np; i += 32) {
        const unsigned long long kk = ((unsigned long long)m.gv()[i] << 32) | ((unsigned long long)m.list()[i] << 16) | m.pv()[i];
        key = kk < key ? kk : key;
    }
    const unsigned kg = (unsigned)(key >> 32);
    const unsigned gmin = __reduce_min_sync(FULL, kg);
    const unsigned kv = (kg == gmin) ? (unsigned)(key & 0xffffffffu) : 0xffffffffu;   // vertex << 16 | neiInP
    const unsigned vmin = __reduce_min_sync(FULL, kv);
    const int minP = (int)gmin;
    const int pp = (int)(vmin >> 16);
    const int ppP = (int)(vmin & 0xffff);
    if (minP + k < max(q, (int)np)) return false;   // src:1624
    int piv, pmin, pval, pidx;
    if (minP + k < tot) {
        // candidates not adjacent to the P pivot (src:1626-1663)
        bits_store(m.ROW(), bits_load<NW>(A + (uint32_t)pp * W, W));
        __syncwarp();
        pmin = INT_MAX; piv = -1; pval = 0; pidx = -1;
        #pragma unroll 1
        for (int i = l; i < (int)nc; i += 32) {
            const uint32_t v = m.list()[np + i];
            if (test_bit(m.ROW(), v)) continue;
            const int g = m.gv()[np + i], p = m.pv()[np + i];
            if (g < pmin) { pmin = g; piv = (int)v; pval = p; pidx = (int)np + i; }
            else if (g == pmin && pval > p) { piv = (int)v; pval = p; pidx = (int)np + i; }
        }
        pivot_tree(pmin, piv, pval, pidx);
    } else {
        // minimum over P (seeded) and C (src:1669-1697)
        pmin = minP; piv = pp; pval = ppP; pidx = -2;
        #pragma unroll 1
        for (int i = l; i < (int)nc; i += 32) {
            const uint32_t v = m.list()[np + i];
            const int g = m.gv()[np + i], p = m.pv()[np + i];
            if (g < pmin) { pmin = g; piv = (int)v; pval = p; pidx = (int)np + i; }
            else if (g == pmin && pval > p) { piv = (int)v; pval = p; pidx = (int)np + i; }
        }
        pivot_tree(pmin, piv, pval, pidx);
        if (pmin >= tot - k) {
            // P ∪ C is a k-plex (src:1698-1717)
            if (tot < q) return false;
            const int nxl = bits_list(X, m.list() + tot);
            #pragma unroll 1
            for (int i = l; i < nxl; i += 32)
                m.gv()[tot + i] = (uint16_t)rowg_popc(A + (uint32_t)m.list()[tot + i] * W, m.PC(), W);
            bits_fill<NW>(m.SAT(), 0u);
            __syncwarp();
            #pragma unroll 1
            for (int i = l; i < tot; i += 32)
                if ((int)m.gv()[i] + k == tot) { const uint32_t u = m.list()[i]; atomicOr(&m.SAT()[u >> 5], 1u << (u & 31)); }
            __syncwarp();
            bool ext = false;
            #pragma unroll 1
            for (int i = l; i < nxl; i += 32) {   // isKplexPC2 src:601-622
                if ((int)m.gv()[tot + i] + k < tot + 1) continue;
                ext |= rowg_covers(A + (uint32_t)m.list()[tot + i] * W, m.SAT(), W);
            }
            if (l == 0) ww.bb() += (unsigned long long)nxl * 4ull * W;
            if (__any_sync(FULL, ext)) return false;
            if (left_maximal(R, m, tot, m.gv(), m.PC(), &ww.bb())) emit_plex<NW>(R, m, tot, sp.hash_on, &ww.cnt(), &ww.hsum());
            return false;
        }
    }
    // ---------------- branch on piv (src:1197-1465)
    if (piv < 0 || pidx < 0) { if (l == 0) raise_error(sp.ctr, KPLEX_ERR_INTERNAL); return false; }
    const uint32_t v = (uint32_t)piv;
    // the include child's rows of v, loaded now so that their latency overlaps the
    // exclude child's write
    const Bits<NW> rowA = bits_load<NW>(A + v * W, W);
    const Bits<NW> rowM2 = bits_ldg<NW>(R.M2() + (uint64_t)v * W, W);
    const Bits<NW> rowM4 = bits_ldg<NW>(R.M4() + (uint64_t)v * W, W);
    {   // exclude child -> this warp's stack
        if (ww.stop - ww.sbot >= sp.stack_depth) { if (l == 0) raise_error(sp.ctr, KPLEX_ERR_INTERNAL); return false; }
        uint32_t* dst = ww.stack + (ww.stop & (sp.stack_depth - 1)) * SW;
        Bits<NW> Cx = C, Xx = X;
        bits_clear(Cx, v);
        bits_set(Xx, v);
        uint32_t* cdst = m.SC() + (ww.stop % STACK_CACHE) * SW;   // shared-memory copy
        if (l == 0) {
            __stcg(dst + 0, t->root); __stcg(dst + 1, np | ((nc - 1) << 16)); __stcg(dst + 2, nx + 1); __stcg(dst + 3, 0u);
            cdst[0] = t->root; cdst[1] = np | ((nc - 1) << 16); cdst[2] = nx + 1; cdst[3] = 0u;
            m.SCT()[ww.stop % STACK_CACHE] = ww.stop;
        }
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            const uint32_t wi = l + 32u * j;
            if (wi < Wt) {
                __stcg(dst + 4 + wi, P.w[j]); __stcg(dst + 4 + Wt + wi, Cx.w[j]); __stcg(dst + 4 + 2 * Wt + wi, Xx.w[j]);
                cdst[4 + wi] = P.w[j]; cdst[4 + Wt + wi] = Cx.w[j]; cdst[4 + 2 * Wt + wi] = Xx.w[j];
            }
        }
        __syncwarp();
        ++ww.stop;
    }
    // include child
    const uint32_t np1 = np + 1;
    Bits<NW> P1 = P;
    bits_set(P1, v);
    bits_store(m.ROW(), rowA);
    bits_store(m.M2(), rowM2);
    bits_store(m.M4(), rowM4);
    bits_fill<NW>(m.SAT(), 0u);
    bits_fill<NW>(m.NC(), 0u);
    bits_fill<NW>(m.NX(), 0u);
    __syncwarp();
    // saturated members of P + v: neiInP' + k == |P'|
    #pragma unroll 1
    for (int i = l; i < (int)np; i += 32) {
        const uint32_t u = m.list()[i];
        const int pu = (int)m.pv()[i] + (int)test_bit(m.ROW(), u);
        if (pu + k == (int)np1) atomicOr(&m.SAT()[u >> 5], 1u << (u & 31));
    }
    if (l == 0 && (int)m.pv()[pidx] + k == (int)np1) atomicOr(&m.SAT()[v >> 5], 1u << (v & 31));
    bits_store(m.P(), P1);
    __syncwarp();
    // C filter: class >= UNLINK2EQUAL and P' + c a k-plex (isKplex3)
    #pragma unroll 1
    for (int i = l; i < (int)nc; i += 32) {
        const uint32_t c = m.list()[np + i];
        if (c == v || !test_bit(m.M2(), c)) continue;
        const int pc = (int)m.pv()[np + i] + (int)test_bit(m.ROW(), c);
        if (pc + k < (int)np1 + 1) continue;
        if (rowg_covers(A + c * W, m.SAT(), W)) atomicOr(&m.NC()[c >> 5], 1u << (c & 31));
    }
    __syncwarp();
    const Bits<NW> C1 = bits_load<NW>(m.NC(), 32 * NW);
    const uint32_t nc1 = (uint32_t)bits_count(C1);
    bits_store(m.PC(), bits_or(P1, C1));
    __syncwarp();
    // upperBound2 over P' (src:1022-1040)
    bool ub = true;
    #pragma unroll 1
    for (int i = l; i <= (int)np; i += 32) {
        const uint32_t u = (i < (int)np) ? m.list()[i] : v;
        if (rowg_popc(A + u * W, m.PC(), W) + k < q) ub = false;
    }
    // rows read below: the exclude record (3), the C filter (nc), the upper bound (np + 1)
    if (!__all_sync(FULL, ub)) {
        if (l == 0) { ++ww.tasks(); ww.bb() += (unsigned long long)(nc + np1 + 3) * 4ull * W; }
        return false;
    }
    // X filter: class >= UNLINK2MORE and P' + x a k-plex
    const int nxl = bits_list(X, m.list());
    #pragma unroll 1
    for (int i = l; i < nxl; i += 32) {
        const uint32_t x = m.list()[i];
        if (!test_bit(m.M4(), x)) continue;
        bool ok;
        const int px = rowg_popc_covers(A + x * W, m.P(), m.SAT(), W, &ok);
        if (ok && px + k >= (int)np1 + 1) atomicOr(&m.NX()[x >> 5], 1u << (x & 31));
    }
    __syncwarp();
    const Bits<NW> X1 = bits_load<NW>(m.NX(), 32 * NW);
    t->nx = (uint32_t)bits_count(X1);
    t->P = P1; t->C = C1; t->X = X1;
    t->np = np1; t->nc = nc1;
    // and the X filter (nxl) and the include record (3)
    if (l == 0) { ww.tasks() += 2; ww.bb() += (unsigned long long)(nc + np1 + nxl + 6) * 4ull * W; }
    return true;
}

// ============================================================== the persistent kernel
template <int NW>
__device__ __forceinline__ void load_record(const uint32_t* src, uint32_t Wt, Node<NW>* t, bool cg) {
    const unsigned l = lane_id();
    if (cg) {
        t->root = __ldcg(src);
        const uint32_t h1 = __ldcg(src + 1);
        t->np = h1 & 0xffff; t->nc = h1 >> 16; t->nx = __ldcg(src + 2);
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            const uint32_t wi = l + 32u * j;
            t->P.w[j] = (wi < Wt) ? __ldcg(src + 4 + wi) : 0u;
            t->C.w[j] = (wi < Wt) ? __ldcg(src + 4 + Wt + wi) : 0u;
            t->X.w[j] = (wi < Wt) ? __ldcg(src + 4 + 2 * Wt + wi) : 0u;
        }
    } else {
        t->root = src[0];
        t->np = src[1] & 0xffff; t->nc = src[1] >> 16; t->nx = src[2];
#pragma unroll
        for (int j = 0; j < NW; ++j) {
            const uint32_t wi = l + 32u * j;
            t->P.w[j] = (wi < Wt) ? src[4 + wi] : 0u;
            t->C.w[j] = (wi < Wt) ? src[4 + Wt + wi] : 0u;
            t->X.w[j] = (wi < Wt) ? src[4 + 2 * Wt + wi] : 0u;
        }
    }
}

// ---------------------------------------------------------------- block queue
// A small LIFO of task records in shared memory, shared by the warps of one
// block.  A warp that holds stacked work hands its oldest record to an idle
// warp of its own block through it, and a producer hands new tasks to it while
// its block has idle warps, with shared-memory atomics only.  The global pool
// is used when the block has no idle warp, and only one warp per block polls
// the global pool at a time, so that an almost empty pool is not hammered by
// every idle warp of the device.
//
// Termination: the counter `work` holds one unit per unclaimed or running
// k-search job, per record in the pool, a block queue or the spill ring, and
// per warp holding work.  A unit is added before a record becomes visible and
// removed (after a fence) only when a job or a warp's work ends; taking a
// record moves its unit to the taker.  So the count is zero exactly when the
// search is finished, and no combination of separately read counters can show
// a finished state while a record is in flight.
constexpr uint32_t BQ_RECORDS = 8;
constexpr uint32_t BQ_HDR = 8;   // lock, count, idle warps, poller token, pad

__host__ __device__ inline uint32_t bq_words(uint32_t slot_words) {
    return BQ_HDR + ((BQ_RECORDS * slot_words + 3u) & ~3u);
}

struct BlockQueue {
    uint32_t* w;
    uint32_t SW;
    __device__ int* lock() const { return reinterpret_cast<int*>(w); }
    __device__ uint32_t* count() const { return w + 1; }
    __device__ uint32_t* idle() const { return w + 2; }
    __device__ int* poller() const { return reinterpret_cast<int*>(w + 3); }
    __device__ uint32_t* rec(uint32_t i) const { return w + BQ_HDR + i * SW; }
    __device__ uint32_t n() const { return *(volatile uint32_t*)count(); }
    __device__ uint32_t idle_warps() const { return *(volatile uint32_t*)idle(); }
};

// lane 0 only; a bounded spin (the lock is held for one record copy)
__device__ __forceinline__ bool bq_lock(const BlockQueue& q) {
    #pragma unroll 1
    for (int i = 0; i < 1 << 14; ++i) {
        if (atomicCAS(q.lock(), 0, 1) == 0) { __threadfence_block(); return true; }
        __nanosleep(32);
    }
    return false;
}
__device__ __forceinline__ void bq_unlock(const BlockQueue& q) {
    __threadfence_block();
    atomicExch(q.lock(), 0);
}

// Pushes one record (SW words from src) if the queue has room; whole warp.
__device__ __forceinline__ bool bq_push(const BlockQueue q, const uint32_t* src, int src_global) {
    const unsigned l = lane_id();
    int slot = -1;
    if (l == 0 && q.n() < BQ_RECORDS && bq_lock(q)) {
        const uint32_t c = q.n();
        if (c < BQ_RECORDS) slot = (int)c;
        else bq_unlock(q);
    }
    slot = __shfl_sync(FULL, slot, 0);
    if (slot < 0) return false;
    uint32_t* dst = q.rec((uint32_t)slot);
    for (unsigned i = l; i < q.SW; i += 32) dst[i] = rec_word(src, src_global, i);
    __threadfence_block();
    __syncwarp();
    if (l == 0) { *(volatile uint32_t*)q.count() = (uint32_t)slot + 1; bq_unlock(q); }
    __syncwarp();
    return true;
}

// Pops the newest record into dst (shared memory, SW words); whole warp.
__device__ __forceinline__ bool bq_pop(const BlockQueue q, uint32_t* dst) {
    const unsigned l = lane_id();
    int slot = -1;
    if (l == 0 && q.n() > 0 && bq_lock(q)) {
        const uint32_t c = q.n();
        if (c > 0) slot = (int)c - 1;
        else bq_unlock(q);
    }
    slot = __shfl_sync(FULL, slot, 0);
    if (slot < 0) return false;
    const uint32_t* src = q.rec((uint32_t)slot);
    #pragma unroll 1
    for (unsigned i = l; i < q.SW; i += 32) dst[i] = src[i];
    __threadfence_block();
    __syncwarp();
    if (l == 0) { *(volatile uint32_t*)q.count() = (uint32_t)slot; bq_unlock(q); }
    __syncwarp();
    return true;
}

template <int NW>
__device__ __forceinline__ void search_body(SearchParams sp, uint32_t nmax) {
    constexpr uint32_t BW = 32 * NW;
    extern __shared__ uint4 smem4[];
    uint32_t* smem = reinterpret_cast<uint32_t*>(smem4);
    const unsigned l = lane_id();
    const unsigned wib = threadIdx.x >> 5;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t SW = sp.slot_words, Wt = sp.Wt;
    const bool producer = (wib == 0);
    const KsLayout KL = ks_layout(nmax, NW);
    const KsSlot<NW> S{smem, KL};
    const BlockQueue BQ{smem + KL.total, SW};
    const BnbSmem m = bnb_smem(smem + KL.total + bq_words(SW) + wib * bnb_smem_words(nmax, SW, sp.a_words, BW), nmax, SW, BW);
    if (threadIdx.x < BQ_HDR) BQ.w[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t* A = nullptr;
    uint32_t same_root = 0;
    uint32_t acc_graph = 0;
    unsigned long long* CT = m.CT();
    if (l < 16) CT[l] = 0ull;
    if (l < STACK_CACHE) m.SCT()[l] = 0xffffffffu;
    __syncwarp();
    // the warp's mbarrier for bulk copies into its shared memory (counter slot 15)
    uint32_t tma_phase = 0;
    bool tma_ok = true;
    if (l == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"((unsigned)__cvta_generic_to_shared(&CT[15])) : "memory");
    __syncwarp();
    WarpWork ww{sp.stacks + (uint64_t)warp * sp.stack_depth * SW, 0u, 0u, CT};
    const unsigned long long resume_at = sp.pause_at / 2 > 0 ? sp.pause_at / 2 : 1;
    bool have = false, counted = false, ks_active = false, paused = false, is_idle = false;
    unsigned long long idle = 0;   // idle iterations counted toward spin_limit
    unsigned spins = 0;            // idle iterations since the warp last had work (backoff)
    // a warp that leaves the idle state (lane 0 keeps the block's idle count)
    auto wake = [&]() {
        if (is_idle) { if (l == 0) atomicSub(BQ.idle(), 1u); is_idle = false; }
        spins = 0;
    };
    Node<NW> t{};
    uint32_t cur_root = 0xffffffffu;
    RootView R{};
    Emitted<NW> e{};

    for (;;) {
        // ---------------- local depth-first work
        if (!have && ww.stop > ww.sbot) {
            --ww.stop;
            const uint32_t cs = ww.stop % STACK_CACHE;
            if (m.SCT()[cs] == ww.stop) load_record<NW>(m.SC() + cs * SW, Wt, &t, false);   // still cached
            else load_record<NW>(ww.stack + (ww.stop & (sp.stack_depth - 1)) * SW, Wt, &t, true);
            have = true;
            __syncwarp();
        }
        if (have) {
            if (ww.stop - ww.sbot >= 2 && (ww.nodes() & 3) == 0) {   // donate the oldest stacked record
                // to an idle warp of this block when there is one, else (every 256
                // nodes) to the global pool when it runs low.  The pool's head and
                // tail share a line that warps taking records hit with atomics: busy
                // warps that read it every 16 nodes spent 15% of the search waiting
                // on it (and reading it every 16 nodes only while it runs low cost
                // 18%: on soc-epinions it runs low nearly all the time).
                int give = 0;
                if (l == 0) {
                    const uint32_t iw = BQ.idle_warps();
                    if (iw > 0 && BQ.n() < iw) give = 1;
                    else if ((ww.nodes() & 255) == 0 && pool_size(sp) < sp.low_water) give = 2;
                }
                give = __shfl_sync(FULL, give, 0);
                if (give) {
                    const uint32_t* src = ww.stack + (ww.sbot & (sp.stack_depth - 1)) * SW;
                    // the record becomes a unit of work before it can be seen (and taken)
                    if (l == 0) { atomicAdd(&sp.ctr->work, 1u); __threadfence(); }
                    __syncwarp();
                    const bool ok = (give == 1) ? bq_push(BQ, src, 1) : pool_push(sp, src, 1);
                    if (ok) ++ww.sbot;
                    else if (l == 0) atomicSub(&sp.ctr->work, 1u);
                }
            }
            if (t.root != cur_root) {
                R = root_view(sp, t.root);
                cur_root = t.root;
                if (R.graph != acc_graph) {   // results are kept per input graph
                    if (l == 0 && (ww.cnt() || ww.hsum())) { atomicAdd(&sp.gcount[acc_graph], ww.cnt()); atomicAdd(&sp.ghash[acc_graph], ww.hsum()); }
                    if (l == 0) { CT[CT_TOT_CNT] += ww.cnt(); CT[CT_TOT_HSUM] += ww.hsum(); ww.cnt() = ww.hsum() = 0; }
                    __syncwarp();
                    acc_graph = R.graph;
                }
                A = R.A;
                same_root = 0;
            } else if (++same_root == sp.stage_after && R.n * R.W <= sp.a_words && tma_ok) {
                // the warp keeps working on this root: one bulk copy (global -> this CTA's shared
                // memory, no multicast) of its adjacency rows, completion on the warp's mbarrier
                const uint32_t bytes = R.n * R.W * 4;
                const unsigned mb = (unsigned)__cvta_generic_to_shared(&CT[15]);
                const unsigned dsts = (unsigned)__cvta_generic_to_shared(m.A());
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (l == 0) {
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mb), "r"(bytes) : "memory");
                    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                                 :: "r"(dsts), "l"(R.A), "r"(bytes), "r"(mb) : "memory");
                }
                uint32_t done = 0;
                for (int it = 0; it < (1 << 22) && !done; ++it)
                    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                                 : "=r"(done) : "r"(mb), "r"(tma_phase) : "memory");
                done = __all_sync(FULL, done);
                if (done) {
                    tma_phase ^= 1u;
                    A = m.A();
                    if (l == 0) ++CT[CT_STAGE];
                } else {   // gave up: keep reading the arena, stage nothing more
                    if (l == 0) raise_error(sp.ctr, KPLEX_ERR_TIMEOUT);
                    tma_ok = false;
                }
            }
            if (l == 0) ++ww.nodes();
            const long long b0 = clock64();
            have = bnb_node<NW>(sp, m, R, A, &t, ww);
            __syncwarp();
            if (l == 0) CT[CT_BNB_CYC] += (unsigned long long)(clock64() - b0);
            if (!have && ww.stop == ww.sbot) {
                ww.stop = ww.sbot = 0;
                if (counted) {   // after this warp's pushes are visible, its unit ends
                    if (l == 0) { __threadfence(); atomicSub(&sp.ctr->holders, 1u); atomicSub(&sp.ctr->work, 1u); }
                    counted = false;
                }
            }
            continue;
        }
        // ---------------- producer: k-search
        if (producer) {
            const unsigned long long ps = pool_size_warp(sp);
            // with spilling on, a full-enough pool sends new tasks to host memory
            // instead of pausing, until the spill ring itself is at its threshold
            int to_host = 0;
            if (sp.spill_on && ps >= sp.pause_at) {
                if (l == 0) to_host = ring_size(spill_ring(sp)) < sp.spill_pause_at;
                to_host = __shfl_sync(FULL, to_host, 0);
            }
            if (paused && ps < resume_at) paused = false;
            if (!paused && ps >= sp.pause_at && !to_host) {
                paused = true;
                if (l == 0) atomicAdd(&sp.ctr->ks_paused, 1u);
            }
            if (!paused) {
                if (!ks_active) {
                    // claim the next k-search job (its unit of work moves from "unclaimed"
                    // to "running"); ks_active tells idle warps that k-search still runs
                    int j = -1;
                    if (l == 0 && *(volatile unsigned*)&sp.ctr->next_root < sp.njobs) {
                        atomicAdd(&sp.ctr->ks_active, 1u);
                        const unsigned c = atomicAdd(&sp.ctr->next_root, 1u);
                        if (c < sp.njobs) j = (int)c;
                        else atomicSub(&sp.ctr->ks_active, 1u);
                    }
                    j = __shfl_sync(FULL, j, 0);
                    if (j >= 0) {
                        // root of job j: the last r with job_base[r] <= j (job_base is
                        // non-decreasing, job_base[0] = 0).  A 32-way search: each lane
                        // probes one point of [lo2, hi2), the ballot of "<= j" is a prefix
                        // of the lanes, and the interval shrinks 32-fold per round (four
                        // dependent loads for a million roots instead of twenty).
                        uint32_t lo2 = 0, hi2 = sp.nroots;
                        while (hi2 - lo2 > 1) {
                            const uint32_t step = (hi2 - lo2 + 31u) >> 5;
                            const uint32_t p = lo2 + (l + 1u) * step;
                            const bool le = p < hi2 && __ldg(sp.job_base + p) <= (uint32_t)j;
                            const uint32_t c = (uint32_t)__popc(__ballot_sync(FULL, le));
                            const uint32_t nlo = lo2 + c * step;
                            hi2 = min(nlo + step, hi2);
                            lo2 = nlo;
                        }
                        const RootDesc rd = sp.roots[lo2];
                        ks_start<NW>(sp, S, lo2, (uint32_t)j - __ldg(sp.job_base + lo2), rd);
                        ks_active = true;
                        wake();
                    }
                }
                if (ks_active) {
                    const long long c0 = clock64();
                    const int got = ks_advance<NW>(sp, S, &e);
                    if (l == 0) CT[CT_KS_CYC] += (unsigned long long)(clock64() - c0);
                    if (got) {
                        if (l == 0) ++CT[CT_KS_TASKS];
                        const uint32_t r = S.root();
                        // stage the record (hdr | P | C | X) in shared memory, then hand it over
                        uint32_t* rec = m.rec();
                        if (l == 0) { rec[0] = r; rec[1] = e.np | (e.nc << 16); rec[2] = e.nx; rec[3] = 0u; }
#pragma unroll
                        for (int j = 0; j < NW; ++j) {
                            const uint32_t wi = l + 32u * j;
                            if (wi < Wt) { rec[4 + wi] = e.P.w[j]; rec[4 + Wt + wi] = e.C.w[j]; rec[4 + 2 * Wt + wi] = e.X.w[j]; }
                        }
                        __syncwarp();
                        bool pushed = false;
                        if (l == 0) { atomicAdd(&sp.ctr->work, 1u); __threadfence(); }   // the task's unit
                        __syncwarp();
                        int local = 0;   // an idle warp of this block takes it directly
                        if (l == 0) local = BQ.idle_warps() > BQ.n();
                        if (__shfl_sync(FULL, local, 0)) pushed = bq_push(BQ, rec, 0);
                        if (!pushed && to_host) {   // spill: the record goes to pinned host memory
                            pushed = ring_push(sp, spill_ring(sp), rec, 0);
                            if (pushed && l == 0) ++CT[CT_SPILL];
                        }
                        if (!pushed) pushed = pool_push(sp, rec, 0);
                        if (!pushed) {   // ring full: keep the task
                            t.root = r; t.np = e.np; t.nc = e.nc; t.nx = e.nx;
                            t.P = e.P; t.C = e.C; t.X = e.X;
                            have = true;
                            wake();
                            if (!counted) { if (l == 0) atomicAdd(&sp.ctr->holders, 1u); counted = true; }
                        }
                    } else {
                        ks_active = false;
                        __syncwarp();
                        if (l == 0) {   // the job's unit ends after its tasks are visible
                            S.root() = 0xffffffffu;
                            __threadfence();
                            atomicSub(&sp.ctr->ks_active, 1u);
                            atomicSub(&sp.ctr->work, 1u);
                        }
                        __syncwarp();
                    }
                    idle = 0;
                    continue;
                }
            }
        }
        // ---------------- consumer: this block's queue, else (one warp per block at a
        // time) the global pool, else refill from the spill ring
        if (!is_idle) { if (l == 0) atomicAdd(BQ.idle(), 1u); is_idle = true; }
        if (bq_pop(BQ, m.rec())) {   // takes over the record's unit of work
            wake();
            load_record<NW>(m.rec(), Wt, &t, false);
            have = true;
            counted = true;
            if (l == 0) atomicAdd(&sp.ctr->holders, 1u);
            idle = 0;
            __syncwarp();
            continue;
        }
        {
            int which = 0;   // 1: main pool, 2: spill ring
            if (l == 0) {
                which = pool_size(sp) > 0 ? 1 : (spill_size(sp) > 0 ? 2 : 0);
                if (which && atomicCAS(BQ.poller(), 0, 1) != 0) which = 0;   // another warp of the block polls
            }
            which = __shfl_sync(FULL, which, 0);
            if (which) {
                const bool got = which == 1 ? pool_pop(sp, m.rec()) : ring_pop(sp, spill_ring(sp), m.rec());
                if (l == 0) atomicExch(BQ.poller(), 0);
                if (got) {
                    wake();
                    if (which == 2 && l == 0) ++CT[CT_REFILL];
                    load_record<NW>(m.rec(), Wt, &t, false);
                    have = true;
                    counted = true;
                    if (l == 0) atomicAdd(&sp.ctr->holders, 1u);
                    idle = 0;
                    __syncwarp();
                    continue;
                }
                __syncwarp();
            }
        }
        // ---------------- idle: exit when nothing is left anywhere
        const long long i0 = clock64();
        int done = 0, others_busy = 0;
        if (l == 0) {
            __threadfence();
            // one counter covers every place work can be (a unit moves, never
            // vanishes, when a record is taken), so zero means finished
            done = *(volatile unsigned*)&sp.ctr->work == 0u;   // a coherent load, not an atomic
            const unsigned live = *(volatile unsigned*)&sp.ctr->ks_active;
            others_busy = *(volatile unsigned*)&sp.ctr->holders > 0 || live > 0;
        }
        done = __shfl_sync(FULL, done, 0);
        others_busy = __shfl_sync(FULL, others_busy, 0);
        if (done && !ks_active) break;
        // waiting while other warps hold work or run k-search ends when they finish
        // (their loops are bounded); the limit counts waits with nobody working
        if (!others_busy || ks_active) ++idle;
        if (idle > sp.spin_limit) {
            if (l == 0) atomicAdd(&sp.ctr->timeouts, 1u);
            if (!ks_active) break;
            paused = false;   // a producer never waits unboundedly for the pool to drain
            idle = 0;
        }
        ++spins;
        __nanosleep(spins < 32 ? 128 : (spins < 512 ? 512 : 2048));
        if (l == 0) CT[CT_IDLE_CYC] += (unsigned long long)(clock64() - i0);
    }
    wake();
    if (l == 0) {
        if (ww.cnt() || ww.hsum()) { atomicAdd(&sp.gcount[acc_graph], ww.cnt()); atomicAdd(&sp.ghash[acc_graph], ww.hsum()); }
        atomicAdd(&sp.ctr->count, CT[CT_TOT_CNT] + ww.cnt());
        atomicAdd(&sp.ctr->hash, CT[CT_TOT_HSUM] + ww.hsum());
        atomicAdd(&sp.ctr->tasks, ww.tasks() + CT[CT_KS_TASKS]);
        atomicAdd(&sp.ctr->ks_tasks, CT[CT_KS_TASKS]);
        atomicAdd(&sp.ctr->nodes, ww.nodes());
        atomicAdd(&sp.ctr->bnb_bytes, ww.bb());
        atomicAdd(&sp.ctr->bnb_done, 1u);
        atomicAdd(&sp.ctr->stage_copies, CT[CT_STAGE]);
        atomicAdd(&sp.ctr->ks_cycles, CT[CT_KS_CYC]);
        atomicAdd(&sp.ctr->spilled, CT[CT_SPILL]);
        atomicAdd(&sp.ctr->refilled, CT[CT_REFILL]);
        atomicAdd(&sp.ctr->bnb_cycles, CT[CT_BNB_CYC]);
        atomicAdd(&sp.ctr->idle_cycles, CT[CT_IDLE_CYC]);
    }
}

// One body, compiled per bitset width (NW words per lane) and register budget:
// MINB blocks of SEARCH_WARPS = 9 warps per SM (2: up to 112 registers, no
// spills, 18 warps per SM; 3: 72, with spills).  Measured on soc-epinions:
// 2 x 9 warps 510 ms, 2 x 8 533 ms, 2 x 10 (96 registers) 519 ms, 3 x 7 563 ms,
// 3 x 6 572 ms.  Roots above 1024 vertices need NW = 2, built for 2 blocks only.
template <int NW, int MINB>
__global__ void __launch_bounds__(32 * SEARCH_WARPS, MINB) search_kernel(SearchParams sp, uint32_t nmax) { search_body<NW>(sp, nmax); }

SearchKernel search_kernel_for(uint32_t nw, int minb) {
    if (nw > 1) return search_kernel<2, 2>;
    return minb == 3 ? search_kernel<1, 3> : search_kernel<1, 2>;
}

uint32_t search_words_per_lane(uint32_t max_w) { return max_w > 32 ? 2u : 1u; }
uint32_t bnb_smem_words_host(uint32_t nmax, uint32_t slot_words, uint32_t a_words, uint32_t nw) {
    return bnb_smem_words(nmax, slot_words, a_words, 32 * nw);
}
uint32_t ks_slot_words_host(uint32_t nmax, uint32_t slot_words, uint32_t nw) {
    return ks_layout(nmax, nw).total + bq_words(slot_words);
}

}  // namespace kplex
