// Warp-level building blocks: reductions, scans, bitset <-> list conversion and
// the task pool (a bounded multi-producer multi-consumer ring whose slots carry
// sequence numbers, after D. Vyukov's published bounded MPMC queue).
#pragma once
#include "device.cuh"

namespace kplex {

constexpr unsigned FULL = 0xffffffffu;

// Warp reductions in one instruction each (the sm_80+ redux.sync unit); warp_sum
// is used for counts, which are never negative.
__device__ __forceinline__ int warp_sum(int v) { return (int)__reduce_add_sync(FULL, (unsigned)v); }
__device__ __forceinline__ unsigned warp_min(unsigned v) { return __reduce_min_sync(FULL, v); }
__device__ __forceinline__ unsigned warp_or(unsigned v) { return __reduce_or_sync(FULL, v); }
// exclusive prefix sum across the warp; *total receives the sum
__device__ __forceinline__ int warp_excl_scan(int v, int* total) {
    const unsigned l = lane_id();
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if ((int)l >= o) x += y;
    }
    *total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// Lane l holds word l of a 32-word group of a bitset whose first bit is
// `base` (0 beyond its length).  Writes the set bits' indices in ascending
// order to list[0..) and returns their count.
__device__ __forceinline__ int bits_to_list(unsigned w, uint16_t* list, unsigned base = 0) {
    // words are visited in order (only the non-zero ones); within a word every
    // lane tests one bit, so all 32 lanes stay active however dense the word is
    const unsigned l = lane_id();
    unsigned nz = __ballot_sync(FULL, w != 0u);
    int off = 0;
    while (nz) {
        const int j = __ffs(nz) - 1;
        nz &= nz - 1;
        const unsigned word = __shfl_sync(FULL, w, j);
        if ((word >> l) & 1u) list[off + __popc(word & ((1u << l) - 1u))] = (uint16_t)(base + j * 32 + l);
        off += __popc(word);
    }
    __syncwarp();
    return off;
}

__device__ __forceinline__ bool test_bit(const uint32_t* bits, unsigned v) { return (bits[v >> 5] >> (v & 31)) & 1u; }

// popcount of (row & mask) over W words (W a multiple of 4, row 16-byte aligned)
__device__ __forceinline__ int row_and_popc(const uint32_t* __restrict__ row, const uint32_t* mask, unsigned W) {
    int c = 0;
    const uint4* r4 = reinterpret_cast<const uint4*>(row);
    const uint4* m4 = reinterpret_cast<const uint4*>(mask);
#pragma unroll 1
    for (unsigned w = 0; w < W / 4; ++w) {
        const uint4 a = __ldg(r4 + w), m = m4[w];
        c += __popc(a.x & m.x) + __popc(a.y & m.y) + __popc(a.z & m.z) + __popc(a.w & m.w);
    }
    return c;
}

// ---------------------------------------------------------------- task pool
// A ring is a control block (head, tail, cap) and one sequence word per slot in
// device memory, plus the record data.  cap is a power of two (a position's slot
// is the position masked).  The data of the main pool is in HBM;
// the spill ring keeps its data in mapped pinned host memory, so only plain
// loads and stores cross the bus (no GPU atomics on host memory) and a
// system-scope fence orders them before the sequence word is published.
struct Ring {
    Pool* ctl;
    uint32_t* seq;
    uint32_t* data;
    int sys;   // data lives in host memory
};

__device__ __forceinline__ Ring main_ring(const SearchParams& sp) { return Ring{sp.pool, sp.pool_seq, sp.pool_data, 0}; }
__device__ __forceinline__ Ring spill_ring(const SearchParams& sp) { return Ring{sp.spill_pool, sp.spill_seq, sp.spill_data, 1}; }

// Word i of a record: from global memory at L2 (it may have been written by
// another SM) or from shared memory.
__device__ __forceinline__ uint32_t rec_word(const uint32_t* src, int src_global, unsigned i) {
    return src_global ? __ldcg(src + i) : src[i];
}

// Enqueue one record of slot_words words copied from src.  Returns false when
// the ring is full or the bounded retry loop gives up; the caller keeps the
// record.
static __device__ __forceinline__ bool ring_push(Ring r, uint32_t slot_words, unsigned long long spin_limit, uint32_t test_stuck,
                                       Counters* ctr, const uint32_t* src, int src_global) {
    Pool* pool = r.ctl;
    const unsigned l = lane_id();
    unsigned long long pos = 0;
    int ok = 0;
    if (l == 0) {
        const unsigned long long cap = pool->cap;
        for (unsigned long long it = 0; it < spin_limit; ++it) {
            pos = atomicAdd(&pool->tail, 0ull);
            const uint32_t seq = atomicAdd(&r.seq[pos & (cap - 1)], 0u);
            const int dif = (int)(seq - (uint32_t)pos);
            if (dif == 0) {
                if (atomicCAS(&pool->tail, pos, pos + 1) == pos) { ok = 1; break; }
            } else if (dif < 0) {
                break;   // full
            }
        }
    }
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) return false;
    pos = __shfl_sync(FULL, pos, 0);
    if (test_stuck) {   // failure-detection test: claim the slot but never publish it
        int stuck = 0;
        if (l == 0) stuck = atomicCAS(&ctr->stuck_once, 0u, 1u) == 0u;
        if (__shfl_sync(FULL, stuck, 0)) return true;
    }
    const unsigned long long slot = pos & (pool->cap - 1);
    uint32_t* dst = r.data + slot * slot_words;
    for (unsigned i = l; i < slot_words; i += 32) __stcg(dst + i, rec_word(src, src_global, i));
    if (r.sys) __threadfence_system(); else __threadfence();
    __syncwarp();
    if (l == 0) atomicExch(&r.seq[slot], (uint32_t)(pos + 1));
    return true;
}

// Dequeue one record into dst (slot_words words).  Returns false if the ring
// looks empty (a record still being published counts as empty).
static __device__ __forceinline__ bool ring_pop(Ring r, uint32_t slot_words, unsigned long long spin_limit, uint32_t* dst) {
    Pool* pool = r.ctl;
    const unsigned l = lane_id();
    unsigned long long pos = 0;
    int ok = 0;
    if (l == 0) {
        const unsigned long long cap = pool->cap;
        for (unsigned long long it = 0; it < spin_limit; ++it) {
            pos = atomicAdd(&pool->head, 0ull);
            const uint32_t seq = atomicAdd(&r.seq[pos & (cap - 1)], 0u);
            const int dif = (int)(seq - (uint32_t)(pos + 1));
            if (dif == 0) {
                if (atomicCAS(&pool->head, pos, pos + 1) == pos) { ok = 1; break; }
            } else if (dif < 0) {
                break;   // empty
            }
        }
    }
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) return false;
    pos = __shfl_sync(FULL, pos, 0);
    const unsigned long long cap = pool->cap;
    const unsigned long long slot = pos & (cap - 1);
    __threadfence();
    const uint32_t* src = r.data + slot * slot_words;
    for (unsigned i = l; i < slot_words; i += 32) dst[i] = __ldcg(src + i);
    __threadfence();
    __syncwarp();
    if (l == 0) atomicExch(&r.seq[slot], (uint32_t)(pos + cap));
    return true;
}

__device__ __forceinline__ unsigned long long ring_size(const Ring& r) {
    const unsigned long long t = *(volatile unsigned long long*)&r.ctl->tail;
    const unsigned long long h = *(volatile unsigned long long*)&r.ctl->head;
    return t > h ? t - h : 0ull;
}

__device__ __forceinline__ bool ring_push(const SearchParams& sp, const Ring& r, const uint32_t* src, int src_global) {
    return ring_push(r, sp.slot_words, sp.spin_limit, sp.test_stuck, sp.ctr, src, src_global);
}
__device__ __forceinline__ bool ring_pop(const SearchParams& sp, const Ring& r, uint32_t* dst) {
    return ring_pop(r, sp.slot_words, sp.spin_limit, dst);
}
__device__ __forceinline__ bool pool_push(const SearchParams& sp, const uint32_t* src, int src_global) {
    return ring_push(sp, main_ring(sp), src, src_global);
}
__device__ __forceinline__ bool pool_pop(const SearchParams& sp, uint32_t* dst) { return ring_pop(sp, main_ring(sp), dst); }
__device__ __forceinline__ unsigned long long pool_size(const SearchParams& sp) { return ring_size(main_ring(sp)); }
__device__ __forceinline__ unsigned long long spill_size(const SearchParams& sp) { return sp.spill_on ? ring_size(spill_ring(sp)) : 0ull; }

// pool_size read once by lane 0 and broadcast, so every lane takes the same branch
__device__ __forceinline__ unsigned long long pool_size_warp(const SearchParams& sp) {
    unsigned long long v = 0;
    if (lane_id() == 0) v = pool_size(sp);
    return __shfl_sync(FULL, v, 0);
}

}  // namespace kplex
