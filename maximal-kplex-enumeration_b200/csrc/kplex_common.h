// Shared host-side definitions: CSR graph, the project's plex hash, and the
// seeded random streams used by the synthetic generator.
//
// The plex hash is defined by this project because the reference never
// materialises an output set (it only increments a counter at
// src/device_funcs.cu:1585 and :1716).  For one maximal k-plex S, written as
// its vertex ids in the ORIGINAL .bin numbering and sorted ascending:
//     x = splitmix64(KPLEX_HASH_SEED ^ |S|);  for v in S: x = splitmix64(x ^ v)
// and the run's hash is the wrapping 64-bit SUM of x over all outputs, so it
// does not depend on the order in which sets are found and a duplicated
// output changes it.
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <string>

#ifdef __CUDACC__
#define KPLEX_HD __host__ __device__ __forceinline__
#else
#define KPLEX_HD inline
#endif

namespace kplex {

constexpr uint64_t KPLEX_HASH_SEED = 0x6b706c6578b200ULL;

// SplitMix64 finaliser (Steele, Lea & Flood 2014; public-domain constants as
// published by S. Vigna).
KPLEX_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

KPLEX_HD uint64_t plex_hash_begin(uint32_t size) { return splitmix64(KPLEX_HASH_SEED ^ (uint64_t)size); }
KPLEX_HD uint64_t plex_hash_step(uint64_t x, uint32_t v) { return splitmix64(x ^ (uint64_t)v); }

// Undirected simple graph in CSR form: neighbour lists sorted ascending,
// every edge stored in both directions (the .bin layout of inc/graph.h:45-62).
struct Csr {
    uint32_t n = 0;
    std::vector<uint32_t> off;   // n + 1
    std::vector<uint32_t> adj;   // off[n] directed entries
    uint32_t deg(uint32_t v) const { return off[v + 1] - off[v]; }
    uint64_t m_directed() const { return off.empty() ? 0 : off[n]; }
};

// xoshiro256** (Blackman & Vigna 2018), seeded through splitmix64.
struct Xoshiro256 {
    uint64_t s[4];
    explicit Xoshiro256(uint64_t seed) {
        uint64_t z = seed;
        for (int i = 0; i < 4; ++i) { s[i] = splitmix64(z); z += 0x9e3779b97f4a7c15ULL; }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, bound) by Lemire's multiply-shift with rejection
    uint64_t below(uint64_t bound) {
        if (bound <= 1) return 0;
        for (;;) {
            unsigned __int128 m = (unsigned __int128)next() * bound;
            uint64_t lo = (uint64_t)m;
            if (lo >= bound || lo >= (uint64_t)(-bound) % bound) return (uint64_t)(m >> 64);
        }
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace kplex
