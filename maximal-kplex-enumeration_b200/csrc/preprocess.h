#pragma once
#include "kplex_common.h"

namespace kplex {
struct Prepped {
    Csr g;                       // pruned graph, ids renumbered in ascending order
    std::vector<int32_t> dpos;   // rank of each pruned vertex in the degeneracy order
    std::vector<int32_t> dseq;   // pruned vertex at each rank
    std::vector<uint32_t> orig;  // pruned id -> id in the input graph
};
int preprocess(const Csr& in, int k, int q, int truss, int threads, Prepped& out);
void weighted_root_owners(const Csr& g, const std::vector<int32_t>& dpos, const std::vector<int32_t>& dseq,
                          uint32_t nroots, uint32_t shards, uint8_t* owner);
}  // namespace kplex
