#pragma once
#include "kplex_common.h"
#include "../../include/kplex.h"

namespace kplex {
int load_bin(const char* path, Csr& g, std::string* err);
int save_bin(const char* path, const Csr& g, std::string* err);
int validate_csr(const Csr& g, std::string* err);

// Seeded synthetic workload (Chung-Lu base graph plus planted dense groups).
struct GenSpec {
    uint64_t seed = 1;
    uint32_t n = 0;
    uint64_t base_edges = 0;   // exact number of undirected Chung-Lu edges
    double exponent = 2.5;     // power-law exponent of the expected degrees
    uint32_t max_degree = 0;   // hard cap on base-graph degree (0: n-1)
    uint32_t groups = 0;       // planted groups
    uint32_t group_min = 0, group_max = 0;  // group size uniform in [min, max]
    double density_min = 1.0, density_max = 1.0;  // internal density uniform in range
};
int generate(const GenSpec& s, Csr& out, std::string* err);
}  // namespace kplex
