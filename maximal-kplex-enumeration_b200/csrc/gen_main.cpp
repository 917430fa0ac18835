// kplex_gen: write a seeded synthetic workload as a .bin graph.
// Named workloads reproduce the benchmark inputs; every field can be overridden.
#include "graph_io.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

using namespace kplex;

static bool preset(const char* name, GenSpec& s) {
    if (!strcmp(name, "small")) {          // Chung-Lu n=2,000, mean degree 10, gamma 2.5, 20 groups of 16 at 0.9
        s = GenSpec{}; s.seed = 1; s.n = 2000; s.base_edges = 10000; s.exponent = 2.5; s.max_degree = 0;
        s.groups = 20; s.group_min = 16; s.group_max = 16; s.density_min = s.density_max = 0.9; return true;
    }
    if (!strcmp(name, "epinions")) {       // n=75,879, 405,740 edges, gamma 2.1, cap 3,044, 200 groups U[40,80] at 0.9
        s = GenSpec{}; s.seed = 2; s.n = 75879; s.base_edges = 405740; s.exponent = 2.1; s.max_degree = 3044;
        s.groups = 200; s.group_min = 40; s.group_max = 80; s.density_min = s.density_max = 0.9; return true;
    }
    if (!strcmp(name, "email")) {          // n=265,214, 364,481 edges, gamma 1.8, cap 7,636, 50 groups U[15,25] at 0.85
        s = GenSpec{}; s.seed = 3; s.n = 265214; s.base_edges = 364481; s.exponent = 1.8; s.max_degree = 7636;
        s.groups = 50; s.group_min = 15; s.group_max = 25; s.density_min = s.density_max = 0.85; return true;
    }
    return false;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <out.bin> <small|epinions|email|custom> [-seed S] [-n N] [-m M] [-exp G] [-cap D] "
                        "[-groups G] [-gmin A] [-gmax B] [-dmin X] [-dmax Y]\n", argv[0]);
        return 1;
    }
    GenSpec s;
    if (!preset(argv[2], s) && strcmp(argv[2], "custom")) { fprintf(stderr, "unknown workload %s\n", argv[2]); return 1; }
    for (int i = 3; i + 1 < argc; i += 2) {
        const char* f = argv[i]; const char* v = argv[i + 1];
        if (!strcmp(f, "-seed")) s.seed = strtoull(v, 0, 10);
        else if (!strcmp(f, "-n")) s.n = (uint32_t)strtoul(v, 0, 10);
        else if (!strcmp(f, "-m")) s.base_edges = strtoull(v, 0, 10);
        else if (!strcmp(f, "-exp")) s.exponent = atof(v);
        else if (!strcmp(f, "-cap")) s.max_degree = (uint32_t)strtoul(v, 0, 10);
        else if (!strcmp(f, "-groups")) s.groups = (uint32_t)strtoul(v, 0, 10);
        else if (!strcmp(f, "-gmin")) s.group_min = (uint32_t)strtoul(v, 0, 10);
        else if (!strcmp(f, "-gmax")) s.group_max = (uint32_t)strtoul(v, 0, 10);
        else if (!strcmp(f, "-dmin")) s.density_min = atof(v);
        else if (!strcmp(f, "-dmax")) s.density_max = atof(v);
        else { fprintf(stderr, "unknown flag %s\n", f); return 1; }
    }
    Csr g; std::string err;
    int rc = generate(s, g, &err);
    if (rc) { fprintf(stderr, "generate: %s\n", err.c_str()); return rc; }
    rc = save_bin(argv[1], g, &err);
    if (rc) { fprintf(stderr, "save: %s\n", err.c_str()); return rc; }
    uint32_t maxd = 0; for (uint32_t v = 0; v < g.n; ++v) maxd = std::max(maxd, g.deg(v));
    printf("wrote %s: n=%u m_directed=%llu max_degree=%u\n", argv[1], g.n, (unsigned long long)g.m_directed(), maxd);
    return 0;
}
