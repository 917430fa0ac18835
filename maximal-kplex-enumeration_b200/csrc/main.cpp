// kplex_main: drop-in for the reference CLI `./main <graph> -k K -q Q -t T -tr {0,1}`
// (main.cu:11-63).  Same usage text, argument handling, exit codes and stdout
// lines (main.cu:30,54; inc/host_funcs.h:1149-1157); two lines are appended:
// the 64-bit count and the order-independent plex hash.  `-dev D` selects a
// CUDA device (an addition; the reference has no such flag).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/kplex.h"

static void usage() { fprintf(stderr, "usage : ./PlexEnum <dataset> -k <k> -q <q> -t <thres> -tr <truss>\n"); }

// main.cu:16-21 tests i == max before incrementing, so a flag in last position
// reads argv[argc] (NULL) and aborts; here it is a usage error (exit 1).
static int check_inc(int i, int max) {
    if (i + 1 >= max) { usage(); exit(1); }
    return i + 1;
}

int main(int argc, char* argv[]) {
    int i = 2;
    if (argc < 6) { usage(); exit(1); }
    printf("file: %s\n", argv[1]);
    kplex_params p;
    memset(&p, 0, sizeof p);
    while (i < argc) {
        if (!strcmp(argv[i], "-k")) { i = check_inc(i, argc); p.k = atoi(argv[i]); }
        else if (!strcmp(argv[i], "-q")) { i = check_inc(i, argc); p.q = atoi(argv[i]); }
        else if (!strcmp(argv[i], "-t")) { i = check_inc(i, argc); p.thres = (float)std::stod(argv[i]); }
        else if (!strcmp(argv[i], "-tr")) { i = check_inc(i, argc); p.truss = atoi(argv[i]); }
        else if (!strcmp(argv[i], "-dev")) { i = check_inc(i, argc); p.device = atoi(argv[i]); }
        else { usage(); exit(1); }
        i++;
    }
    printf("k=%d,q=%d,thres=%f, truss: %d\n", p.k, p.q, p.thres, p.truss);
    fflush(stdout);
    kplex_result r;
    const int rc = kplex_enumerate_file(argv[1], &p, &r);
    if (rc != KPLEX_OK) {
        fprintf(stderr, "error %d (%s): %s\n", rc, kplex_status_string(rc), kplex_last_error());
        return rc;
    }
    printf("Maximal k-Plexes (64-bit): %llu\n", (unsigned long long)r.count);
    printf("Plex hash: 0x%016llx\n", (unsigned long long)r.hash);
    return 0;
}
