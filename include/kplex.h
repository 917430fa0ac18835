/* kplex.h — C ABI of libkplex.so, the B200 (sm_100a) maximal k-plex enumerator.
 *
 * The reference (CudaPlex) has no library API: its drop-in surface is the CLI
 * `./main <graph> -k K -q Q -t T -tr {0,1}` (main.cu:11-55), the .bin graph
 * format (inc/graph.h:45-62) and the internal entry
 * `void decomposableSearch(const graph<int>&)` (inc/host_funcs.h:722), which
 * reads the globals k, lb(=q), thres, truss, bd(=q-k) (inc/kPlexEnum.h:20-24).
 * Every entry point below names the reference interface it replaces.
 *
 * Conventions: plain pointers and sizes only; buffers are owned by the caller;
 * every function returns a status (KPLEX_OK = 0) instead of exiting (the
 * reference calls exit() on CUDA and IO errors, gpu_memory_allocation.h:1-8,
 * utils.h:24-33).  Calls are thread-compatible: one call at a time per CUDA
 * device; device memory is cached inside the library between calls.
 */
#ifndef KPLEX_H
#define KPLEX_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define KPLEX_OK             0
#define KPLEX_ERR_PARAM      1  /* unsupported k/q/t combination or bad argument */
#define KPLEX_ERR_IO         2  /* file cannot be opened/written */
#define KPLEX_ERR_FORMAT     3  /* .bin inconsistent with its header, unsorted lists, ids >= n */
#define KPLEX_ERR_CUDA       4  /* a CUDA runtime call failed */
#define KPLEX_ERR_NOMEM      5  /* device or host allocation failed / budget too small */
#define KPLEX_ERR_CAPACITY   6  /* a root's 2-hop subgraph exceeds 1024 vertices (the reference's
                                   MAX_BLK_SIZE, inc/common.h:8) or its left set 8192 */
#define KPLEX_ERR_TIMEOUT    7  /* a bounded device-side wait gave up */
#define KPLEX_ERR_NO_DEVICE  8  /* no CUDA device / extension not usable */
#define KPLEX_ERR_INTERNAL   9  /* device-side consistency check failed */

/* kplex_params.flags */
#define KPLEX_FLAG_QUIET        0x1u  /* no stdout lines from the library */
#define KPLEX_FLAG_NO_HASH      0x2u  /* skip the per-output hash (count only) */
#define KPLEX_FLAG_SPILL_HOST   0x4u  /* when the device task pool reaches thres * pool_slots, k-search writes
                                         further tasks to pinned host memory (up to 4x the pool) instead of
                                         pausing, and idle warps refill from there (the reference declares
                                         spillToHost/reFillTasks, host:168-251, but never calls them) */
#define KPLEX_FLAG_TEST_NO_WAIT 0x8u  /* test hook: branch warps give up every bounded wait at once, so the
                                         run must end with KPLEX_ERR_TIMEOUT instead of hanging */
#define KPLEX_FLAG_SHARD_WEIGHTED 0x10u /* with shard_count > 1: this call searches the roots that
                                         kplex_partition_roots assigns to shard_index (cost-weighted)
                                         instead of r % shard_count == shard_index */

/* Run parameters: the reference's CLI flags (main.cu:31-53) plus device knobs. */
typedef struct {
    int k;                  /* -k : each vertex may miss at most k-1 others (k >= 2) */
    int q;                  /* -q : minimum size of a reported k-plex (lb) */
    float thres;            /* -t : pause-and-resume threshold, fraction of the task pool (0,1] */
    int truss;              /* -tr: 1 = (q-2k)-truss pruning before the degeneracy order */
    uint32_t flags;         /* KPLEX_FLAG_* */
    int device;             /* CUDA device ordinal */
    uint64_t pool_slots;    /* task-pool capacity in records (0 = default 4,194,304, the reference's MAX_CAP) */
    uint32_t omp_threads;   /* host threads for preprocessing (0 = all) */
    uint32_t shard_index;   /* multi-GPU root sharding: this call searches the roots whose */
    uint32_t shard_count;   /* degeneracy rank r has r % shard_count == shard_index (0/0 = all) */
    uint32_t blocks_per_sm; /* persistent search kernel: 9-warp blocks per SM, 2 or 3 (0 = 2) */
    int32_t stage_after;    /* branch nodes a warp processes on one root before it copies the root's
                               adjacency matrix to shared memory (0 = 8, < 0 = never) */
    uint32_t root_begin;    /* search only the roots of degeneracy rank r in [root_begin, root_end) */
    uint32_t root_end;      /* (0/0 = all; combined with the shard rule above; a bounded, stated
                               subset of a graph too large to enumerate whole) */
} kplex_params;

/* Results.  count/hash are the parity outputs; the rest mirrors the
 * reference's printed lines (inc/host_funcs.h:1149-1157) and adds timings. */
typedef struct {
    uint64_t count;         /* number of maximal k-plexes of size >= q */
    uint64_t hash;          /* order-independent 64-bit hash of the sorted vertex sets (original ids) */
    uint64_t valid_roots;   /* "Total Valid Blocks" */
    uint64_t tasks;         /* "Total tasks generated": kSearch tasks + branch children */
    uint64_t nodes;         /* branch-and-bound nodes processed on the device */
    uint32_t pn, pm;        /* vertices / directed edges after (q-k)-core (and truss) pruning */
    uint32_t max_local_n;   /* largest root subgraph |{root} u C1 u C2| */
    uint32_t max_left;      /* largest root left set */
    uint32_t pauses;        /* kSearch pause/resume cycles */
    uint32_t spilled;       /* task records written to pinned host memory (KPLEX_FLAG_SPILL_HOST) */
    double ms_preprocess;   /* host core/truss/degeneracy */
    double ms_device;       /* device search: decomposition + k-search + branch-and-bound */
    double ms_ref_region;   /* preprocess + device search: the reference's "Total Time Elapsed" region */
    double ms_total;        /* whole call, including uploads and allocation */
    int status;
    uint32_t gpu_launches;  /* kernels launched by this call */
    double ms_decompose;    /* device time of the decomposition kernel */
    double ms_ksearch;      /* device time of the k-search launches */
    double ms_bnb;          /* device time of the branch-and-bound launches */
    uint64_t bnb_bytes;     /* algorithmic bytes of branch-and-bound: 12W per node and per child
                               record (P, C, X bitsets of W words) + 4W per adjacency row read */
    uint64_t roots_bytes;   /* algorithmic bytes of decomposition: CSR words read + bit matrices written */
    uint64_t ks_tasks;      /* tasks emitted by k-search (the rest of `tasks` are branch children) */
    uint64_t stage_copies;  /* root adjacency matrices copied into shared memory */
    double ks_warp_ms;      /* k-search time summed over producer warps (diagnostic) */
    double bnb_warp_ms;     /* branch-and-bound time summed over warps (diagnostic) */
    double idle_warp_ms;    /* time warps spent finding no work, summed (diagnostic) */
    uint32_t search_warps;  /* warps of the persistent search kernel */
} kplex_result;

/* A CSR graph owned by the library (kplex_load_bin / kplex_generate). */
typedef struct {
    uint32_t n;
    uint64_t m_directed;    /* = offsets[n] = 2|E| */
    uint32_t* offsets;      /* n + 1 */
    uint32_t* neighbors;    /* m_directed, each list strictly ascending */
} kplex_graph;

/* Seeded synthetic workload: Chung-Lu base graph with an exact edge count
 * plus planted dense groups (project-defined; replaces the reference's
 * shipped datasets when those are not available). */
typedef struct {
    uint64_t seed;
    uint32_t n;
    uint64_t base_edges;
    double exponent;
    uint32_t max_degree;
    uint32_t groups, group_min, group_max;
    double density_min, density_max;
} kplex_gen_spec;

/* Replaces graph<intT>::graph(path) (inc/graph.h:37-65). Caller frees with kplex_free_graph. */
int kplex_load_bin(const char* path, kplex_graph* out);
/* Inverse of kplex_load_bin; the layout of writeBinaryGraph (inc/graphIO.h:13-27). */
int kplex_save_bin(const char* path, const kplex_graph* g);
/* Replaces graph<intT>::del() (inc/graph.h:78-87). */
void kplex_free_graph(kplex_graph* g);
/* Project-written generator (no reference counterpart). */
int kplex_generate(const kplex_gen_spec* spec, kplex_graph* out);

/* Replaces decomposableSearch(g) (inc/host_funcs.h:722-1161) with the globals
 * k/lb/thres/truss passed in `p`.  Inputs are host CSR arrays owned by the
 * caller.  Runs the host preprocessing (core, truss, degeneracy) and the
 * device search on p->device; fills *out and returns out->status. */
int kplex_enumerate_csr(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n,
                        uint64_t m_directed, const kplex_params* p, kplex_result* out);

/* Replaces main.cu:56-61 (load + decomposableSearch) for a .bin path. */
int kplex_enumerate_file(const char* path, const kplex_params* p, kplex_result* out);

/* Two-stage form used to time the device search alone: kplex_prepare runs the
 * host preprocessing and uploads the pruned graph (handle returned in *h);
 * kplex_search runs decomposition + k-search + branch-and-bound on it and may
 * be called repeatedly; kplex_release frees the handle.  No reference
 * counterpart (the reference fuses these in decomposableSearch). */
typedef struct kplex_prepared kplex_prepared;
int kplex_prepare(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n,
                  uint64_t m_directed, const kplex_params* p, kplex_prepared** h, kplex_result* out);
int kplex_search(kplex_prepared* h, kplex_result* out);
void kplex_release(kplex_prepared* h);

/* Host preprocessing only (no device): (q-k)-core (inc/host_funcs.h:16-122),
 * optional (q-2k)-truss (inc/host_funcs.h:761-823, 463-559) and the degeneracy
 * order (inc/degeneracy.h + inc/host_funcs.h:829-851).  Output buffers are
 * caller-owned and sized n+1 (out_off), m_directed (out_adj) and n (the rest).
 * Returns the pruned vertex count pn (>= 0) or -status. */
long long kplex_preprocess_csr(const uint32_t* offsets, const uint32_t* neighbors, uint32_t n, uint64_t m_directed,
                               int k, int q, int truss, uint32_t omp_threads,
                               uint32_t* out_off, uint32_t* out_adj, int32_t* out_dpos, int32_t* out_dseq,
                               uint32_t* out_orig, uint64_t* out_m);

/* No reference counterpart: added for callers that cannot allocate device memory
 * (device memory fully reserved by another allocator, a fixed memory plan with
 * no allocation on the request path, or no tolerance for the synchronisation
 * an allocation can cause).  Runs decomposition + k-search + branch-and-bound
 * with every scratch buffer carved from one 64 MiB __device__ array inside the
 * library; calls no cudaMalloc/cudaFree.  Inputs are the pruned graph from
 * kplex_preprocess_csr in caller-owned device buffers (offsets, neighbors,
 * dpos, dseq, pruned->input ids, pn vertices); the result goes to *out.
 * Graphs whose scratch exceeds 64 MiB are rejected with KPLEX_ERR_NOMEM.  The
 * first call on a device looks up the array's device address (make it before
 * any stream capture); calls share the array, so calls that overlap on one
 * GPU race.  The inputs must be complete when the call starts (it runs on
 * cudaStreamPerThread); p->device is made current during the call and the
 * caller's device is restored.  ms_device is not measured (0). */
int kplex_search_noalloc(const uint32_t* d_offsets, const uint32_t* d_neighbors, const int32_t* d_dpos,
                         const int32_t* d_dseq, const uint32_t* d_orig, uint32_t pn,
                         const kplex_params* p, kplex_result* out);

/* Batched enumeration (no reference counterpart; the reference handles one
 * graph per process).  Each job is an independent graph with its own k, q and
 * truss setting; thres, flags, device and pool size come from `common`.  All
 * jobs' roots are decomposed and searched together in one persistent launch,
 * and per_job[i] receives job i's count, hash, valid roots, pn and pm
 * (per_job may be NULL); *total receives the sums and timings.  Results are
 * identical to separate kplex_enumerate_csr calls. */
typedef struct {
    const uint32_t* offsets;
    const uint32_t* neighbors;
    uint32_t n;
    uint64_t m_directed;
    int k, q, truss;
} kplex_job;
int kplex_enumerate_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common,
                          kplex_result* per_job, kplex_result* total);
/* Two-stage batch: preprocess and upload once, then search (repeatable). */
int kplex_prepare_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common,
                        kplex_prepared** h, kplex_result* total);
int kplex_search_batch(kplex_prepared* h, kplex_result* per_job, kplex_result* total);

/* Request server (no reference counterpart; the reference runs one graph per
 * process).  Requests (one graph with its own k, q, truss) are submitted as
 * they arrive and complete asynchronously.  `slots` worker threads each own a
 * CUDA stream and a device workspace (arena, task pool, branch stacks, spill
 * ring); a free slot admits every waiting request that fits the device-memory
 * budget (up to max_batch) and enumerates them as one batched launch, so
 * requests arriving while others run join the next launch and launches of
 * different slots overlap on the device.  A request's result is the same as
 * kplex_enumerate_csr's on its graph. */
typedef struct kplex_server kplex_server;
typedef struct {
    int device;
    uint32_t slots;          /* concurrent launches (streams), 0 -> 2 */
    uint32_t max_batch;      /* requests per launch, 0 -> 1024 */
    uint64_t mem_budget;     /* device bytes for workspaces + admitted requests (spill ring
                                included), 0 -> 16 GiB */
    uint32_t split_grid;     /* 1: each launch gets 1/slots of the SMs; 0: the whole device */
    float thres;             /* pause threshold, as kplex_params.thres (0 -> 0.25) */
    uint32_t flags;          /* KPLEX_FLAG_* applied to every launch */
    uint64_t pool_slots;     /* as kplex_params.pool_slots */
    uint64_t large_bytes;    /* a request whose device estimate reaches this runs in a launch of its own,
                                so small requests never wait inside a launch for a large one
                                (0 -> 32 MiB, UINT64_MAX -> never) */
} kplex_server_config;

typedef struct {
    uint64_t tag;            /* the submitter's request id */
    int status;
    uint32_t batch_size;     /* requests in the launch that served it */
    uint64_t count, hash;
    uint64_t valid_roots;
    uint32_t pn, slot;
    double ms_queue;         /* submit -> launch start (admission wait) */
    double ms_service;       /* launch start -> results on the host (preprocess, upload, search) */
    double ms_latency;       /* submit -> completion */
} kplex_completion;

typedef struct {
    uint64_t submitted, completed, rejected, launches;
    uint64_t device_bytes;        /* workspaces + in-flight requests now */
    uint64_t peak_device_bytes;
    uint32_t max_concurrent;      /* most launches in flight at once */
    uint32_t max_batch_seen;
} kplex_server_stats;

int kplex_server_create(const kplex_server_config* cfg, kplex_server** out);
/* Copies the job's CSR; returns KPLEX_OK, or KPLEX_ERR_PARAM / KPLEX_ERR_NOMEM (the
 * request alone exceeds the budget) without queueing it. */
int kplex_server_submit(kplex_server* s, const kplex_job* job, uint64_t tag);
/* Moves up to `max` completions into out; waits up to timeout_ms (-1: until one
 * arrives or nothing is pending) for the first.  Returns the number moved. */
int kplex_server_poll(kplex_server* s, kplex_completion* out, uint32_t max, int timeout_ms);
/* Waits until every submitted request has completed; KPLEX_ERR_TIMEOUT after timeout_ms (-1: no limit). */
int kplex_server_drain(kplex_server* s, int timeout_ms);
int kplex_server_stats_get(kplex_server* s, kplex_server_stats* out);
/* Finishes queued requests, joins the workers and frees the workspaces. */
void kplex_server_destroy(kplex_server* s);

/* Autotuner for batched runs (no reference counterpart): enumerates a
 * deterministic sample of `sample` jobs (every njobs/sample-th) under each
 * candidate schedule (blocks per SM, shared-memory staging point, task-pool
 * capacity, pause threshold), keeps the fastest by device time, and writes it
 * to *best (= *common with the tuned fields replaced).  The sample's counts
 * must agree across candidates, or KPLEX_ERR_INTERNAL is returned.
 * *best_ms receives the winner's device time on the sample. */
int kplex_autotune_batch(const kplex_job* jobs, uint32_t njobs, const kplex_params* common, uint32_t sample,
                         kplex_params* best, double* best_ms);

/* Cost-weighted partition of the roots over `shards` processes (no reference
 * counterpart; the reference runs on one GPU).  Input: the pruned graph and
 * degeneracy order from kplex_preprocess_csr.  owner_out[r] (one byte per root
 * rank r < pn - q + 2) receives the shard that searches root r: roots are taken
 * largest estimated cost first ((later neighbours + 1)^2) and given to the least
 * loaded shard, so every process computes the same assignment.  Returns the
 * number of roots, or -status.  KPLEX_FLAG_SHARD_WEIGHTED makes a search use it. */
long long kplex_partition_roots(const uint32_t* offsets, const uint32_t* neighbors, const int32_t* dpos,
                                const int32_t* dseq, uint32_t pn, int q, uint32_t shards, uint8_t* owner_out);

const char* kplex_status_string(int status);
/* Text of the last failure on the calling thread (CUDA message, parse error, ...). */
const char* kplex_last_error(void);
int kplex_version(void);
/* 1 if a CUDA device is visible and the sm_100a kernels can run on it. */
int kplex_device_ok(int device);

#ifdef __cplusplus
}
#endif
#endif /* KPLEX_H */
