// Device-side layout shared by the decomposition, k-search and branch kernels.
//
// HBM layout (all per search, sized on the host):
//   roots[R]        RootDesc per root rank r < pn - q + 2 (inc: src/device_funcs.cu:44-45)
//   arena           u32 words; each valid root owns one contiguous block:
//                     A  [n][W]   adjacency bits of the root's local subgraph
//                     M2 [n][W]   pair class >= UNLINK2EQUAL (src:1751-1853, used by
//                                 updateCand13/23 and the include filter)
//                     M4 [n][W]   pair class >= UNLINK2MORE (the X filter, src:1396-1404)
//                     LA [n][WL]  adjacency from local vertices to the root's left set
//                     LT [nl][W]  the transpose of LA
//                     sorig [n]   original ids of the local vertices, ascending
//                     srank [n]   position of each local vertex in sorig (u32)
//   pool            bounded MPMC ring of task records (the reference's queue A;
//                   host:953-957) shared by the k-search and branch kernels
//   stacks          one depth-first stack of task records per branch warp
// A task record is TaskHdr followed by the P, C and X bitsets (Wt words each).
// Local vertex ids: 0 = root, [1, hop) = C1, [hop, n) = C2 (as in the reference).
#pragma once
#include <cstdint>
#include "kplex_common.h"
#include "../../include/kplex.h"

namespace kplex {

// The reference keeps at most MAX_BLK_SIZE = 1024 one-hop neighbours of a root
// (inc/common.h:8): 1023 later and 1024 earlier ones in CSR order, dropping the
// rest (src:87-131).  That truncation is part of its results and is kept.
constexpr int REF_BLK = 1024;
// A root's local subgraph (root, C1, C2) may hold up to MAX_LOCAL vertices.  The
// reference overruns its 1024-entry buffers beyond REF_BLK (src:255); here a
// warp keeps one bitset word per lane up to 1024 vertices and two beyond.
constexpr int MAX_LOCAL = 2048;
constexpr int MAX_WORDS = MAX_LOCAL / 32;
// The left set (earlier-ordered vertices that may extend an output) is only
// read by the maximality check, so it may be larger than the local subgraph;
// the reference's left buffers and its 1024-bit `uni` mask stop at 1024
// (src:117-121, 262, 706-841).
constexpr int MAX_LEFT = 8192;
constexpr int MAX_LEFT_WORDS = MAX_LEFT / 32;
// The reference's k-search stack holds 1000 frames (inc/common.h:15 MAX_DEPTH) and
// abandons the rest of a root when it would go deeper (src:1987-1991), losing
// results on roots with about 1000 or more C2 vertices.  A path pushes at most
// one frame per C2 vertex plus a leaf frame, so n + 8 frames (n = the root's
// local vertices) never fill and no root is abandoned here.
constexpr int KS_MAX_DEPTH = MAX_LOCAL + 8;
constexpr int MAX_K = 32;
// warps per block of the persistent search kernel: one k-search producer and
// SEARCH_WARPS - 1 branch-and-bound consumers
constexpr int SEARCH_WARPS = 9;

// root flags
enum : uint32_t {
    ROOT_VALID = 1u,       // |blk| >= q: counted in "Total Valid Blocks"
    ROOT_TRUNCATED = 2u,   // more than 1023 later or 1024 earlier neighbours (reference drops extras)
    ROOT_OVERSIZED = 4u,   // n beyond MAX_LOCAL or |left| beyond MAX_LEFT: the run fails
    ROOT_SKIPPED = 8u,     // C1 smaller than q-k after peeling (src:148)
};

struct RootDesc {
    uint32_t n, hop, nleft, W;   // W: words per local row, multiple of 4
    uint32_t WL, flags, gid, graph;
    uint64_t base;               // word offset of the root's block in the arena
    int32_t k, q;                // the parameters of the root's graph
};

// One input graph of a search (a single-graph search has one).  Vertices of
// graph g are [vbase, vbase + pn) in the concatenated pruned CSR; its roots are
// [root_base, root_base + nroots).
struct GraphInfo {
    uint32_t vbase, pn, root_base, nroots;
    int32_t k, q;
    uint32_t pad[2];
};

struct TaskHdr {
    uint32_t root;
    uint16_t np, nc;
    uint16_t nx, pad0;
    uint32_t pad1;
};
static_assert(sizeof(TaskHdr) == 16, "task header is one uint4");

// Global counters and flags, one per search.
struct Counters {
    unsigned long long count;      // maximal k-plexes found
    unsigned long long hash;       // wrapping sum of plex hashes
    unsigned long long tasks;      // kSearch tasks + branch children ("Total tasks generated")
    unsigned long long nodes;      // branch nodes processed
    unsigned long long bnb_bytes;  // algorithmic bytes of branch nodes (roofline accounting)
    unsigned long long arena_top;  // words bump-allocated in the arena
    unsigned int valid_roots;
    unsigned int max_n, max_left, max_w, max_nw;
    unsigned int truncated, oversized, depth_capped;
    unsigned int error;            // KPLEX_ERR_* raised on the device (first one wins)
    // the counters that many warps update during the search each start a line of
    // their own, so that atomics on one do not queue behind atomics on another
    alignas(128) unsigned int next_root;   // k-search job dispenser
    unsigned int ks_paused;        // k-search warps that stopped at the pause threshold
    unsigned int ks_active;        // k-search slots holding an unfinished root
    alignas(128) unsigned int holders;     // warps holding work now (the idle-wait heuristic)
    alignas(128) unsigned int work;            // outstanding work units: unclaimed k-search jobs, running jobs,
                                   // records in the pool / block queues / spill ring, warps holding work
    alignas(128) unsigned int bnb_done;    // branch warps that exited
    unsigned int timeouts;         // bounded waits that gave up
    unsigned int decomp_next;      // decomposition root dispenser
    unsigned int pad[2];
    unsigned long long roots_bytes; // algorithmic bytes of the decomposition
    unsigned long long ks_tasks;   // tasks emitted by k-search
    unsigned int stuck_once;       // test hook: one pool slot claimed and never published
    unsigned long long stage_copies;  // adjacency matrices copied to shared memory
    unsigned long long ks_cycles;  // SM cycles producers spent in k-search
    unsigned long long spilled;    // records written to the host spill ring
    unsigned long long refilled;   // records read back from it
    unsigned long long bnb_cycles;   // SM cycles warps spent in branch-and-bound nodes
    unsigned long long idle_cycles;  // SM cycles warps spent finding no work
};

// Vyukov bounded MPMC ring: each slot carries a sequence number so that a
// producer and a consumer never touch the same record concurrently.
// head, tail and the read-only capacity are on separate lines: takers hit the
// head with atomics, givers the tail.
struct Pool {
    alignas(128) unsigned long long head;   // next slot to dequeue
    alignas(128) unsigned long long tail;   // next slot to enqueue
    alignas(128) unsigned long long cap;    // slots
    unsigned long long pad;
};

struct SearchParams {
    uint32_t nroots;           // roots over all graphs
    uint32_t pn;               // largest pruned vertex count of any graph (scratch sizing)
    const uint32_t* off;       // pruned CSR
    const uint32_t* adj;
    const int32_t* dpos;
    const int32_t* dseq;
    const uint32_t* orig;      // pruned id -> input id
    RootDesc* roots;
    uint32_t* arena;
    unsigned long long arena_cap;  // words
    Counters* ctr;
    Pool* pool;
    uint32_t* pool_seq;        // per slot sequence (u64 position folded to 32 bits)
    uint32_t* pool_data;       // cap * slot_words
    uint32_t slot_words;       // 4 + 3 * Wt
    Pool* spill_pool;          // spill ring: control + sequence words in HBM,
    uint32_t* spill_seq;       // record data in mapped pinned host memory
    uint32_t* spill_data;
    uint32_t spill_on;
    unsigned long long spill_pause_at;   // producers pause when the spill ring holds this many
    uint32_t Wt;               // words per bitset in a task record
    unsigned long long pause_at;   // k-search pauses when the pool holds this many records
    uint32_t* warp_scratch;    // decomposition per-warp scratch
    uint64_t scratch_words;    // words per warp
    uint32_t* ks_slots;        // k-search per-warp state (KS_WORDS each), kept across pauses
    uint32_t* stacks;          // branch stacks: warps * stack_depth * slot_words
    uint32_t stack_depth;      // records per warp stack, a power of two
    uint32_t nwarps;           // branch warps launched
    uint32_t low_water;        // a branch warp donates work when the pool holds fewer records
    uint32_t hash_on;
    uint32_t shard_index, shard_count;
    uint32_t root_begin, root_end;   // roots of rank r outside [root_begin, root_end) are skipped
    const uint8_t* root_owner;       // cost-weighted shards: root r is searched iff root_owner[r] == shard_index
    uint32_t test_stuck;       // test hook: the first push claims a slot and never publishes it
    const GraphInfo* graphs;   // ngraphs entries
    uint32_t ngraphs;
    unsigned long long* gcount;   // per graph: maximal k-plexes
    unsigned long long* ghash;    // per graph: hash sum
    unsigned int* gvalid;         // per graph: valid roots
    uint32_t a_words;          // per-warp shared-memory copy of a root's A (0: read A from the arena)
    uint32_t stage_after;      // nodes on one root before its A is copied to shared memory
    const uint32_t* job_base;  // k-search jobs: root r owns jobs [job_base[r], job_base[r+1])
    uint32_t njobs;
    unsigned long long spin_limit;   // iterations for any bounded wait
};

// The persistent search kernel, one instantiation per bitset width (words per
// lane, 1 or 2) and blocks per SM (2 or 3): search.cu.
using SearchKernel = void (*)(SearchParams, uint32_t);
SearchKernel search_kernel_for(uint32_t words_per_lane, int blocks_per_sm);
uint32_t search_words_per_lane(uint32_t max_w);   // 2 when a root's rows exceed 32 words
uint32_t bnb_smem_words_host(uint32_t nmax, uint32_t slot_words, uint32_t a_words, uint32_t words_per_lane);
uint32_t ks_slot_words_host(uint32_t nmax, uint32_t slot_words, uint32_t words_per_lane);

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ void raise_error(Counters* c, unsigned code) { atomicCAS(&c->error, 0u, code); }

}  // namespace kplex
