// qc_device.h -- types shared by the host code and the expansion kernel.
//
// Device data layout (all in HBM, one set per context):
//   * graph CSR (int64 offsets, int32 sorted rows) and 2-hop CSR;
//   * md[k] = ceil(gamma*(k-1)) and ubt[d] = floor(d/gamma) tables, computed
//     on the host in double exactly as the reference does (main.cu:526-533,
//     main.cu:1905), so every device test is an integer comparison;
//   * a task-record arena: each record holds one branch-and-bound node as
//     its vertex ids plus its induced 1-hop and 2-hop adjacency as bit
//     matrices (row v = W words), so children never re-read the CSR;
//   * a LIFO stack of work items (record + branch range) with per-slot
//     hand-off flags, a control block (counters, status) and a flat buffer
//     of emitted vertex sets [k, id_1..id_k].
#pragma once
#include <stdint.h>

namespace qcb {

__host__ __device__ inline int clz64(unsigned long long x)
{
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

constexpr int kWarp = 32;
constexpr int kStackShards = 32;       // shared-stack shards (one per lane of a scanning warp)
constexpr int kArenaClasses = 4 * 40; // arena size classes (see arena_class)
constexpr int kArenaShards = 32;       // free lists per class, selected by block

// status bits written by the device
enum : int {
    ST_OK = 0,
    ST_TASK_OVERFLOW = 1,   // arena or stack exhausted
    ST_RESULT_OVERFLOW = 2, // emitted-set buffer exhausted
    ST_ITER_LIMIT = 4,      // a bounded wait gave up
    ST_TOO_LARGE = 8,       // task larger than the workspace supports
    ST_DEADLINE = 16,       // the run's time budget ran out
    ST_CHECK = 32           // a self-check caught a bad record offset or header
};

// Control block of a launch.  Words that many warps touch at once sit on
// their own 128-byte lines, so reads of one do not queue behind atomics on
// another.
struct Control {
    // capacities (written by the host, read-only on the device)
    unsigned long long arena_cap;
    unsigned long long result_cap;
    unsigned long long set_cap;    // capacity of the set-start array
    int stack_cap;                 // slots per shard; shard s owns slots [s*cap, (s+1)*cap)
    alignas(128) int stack_top[kStackShards]; // entries pushed on each shard of the shared stack
    alignas(128) int stack_bot[kStackShards]; // entries taken from the bottom (FIFO shards only)
    alignas(128) int pending;      // items on the shared stack + warps holding work
    alignas(128) int idle_warps;   // warps looking for work on the shared stack
    alignas(128) int status;
    alignas(128) unsigned long long arena_top; // bytes of record blocks handed out
    alignas(128) unsigned long long result_top; // ints of emitted sets written
    unsigned long long emitted;
    alignas(128) unsigned long long tasks, branches, children;
    unsigned long long lookahead_hits;
    unsigned long long parent_vertices, p_rows, child_vertices;
    int max_task;
    int active_warps;              // warps still inside the work loop
    unsigned long long t_start;    // globaltimer at the launch's start (0 until a warp sets it)
    unsigned long long wait_fail_where; // diagnostic: which wait gave up
    unsigned long long check_site;      // first failed self-check: site id
    unsigned long long check_value;     //   ... and the offending value
    int root_t, root_cov;          // the root task's size and covered count (device set-up)
    alignas(128) unsigned long long free_head[kArenaClasses * kArenaShards]; // [tag:24 | offset/16+1:40]
};

struct WorkItem {
    unsigned long long rec; // byte offset of the task record in the arena
    int q_lo;               // first branch position, -1: fresh task
    int q_hi;               // last branch position (inclusive)
};

// One slot of the shared stack: a branch range of one task, or a bundle of
// up to kBundle fresh tasks that a busy warp donated at once (a warp that
// takes it runs the first and keeps the rest on its own stack).
constexpr int kBundle = 6;
struct StackEntry {
    unsigned long long rec[kBundle];
    int32_t n;    // records in the entry, 1..kBundle
    int32_t q_lo; // with n == 1: branch range, q_lo = -1 for a fresh task
    int32_t q_hi;
    int32_t pad;
};

// Task record header; the record continues with
//   int32 ids[t]            (padded to 16 B)
//   int32 l2[t]             (lookahead 2-hop counts; 0 until computed)
//   uint32 A1[t][W]         (A1[v] bit w: w in N(v))
//   uint32 A2[t][W]         (A2[v] bit w: w in N2(v))
// and, in a record of at most 32 vertices written by the register path
// (flag kFlagRanked), at rec_ranks_off(): uint8 ranks[t], the number of the
// task's vertices with a larger id than vertex i.
struct TaskHdr {
    int32_t t;    // vertices
    int32_t m;    // members are positions [0, m)
    int32_t cov;  // covered candidates right after the members (root only)
    int32_t W;    // words per bit row
    int32_t refs; // work items that still reference this record
    int32_t cls;  // arena size class of the record's block
    int32_t inst; // instance (batched runs) whose rules apply
    int32_t flags; // kFlagShardRoot, kFlagRanked
};
constexpr int32_t kFlagShardRoot = 1; // the root of a search split by its branches (ExpandParams)
constexpr int32_t kFlagRanked = 2;    // id ranks stored at rec_ranks_off()

// Arena blocks come in size classes: four steps per power of two from
// 256 B (2^(e-1) + s*2^(e-3), s = 1..4).  Freed blocks go to a lock-free
// free list per class (see expand_kernel.cuh).

__host__ __device__ inline int arena_class(unsigned long long bytes)
{
    if (bytes <= 256) return 0;
    int e = 64 - clz64(bytes - 1); // 2^(e-1) < bytes <= 2^e
    unsigned long long half = 1ull << (e - 1), q = 1ull << (e - 3);
    int s = (int)((bytes - half + q - 1) / q); // 1..4
    return (e - 9) * 4 + s;                    // e = 9 -> classes 1..4 (257..512 B)
}
__host__ __device__ inline unsigned long long arena_class_bytes(int c)
{
    if (c == 0) return 256;
    int e = (c - 1) / 4 + 9, s = (c - 1) % 4 + 1;
    return (1ull << (e - 1)) + (unsigned long long)s * (1ull << (e - 3));
}

__host__ __device__ inline uint64_t align16(uint64_t x) { return (x + 15) & ~uint64_t(15); }
__host__ __device__ inline int words_for(int t) { return (t + 31) >> 5; }
__host__ __device__ inline uint64_t rec_ids_off() { return sizeof(TaskHdr); }
__host__ __device__ inline uint64_t rec_l2_off(int t) { return sizeof(TaskHdr) + align16(4ull * t); }
__host__ __device__ inline uint64_t rec_a1_off(int t) { return rec_l2_off(t) + align16(4ull * t); }
__host__ __device__ inline uint64_t rec_a2_off(int t, int W) {
    return rec_a1_off(t) + align16(4ull * t * W);
}
__host__ __device__ inline uint64_t rec_bytes(int t, int W) {
    return rec_a2_off(t, W) + align16(4ull * t * W);
}
// Every record of at most 32 vertices gets a block of one size, that of a
// 32-vertex record and its ranks, so a block freed by any small task can hold
// any small child (children are smaller than their parents, and per-size
// classes would leave the freed blocks in the wrong class).
__host__ __device__ inline uint64_t rec_ranks_off() { return rec_bytes(32, 1); }
__host__ __device__ inline uint64_t rec_block_bytes(int t, int W) {
    return W == 1 ? rec_ranks_off() + 32 : rec_bytes(t, W);
}

// Per-instance rules: the gamma tables and CSR offsets of one mining
// instance (a batched launch carries one entry per instance).
struct Rules {
    const int32_t* md;   // md[0 .. mdlen)
    const int32_t* ubt;  // floor(d / gamma), d in [0 .. mdlen)
    const int64_t* off;  // 1-hop offsets (degrees for the work counters)
    const int64_t* off2; // 2-hop offsets
    const int32_t* adj;  // 1-hop rows (read when the root record is built)
    const int32_t* adj2; // 2-hop rows
    int32_t mdlen;
    int32_t min_size;
    int32_t vbase;       // added to vertex ids when sets are emitted
    int32_t n;           // vertices of the instance (ids must be below it)
    const int32_t* md_s;  // shared-memory copies of md / ubt [0, kTabCache) (set on the
    const int32_t* ubt_s; //   device per warp; null in the table uploaded by the host)
    int32_t md_min;       // md[min_size] (set on the device with md_s)
    int32_t pad_;
};

constexpr int32_t kFreeMagic = 0x7ee7f00d; // refs of a block on a free list

struct ExpandParams {
    const Rules* rules;  // indexed by TaskHdr::inst
    int32_t nrules;
    Control* ctl;
    char* arena;
    StackEntry* stack;
    int32_t* slot;       // 0 free, 1 full, 2 being written, 3 being read
    int32_t* results;
    unsigned long long* set_starts; // start offset (in results) of every emitted set
    char* ws;            // per-warp workspace
    int64_t ws_stride;   // bytes per warp
    unsigned long long arena_cap; // bytes of the record arena
    int32_t smem_t;      // tasks of 33..smem_t vertices are staged in shared memory (0: none)
    int32_t max_t;       // largest task the workspace holds
    int32_t split;       // branches per work item before splitting
    int32_t small_path;  // 1: tasks of <= 32 vertices use the register path
    int64_t wait_ns;     // give up a wait after this long without progress
    int32_t shared_fifo; // 1: idle warps take the oldest shared-stack entry, 0: the newest
    int32_t shard;       // a search split by the root's branches: branch i of the root
    int32_t nshards;     //   (counted from the first branched) belongs to shard i % nshards
    unsigned long long time_limit_ns; // stop this long after the launch began (0: none); the
                                      // start is the first warp's globaltimer read, kept in
                                      // Control::t_start, so a replayed launch times itself
};

// Work counters a warp accumulates privately and adds to the control block
// once, when it leaves the work loop.
struct WarpCount {
    unsigned long long tasks, branches, children, lookahead_hits;
    unsigned long long parent_vertices, p_rows, child_vertices;
    unsigned long long max_task;
};

// Blocks a warp keeps on its private free lists before it hands further
// frees to the shared lists.
constexpr int kPrivateFreeCap = 64;

// Blocks of the small-record class (section below) a warp keeps in shared
// memory, taken and returned without touching the arena.
constexpr int kSmallFree = 32;

// Entries of the gamma tables (md, ubt) a warp keeps in shared memory; the
// tests of tasks up to this size never look further.
constexpr int kTabCache = 128;

// Fresh child tasks a warp keeps on its own stack (run depth first by the
// warp itself) before it pushes further children to the shared stack.
constexpr int kLocalStack = 48;

// Sets of at most 32 vertices a warp has found, kept in shared memory and
// appended to the result buffer together (one reservation for many sets).
constexpr int kEmitInts = 256;
constexpr int kEmitSets = 64;

// A fresh task on a warp's own stack.  A child the warp wrote itself carries
// its header (t > 0), so taking it needs no read of the record's header; a
// task taken from a donated bundle has t = 0 and is read and checked.
struct LocalTask {
    unsigned long long rec;
    int32_t t, m, W, cls, inst, flags;
};

// The register path's copy of the newest child a warp wrote (one lane's
// vertex each): taken from shared memory instead of the arena when that
// child is the warp's next task.
struct HotLane {
    int32_t id;
    uint32_t a1, a2;
    int32_t rank;
};

// Per-warp state in shared memory: everything a warp touches on every task.
struct WarpSmem {
    WarpCount cnt;
    LocalTask lstack[kLocalStack]; // this warp's own fresh child tasks
    int32_t lcount;                // entries on lstack
    int32_t hungry;                // idle warps seen when the previous item started
    int32_t stat;                  // run status seen when the previous item started
    int32_t tab_inst;            // instance whose gamma tables are cached (-1: none)
    unsigned long long fhead[kArenaClasses]; // private free lists: offset/16+1, 0 = empty
    int32_t fcount[kArenaClasses];
    unsigned long long sfree[kSmallFree]; // free blocks of the small-record class
    int32_t nsfree, pad2_;
    unsigned long long hot_rec;    // record whose copy is in hot (~0: none)
    HotLane hot[32];
    int32_t md[kTabCache];
    int32_t ubt[kTabCache];
    int32_t ebuf[kEmitInts];       // buffered sets, [k, ids..] each
    int32_t eset[kEmitSets];       // start of each buffered set in ebuf
    int32_t en, es;                // ints and sets buffered
    unsigned long long deadline;   // globaltimer value to stop at (0: none)
    unsigned long long stage_bar;  // mbarrier of this warp's bulk copies into its stage buffer
    int32_t stage_phase;           // parity of the next completion of stage_bar
    int32_t pad_;
};

// Per-warp workspace (global memory) for the bit-matrix path, tasks of up
// to max_t vertices.
struct WsLayout {
    int64_t indeg, exdeg, aux, vlist, hist, pref_cnt, pref_sum, sel, key_hi, key_lo, masks;
    int64_t total;
};

// Children of at most this many vertices are ordered by counting ranks, larger
// ones by a bitonic sort of their keys.
constexpr int kRankOrderMax = 256;

// Every array is indexed by a position below max_t, the histograms and their
// prefixes by a bin up to max_t + 1; the sort keys of a child larger than
// kRankOrderMax pad to a power of two.  No slack beyond that: a workspace of
// 160 vertices then fits 8 warps within the 196 KB shared-memory carve-out.
__host__ __device__ inline WsLayout ws_layout(int max_t)
{
    WsLayout L;
    int64_t t = max_t + 2;
    int64_t tp = max_t;
    if (max_t > kRankOrderMax) {
        tp = 1;
        while (tp < max_t) tp <<= 1;
    }
    int64_t W = words_for(max_t) + 2;
    int64_t o = 0;
    L.indeg = o;    o += align16(4 * t);
    L.exdeg = o;    o += align16(4 * t);
    L.aux = o;      o += align16(4 * t);
    L.vlist = o;    o += align16(4 * t);
    L.hist = o;     o += align16(4 * (t + 2));
    L.pref_cnt = o; o += align16(4 * (t + 2));
    L.pref_sum = o; o += align16(8 * (t + 2));
    L.sel = o;      o += align16(4 * tp);
    L.key_hi = o;   o += align16(8 * tp);
    L.key_lo = o;   o += align16(8 * tp);
    L.masks = o;    o += align16(4 * W * 12);
    L.total = align16(o);
    return L;
}

// Shared memory of one warp: its WarpSmem, then (when tasks of up to smem_t
// vertices are staged) a workspace laid out by ws_layout(smem_t) and a buffer
// for one record body of smem_t vertices.
__host__ __device__ inline uint64_t warp_smem_bytes(int smem_t)
{
    uint64_t b = align16(sizeof(WarpSmem));
    if (smem_t > 0)
        b += (uint64_t)ws_layout(smem_t).total + rec_bytes(smem_t, words_for(smem_t)) - rec_ids_off();
    return align16(b);
}

} // namespace qcb
