// expand_kernel.cuh -- persistent branch-and-bound expansion (device code).
//
// One warp works on one work item at a time: a task (a node of the
// set-enumeration tree) or a range of its branches.  A task carries its own
// induced adjacency as bit matrices, so every degree in the reference's
// rules becomes popc(row & mask) over ceil(t/32) words instead of a binary
// search in the global CSR (reference: d_bsearch_array, main.cu:4339).
//
// Rules implemented (plain set semantics of the reference's host routines;
// each function names the routine it follows):
//   lookahead            main.cu:1349-1405 / 3405-3471
//   remove-one threshold main.cu:1408-1462 / 3474-3515
//   add one + diameter   main.cu:1465-1523, 1709-1732
//   degree pruning       main.cu:1735-1855
//   lower/upper bounds   main.cu:1857-1972
//   critical vertices    main.cu:1526-1707
//   clique check         main.cu:1974-1995
//   Q enumeration order  main.cu:2059-2104
//   validity tests       main.cu:2144-2198
// The scheduler (a LIFO stack of work items with atomics, bounded waits and
// an outstanding-work counter) replaces the reference's host level loop,
// transfer_buffers and fill_from_buffer (main.cu:606-678, 3251-3398).
#pragma once
#include "qc_device.h"

namespace qcb {

#define QC_FULL 0xffffffffu

// Inlining of the large-task path's and the register path's routines, left to
// the compiler unless a build sets these (__noinline__ keeps one copy of a
// routine that several call sites share, which shrinks the kernel's code).
//
// The loops in those routines are kept rolled (`#pragma unroll 1`): the warps
// of an SM run the large-task path, the register path and the scheduler at
// once, and their code together overflows the instruction cache (instruction
// fetch is the batched workload's top stall).  Rolled, the batch of 64
// instances takes 113 ms instead of 137; config 1 is unchanged (1.14 against
// 1.15 ms).  Left to the compiler: the loops over a row's words (the degree
// counts of a branch and the child's row compaction), which stream the rows
// of tasks of thousands of vertices with several loads in flight, the child's
// rank count over its keys, and the scheduler's loops (rolling those too made
// config 1 1.4 times slower).
#ifndef QC_BIG_FN
#define QC_BIG_FN
#endif
#ifndef QC_SMALL_FN
#define QC_SMALL_FN
#endif
#ifndef QC_PRUNE_FN
#define QC_PRUNE_FN QC_BIG_FN
#endif
#ifndef QC_BOUNDS_FN
#define QC_BOUNDS_FN QC_BIG_FN
#endif

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// warp reductions: one redux instruction on the device, shuffles in the
// CPU emulator
__device__ __forceinline__ int wsum(int x)
{
#ifdef QC_EMULATION
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(QC_FULL, x, o);
    return x;
#else
    return __reduce_add_sync(QC_FULL, x);
#endif
}
__device__ __forceinline__ long long wsum64(long long x)
{
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(QC_FULL, x, o);
    return x;
}
__device__ __forceinline__ int wmin(int x)
{
#ifdef QC_EMULATION
    for (int o = 16; o; o >>= 1) {
        int y = __shfl_xor_sync(QC_FULL, x, o);
        x = y < x ? y : x;
    }
    return x;
#else
    return __reduce_min_sync(QC_FULL, x);
#endif
}
__device__ __forceinline__ int wmax(int x)
{
#ifdef QC_EMULATION
    for (int o = 16; o; o >>= 1) {
        int y = __shfl_xor_sync(QC_FULL, x, o);
        x = y > x ? y : x;
    }
    return x;
#else
    return __reduce_max_sync(QC_FULL, x);
#endif
}
// inclusive prefix sum across lanes
__device__ __forceinline__ int wscan(int x)
{
    int lane = lane_id();
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(QC_FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}
__device__ __forceinline__ long long wscan64(long long x)
{
    int lane = lane_id();
    for (int o = 1; o < 32; o <<= 1) {
        long long y = __shfl_up_sync(QC_FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__device__ __forceinline__ bool bit(const uint32_t* a, int v) { return (a[v >> 5] >> (v & 31)) & 1u; }

// Task records are written by one SM and read by another after a hand-off
// through the work stack, and their blocks are recycled; every read of record
// content in global memory goes through L2 (ld.global.cg) so no SM can see a
// stale L1 copy of a block's previous contents.  A record staged in shared
// memory is read there.
__device__ __forceinline__ uint32_t rec_ld(const uint32_t* p) { return __isGlobal(p) ? __ldcg(p) : *p; }
__device__ __forceinline__ int32_t rec_ld(const int32_t* p) { return __isGlobal(p) ? __ldcg(p) : *p; }
__device__ __forceinline__ uint8_t rec_ld(const uint8_t* p) { return __isGlobal(p) ? __ldcg(p) : *p; }
__device__ __forceinline__ bool rec_bit(const uint32_t* a, int v) { return (rec_ld(a + (v >> 5)) >> (v & 31)) & 1u; }

// |record row & mask| over W words (row in a task record, mask in the workspace)
__device__ __forceinline__ int popc_and(const uint32_t* row, const uint32_t* mask, int W)
{
    int s = 0;
    for (int w = 0; w < W; w++) {
        const uint32_t mw = mask[w]; // the same in every lane: skipping a zero word never diverges
        if (mw) s += __popc(rec_ld(row + w) & mw);
    }
    return s;
}

// warp-cooperative bitset helpers over W words
__device__ __forceinline__ void bs_copy(uint32_t* d, const uint32_t* s, int W)
{
    for (int w = lane_id(); w < W; w += 32) d[w] = s[w];
    __syncwarp();
}
__device__ __forceinline__ void bs_zero(uint32_t* d, int W)
{
    for (int w = lane_id(); w < W; w += 32) d[w] = 0;
    __syncwarp();
}
// bits [lo, hi) of word w as a mask
__device__ __forceinline__ uint32_t range_word(int w, int lo, int hi)
{
    int a = lo - w * 32, b = hi - w * 32; // the range relative to the word
    a = a < 0 ? 0 : (a > 32 ? 32 : a);
    b = b < 0 ? 0 : (b > 32 ? 32 : b);
    if (b <= a) return 0u;
    const uint32_t upto_b = b >= 32 ? ~0u : ((1u << b) - 1u);
    const uint32_t below_a = a >= 32 ? ~0u : ((1u << a) - 1u);
    return upto_b & ~below_a;
}

// d = bits [lo, hi)
__device__ __forceinline__ void bs_range(uint32_t* d, int W, int lo, int hi)
{
    for (int w = lane_id(); w < W; w += 32) d[w] = range_word(w, lo, hi);
    __syncwarp();
}
__device__ __forceinline__ int bs_count(const uint32_t* a, int W)
{
    int s = 0;
    for (int w = lane_id(); w < W; w += 32) s += __popc(a[w]);
    return wsum(s);
}
__device__ __forceinline__ bool bs_empty(const uint32_t* a, int W)
{
    int nz = 0;
    for (int w = lane_id(); w < W; w += 32) nz |= (a[w] != 0);
    return !__any_sync(QC_FULL, nz);
}

// ------------------------------------------------------------------
// per-warp state
// ------------------------------------------------------------------

struct TaskView {
    int t, m, cov, W, inst, flags;
    const int32_t* ids;
    int32_t* l2;
    const uint32_t* A1;
    const uint32_t* A2;
    int32_t* l2g;      // the record's l2 array in the arena (== l2 unless staged)
    unsigned long long rec;
};

// view of a record whose header fields were read once (through L2) and
// validated when the work item was dequeued
__device__ __forceinline__ TaskView task_view(char* arena, unsigned long long rec, const TaskHdr& h)
{
    TaskView T;
    T.t = h.t;
    T.m = h.m;
    T.cov = h.cov;
    T.W = h.W;
    T.inst = h.inst;
    T.flags = h.flags;
    T.ids = (const int32_t*)(arena + rec + rec_ids_off());
    T.l2 = (int32_t*)(arena + rec + rec_l2_off(T.t));
    T.A1 = (const uint32_t*)(arena + rec + rec_a1_off(T.t));
    T.A2 = (const uint32_t*)(arena + rec + rec_a2_off(T.t, T.W));
    T.l2g = T.l2;
    T.rec = rec;
    return T;
}


// A warp's workspace: one base pointer and the byte offsets of its arrays
// (laid out by ws_layout), so the whole view fits in a few registers.
struct Ws {
    WarpSmem* sm; // per-warp state in shared memory
    char* b;      // workspace base (global or shared memory)
    int32_t o_exdeg, o_aux, o_vlist, o_hist, o_pcnt, o_psum, o_sel, o_khi, o_klo, o_masks;
    int32_t wm;   // words per mask
    __device__ __forceinline__ int32_t* indeg() const { return (int32_t*)b; }
    __device__ __forceinline__ int32_t* exdeg() const { return (int32_t*)(b + o_exdeg); }
    __device__ __forceinline__ int32_t* aux() const { return (int32_t*)(b + o_aux); }
    // compacted vertex positions (see compact)
    __device__ __forceinline__ int32_t* vlist() const { return (int32_t*)(b + o_vlist); }
    __device__ __forceinline__ int32_t* hist() const { return (int32_t*)(b + o_hist); }
    __device__ __forceinline__ int32_t* pcnt() const { return (int32_t*)(b + o_pcnt); }
    __device__ __forceinline__ long long* psum() const { return (long long*)(b + o_psum); }
    __device__ __forceinline__ int32_t* sel() const { return (int32_t*)(b + o_sel); }
    __device__ __forceinline__ unsigned long long* khi() const { return (unsigned long long*)(b + o_khi); }
    __device__ __forceinline__ unsigned long long* klo() const { return (unsigned long long*)(b + o_klo); }
    __device__ __forceinline__ uint32_t* mk(int i) const { return (uint32_t*)(b + o_masks) + i * wm; }
};

// workspace arrays laid out by ws_layout(max_t) from base b (global or shared)
__device__ __forceinline__ Ws ws_view(char* b, int max_t, WarpSmem* sm)
{
    WsLayout L = ws_layout(max_t);
    Ws w;
    w.sm = sm;
    w.b = b + L.indeg;
    w.o_exdeg = (int32_t)(L.exdeg - L.indeg);
    w.o_aux = (int32_t)(L.aux - L.indeg);
    w.o_vlist = (int32_t)(L.vlist - L.indeg);
    w.o_hist = (int32_t)(L.hist - L.indeg);
    w.o_pcnt = (int32_t)(L.pref_cnt - L.indeg);
    w.o_psum = (int32_t)(L.pref_sum - L.indeg);
    w.o_sel = (int32_t)(L.sel - L.indeg);
    w.o_khi = (int32_t)(L.key_hi - L.indeg);
    w.o_klo = (int32_t)(L.key_lo - L.indeg);
    w.o_masks = (int32_t)(L.masks - L.indeg);
    w.wm = words_for(max_t) + 2;
    return w;
}

// mask slots
enum { MK_M = 0, MK_C = 1, MK_PRE = 2, MK_D = 3, MK_R = 4, MK_X = 5, MK_K = 6, MK_CA = 7,
       MK_T = 8, MK_U = 9 };

struct Bounds {
    int U, L, med;
};

// ------------------------------------------------------------------
// gamma tables (main.cu:526-533, 2144-2151)
// ------------------------------------------------------------------

// Each warp keeps shared-memory copies of entries [0, kTabCache) of md and
// ubt, padded past the table's end with its last entry.  A lookup clamps the
// index to the table and reads the copy or, past it, the global table; both
// loads are plain predicated instructions (no call, no divergent branch).
__device__ __forceinline__ int tab_far(const int32_t* tab_s, const int32_t* tab, int len, int k)
{
    k = k < 0 ? 0 : (k >= len ? len - 1 : k);
    return k < kTabCache ? tab_s[k] : __ldg(tab + k);
}
// `Near` lookups read the copy alone: on the register path members and
// candidates number at most 32, so every index is below 96, and an index at
// or below min_size goes through md_min.
__device__ __forceinline__ int tab_near(const int32_t* tab, int k)
{
    k = k < 0 ? 0 : (k >= kTabCache ? kTabCache - 1 : k);
    return tab[k];
}
template <bool Near = false>
__device__ __forceinline__ int md_at(const Rules& R, int k)
{
    if (Near) return tab_near(R.md_s, k);
    return tab_far(R.md_s, R.md, R.mdlen, k);
}
template <bool Near = false>
__device__ __forceinline__ int mindeg(const Rules& R, int k)
{
    if (Near) return k < R.min_size ? R.md_min : tab_near(R.md_s, k);
    return md_at(R, k < R.min_size ? R.min_size : k);
}
template <bool Near = false>
__device__ __forceinline__ int ubt_at(const Rules& R, int d)
{
    if (Near) return tab_near(R.ubt_s, d);
    return tab_far(R.ubt_s, R.ubt, R.mdlen, d);
}

// main.cu:2167-2178
template <bool Near = false>
__device__ __forceinline__ bool cand_valid(const Rules& R, int in, int ex, int m,
                                           const Bounds& b)
{
    int tot = in + ex;
    if (tot < R.md_min) return false;
    if (tot < mindeg<Near>(R, m + ex + 1)) return false;
    if (tot < b.med) return false;
    if (in + b.U - 1 < md_at<Near>(R, m + b.L)) return false;
    if (tot < mindeg<Near>(R, m + b.L)) return false;
    return true;
}
// main.cu:2180-2198
template <bool Near = false>
__device__ __forceinline__ bool vert_extendable(const Rules& R, int in, int ex, int m,
                                                const Bounds& b)
{
    int tot = in + ex;
    if (tot < R.md_min) return false;
    if (tot < mindeg<Near>(R, m + ex)) return false;
    if (tot < b.med) return false;
    if (ex == 0 && in < mindeg<Near>(R, m + ex)) return false;
    if (in + b.U < md_at<Near>(R, m + b.U)) return false;
    if (tot < mindeg<Near>(R, m + b.L)) return false;
    return true;
}

// ------------------------------------------------------------------
// candidate indegree histogram -> S(k) = sum of the k largest
// ------------------------------------------------------------------

// Build the histogram of indeg over the vertices in mask `cm` (optionally
// only those passing validity under `b`), then prefix tables over bins in
// descending value order: pcnt[j] = #values > vmax-j, psum[j] = their sum.
// Values are bounded by vmax (members count).  Returns the number of values.
__device__ QC_BOUNDS_FN int build_hist(const ExpandParams& P, const Rules& R, Ws& ws, const uint32_t* cm, int t, int vmax,
                          bool filter_valid, int m, const Bounds& b)
{
    int lane = lane_id();
    #pragma unroll 1
    for (int j = lane; j <= vmax + 1; j += 32) ws.hist()[j] = 0;
    __syncwarp();
    int cnt = 0;
    #pragma unroll 1
    for (int base = 0; base < t; base += 32) {
        const uint32_t cw = cm[base >> 5];
        if (cw == 0) continue; // no vertex of this chunk (the word is the same in every lane)
        int v = base + lane;
        int j = -1;
        if (v < t && ((cw >> lane) & 1u)) {
            int in = ws.indeg()[v];
            if (!filter_valid || cand_valid(R, in, ws.exdeg()[v], m, b)) {
                j = vmax - (in > vmax ? vmax : (in < 0 ? 0 : in));
                cnt++;
            }
        }
        // one shared-memory add per distinct bin of the 32 lanes (many lanes
        // share a degree, and their adds would otherwise queue on one word)
        const unsigned peers = __match_any_sync(QC_FULL, j);
        if (j >= 0 && (peers & ((1u << lane) - 1u)) == 0) atomicAdd(&ws.hist()[j], __popc(peers));
    }
    __syncwarp();
    // exclusive prefix over bins 0..vmax+1
    int carry = 0;
    long long carry_s = 0;
    #pragma unroll 1
    for (int base = 0; base <= vmax + 1; base += 32) {
        int j = base + lane;
        int c = (j <= vmax + 1) ? ws.hist()[j] : 0;
        long long s = (j <= vmax) ? (long long)c * (vmax - j) : 0;
        int ic = wscan(c);
        // the sums stay below t * vmax: 32 bits hold them below 46,341 vertices
        long long is = t < 46341 ? (long long)wscan((int)s) : wscan64(s);
        if (j <= vmax + 1) {
            ws.pcnt()[j] = carry + ic - c;
            ws.psum()[j] = carry_s + is - s;
        }
        carry += __shfl_sync(QC_FULL, ic, 31);
        carry_s += __shfl_sync(QC_FULL, is, 31);
    }
    __syncwarp();
    return wsum(cnt);
}

// sum of the k largest values (0 <= k <= total)
__device__ __forceinline__ long long top_sum(const Ws& ws, int vmax, int k)
{
    // largest bin j in [0, vmax+1] with pcnt[j] <= k
    int lo = 0, hi = vmax + 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ws.pcnt()[mid] <= k) lo = mid;
        else hi = mid - 1;
    }
    if (lo > vmax) return ws.psum()[vmax + 1];
    return ws.psum()[lo] + (long long)(k - ws.pcnt()[lo]) * (vmax - lo);
}

// The lower bound's search (main.cu:1877-1890): the first L >= mindeg(m) -
// min_in with !(L <= min_in_ex && min_in + L < md[m+L]), for members whose
// smallest indegree is min_in (min_in_ex: the smallest exdegree among them).
__device__ __forceinline__ int lower_start(const Rules& R, int m, int min_in, int min_in_ex)
{
    const int lane = lane_id();
    int lb = mindeg(R, m) - min_in;
    for (int base = lb;; base += 32) {
        int L = base + lane;
        bool cont = (L <= min_in_ex) && (min_in + L < md_at(R, m + L));
        unsigned stop = __ballot_sync(QC_FULL, !cont);
        if (stop) return base + __ffs(stop) - 1;
    }
}

// ------------------------------------------------------------------
// lower / upper bounds (main.cu:1857-1972).  Members: mask mm (m of them).
// The candidate histogram must be built.  Returns true when invalid.
// ------------------------------------------------------------------

__device__ QC_BOUNDS_FN bool lu_bounds(const ExpandParams& P, const Rules& R, Ws& ws, const uint32_t* mm, int t, int m,
                          int ncand, int vmax, Bounds& b)
{
    int lane = lane_id();
    // one pass over the members: this lane's smallest indegree and, among
    // its members with that indegree, the smallest exdegree
    int mi = 0x7fffffff, mt = 0x7fffffff, me = 0x7fffffff;
    long long si = 0;
    #pragma unroll 1
    for (int base = 0; base < t; base += 32) {
        const uint32_t mw = mm[base >> 5];
        if (mw == 0) continue;
        int v = base + lane;
        if (v < t && ((mw >> lane) & 1u)) {
            int in = ws.indeg()[v], ex = ws.exdeg()[v];
            if (in < mi) {
                mi = in;
                me = ex;
            } else if (in == mi && ex < me) {
                me = ex;
            }
            mt = in + ex < mt ? in + ex : mt;
            si += in;
        }
    }
    int min_in = wmin(mi);
    int min_tot = wmin(mt);
    // a sum of at most t indegrees below t: 32 bits hold it below 46,341 vertices
    long long sum_in = t < 46341 ? (long long)wsum((int)si) : wsum64(si);
    int min_in_ex = wmin(mi == min_in ? me : 0x7fffffff);

    bool invalid = false;
    b.med = mindeg(R, m + 1);
    if (min_in < md_at(R, m)) {
        int lb = lower_start(R, m, min_in, min_in_ex);
        if (min_in + lb < md_at(R, m + lb)) {
            lb = ncand + 1;
            invalid = true;
        }
        int ub = ubt_at(R, min_tot) + 1 - m;
        if (ub > ncand) ub = ncand;
        if (lb < ub) {
            // first k in [lb, ub] with k == ub || sum_in + S(k) >= m*md[m+k]
            int idx = ub;
            #pragma unroll 1
            for (int base = lb; base <= ub; base += 32) {
                int k = base + lane;
                bool ok = false;
                if (k <= ub) {
                    ok = (k == ub) ||
                         (sum_in + top_sum(ws, vmax, k) >= (long long)m * md_at(R, m + k));
                }
                unsigned bal = __ballot_sync(QC_FULL, ok);
                if (bal) {
                    idx = base + __ffs(bal) - 1;
                    break;
                }
            }
            if (sum_in + top_sum(ws, vmax, idx) < (long long)m * md_at(R, m + idx)) {
                lb = ub + 1;
                invalid = true;
            } else {
                lb = idx;
                int tub = idx;
                #pragma unroll 1
                for (int base = idx + 1; base <= ub; base += 32) {
                    int k = base + lane;
                    bool ok = (k <= ub) &&
                              (sum_in + top_sum(ws, vmax, k) >= (long long)m * md_at(R, m + k));
                    int best = wmax(ok ? k : -1);
                    if (best > tub) tub = best;
                }
                if (ub > tub) ub = tub;
                if (lb > 1) b.med = mindeg(R, m + lb);
            }
        }
        b.U = ub;
        b.L = lb;
    } else {
        b.U = ncand;
        b.L = m < R.min_size ? R.min_size - m : 0;
    }
    if (m + b.U < R.min_size) invalid = true;
    if (b.U < 0 || b.U < b.L) invalid = true;
    return invalid;
}

// every member extendable? (main.cu:1749-1753)
__device__ QC_BIG_FN bool members_ok(const ExpandParams& P, const Rules& R, Ws& ws, const uint32_t* mm, int t, int m,
                           const Bounds& b)
{
    int lane = lane_id();
    int bad = 0;
    #pragma unroll 1
    for (int base = 0; base < t; base += 32) {
        const uint32_t mw = mm[base >> 5];
        if (mw == 0) continue;
        int v = base + lane;
        if (v < t && ((mw >> lane) & 1u) && !vert_extendable(R, ws.indeg()[v], ws.exdeg()[v], m, b)) bad = 1;
    }
    return !__any_sync(QC_FULL, bad);
}

// positions v < t set in `mask`, ascending, into ws.vlist(); returns their number.
// Loops over the list keep all 32 lanes busy however sparse the mask is.
__device__ int compact(Ws& ws, const uint32_t* mask, int t)
{
    int lane = lane_id();
    int n = 0;
    for (int base = 0; base < t; base += 32) {
        const uint32_t mw = mask[base >> 5];
        if (mw == 0) continue;
        int v = base + lane;
        bool in = v < t && ((mw >> lane) & 1u);
        unsigned bal = __ballot_sync(QC_FULL, in);
        if (in) ws.vlist()[n + __popc(bal & ((1u << lane) - 1u))] = v;
        n += __popc(bal);
    }
    __syncwarp();
    return n;
}

// exdeg[v] = |N(v) & R| for v in mask `who`
__device__ QC_BIG_FN void recount_exdeg(const TaskView& T, Ws& ws, const uint32_t* who, const uint32_t* R)
{
    int n = compact(ws, who, T.t);
    #pragma unroll 1
    for (int i = lane_id(); i < n; i += 32) {
        int v = ws.vlist()[i];
        ws.exdeg()[v] = popc_and(T.A1 + (int64_t)v * T.W, R, T.W);
    }
    __syncwarp();
}

// out = {v in in_mask : cand_valid(v)} ; rem = in_mask \ out
__device__ QC_BIG_FN void filter_valid(const ExpandParams& P, const Rules& R, Ws& ws, const uint32_t* in_mask, int t, int W,
                             int m, const Bounds& b, uint32_t* out, uint32_t* rem)
{
    int lane = lane_id();
    #pragma unroll 1
    for (int base = 0; base < t; base += 32) {
        const uint32_t iw = in_mask[base >> 5];
        if (iw == 0) {
            if (lane == 0) {
                out[base >> 5] = 0;
                if (rem) rem[base >> 5] = 0;
            }
            continue;
        }
        int v = base + lane;
        bool in = v < t && ((iw >> lane) & 1u);
        bool ok = in && cand_valid(R, ws.indeg()[v], ws.exdeg()[v], m, b);
        unsigned bo = __ballot_sync(QC_FULL, ok);
        unsigned br = __ballot_sync(QC_FULL, in && !ok);
        if (lane == 0) {
            out[base >> 5] = bo;
            if (rem) rem[base >> 5] = br;
        }
    }
    #pragma unroll 1
    for (int w = words_for(t) + lane; w < W; w += 32) {
        out[w] = 0;
        if (rem) rem[w] = 0;
    }
    __syncwarp();
}

// ------------------------------------------------------------------
// iterative degree pruning (main.cu:1735-1855)
// Entry: indeg/exdeg valid for M u Call with exdeg relative to Call.
// D = diameter survivors (label 0).  On success R holds the candidates.
// Returns 1 on invalid bounds or a non-extendable member, 0 when the
// fixpoint is reached, and, with may_switch, 2 when a further round is due
// and the members and remaining candidates Rm number at most 32: the caller
// then runs the rest of the branch on the register path.
// ------------------------------------------------------------------

enum { DP_DONE = 0, DP_INVALID = 1, DP_SWITCH = 2 };

__device__ QC_PRUNE_FN int degree_prune(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws, const uint32_t* M,
                            int m, const uint32_t* Call, const uint32_t* D, uint32_t* Rm,
                            Bounds& b, bool may_switch)
{
    const int t = T.t, W = T.W;
    uint32_t* X = ws.mk(MK_X);
    uint32_t* who = ws.mk(MK_U);
    Bounds dummy = {0, 0, 0};
    int nc = build_hist(P, R, ws, D, t, m, false, m, dummy);
    if (lu_bounds(P, R, ws, M, t, m, nc, m, b)) return DP_INVALID;
    if (!members_ok(P, R, ws, M, t, m, b)) return DP_INVALID;
    filter_valid(P, R, ws, D, t, W, m, b, Rm, nullptr);
    // X = Call \ Rm
    #pragma unroll 1
    for (int w = lane_id(); w < W; w += 32) X[w] = Call[w] & ~Rm[w];
    __syncwarp();
    while (!bs_empty(Rm, W) && !bs_empty(X, W)) {
        if (may_switch && m + bs_count(Rm, W) <= 32) return DP_SWITCH;
        #pragma unroll 1
        for (int w = lane_id(); w < W; w += 32) who[w] = M[w] | Rm[w];
        __syncwarp();
        recount_exdeg(T, ws, who, Rm);
        int nv = build_hist(P, R, ws, Rm, t, m, true, m, b);
        if (lu_bounds(P, R, ws, M, t, m, nv, m, b)) return DP_INVALID;
        if (!members_ok(P, R, ws, M, t, m, b)) return DP_INVALID;
        // Rm' = valid(Rm), X = Rm \ Rm'
        filter_valid(P, R, ws, Rm, t, W, m, b, ws.mk(MK_T), X);
        bs_copy(Rm, ws.mk(MK_T), W);
    }
    return DP_DONE;
}

// ------------------------------------------------------------------
// emission and allocation
// ------------------------------------------------------------------

__device__ __forceinline__ void set_status(const ExpandParams& P, int bits)
{
    atomicOr(&P.ctl->status, bits);
}

// record the first failed self-check (site, value) and stop the run
__device__ __forceinline__ void check_fail(const ExpandParams& P, unsigned long long site,
                                           unsigned long long value)
{
    if (atomicCAS(&P.ctl->check_site, 0ull, site) == 0ull) P.ctl->check_value = value;
    set_status(P, ST_CHECK);
}

// write the ids of the vertices in mask `mm` (count k) as one set
__device__ QC_BIG_FN void emit_mask(const ExpandParams& P, const Rules& R, const TaskView& T, const uint32_t* mm, int k)
{
    int lane = lane_id();
    unsigned long long at = 0;
    if (lane == 0) {
        at = atomicAdd(&P.ctl->result_top, (unsigned long long)(k + 1));
        unsigned long long idx = atomicAdd(&P.ctl->emitted, 1ull);
        if (at + k + 1 > P.ctl->result_cap || idx >= P.ctl->set_cap) {
            set_status(P, ST_RESULT_OVERFLOW);
            at = ~0ull;
        } else {
            P.set_starts[idx] = at;
        }
    }
    at = __shfl_sync(QC_FULL, at, 0);
    if (at == ~0ull) return;
    if (lane == 0) P.results[at] = k;
    int written = 0;
    #pragma unroll 1
    for (int base = 0; base < T.t; base += 32) {
        int v = base + lane;
        bool in = v < T.t && bit(mm, v);
        unsigned bal = __ballot_sync(QC_FULL, in);
        if (in) {
            int r = __popc(bal & ((1u << lane) - 1u));
            P.results[at + 1 + written + r] = rec_ld(T.ids + v) + R.vbase;
        }
        written += __popc(bal);
    }
}

// clique check (main.cu:1974-1995): every member has indeg >= md[m]
__device__ QC_BIG_FN void check_clique(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws, const uint32_t* mm,
                             int m)
{
    int lane = lane_id();
    int need = md_at(R, m);
    int bad = 0;
    #pragma unroll 1
    for (int base = 0; base < T.t; base += 32) {
        int v = base + lane;
        if (v < T.t && bit(mm, v) && ws.indeg()[v] < need) bad = 1;
    }
    if (!__any_sync(QC_FULL, bad)) emit_mask(P, R, T, mm, m);
}

// ------------------------------------------------------------------
// work stack: push / pop with per-slot hand-off and bounded waits
// ------------------------------------------------------------------

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
#ifdef QC_EMULATION
    t = emu_globaltimer();
#else
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
#endif
    return t;
}

// the shard a warp pushes to and starts its scans from
__device__ __forceinline__ int home_shard() { return (int)((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) % kStackShards); }

// Shared-stack shards.  Each shard is a stack (idle warps take the newest
// entry: depth first, few live tasks) or, with P.shared_fifo, a ring whose
// oldest entry is taken first (the shallowest donated tasks, which head the
// largest subtrees, start first: better when many independent instances
// keep every warp busy).  reserve_push returns the slot a new entry of shard
// `shard` goes to, or -1 when the shard is full.
__device__ __forceinline__ long long reserve_push(const ExpandParams& P, int shard)
{
    const int cap = P.ctl->stack_cap;
    const int idx = atomicAdd(&P.ctl->stack_top[shard], 1);
    if (P.shared_fifo) {
        // indices count up for the whole run; cap is a power of two, so the
        // slot (idx mod cap) stays right when the 32-bit count wraps.  Takers
        // may have claimed this index and later ones already (they wait for
        // the writes), so the distance to the bottom is taken as signed.
        if ((int)((unsigned)idx - (unsigned)*(volatile int*)&P.ctl->stack_bot[shard]) >= cap)
            return -1;
        return (long long)shard * cap + ((unsigned)idx & (unsigned)(cap - 1));
    }
    if (idx >= cap) return -1;
    return (long long)shard * cap + idx;
}

// lane-0 only: one entry onto shard `shard` of the shared stack
__device__ bool push_entry(const ExpandParams& P, const StackEntry& e, int shard)
{
    atomicAdd(&P.ctl->pending, 1);
    const long long at = reserve_push(P, shard);
    if (at < 0) {
        set_status(P, ST_TASK_OVERFLOW);
        atomicSub(&P.ctl->pending, 1);
        return false;
    }
    unsigned long long t0 = now_ns();
    unsigned spins = 0;
    while (atomicCAS(&P.slot[at], 0, 2) != 0) {
        if ((++spins & 255u) == 0) {
            if (now_ns() - t0 > (unsigned long long)P.wait_ns || P.ctl->status) {
                set_status(P, ST_ITER_LIMIT);
                P.ctl->wait_fail_where = 1;
                return false;
            }
        }
        __nanosleep(64);
    }
    P.stack[at] = e;
    __threadfence();
    atomicExch(&P.slot[at], 1);
    return true;
}

__device__ bool push_item(const ExpandParams& P, const WorkItem& it)
{
    StackEntry e;
    for (int i = 0; i < kBundle; i++) e.rec[i] = 0;
    e.rec[0] = it.rec;
    e.n = 1;
    e.q_lo = it.q_lo;
    e.q_hi = it.q_hi;
    e.pad = 0;
    return push_entry(P, e, home_shard());
}

// Whole warp: push `count` branch ranges of record `rec`, range c (covering
// the `split` branches ending at hi_first - c*split, not below q_lo) onto
// shard (home + c) mod S, so that many waiting warps can take them at once
// instead of queueing on one shard's top.  Every lane pushes a share.
// Returns false when a shard is full (the run then stops with
// ST_TASK_OVERFLOW) or a slot wait gave up.
__device__ QC_SMALL_FN bool push_ranges(const ExpandParams& P, unsigned long long rec, int q_lo, int hi_first,
                            int split, int count)
{
    const int lane = lane_id();
    const int home = home_shard();
    if (lane == 0) atomicAdd(&P.ctl->pending, count);
    __syncwarp();
    int ok = 1;
    #pragma unroll 1
    for (int c = lane; c < count; c += 32) {
        const int shard = (home + c) % kStackShards;
        const long long at = reserve_push(P, shard);
        if (at < 0) {
            set_status(P, ST_TASK_OVERFLOW);
            atomicSub(&P.ctl->pending, 1);
            ok = 0;
            continue;
        }
        unsigned long long t0 = now_ns();
        unsigned spins = 0;
        bool got = true;
        while (atomicCAS(&P.slot[at], 0, 2) != 0) {
            if ((++spins & 255u) == 0 &&
                (now_ns() - t0 > (unsigned long long)P.wait_ns || *(volatile int*)&P.ctl->status)) {
                set_status(P, ST_ITER_LIMIT);
                P.ctl->wait_fail_where = 4;
                got = false;
                break;
            }
            __nanosleep(64);
        }
        if (!got) {
            ok = 0;
            continue;
        }
        const int hi = hi_first - c * split;
        StackEntry e;
        #pragma unroll 1
        for (int i = 0; i < kBundle; i++) e.rec[i] = 0;
        e.rec[0] = rec;
        e.n = 1;
        e.q_hi = hi;
        e.q_lo = hi - split + 1 < q_lo ? q_lo : hi - split + 1;
        e.pad = 0;
        P.stack[at] = e;
        __threadfence();
        atomicExch(&P.slot[at], 1);
    }
    return __all_sync(QC_FULL, ok);
}

// lane 0: read the entry at index idx of shard s once its writer is done
__device__ int take_slot(const ExpandParams& P, int s, int idx, StackEntry& out)
{
    long long at;
    if (P.shared_fifo) {
        at = (long long)s * P.ctl->stack_cap + ((unsigned)idx & (unsigned)(P.ctl->stack_cap - 1));
    } else {
        // a failed push (shard full) leaves the top above the capacity; such
        // an index has no slot behind it
        if (idx >= P.ctl->stack_cap) {
            set_status(P, ST_TASK_OVERFLOW);
            return -1;
        }
        at = (long long)s * P.ctl->stack_cap + idx;
    }
    unsigned long long t1 = now_ns();
    unsigned s2 = 0;
    while (atomicCAS(&P.slot[at], 1, 3) != 1) {
        if ((++s2 & 255u) == 0) {
            // a run that is stopping may leave reserved slots unwritten
            if (*(volatile int*)&P.ctl->status) return -1;
            if (now_ns() - t1 > (unsigned long long)P.wait_ns) {
                set_status(P, ST_ITER_LIMIT);
                P.ctl->wait_fail_where = 2;
                return -1;
            }
        }
        __nanosleep(32);
    }
    __threadfence();
    const volatile StackEntry* src = &P.stack[at];
    out.n = src->n;
    out.q_lo = src->q_lo;
    out.q_hi = src->q_hi;
    for (int i = 0; i < kBundle; i++) out.rec[i] = src->rec[i];
    __threadfence();
    atomicExch(&P.slot[at], 0);
    return 1;
}

// Whole warp: take one entry from the shared stack.  The lanes read all
// shard tops in one coalesced load and lane 0 claims the first non-empty
// shard at or after the warp's home shard.  Returns (in every lane) 1 with
// the entry in lane 0's `out`, 0 when the stack is empty and no warp holds
// work, -1 on error or abort.
#ifndef QC_IDLE_BACKOFF_MAX
#define QC_IDLE_BACKOFF_MAX 4096
#endif
constexpr unsigned kIdleBackoffMax = QC_IDLE_BACKOFF_MAX; // ns

__device__ int pop_shared(const ExpandParams& P, StackEntry& out, unsigned long long deadline)
{
    const int lane = lane_id();
    const int home = home_shard();
    unsigned long long t0 = now_ns();
    unsigned spins = 0;
    unsigned backoff = 64;
    int last_pending = -1;
    for (;;) {
        int act = 0;
        if (lane == 0) {
            if (*(volatile int*)&P.ctl->status) act = -1;
            else if (deadline && now_ns() > deadline) {
                set_status(P, ST_DEADLINE);
                act = -1;
            }
        }
        if (__shfl_sync(QC_FULL, act, 0) < 0) return -1;
        int top = *(volatile int*)&P.ctl->stack_top[lane];
        const int bot = P.shared_fifo ? *(volatile int*)&P.ctl->stack_bot[lane] : 0;
        unsigned ne = __ballot_sync(QC_FULL, (int)((unsigned)top - (unsigned)bot) > 0);
        if (ne) {
            unsigned rot = home ? ((ne >> home) | (ne << (32 - home))) : ne;
            int s = (home + __ffs(rot) - 1) & 31;
            int got = 0;
            if (P.shared_fifo) {
                // the oldest entry of the shard
                const int bs = __shfl_sync(QC_FULL, bot, s);
                if (lane == 0 && atomicCAS(&P.ctl->stack_bot[s], bs, bs + 1) == bs)
                    got = take_slot(P, s, bs, out);
            } else {
                const int ts = __shfl_sync(QC_FULL, top, s);
                if (lane == 0 && atomicCAS(&P.ctl->stack_top[s], ts, ts - 1) == ts)
                    got = take_slot(P, s, ts - 1, out);
            }
            got = __shfl_sync(QC_FULL, got, 0);
            if (got != 0) return got;
            // lost the race for that top: wait a short, warp-dependent time so
            // the losers do not retry in lock step
            unsigned jitter = (unsigned)((blockIdx.x * 37u + (threadIdx.x >> 5) * 11u + spins) & 255u);
            __nanosleep(32 + jitter);
            spins++;
            continue;
        }
        int done = 0;
        if (lane == 0) {
            int pend = *(volatile int*)&P.ctl->pending;
            if (pend == 0) done = 1;
            else {
                if (pend != last_pending) {
                    last_pending = pend;
                    t0 = now_ns();
                }
                if ((++spins & 15u) == 0 && now_ns() - t0 > (unsigned long long)P.wait_ns) {
                    set_status(P, ST_ITER_LIMIT);
                    P.ctl->wait_fail_where = 3;
                    done = -1;
                }
            }
        }
        done = __shfl_sync(QC_FULL, done, 0);
        if (done == 1) return 0;
        if (done < 0) return -1;
        // idle: back off (64 ns doubling to kIdleBackoffMax) so waiting warps
        // leave the issue slots and the tops' cache line to the working ones
        __nanosleep(backoff);
        backoff = backoff < kIdleBackoffMax ? backoff * 2 : kIdleBackoffMax;
    }
}

// Whole warp.  While it waits the warp is counted in `idle_warps`, which
// busy warps read to decide whether to donate.  The first task of a popped
// bundle becomes the warp's item (in lane 0), the others go on its own stack
// (it holds no work when it pops, so they fit).
__device__ QC_SMALL_FN int pop_item(const ExpandParams& P, Ws& ws, WorkItem& out)
{
    const int lane = lane_id();
    if (lane == 0) atomicAdd(&P.ctl->idle_warps, 1);
    StackEntry e;
    int r = pop_shared(P, e, ws.sm->deadline);
    if (lane == 0) {
        atomicSub(&P.ctl->idle_warps, 1);
        if (r > 0) {
            if (e.n < 1 || e.n > kBundle || (e.n > 1 && e.q_lo >= 0)) {
                check_fail(P, 16, (unsigned long long)e.n); // a malformed stack entry
                r = -1;
            } else {
                out.rec = e.rec[0];
                out.q_lo = e.q_lo;
                out.q_hi = e.q_hi;
                #pragma unroll 1
                for (int i = e.n - 1; i >= 1 && ws.sm->lcount < kLocalStack; i--) {
                    LocalTask lt{};
                    lt.rec = e.rec[i]; // header read and checked when taken
                    ws.sm->lstack[ws.sm->lcount++] = lt;
                }
            }
        }
    }
    return __shfl_sync(QC_FULL, r, 0);
}

// lane 0: hand a freshly written child to the scheduler.  Children go to the
// warp's own stack in shared memory (run depth first by this warp, no
// atomics); only when that stack is full does a child go to the shared one.
// `pending` counts shared-stack items plus warps that hold work, so local
// children change it only when they are donated (push_item).
__device__ void schedule_child(const ExpandParams& P, Ws& ws, unsigned long long rec, int t, int m,
                               int W, int cls, int inst, int flags)
{
    if (ws.sm->lcount < kLocalStack) {
        LocalTask lt;
        lt.rec = rec;
        lt.t = t;
        lt.m = m;
        lt.W = W;
        lt.cls = cls;
        lt.inst = inst;
        lt.flags = flags;
        ws.sm->lstack[ws.sm->lcount++] = lt;
        return;
    }
    // published to other warps: push_entry fences the record before the hand-off
    WorkItem it;
    it.rec = rec;
    it.q_lo = -1;
    it.q_hi = -1;
    push_item(P, it);
}

// waiting warps from which a small task's children are donated between its
// branches, not only between items
#ifndef QC_EAGER_HUNGRY
#define QC_EAGER_HUNGRY 4
#endif
constexpr int kEagerHungry = QC_EAGER_HUNGRY;
// tasks a warp keeps on its own stack when it donates between a small task's
// branches (it has branches left to run, so it may give away all of them)
#ifndef QC_EAGER_KEEP
#define QC_EAGER_KEEP 1
#endif
constexpr int kEagerKeep = QC_EAGER_KEEP;

// Whole warp: while other warps wait for work, hand them all but the newest
// task of this warp's own stack, oldest (shallowest, usually largest) first,
// in bundles sized so each waiting warp can take one.  Lane b pushes bundle b
// to shard (home + b), so the pushes' round trips overlap.
__device__ QC_SMALL_FN void donate(const ExpandParams& P, Ws& ws, int keep = 1)
{
    const int lane = lane_id();
    __syncwarp(); // lane 0's stack and counters written before the call
    const int n = ws.sm->lcount;
    // read when the previous item started (the read overlapped its work)
    const int hungry = ws.sm->hungry;
    if (n <= keep || hungry <= 0) return;
    const int give = n - keep;
    int per = (give + hungry - 1) / hungry;
    per = per < 1 ? 1 : (per > kBundle ? kBundle : per);
    int nb = (give + per - 1) / per;
    nb = nb > 8 ? 8 : nb;
    bool pushed = false;
    if (lane < nb) {
        const int first = lane * per;
        const int k = give - first < per ? give - first : per;
        StackEntry e;
        #pragma unroll 1
        for (int i = 0; i < kBundle; i++) e.rec[i] = i < k ? ws.sm->lstack[first + i].rec : 0ull;
        e.n = k;
        e.q_lo = -1;
        e.q_hi = -1;
        e.pad = 0;
        pushed = push_entry(P, e, (home_shard() + lane) % kStackShards);
    }
    const unsigned ok = __ballot_sync(QC_FULL, pushed);
    __syncwarp();
    if (lane == 0) {
        // keep, in order, the tasks of bundles that were not pushed (a failed
        // push has stopped the run) and the tasks past the last bundle
        int keep = 0;
        #pragma unroll 1
        for (int i = 0; i < n; i++) {
            const int b = i / per;
            if (i < give && b < nb && ((ok >> b) & 1u)) continue;
            ws.sm->lstack[keep++] = ws.sm->lstack[i];
        }
        ws.sm->lcount = keep;
        ws.sm->hungry = hungry > nb ? hungry - nb : 0;
    }
    __syncwarp();
}

// ------------------------------------------------------------------
// record arena: size classes with lock-free free lists (lane 0 only)
// A list head packs a 24-bit tag (bumped on every change, against ABA) and
// the block offset / 16 + 1 (0 = empty); a free block's first 8 bytes hold
// the next block in the same encoding without the tag.
// ------------------------------------------------------------------

constexpr unsigned long long kOffMask = (1ull << 40) - 1;

// the size class of every record of at most 32 vertices (rec_block_bytes)
__device__ __forceinline__ int small_class() { return arena_class(rec_bytes(32, 1)); }

__device__ unsigned long long arena_block(const ExpandParams& P, Ws& ws, unsigned long long bytes, int& cls)
{
    cls = arena_class(bytes);
    if (cls >= kArenaClasses) {
        set_status(P, ST_TOO_LARGE);
        return ~0ull;
    }
    unsigned long long size = arena_class_bytes(cls);
    // small records: this warp's array of free blocks in shared memory
    if (cls == small_class() && ws.sm->nsfree > 0) {
        const unsigned long long off = ws.sm->sfree[--ws.sm->nsfree];
        if ((off & 15ull) != 0 || off + size > P.arena_cap) {
            check_fail(P, 13, off); // a free block outside the arena
            return ~0ull;
        }
        return off;
    }
    // this warp's own free list: blocks it freed itself, no other warp touches it
    if (ws.sm->fcount[cls] > 0) {
        unsigned long long off = (ws.sm->fhead[cls] - 1) * 16;
        if (ws.sm->fhead[cls] == 0 || off + size > P.arena_cap) {
            check_fail(P, 13, off); // a private list that points outside the arena
            return ~0ull;
        }
        ws.sm->fhead[cls] = *(unsigned long long*)(P.arena + off) & kOffMask;
        ws.sm->fcount[cls]--;
        ((TaskHdr*)(P.arena + off))->refs = 0;
        return off;
    }
    unsigned long long* head = &P.ctl->free_head[cls * kArenaShards + (blockIdx.x % kArenaShards)];
    for (int tries = 0; tries < 256; tries++) {
        unsigned long long h = *(volatile unsigned long long*)head;
        unsigned long long idx = h & kOffMask;
        if (idx == 0) break;
        unsigned long long off = (idx - 1) * 16;
        {
            unsigned long long lim0 = *(volatile unsigned long long*)&P.ctl->arena_top;
            if (lim0 > P.ctl->arena_cap) lim0 = P.ctl->arena_cap;
            if (off + size > lim0) {
                check_fail(P, 12, off); // a list head outside the arena: never read through it
                return ~0ull;
            }
        }
        // acquire: the block's link word must be read after the head that
        // published it, or a stale link could be installed as the new head
        __threadfence();
        unsigned long long next = *(volatile unsigned long long*)(P.arena + off) & kOffMask;
        unsigned long long nh = (((h >> 40) + 1) << 40) | next;
        if (atomicCAS(head, h, nh) == h) {
            unsigned long long lim = *(volatile unsigned long long*)&P.ctl->arena_top;
            if (lim > P.ctl->arena_cap) lim = P.ctl->arena_cap;
            if ((off & 15ull) != 0 || off + size > lim || (next && (next - 1) * 16 + 16 > lim)) {
                check_fail(P, 7, off); // a corrupted list: report it, never write through it
                return ~0ull;
            }
            int mark = ((volatile TaskHdr*)(P.arena + off))->refs;
            if (mark != kFreeMagic) {
                check_fail(P, 9, off); // handed out a block that is not free
                return ~0ull;
            }
            ((volatile TaskHdr*)(P.arena + off))->refs = 0;
            __threadfence();
            return off;
        }
    }
    unsigned long long at = atomicAdd(&P.ctl->arena_top, size);
    if (at + size > P.ctl->arena_cap) {
        set_status(P, ST_TASK_OVERFLOW);
        return ~0ull;
    }
    return at;
}

// lane 0: a block for a record of `bytes` (class in `cls`); ~0 on failure.
// A reused block's old contents no longer stand for the warp's newest child.
__device__ unsigned long long arena_alloc(const ExpandParams& P, Ws& ws, unsigned long long bytes, int& cls)
{
    const unsigned long long off = arena_block(P, ws, bytes, cls);
    if (off == ws.sm->hot_rec) ws.sm->hot_rec = ~0ull;
    return off;
}

// lane 0: return a block.  It goes to this warp's private list (reused by the
// warp's next allocation of the class, without atomics) until that list holds
// kPrivateFreeCap blocks; beyond that, to the shared lock-free list.
__device__ void arena_free(const ExpandParams& P, Ws& ws, unsigned long long off, int cls)
{
    if (cls == small_class() && ws.sm->nsfree < kSmallFree) {
        ((TaskHdr*)(P.arena + off))->refs = kFreeMagic; // a stale item on it fails its check
        ws.sm->sfree[ws.sm->nsfree++] = off;
        return;
    }
    if (ws.sm->fcount[cls] < kPrivateFreeCap) {
        *(unsigned long long*)(P.arena + off) = ws.sm->fhead[cls];
        ((TaskHdr*)(P.arena + off))->refs = kFreeMagic;
        ws.sm->fhead[cls] = off / 16 + 1;
        ws.sm->fcount[cls]++;
        return;
    }
    unsigned long long* head = &P.ctl->free_head[cls * kArenaShards + (blockIdx.x % kArenaShards)];
    for (int tries = 0; tries < (1 << 20); tries++) {
        unsigned long long h = *(volatile unsigned long long*)head;
        *(volatile unsigned long long*)(P.arena + off) = h & kOffMask;
        ((volatile TaskHdr*)(P.arena + off))->refs = kFreeMagic;
        __threadfence();
        unsigned long long nh = (((h >> 40) + 1) << 40) | (off / 16 + 1);
        if (atomicCAS(head, h, nh) == h) return;
    }
    // contention beyond any plausible bound: keep the block (a leak, not a fault)
}

// a work item on this record is finished; the last one frees the block.
// `sole`: no other work item ever referenced the record (a task processed
// whole by one warp), so the reference count needs no atomic.
// `hv` is the record's header as validated when the item was dequeued.
__device__ void release_record(const ExpandParams& P, Ws& ws, unsigned long long rec, bool sole,
                               const TaskHdr& hv)
{
    TaskHdr* h = (TaskHdr*)(P.arena + rec);
    int cls = hv.cls;
    if (sole) {
        if (hv.refs != 1) {
            check_fail(P, 14, rec); // a record thought to be private has other users
            return;
        }
        arena_free(P, ws, rec, cls);
        return;
    }
    __threadfence();
    int before = atomicSub(&h->refs, 1);
    if (before == 1) arena_free(P, ws, rec, cls);
    else if (before < 1 || before == kFreeMagic) check_fail(P, 10, rec); // released too often
}

// ------------------------------------------------------------------
// child task: Q-sort (main.cu:2059-2104) and compacted matrices
// ------------------------------------------------------------------

// key: members first; then indeg desc, exdeg desc, l2 desc, id desc.
__device__ __forceinline__ bool key_less(unsigned long long ah, unsigned long long al,
                                         unsigned long long bh, unsigned long long bl)
{
    return ah < bh || (ah == bh && al < bl);
}

// Warp bitonic sort of n (key_hi, key_lo, sel) entries in the workspace.
__device__ QC_BIG_FN void sort_keys(Ws& ws, int n)
{
    int lane = lane_id();
    int N = 1;
    while (N < n) N <<= 1;
    #pragma unroll 1
    for (int i = n + lane; i < N; i += 32) {
        ws.khi()[i] = ~0ull;
        ws.klo()[i] = ~0ull;
        ws.sel()[i] = -1;
    }
    __syncwarp();
    #pragma unroll 1
    for (int k = 2; k <= N; k <<= 1) {
        #pragma unroll 1
        for (int j = k >> 1; j > 0; j >>= 1) {
            #pragma unroll 1
            for (int i = lane; i < N; i += 32) {
                int p = i ^ j;
                if (p > i) {
                    bool up = (i & k) == 0;
                    unsigned long long ah = ws.khi()[i], al = ws.klo()[i];
                    unsigned long long bh = ws.khi()[p], bl = ws.klo()[p];
                    bool gt = key_less(bh, bl, ah, al);
                    if (gt == up) {
                        ws.khi()[i] = bh; ws.klo()[i] = bl;
                        ws.khi()[p] = ah; ws.klo()[p] = al;
                        int s = ws.sel()[i]; ws.sel()[i] = ws.sel()[p]; ws.sel()[p] = s;
                    }
                }
            }
            __syncwarp();
        }
    }
}

__device__ QC_BIG_FN void write_child(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws, const uint32_t* M,
                            int m, const uint32_t* Rm, int nr)
{
    int lane = lane_id();
    int tc = m + nr;
    if (tc > P.max_t) {
        if (lane == 0) set_status(P, ST_TOO_LARGE);
        return;
    }
    // gather (key, position)
    int written = 0;
    #pragma unroll 1
    for (int base = 0; base < T.t; base += 32) {
        int v = base + lane;
        bool isM = v < T.t && bit(M, v);
        bool isR = v < T.t && bit(Rm, v);
        bool in = isM || isR;
        unsigned bal = __ballot_sync(QC_FULL, in);
        if (in) {
            int r = written + __popc(bal & ((1u << lane) - 1u));
            unsigned long long cls = isM ? 0ull : 1ull;
            unsigned long long in_k = 0xffffull - (unsigned long long)ws.indeg()[v];
            unsigned long long ex_k = 0xffffull - (unsigned long long)ws.exdeg()[v];
            unsigned long long l2_k = 0xffffull - (unsigned long long)rec_ld(T.l2 + v);
            ws.khi()[r] = (cls << 48) | (in_k << 32) | (ex_k << 16) | l2_k;
            ws.klo()[r] = 0xffffffffull - (unsigned long long)(unsigned)rec_ld(T.ids + v);
            ws.sel()[r] = v;
        }
        written += __popc(bal);
    }
    __syncwarp();
    // The child's order.  A child of up to kRankOrderMax vertices: each
    // vertex's place is the number of smaller keys (the keys are distinct:
    // they end in the id), with the keys read by all lanes at once; a larger
    // one: the bitonic sort of the keys.
    const int32_t* order = ws.sel();
    if (tc <= kRankOrderMax) {
        int32_t* dst = ws.vlist();
        #pragma unroll 1
        for (int e = lane; e < tc; e += 32) {
            const unsigned long long h = ws.khi()[e], l = ws.klo()[e];
            int r = 0;
            for (int j = 0; j < tc; j++) {
                const unsigned long long hj = ws.khi()[j], lj = ws.klo()[j];
                r += (hj < h || (hj == h && lj < l)) ? 1 : 0;
            }
            dst[r] = ws.sel()[e];
        }
        __syncwarp();
        order = dst;
    } else {
        sort_keys(ws, tc);
    }
    int Wc = words_for(tc);
    unsigned long long bytes = rec_block_bytes(tc, Wc);
    unsigned long long at = 0;
    int cls = 0;
    if (lane == 0) at = arena_alloc(P, ws, bytes, cls);
    at = __shfl_sync(QC_FULL, at, 0);
    if (at == ~0ull) return;
    char* rec = P.arena + at;
    if (lane == 0) {
        TaskHdr* h = (TaskHdr*)rec;
        h->t = tc;
        h->m = m;
        h->cov = 0;
        h->W = Wc;
        h->refs = 1;
        h->cls = cls;
        h->inst = T.inst;
        h->flags = 0;
    }
    int32_t* cid = (int32_t*)(rec + rec_ids_off());
    int32_t* cl2 = (int32_t*)(rec + rec_l2_off(tc));
    uint32_t* c1 = (uint32_t*)(rec + rec_a1_off(tc));
    uint32_t* c2 = (uint32_t*)(rec + rec_a2_off(tc, Wc));
    #pragma unroll 1
    for (int i = lane; i < tc; i += 32) {
        cid[i] = rec_ld(T.ids + order[i]);
        cl2[i] = 0;
    }
    // compacted rows: child bit j of row i = parent bit order[j] of row
    // order[i].  A parent of at most 8 words a row: lane r takes child row
    // i0 + r, holds its parent row's words in registers and picks the child's
    // columns from them, the columns' parent positions passed round the warp.
    if (T.W <= 8) {
        #pragma unroll 1
        for (int i0 = 0; i0 < tc; i0 += 32) {
            const int row = i0 + lane;
            const int src = row < tc ? order[row] : -1;
            uint32_t a1w[8], a2w[8];
#pragma unroll
            for (int w = 0; w < 8; w++) {
                const bool ok = src >= 0 && w < T.W;
                a1w[w] = ok ? rec_ld(T.A1 + (int64_t)src * T.W + w) : 0u;
                a2w[w] = ok ? rec_ld(T.A2 + (int64_t)src * T.W + w) : 0u;
            }
            for (int cw = 0; cw < Wc; cw++) {
                const int jn = tc - cw * 32 < 32 ? tc - cw * 32 : 32;
                const int my_col = lane < jn ? order[cw * 32 + lane] : 0;
                uint32_t o1 = 0, o2 = 0;
                for (int b = 0; b < jn; b++) {
                    const int pj = __shfl_sync(QC_FULL, my_col, b);
                    const int pw = pj >> 5, pb = pj & 31;
                    uint32_t x1 = a1w[0], x2 = a2w[0];
#pragma unroll
                    for (int w = 1; w < 8; w++)
                        if (pw == w) {
                            x1 = a1w[w];
                            x2 = a2w[w];
                        }
                    o1 |= ((x1 >> pb) & 1u) << b;
                    o2 |= ((x2 >> pb) & 1u) << b;
                }
                if (row < tc) {
                    c1[(int64_t)row * Wc + cw] = o1;
                    c2[(int64_t)row * Wc + cw] = o2;
                }
            }
        }
    } else {
        // Column word w: lane k holds the parent column order[w*32+k]; rows go by in
        // groups of 32 (lane r holds the parent row of child row i0+r), and the
        // reads of different rows do not depend on each other.
        for (int w = 0; w < Wc; w++) {
            const int j = w * 32 + lane;
            const int pj = j < tc ? order[j] : 0;
            const int pw = pj >> 5, pb = pj & 31;
            const bool col = j < tc;
            #pragma unroll 1
            for (int i0 = 0; i0 < tc; i0 += 32) {
                const int rows = tc - i0 < 32 ? tc - i0 : 32;
                const int my_row = lane < rows ? order[i0 + lane] : 0;
                unsigned o1 = 0, o2 = 0;
    #pragma unroll 4
                for (int r = 0; r < rows; r++) {
                    const int64_t base = (int64_t)__shfl_sync(QC_FULL, my_row, r) * T.W + pw;
                    const uint32_t x1 = col ? rec_ld(T.A1 + base) : 0u;
                    const uint32_t x2 = col ? rec_ld(T.A2 + base) : 0u;
                    const unsigned w1 = __ballot_sync(QC_FULL, (x1 >> pb) & 1u);
                    const unsigned w2 = __ballot_sync(QC_FULL, (x2 >> pb) & 1u);
                    if (lane == r) {
                        o1 = w1;
                        o2 = w2;
                    }
                }
                if (lane < rows) {
                    c1[(int64_t)(i0 + lane) * Wc + w] = o1;
                    c2[(int64_t)(i0 + lane) * Wc + w] = o2;
                }
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        ws.sm->cnt.children++;
        ws.sm->cnt.child_vertices += (unsigned long long)tc;
        schedule_child(P, ws, at, tc, m, Wc, cls, T.inst, 0);
    }
    __syncwarp();
}

// ------------------------------------------------------------------
// one branch: add parent position q (main.cu:1086-1178)
// ------------------------------------------------------------------

__device__ void branch_rest_small(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws,
                                  const uint32_t* M, int m1, const uint32_t* Rm, const Bounds& b);

__device__ QC_BIG_FN void expand_branch(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws, int q)
{
    const int t = T.t, W = T.W;
    int lane = lane_id();
    uint32_t* M = ws.mk(MK_M);
    uint32_t* PRE = ws.mk(MK_PRE);
    uint32_t* D = ws.mk(MK_D);
    uint32_t* Rm = ws.mk(MK_R);
    uint32_t* CA = ws.mk(MK_CA);
    uint32_t* Kc = ws.mk(MK_K);

    // members M u {q}; candidates before q
    bs_range(M, W, 0, T.m);
    if (lane == 0) M[q >> 5] |= 1u << (q & 31);
    __syncwarp();
    bs_range(PRE, W, T.m, q);
    int m1 = T.m + 1;
    // diameter pruning (main.cu:1709-1732): PRE & N2(q)
    const uint32_t* r2q = T.A2 + (int64_t)q * W;
    #pragma unroll 1
    for (int w = lane; w < W; w += 32) D[w] = PRE[w] & rec_ld(r2q + w);
    __syncwarp();
    if (lane == 0) {
        ws.sm->cnt.branches++;
        ws.sm->cnt.parent_vertices += (unsigned long long)(q + 1);
    }
    // degrees for members and PRE (add one vertex, main.cu:1465-1492); only the
    // members and the candidates that survive the diameter test are ever read
    {
        uint32_t* MD = ws.mk(MK_U);
        #pragma unroll 1
        for (int w = lane; w < W; w += 32) MD[w] = M[w] | D[w];
        __syncwarp();
        int n = compact(ws, MD, t);
        // members are positions [0, m) and q, the earlier candidates [m, q):
        // both counts come from the row's words up to q's, read once
        const int mt = T.m, qw = q >> 5;
        #pragma unroll 1
        for (int i = lane; i < n; i += 32) {
            int v = ws.vlist()[i];
            const uint32_t* row = T.A1 + (int64_t)v * W;
            int in = 0, ex = 0;
            for (int w = 0; w <= qw; w++) {
                const uint32_t x = rec_ld(row + w);
                in += __popc(x & range_word(w, 0, mt));
                ex += __popc(x & range_word(w, mt, q));
            }
            in += (int)((rec_ld(row + qw) >> (q & 31)) & 1u);
            ws.indeg()[v] = in;
            ws.exdeg()[v] = ex;
        }
        __syncwarp();
    }

    Bounds b = {0, 0, 0};
    const int dp = degree_prune(P, R, T, ws, M, m1, PRE, D, Rm, b, P.small_path != 0);
    if (dp == DP_INVALID) {
        if (m1 >= R.min_size) check_clique(P, R, T, ws, M, m1);
        return;
    }
    // the rest on the register path once members and candidates fit a warp
    // (a converged pruning repeats one round there, which removes nothing)
    if (dp == DP_SWITCH || (P.small_path && m1 + bs_count(Rm, W) <= 32)) {
        branch_rest_small(P, R, T, ws, M, m1, Rm, b);
        return;
    }

    // critical-vertex pruning (main.cu:1526-1707)
    int critv = md_at(R, m1 + b.L);
    #pragma unroll 1
    for (int base = 0; base < t; base += 32) {
        int v = base + lane;
        bool k = v < t && bit(M, v) && ws.indeg()[v] + ws.exdeg()[v] == critv && ws.exdeg()[v] > 0;
        unsigned bal = __ballot_sync(QC_FULL, k);
        if (lane == 0) Kc[base >> 5] = bal;
    }
    #pragma unroll 1
    for (int w = words_for(t) + lane; w < W; w += 32) Kc[w] = 0;
    __syncwarp();
    // CA = R & OR over critical members of A1 rows
    #pragma unroll 1
    for (int w = lane; w < W; w += 32) {
        uint32_t acc = 0;
        #pragma unroll 1
        for (int base = 0; base < t; base += 32) {
            uint32_t kw = Kc[base >> 5];
            while (kw) {
                int v = base + __ffs(kw) - 1;
                kw &= kw - 1;
                acc |= rec_ld(T.A1 + (int64_t)v * W + w);
            }
        }
        CA[w] = acc & Rm[w];
    }
    __syncwarp();
    int nca = bs_count(CA, W);
    int m2 = m1;
    uint32_t* C2 = ws.mk(MK_C);
    uint32_t* D2 = ws.mk(MK_D);
    if (nca > 0) {
        // add the critical-adjacent candidates; 2-hop counts to them
        int bad = 0;
        #pragma unroll 1
        for (int base = 0; base < t; base += 32) {
            int v = base + lane;
            if (v < t && (bit(M, v) || bit(Rm, v))) {
                int d = popc_and(T.A1 + (int64_t)v * W, CA, W);
                ws.indeg()[v] += d;
                ws.exdeg()[v] -= d;
                int a = popc_and(T.A2 + (int64_t)v * W, CA, W);
                ws.aux()[v] = a;
                if (bit(M, v) && a != nca) bad = 1;
                if (bit(CA, v) && a < nca - 1) bad = 1;
            }
        }
        if (__any_sync(QC_FULL, bad)) return;
        #pragma unroll 1
        for (int w = lane; w < W; w += 32) {
            M[w] |= CA[w];
            C2[w] = Rm[w] & ~CA[w];
        }
        __syncwarp();
        m2 = m1 + nca;
        // diameter pruning against the added vertices (main.cu:1689-1697)
        #pragma unroll 1
        for (int base = 0; base < t; base += 32) {
            int v = base + lane;
            bool in = v < t && bit(C2, v) && ws.aux()[v] == nca;
            unsigned bal = __ballot_sync(QC_FULL, in);
            if (lane == 0) D2[base >> 5] = bal;
        }
        #pragma unroll 1
        for (int w = words_for(t) + lane; w < W; w += 32) D2[w] = 0;
        __syncwarp();
    } else {
        bs_copy(C2, Rm, W);
        bs_copy(D2, Rm, W);
    }
    uint32_t* R2 = ws.mk(MK_R);
    Bounds b2 = {0, 0, 0};
    bool fail2 = degree_prune(P, R, T, ws, M, m2, C2, D2, R2, b2, false) == DP_INVALID;
    if (m2 >= R.min_size) check_clique(P, R, T, ws, M, m2);
    if (fail2) return;
    int nr = bs_count(R2, W);
    if (nr > 0) write_child(P, R, T, ws, M, m2, R2, nr);
}

// ------------------------------------------------------------------
// register-resident path for tasks of at most 32 vertices (the bulk of the
// search tree): lane v holds vertex v's id, 1-hop row and 2-hop row; every
// vertex set is one 32-bit word, identical in all lanes.
// ------------------------------------------------------------------

__device__ __forceinline__ int rmin(int x)
{
#ifdef QC_EMULATION
    return wmin(x);
#else
    return __reduce_min_sync(QC_FULL, x);
#endif
}
__device__ __forceinline__ int rmax(int x)
{
#ifdef QC_EMULATION
    return wmax(x);
#else
    return __reduce_max_sync(QC_FULL, x);
#endif
}
__device__ __forceinline__ int radd(int x)
{
#ifdef QC_EMULATION
    return wsum(x);
#else
    return __reduce_add_sync(QC_FULL, x);
#endif
}
__device__ __forceinline__ unsigned ror(unsigned x)
{
#ifdef QC_EMULATION
    for (int o = 16; o; o >>= 1) x |= __shfl_xor_sync(QC_FULL, x, o);
    return x;
#else
    return __reduce_or_sync(QC_FULL, x);
#endif
}

__device__ __forceinline__ bool in_set(unsigned s, int lane) { return (s >> lane) & 1u; }
__device__ __forceinline__ unsigned low_mask(int k) { return k >= 32 ? ~0u : ((1u << k) - 1u); }

struct SmallTask {
    int t, m, cov, inst, id, l2;
    unsigned a1, a2;
    int rows; // deg + |N2| of this lane's vertex (work accounting only)
    int idr;  // lanes of the task with a larger id than this lane's
};

// Sum of the k largest values `in` of the lanes in `cs` (0 for k = 0, all
// of them for k >= popc(cs)), for each lane's own k: a radix select over the
// values' bits (values 0..63) on six ballots, with no data exchange between
// the lanes after them.  The select keeps `gt` (lanes whose value is above
// the k-th largest) and narrows `eq` to the lanes equal to it so far.
__device__ __forceinline__ int top_k_sum(unsigned cs, int in, int k)
{
    const bool c = in_set(cs, lane_id());
    unsigned B[6];
#pragma unroll
    for (int b = 0; b < 6; b++) B[b] = __ballot_sync(QC_FULL, c && ((in >> b) & 1));
    unsigned eq = cs, gt = 0;
    int x = 0;
#pragma unroll
    for (int b = 5; b >= 0; b--) {
        const unsigned hi = eq & B[b];
        if (__popc(gt) + __popc(hi) >= k) {
            x |= 1 << b;
            eq = hi;
        } else {
            gt |= hi;
            eq &= ~B[b];
        }
    }
    int sum = 0;
#pragma unroll
    for (int b = 0; b < 6; b++) sum += __popc(gt & B[b]) << b;
    return sum + (k - __popc(gt)) * x;
}

// LU bounds (main.cu:1857-1972) for members set M (m of them) and the
// candidate indegree multiset given by lanes in `cs` with value `in`.
__device__ QC_SMALL_FN bool lu_small(const ExpandParams& P, const Rules& R, unsigned M, int m, unsigned cs, int in, int ex,
                         Bounds& b)
{
    int lane = lane_id();
    bool mem = in_set(M, lane);
    int min_in = rmin(mem ? in : 0x7fffffff);
    int min_tot = rmin(mem ? in + ex : 0x7fffffff);
    int sum_in = radd(mem ? in : 0);
    int min_in_ex = rmin(mem && in == min_in ? ex : 0x7fffffff);
    int ncand = __popc(cs);
    bool invalid = false;
    b.med = mindeg<true>(R, m + 1);
    if (min_in < md_at<true>(R, m)) {
        int lb = mindeg<true>(R, m) - min_in;
        #pragma unroll 1
        for (int base = lb;; base += 32) {
            int L = base + lane;
            bool cont = (L <= min_in_ex) && (min_in + L < md_at<true>(R, m + L));
            unsigned stop = __ballot_sync(QC_FULL, !cont);
            if (stop) {
                lb = base + __ffs(stop) - 1;
                break;
            }
        }
        if (min_in + lb < md_at<true>(R, m + lb)) {
            lb = ncand + 1;
            invalid = true;
        }
        int ub = ubt_at<true>(R, min_tot) + 1 - m;
        if (ub > ncand) ub = ncand;
        if (lb < ub) {
            // S(k) for k = lane: sum of the k largest candidate indegrees
            // (indegrees within at most 32 members: 0..31)
            const int excl = top_k_sum(cs, in, lane);
            // g(k) for k in [lb, ub] (ub <= 31): k == ub or sum_in + S(k) >= m*md[m+k]
            int k = lane;
            long long Sk = excl;
            bool g = (k >= lb && k <= ub) &&
                     (k == ub || (long long)sum_in + Sk >= (long long)m * md_at<true>(R, m + k));
            unsigned bal = __ballot_sync(QC_FULL, g);
            int idx = bal ? __ffs(bal) - 1 : ub;
            // idx <= ub <= ncand < 32: a task of at most 32 vertices has a member
            long long Sidx = __shfl_sync(QC_FULL, excl, idx & 31);
            if ((long long)sum_in + Sidx < (long long)m * md_at<true>(R, m + idx)) {
                lb = ub + 1;
                invalid = true;
            } else {
                lb = idx;
                bool g2 = (k > idx && k <= ub) &&
                          ((long long)sum_in + Sk >= (long long)m * md_at<true>(R, m + k));
                unsigned b2 = __ballot_sync(QC_FULL, g2);
                int tub = b2 ? 31 - __clz(b2) : idx;
                if (ub > tub) ub = tub;
                if (lb > 1) b.med = mindeg<true>(R, m + lb);
            }
        }
        b.U = ub;
        b.L = lb;
    } else {
        b.U = ncand;
        b.L = m < R.min_size ? R.min_size - m : 0;
    }
    if (m + b.U < R.min_size) invalid = true;
    if (b.U < 0 || b.U < b.L) invalid = true;
    return invalid;
}

// the rounds of the degree pruning fixpoint after the first: entered with
// the surviving candidates Rm and the removed set X (non-empty), both words
__device__ QC_SMALL_FN bool prune_loop_small(const ExpandParams& P, const Rules& R, unsigned a1, unsigned M, int m,
                                 unsigned& Rm, unsigned X, int in, int& ex, Bounds& b)
{
    int lane = lane_id();
    while (Rm && X) {
        ex = __popc(a1 & Rm);
        unsigned V = __ballot_sync(QC_FULL, in_set(Rm, lane) && cand_valid<true>(R, in, ex, m, b));
        if (lu_small(P, R, M, m, V, in, ex, b)) return true;
        if (__any_sync(QC_FULL, in_set(M, lane) && !vert_extendable<true>(R, in, ex, m, b))) return true;
        unsigned R2 = __ballot_sync(QC_FULL, in_set(Rm, lane) && cand_valid<true>(R, in, ex, m, b));
        X = Rm & ~R2;
        Rm = R2;
    }
    return false;
}

// degree pruning fixpoint (main.cu:1735-1855) on words; `ex` is updated in place
__device__ bool prune_small(const ExpandParams& P, const Rules& R, unsigned a1, unsigned M, int m, unsigned Call,
                            unsigned D, unsigned& Rm, int in, int& ex, Bounds& b)
{
    int lane = lane_id();
    if (lu_small(P, R, M, m, D, in, ex, b)) return true;
    if (__any_sync(QC_FULL, in_set(M, lane) && !vert_extendable<true>(R, in, ex, m, b))) return true;
    Rm = __ballot_sync(QC_FULL, in_set(D, lane) && cand_valid<true>(R, in, ex, m, b));
    return prune_loop_small(P, R, a1, M, m, Rm, Call & ~Rm, in, ex, b);
}

// Whole warp: append the buffered sets to the result buffer under one
// reservation of result ints and one of set indices.
__device__ QC_SMALL_FN void emit_flush(const ExpandParams& P, Ws& ws)
{
    const int lane = lane_id();
    __syncwarp();
    const int n = ws.sm->en, ns = ws.sm->es;
    if (n == 0) return;
    unsigned long long at = 0, idx = 0;
    if (lane == 0) {
        at = atomicAdd(&P.ctl->result_top, (unsigned long long)n);
        idx = atomicAdd(&P.ctl->emitted, (unsigned long long)ns);
        if (at + n > P.ctl->result_cap || idx + ns > P.ctl->set_cap) {
            set_status(P, ST_RESULT_OVERFLOW);
            at = ~0ull;
        }
    }
    at = __shfl_sync(QC_FULL, at, 0);
    idx = __shfl_sync(QC_FULL, idx, 0);
    if (at != ~0ull) {
        #pragma unroll 1
        for (int i = lane; i < n; i += 32) P.results[at + i] = ws.sm->ebuf[i];
        #pragma unroll 1
        for (int j = lane; j < ns; j += 32) P.set_starts[idx + j] = at + ws.sm->eset[j];
    }
    __syncwarp();
    if (lane == 0) {
        ws.sm->en = 0;
        ws.sm->es = 0;
    }
    __syncwarp();
}

// Whole warp: buffer the set of lanes in S (ids `id`, at most 32 of them)
__device__ void emit_small(const ExpandParams& P, const Rules& R, Ws& ws, unsigned S, int id)
{
    const int lane = lane_id();
    const int k = __popc(S);
    if (ws.sm->en + k + 1 > kEmitInts || ws.sm->es >= kEmitSets) emit_flush(P, ws);
    const int base = ws.sm->en;
    __syncwarp(); // every lane has read `en` before lane 0 moves it
    if (in_set(S, lane)) ws.sm->ebuf[base + 1 + __popc(S & low_mask(lane))] = id + R.vbase;
    if (lane == 0) {
        ws.sm->ebuf[base] = k;
        ws.sm->eset[ws.sm->es] = base;
        ws.sm->en = base + k + 1;
        ws.sm->es += 1;
    }
    __syncwarp();
}

__device__ __forceinline__ void clique_small(const ExpandParams& P, const Rules& R, Ws& ws, unsigned M, int m, int in,
                                             int id)
{
    int lane = lane_id();
    int need = md_at<true>(R, m);
    if (!__any_sync(QC_FULL, in_set(M, lane) && in < need)) emit_small(P, R, ws, M, id);
}

// child record of the vertices in M2 | R2, Q-sorted, matrices compacted
__device__ QC_SMALL_FN void child_small(const ExpandParams& P, const Rules& R, Ws& ws, const SmallTask& T, unsigned M2, int m2,
                            unsigned R2, int in, int ex)
{
    int lane = lane_id();
    unsigned S = M2 | R2;
    int tc = __popc(S);
    // child order (main.cu cmp of the Q sort): members first, then indegree,
    // exdegree and two-hop count descending, then id descending.  Within a
    // task of at most 32 vertices each count is 0..31 and T.idr ranks the ids,
    // so the whole key and the source lane fit one 32-bit word.
    unsigned key = ~0u;
    if (in_set(S, lane)) {
        const unsigned cls = in_set(M2, lane) ? 0u : 1u;
        key = (cls << 25) | ((unsigned)(31 - in) << 20) | ((unsigned)(31 - ex) << 15) |
              ((unsigned)(31 - T.l2) << 10) | ((unsigned)T.idr << 5) | (unsigned)lane;
    }
    // bitonic sort ascending
    #pragma unroll 1
    for (int k = 2; k <= 32; k <<= 1)
        #pragma unroll 1
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned o = __shfl_xor_sync(QC_FULL, key, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            const bool take_min = (lower == up);
            if (take_min != (key < o)) key = o;
        }
    int src = (int)(key & 31u);
    unsigned sa1 = __shfl_sync(QC_FULL, T.a1, src);
    unsigned sa2 = __shfl_sync(QC_FULL, T.a2, src);
    int sid = __shfl_sync(QC_FULL, T.id, src);
    // the child's id ranks from the parent's: a rank counts the larger ids,
    // parent ranks are distinct, so a child vertex's rank counts the child's
    // parent ranks below its own
    const int prank = __shfl_sync(QC_FULL, T.idr, src);
    const unsigned ranks = ror(lane < tc ? 1u << prank : 0u);
    const int crank = __popc(ranks & ((1u << prank) - 1u));
    unsigned c1 = 0, c2 = 0;
    for (int j = 0; j < tc; j++) {
        int pj = __shfl_sync(QC_FULL, src, j);
        c1 |= ((sa1 >> pj) & 1u) << j;
        c2 |= ((sa2 >> pj) & 1u) << j;
    }
    unsigned long long bytes = rec_block_bytes(tc, 1);
    unsigned long long at = 0;
    int cls = 0;
    if (lane == 0) at = arena_alloc(P, ws, bytes, cls);
    at = __shfl_sync(QC_FULL, at, 0);
    if (at == ~0ull) return;
    char* rec = P.arena + at;
    if (lane == 0) {
        TaskHdr* h = (TaskHdr*)rec;
        h->t = tc;
        h->m = m2;
        h->cov = 0;
        h->W = 1;
        h->refs = 1;
        h->cls = cls;
        h->inst = T.inst;
        h->flags = kFlagRanked;
    }
    if (lane < tc) {
        ((int32_t*)(rec + rec_ids_off()))[lane] = sid;
        ((int32_t*)(rec + rec_l2_off(tc)))[lane] = 0;
        ((uint32_t*)(rec + rec_a1_off(tc)))[lane] = c1;
        ((uint32_t*)(rec + rec_a2_off(tc, 1)))[lane] = c2;
        ((uint8_t*)(rec + rec_ranks_off()))[lane] = (uint8_t)crank;
    }
    // the copy the warp reads if this child is its next task
    ws.sm->hot[lane] = HotLane{sid, c1, c2, crank};
    __syncwarp();
    if (lane == 0) {
        ws.sm->hot_rec = at;
        ws.sm->cnt.children++;
        ws.sm->cnt.child_vertices += (unsigned long long)tc;
        schedule_child(P, ws, at, tc, m2, 1, cls, T.inst, kFlagRanked);
    }
    __syncwarp();
}

__device__ void branch_tail_small(const ExpandParams& P, const Rules& R, Ws& ws, const SmallTask& T,
                                  unsigned M1, int m1, unsigned Rm, int in, int ex, const Bounds& b);

__device__ void branch_small(const ExpandParams& P, const Rules& R, Ws& ws, const SmallTask& T, int q)
{
    int lane = lane_id();
    unsigned Mm = low_mask(T.m);
    unsigned M1 = Mm | (1u << q);
    int m1 = T.m + 1;
    unsigned PRE = low_mask(q) & ~Mm;
    int in = __popc(T.a1 & M1);
    int ex = __popc(T.a1 & PRE);
    unsigned r2q = __shfl_sync(QC_FULL, T.a2, q);
    unsigned D = PRE & r2q;
    {
        const int rows = __shfl_sync(QC_FULL, T.rows, q);
        if (lane == 0) {
            ws.sm->cnt.branches++;
            ws.sm->cnt.parent_vertices += (unsigned long long)(q + 1);
            ws.sm->cnt.p_rows += (unsigned long long)rows;
        }
    }
    // too few candidates survive the diameter test for any set of min_size
    // (the bounds test finds U <= |D| too small; no clique, m1 < min_size)
    if (m1 + __popc(D) < R.min_size) return;
    Bounds b = {0, 0, 0};
    unsigned Rm = 0;
    if (prune_small(P, R, T.a1, M1, m1, PRE, D, Rm, in, ex, b)) {
        if (m1 >= R.min_size) clique_small(P, R, ws, M1, m1, in, T.id);
        return;
    }
    branch_tail_small(P, R, ws, T, M1, m1, Rm, in, ex, b);
}

// The rest of a branch once its first degree pruning has converged: members
// M1 (m1 of them), candidates Rm, bounds b, degrees in/ex of this lane's
// vertex.  Critical vertices, second pruning, clique check, child.
__device__ QC_SMALL_FN void branch_tail_small(const ExpandParams& P, const Rules& R, Ws& ws, const SmallTask& T,
                                  unsigned M1, int m1, unsigned Rm, int in, int ex, const Bounds& b)
{
    int lane = lane_id();
    // critical vertices (main.cu:1526-1707)
    int critv = md_at<true>(R, m1 + b.L);
    unsigned K = __ballot_sync(QC_FULL, in_set(M1, lane) && in + ex == critv && ex > 0);
    unsigned CA = Rm & ror(in_set(K, lane) ? T.a1 : 0u);
    int nca = __popc(CA);
    unsigned M2 = M1, C2 = Rm, D2 = Rm;
    int m2 = m1;
    if (nca > 0) {
        int d = __popc(T.a1 & CA);
        in += d;
        ex -= d;
        int adj = __popc(T.a2 & CA);
        bool bad = (in_set(M1, lane) && adj != nca) || (in_set(CA, lane) && adj < nca - 1);
        if (__any_sync(QC_FULL, bad)) return;
        M2 = M1 | CA;
        m2 = m1 + nca;
        C2 = Rm & ~CA;
        D2 = __ballot_sync(QC_FULL, in_set(C2, lane) && adj == nca);
    }
    Bounds b2 = {0, 0, 0};
    unsigned R2 = 0;
    bool fail2 = prune_small(P, R, T.a1, M2, m2, C2, D2, R2, in, ex, b2);
    if (m2 >= R.min_size) clique_small(P, R, ws, M2, m2, in, T.id);
    if (fail2) return;
    if (R2) child_small(P, R, ws, T, M2, m2, R2, in, ex);
}

// A branch of a task over 32 vertices whose members M (m1 of them) and
// remaining candidates Rm number at most 32 while its degree pruning has
// rounds to go: the set S = M u Rm, in ascending positions, is compacted into
// the register form (lane i holds the i-th vertex of S and its 1-hop and 2-hop
// rows restricted to S) and the rest of the branch runs there.  Within S the
// children's order keys need ranks: of the ids, and of the task's lookahead
// 2-hop counts (which may exceed 31 in a large task).
__device__ QC_SMALL_FN void branch_rest_small(const ExpandParams& P, const Rules& R, const TaskView& T, Ws& ws,
                                  const uint32_t* M, int m1, const uint32_t* Rm, const Bounds& b)
{
    const int lane = lane_id();
    const int W = T.W;
    uint32_t* S = ws.mk(MK_U);
    #pragma unroll 1
    for (int w = lane; w < W; w += 32) S[w] = M[w] | Rm[w];
    __syncwarp();
    const int n = compact(ws, S, T.t); // m1 + |Rm| <= 32
    const bool act = lane < n;
    const int pos = act ? ws.vlist()[lane] : 0;
    SmallTask C;
    C.t = n;
    C.m = m1;
    C.cov = 0;
    C.inst = T.inst;
    C.rows = 0;
    C.id = act ? rec_ld(T.ids + pos) : -1;
    const int l2v = act ? rec_ld(T.l2 + pos) : -1;
    const uint32_t* r1 = T.A1 + (int64_t)pos * W;
    const uint32_t* r2 = T.A2 + (int64_t)pos * W;
    unsigned a1 = 0, a2 = 0;
    #pragma unroll 1
    for (int j = 0; j < n; j++) {
        const int pj = __shfl_sync(QC_FULL, pos, j);
        if (act) {
            a1 |= ((rec_ld(r1 + (pj >> 5)) >> (pj & 31)) & 1u) << j;
            a2 |= ((rec_ld(r2 + (pj >> 5)) >> (pj & 31)) & 1u) << j;
        }
    }
    C.a1 = a1;
    C.a2 = a2;
    int idr = 0, l2r = 0;
    #pragma unroll 1
    for (int j = 0; j < 32; j++) {
        const int oid = __shfl_sync(QC_FULL, C.id, j);
        const int ol2 = __shfl_sync(QC_FULL, l2v, j);
        if (j < n) {
            idr += oid > C.id ? 1 : 0;
            l2r += ol2 > l2v ? 1 : 0;
        }
    }
    C.idr = idr;
    C.l2 = 31 - l2r; // the child key orders by 31 - l2: the largest count first
    const unsigned Mc = __ballot_sync(QC_FULL, act && bit(M, pos));
    unsigned Rc = __ballot_sync(QC_FULL, act && bit(Rm, pos));
    int in = __popc(a1 & Mc);
    int ex = 0; // recounted by the next round
    Bounds bb = b;
    // the pending round: its removed set is non-empty (the big loop's test)
    if (prune_loop_small(P, R, a1, Mc, m1, Rc, ~0u, in, ex, bb)) {
        if (m1 >= R.min_size) clique_small(P, R, ws, Mc, m1, in, C.id);
        return;
    }
    branch_tail_small(P, R, ws, C, Mc, m1, Rc, in, ex, bb);
}

// Branches of a small task handed to waiting warps: a fresh task with at
// least this many branches is split when other warps wait for work.
#ifndef QC_SMALL_SPLIT_MIN
#define QC_SMALL_SPLIT_MIN 8
#endif
constexpr int kSmallSplitMin = QC_SMALL_SPLIT_MIN;
// waiting warps needed before a small task splits
#ifndef QC_SMALL_SPLIT_HUNGRY
#define QC_SMALL_SPLIT_HUNGRY 2
#endif
constexpr int kSmallSplitHungry = QC_SMALL_SPLIT_HUNGRY;
// at most this many branch ranges pushed by one task
constexpr int kSmallSplitMax = 16;
// fewest branches in one handed-out range
#ifndef QC_SMALL_SPLIT_PER
#define QC_SMALL_SPLIT_PER 4
#endif
constexpr int kSmallSplitPer = QC_SMALL_SPLIT_PER;

// A task of at most 32 vertices on the register path.  A fresh task
// (q_lo < 0) runs its lookahead and finds its branch range; when other warps
// wait for work it keeps the first part of its branches and pushes the rest
// as branch ranges (the record's l2 counts are written back first, since the
// children's order reads them).  A branch-range item (q_lo >= 0) of a split
// task runs its branches only.  Returns true when this call pushed branch
// ranges of the record, which is then shared.
__device__ QC_SMALL_FN bool process_small(const ExpandParams& P, const Rules& R, Ws& ws, const TaskView& V,
                              int q_lo, int q_hi, bool sroot, bool hot)
{
    int lane = lane_id();
    SmallTask T;
    T.t = V.t;
    T.m = V.m;
    T.cov = V.cov;
    T.inst = V.inst;
    bool act = lane < T.t;
    // id ranks among the task's ids, largest first (the children's order):
    // stored by the register path's writer, else counted below
    const bool ranked = hot || (V.flags & kFlagRanked) != 0;
    if (hot) {
        // the child this warp wrote last, from its copy in shared memory (a
        // fresh child: its l2 counts are still zero)
        const HotLane h = ws.sm->hot[lane];
        T.id = act ? h.id : -1;
        T.a1 = act ? h.a1 : 0u;
        T.a2 = act ? h.a2 : 0u;
        T.l2 = 0;
        T.idr = h.rank;
    } else {
        T.id = act ? rec_ld(V.ids + lane) : -1;
        T.a1 = act ? rec_ld(V.A1 + lane) : 0u;
        T.a2 = act ? rec_ld(V.A2 + lane) : 0u;
        T.l2 = act ? rec_ld(V.l2 + lane) : 0;
        T.idr = ranked && act ? (int)rec_ld((const uint8_t*)V.ids - rec_ids_off() + rec_ranks_off() + lane)
                              : 0;
    }
    if (__any_sync(QC_FULL, act && (T.id < 0 || T.id >= R.n))) {
        if (lane == 0) check_fail(P, 8, V.rec); // a vertex id outside the instance
        return false;
    }
    // issued now, first read by a branch after the lookahead has run
    T.rows = act ? (int)((R.off[T.id + 1] - R.off[T.id]) + (R.off2[T.id + 1] - R.off2[T.id])) : 0;
    const int t = T.t, m = T.m;
    unsigned Mm = low_mask(m), Cm = low_mask(t) & ~Mm;
    int in = __popc(T.a1 & Mm), ex = __popc(T.a1 & Cm);
    int qlo = q_lo, qhi = q_hi;
    bool pushed = false;
    if (q_lo < 0) {
        if (lane == 0) {
            ws.sm->cnt.tasks++;
            if ((unsigned long long)t > ws.sm->cnt.max_task) ws.sm->cnt.max_task = t;
        }
        // lookahead (main.cu:1349-1405)
        int need_t = md_at<true>(R, t);
        if (!__any_sync(QC_FULL, in_set(Mm, lane) && in + ex < need_t)) {
            int nc = t - m;
            if (in_set(Cm, lane)) T.l2 = __popc(T.a2 & Cm);
            bool bad = in_set(Cm, lane) && (T.l2 < nc - 1 || in + ex < need_t);
            if (!__any_sync(QC_FULL, bad)) {
                if (lane == 0) ws.sm->cnt.lookahead_hits++;
                if (!sroot || P.shard == 0) emit_small(P, R, ws, low_mask(t), T.id);
                return false;
            }
        }
        // branches run until a member would fail on removal (main.cu:1092-1099)
        int need = mindeg<true>(R, m);
        int pos = 0;
        if (in_set(Mm, lane)) {
            int k = need - in;
            if (k > 0) {
                unsigned x = T.a1 & Cm;
                #pragma unroll 1
                for (int s = 1; s < k; s++) x &= x - 1;
                pos = x ? __ffs(x) - 1 : t - 1;
            }
        }
        qlo = rmax(pos);
        qlo = qlo > m + T.cov ? qlo : m + T.cov;
        if (qlo > t - 1) return false;
        // run status as read when the previous item started (no round trip here)
        if (ws.sm->stat) return false;
        qhi = t - 1;
        // hand branch ranges to waiting warps (the waiting count was read when
        // this item started): nb branches in parts of `per`, this warp keeping
        // the first part (the highest positions, branched first)
        const int nb = qhi - qlo + 1;
        const int hungry = ws.sm->hungry;
        if (hungry >= kSmallSplitHungry && nb >= kSmallSplitMin) {
            int parts = hungry + 1;
            parts = parts > nb / kSmallSplitPer ? nb / kSmallSplitPer : parts;
            parts = parts > kSmallSplitMax + 1 ? kSmallSplitMax + 1 : parts;
            const int per = (nb + parts - 1) / parts;
            const int extra = (nb - per + per - 1) / per;
            if (extra > 0) {
                // the l2 counts of this task's record as the lookahead left them
                if (act) ((int32_t*)V.l2)[lane] = T.l2;
                __syncwarp();
                __threadfence();
                if (lane == 0) atomicAdd(&((TaskHdr*)(P.arena + V.rec))->refs, extra);
                __syncwarp();
                push_ranges(P, V.rec, qlo, qhi - per, per, extra);
                __syncwarp();
                if (lane == 0) ws.sm->hungry = hungry > extra ? hungry - extra : 0;
                __syncwarp();
                qlo = qhi - per + 1;
                pushed = true;
            }
        }
    } else if (ws.sm->stat) {
        return false;
    }
    if (!ranked) {
        #pragma unroll 1
        for (int j = 0; j < 32; j++) {
            const int o = __shfl_sync(QC_FULL, T.id, j);
            T.idr += (j < t && o > T.id) ? 1 : 0;
        }
    }
    #pragma unroll 1
    for (int q = qhi; q >= qlo; q--) {
        // a sharded search's root: only this shard's branches
        if (sroot && (t - 1 - q) % P.nshards != P.shard) continue;
        branch_small(P, R, ws, T, q);
        // children of this task can go to waiting warps before its last branch
        // when many warps wait (not for the odd one that will soon get work)
        if (q > qlo && ws.sm->hungry >= kEagerHungry) donate(P, ws, kEagerKeep);
    }
    return pushed;
}

#ifndef QC_EMULATION
__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}
// this warp's mbarrier for its bulk copies (one arrival: lane 0's)
__device__ __forceinline__ void stage_bar_init(WarpSmem* sm)
{
    if (lane_id() == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&sm->stage_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sm->stage_phase = 0;
    }
    __syncwarp();
}
// has the bulk copy of the given parity landed?
__device__ __forceinline__ bool stage_bar_done(WarpSmem* sm, int phase)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_addr(&sm->stage_bar)), "r"(phase)
                 : "memory");
    return ok != 0;
}
#endif

// Copy a record's body (ids, l2, A1, A2) into this warp's shared-memory
// buffer and point the view there.  On the device one bulk copy by the TMA
// unit (cp.async.bulk, global -> shared, completing on the warp's mbarrier;
// the body and both addresses are 16-byte multiples); in the CPU emulator
// 16-byte loads through L2.  Returns false if the copy did not land within
// the run's wait limit (the run then stops).
__device__ QC_BIG_FN bool stage_record(const ExpandParams& P, WarpSmem* sm, TaskView& T, char* buf)
{
    const char* src = P.arena + T.rec + rec_ids_off();
    const uint64_t body = rec_bytes(T.t, T.W) - rec_ids_off(); // multiple of 16
#if !defined(QC_EMULATION) && !defined(QC_STAGE_LOOP)
    const int phase = sm->stage_phase;
    if (lane_id() == 0) {
        // earlier reads of the buffer (generic proxy) and the record's writes
        // by other warps ordered before the copy (async proxy)
        asm volatile("fence.proxy.async;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_addr(&sm->stage_bar)), "r"((unsigned)body) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_addr(buf)), "l"(src), "r"((unsigned)body), "r"(smem_addr(&sm->stage_bar))
                     : "memory");
    }
    bool done = stage_bar_done(sm, phase);
    if (!done) {
        const unsigned long long t0 = now_ns();
        while (!(done = stage_bar_done(sm, phase))) {
            if (now_ns() - t0 > (unsigned long long)P.wait_ns) break;
        }
    }
    if (!__all_sync(QC_FULL, done)) {
        if (lane_id() == 0) {
            set_status(P, ST_ITER_LIMIT);
            P.ctl->wait_fail_where = 5;
        }
        // the copy may still land: wait for it once more, again bounded,
        // before the buffer can be reused
        const unsigned long long t1 = now_ns();
        while (!stage_bar_done(sm, phase) && now_ns() - t1 <= (unsigned long long)P.wait_ns) {
        }
        return false;
    }
    __syncwarp();
    if (lane_id() == 0) sm->stage_phase = phase ^ 1;
    __syncwarp();
#else
    const uint4* s4 = (const uint4*)src;
    uint4* d4 = (uint4*)buf;
    #pragma unroll 1
    for (uint64_t i = lane_id(); i < body / 16; i += 32) d4[i] = __ldcg(s4 + i);
    __syncwarp();
#endif
    char* b = buf - rec_ids_off(); // same offsets as in the record
    T.ids = (const int32_t*)(b + rec_ids_off());
    T.l2 = (int32_t*)(b + rec_l2_off(T.t));
    T.A1 = (const uint32_t*)(b + rec_a1_off(T.t));
    T.A2 = (const uint32_t*)(b + rec_a2_off(T.t, T.W));
    return true;
}

// ------------------------------------------------------------------
// a work item: fresh task (lookahead, branch range) or a branch range
// ------------------------------------------------------------------

// Returns true when other work items (branch ranges pushed here or earlier)
// share the record, so its release must go through the reference count.
//
// Tasks of 33..P.smem_t vertices run with their record and workspace in this
// warp's shared memory (`wss`, `stage`); larger ones use the global
// workspace `wsg` and read the record through L2.
__device__ bool process_item(const ExpandParams& P, Ws& wsg, Ws& wss, char* stage, const WorkItem& it,
                             const TaskHdr& hv, bool hot)
{
    TaskView T = task_view(P.arena, it.rec, hv);
    const int t = T.t, W = T.W, m = T.m;
    int lane = lane_id();
    const bool staged = stage != nullptr && t > 32 && t <= P.smem_t && t <= P.max_t;
    if (staged && !stage_record(P, wss.sm, T, stage)) return it.q_lo >= 0; // the run is stopping
    Ws ws = staged ? wss : wsg;
    Rules R = P.rules[T.inst];
    if (ws.sm->tab_inst != T.inst) {
        // refresh this warp's shared copy of the instance's gamma tables
        for (int k = lane; k < kTabCache; k += 32) {
            int kk = k < R.mdlen ? k : R.mdlen - 1;
            ws.sm->md[k] = __ldg(R.md + kk);
            ws.sm->ubt[k] = __ldg(R.ubt + kk);
        }
        __syncwarp();
        if (lane == 0) ws.sm->tab_inst = T.inst;
        __syncwarp();
    }
    R.md_s = ws.sm->md;
    R.ubt_s = ws.sm->ubt;
    R.md_min = md_at(R, R.min_size);
    bool shared = it.q_lo >= 0;
    if (!(t <= 32 && P.small_path)) { // the register path checks its own ids
        int bad = 0;
        for (int v = lane; v < t; v += 32) {
            int id = rec_ld(T.ids + v);
            if (id < 0 || id >= R.n) bad = 1;
        }
        if (__any_sync(QC_FULL, bad)) {
            if (lane == 0) check_fail(P, 8, it.rec);
            return shared;
        }
    }
    if (t > P.max_t) {
        if (lane == 0) set_status(P, ST_TOO_LARGE);
        return shared;
    }
    int q_lo = it.q_lo, q_hi = it.q_hi;
    // the root of a search split by its branches: this launch expands only the
    // branches of its own shard (and emits an accepted root in shard 0 only)
    const bool sroot = (hv.flags & kFlagShardRoot) != 0 && P.nshards > 1;
    if (t <= 32 && P.small_path) {
        if (process_small(P, R, ws, T, q_lo, q_hi, sroot, hot)) shared = true;
        return shared;
    }
    if (q_lo < 0) {
        if (lane == 0) {
            ws.sm->cnt.tasks++;
            if ((unsigned long long)t > ws.sm->cnt.max_task) ws.sm->cnt.max_task = t;
        }
        uint32_t* MM = ws.mk(MK_M);
        uint32_t* CC = ws.mk(MK_C);
        bs_range(MM, W, 0, m);
        bs_range(CC, W, m, t);
        int nc = t - m;
        // task degrees
        for (int base = 0; base < t; base += 32) {
            int v = base + lane;
            if (v < t) {
                const uint32_t* row = T.A1 + (int64_t)v * W;
                ws.indeg()[v] = popc_and(row, MM, W);
                ws.exdeg()[v] = popc_and(row, CC, W);
            }
        }
        __syncwarp();
        // lookahead (main.cu:1349-1405)
        int need_t = md_at(R, t);
        int bad = 0;
        for (int v = lane; v < m; v += 32)
            if (ws.indeg()[v] + ws.exdeg()[v] < need_t) bad = 1;
        if (!__any_sync(QC_FULL, bad)) {
            int bad2 = 0;
            for (int v = m + lane; v < t; v += 32) {
                int l2 = popc_and(T.A2 + (int64_t)v * W, CC, W);
                T.l2[v] = l2;
                if (T.l2g != T.l2) T.l2g[v] = l2; // branch items on other warps read the arena
                if (l2 < nc - 1 || ws.indeg()[v] + ws.exdeg()[v] < need_t) bad2 = 1;
            }
            __syncwarp();
            if (!__any_sync(QC_FULL, bad2)) {
                uint32_t* all = ws.mk(MK_T);
                bs_range(all, W, 0, t);
                if (lane == 0) ws.sm->cnt.lookahead_hits++;
                if (!sroot || P.shard == 0) emit_mask(P, R, T, all, t);
                return shared;
            }
        }
        // branches executed before a member fails on removal (main.cu:1092-1099)
        int need = mindeg(R, m);
        int qmax = m + T.cov;
        // lane per member: position of its k-th candidate neighbour (t-1 if it
        // has fewer), scanning its own row word by word
        for (int v0 = 0; v0 < m; v0 += 32) {
            const int v = v0 + lane;
            int pos = -1;
            if (v < m) {
                const int k = need - ws.indeg()[v];
                if (k > 0) {
                    const uint32_t* row = T.A1 + (int64_t)v * W;
                    pos = t - 1;
                    int seen = 0;
                    for (int w = 0; w < W; w++) {
                        uint32_t x = rec_ld(row + w) & CC[w];
                        const int c = __popc(x);
                        if (seen + c >= k) {
                            for (int r = k - seen; r > 1; r--) x &= x - 1; // drop the lower ones
                            pos = w * 32 + __ffs(x) - 1;
                            break;
                        }
                        seen += c;
                    }
                }
            }
            const int best = wmax(pos);
            qmax = best > qmax ? best : qmax;
        }
        q_lo = qmax > t - 1 ? t - 1 : qmax;
        q_hi = t - 1;
        if (m + T.cov >= t) return shared; // no branchable candidate
        int nb = q_hi - q_lo + 1;
        // branches per item: as configured, else one for a task of up to 256
        // vertices (its branches start at once) and two above (a huge root's
        // thousands of branches would otherwise crowd out its own children)
        const int split = P.split > 0 ? P.split : (t <= 256 ? 1 : 2);
        if (nb > split) {
            __syncwarp();
            __threadfence();
            // every range but the first goes to the shared stack, all at once;
            // the references are counted before any range is published
            const int extra = (q_hi - split - q_lo) / split + 1;
            if (lane == 0) atomicAdd(&((TaskHdr*)(P.arena + it.rec))->refs, extra);
            __syncwarp();
            push_ranges(P, it.rec, q_lo, q_hi - split, split, extra);
            __syncwarp();
            q_lo = q_hi - split + 1;
            shared = true;
        }
    }
    // deg + |N2| of every branch vertex (work accounting only): loads issued
    // here, summed after the branches
    long long rows = 0;
    for (int q = q_lo + lane; q <= q_hi; q += 32) {
        if (sroot && (t - 1 - q) % P.nshards != P.shard) continue;
        const int pid = rec_ld(T.ids + q);
        if (pid >= 0 && pid < R.n)
            rows += (R.off[pid + 1] - R.off[pid]) + (R.off2[pid + 1] - R.off2[pid]);
    }
    for (int q = q_hi; q >= q_lo; q--) {
        if (sroot && (t - 1 - q) % P.nshards != P.shard) continue;
        int stop = 0;
        if (lane == 0) stop = *(volatile int*)&P.ctl->status;
        if (__shfl_sync(QC_FULL, stop, 0)) break;
        if (ws.sm->deadline && now_ns() > ws.sm->deadline) {
            if (lane == 0) set_status(P, ST_DEADLINE);
            break;
        }
        expand_branch(P, R, T, ws, q);
    }
    rows = wsum64(rows);
    if (lane == 0) ws.sm->cnt.p_rows += (unsigned long long)rows;
    return shared;
}


// Self-check of a dequeued work item before any lane reads its record: the
// offset must be 16-byte aligned and inside the written arena, and the
// header must describe a record that fits there.  A failure records the
// site and value and the item is skipped instead of being dereferenced.
// The header is read once, through L2, into `hv`; the warp uses only those
// validated values.
__device__ bool item_ok(const ExpandParams& P, const WorkItem& it, TaskHdr& hv)
{
    const unsigned long long lim = P.arena_cap;
    unsigned long long site = 0, val = it.rec;
    if ((it.rec & 15ull) != 0) site = 1;
    else if (it.rec + sizeof(TaskHdr) > lim) site = 2;
    else {
        const volatile TaskHdr* h = (const volatile TaskHdr*)(P.arena + it.rec);
        int t = h->t, W = h->W, m = h->m, inst = h->inst, cov = h->cov, cls = h->cls,
            refs = h->refs;
        hv.t = t;
        hv.W = W;
        hv.m = m;
        hv.inst = inst;
        hv.flags = h->flags;
        hv.cov = cov;
        hv.cls = cls;
        hv.refs = refs;
        if (t < 1 || t > P.max_t || W != words_for(t) || m < 0 || m > t || cov < 0 || m + cov > t ||
            cls < 0 || cls >= kArenaClasses || refs < 1 || refs == kFreeMagic) {
            site = 3;
            val = ((unsigned long long)(unsigned)t << 32) | (unsigned)W;
        } else if (it.rec + rec_bytes(t, W) > lim) site = 4;
        else if (inst < 0 || inst >= P.nrules) site = 5;
        else if (it.q_lo >= 0 && (it.q_hi >= t || it.q_lo > it.q_hi)) site = 6;
    }
    if (site) {
        if (atomicCAS((unsigned long long*)&P.ctl->check_site, 0ull, site) == 0ull)
            P.ctl->check_value = val;
        set_status(P, ST_CHECK);
        return false;
    }
    return true;
}

// ------------------------------------------------------------------
// the persistent kernel
// ------------------------------------------------------------------

#ifndef QC_EMULATION
extern __shared__ __align__(16) unsigned char qc_dyn_smem[];
__device__ __forceinline__ unsigned char* dyn_smem() { return qc_dyn_smem; }
#else
__device__ __forceinline__ unsigned char* dyn_smem() { return emu_dyn_smem(); }
#endif

// dynamic shared memory the kernel needs per block of `warps` warps when
// tasks of up to smem_t vertices are staged in shared memory
__host__ __device__ inline size_t expand_smem_bytes(int warps, int smem_t)
{
    return warp_smem_bytes(smem_t) * (size_t)warps;
}

#ifndef QC_EMULATION
__global__ void __launch_bounds__(256, 2) expand_kernel(ExpandParams P)
#else
__global__ void expand_kernel(ExpandParams P)
#endif
{
    int lane = lane_id();
    int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    char* base = (char*)dyn_smem() + (size_t)(threadIdx.x >> 5) * warp_smem_bytes(P.smem_t);
    WarpSmem* sm = (WarpSmem*)base;
    Ws ws = ws_view(P.ws + (int64_t)warp_global * P.ws_stride, P.max_t, sm);
    Ws wss = ws;
    char* stage = nullptr;
    if (P.smem_t > 0) {
        char* sb = base + align16(sizeof(WarpSmem));
        wss = ws_view(sb, P.smem_t, sm);
        stage = sb + ws_layout(P.smem_t).total;
    }
    if (lane == 0) {
        sm->lcount = 0;
        sm->hungry = 0;
        sm->stat = 0;
        sm->tab_inst = -1;
        sm->en = 0;
        sm->es = 0;
        sm->cnt = WarpCount{};
        sm->deadline = 0;
        if (P.time_limit_ns) {
            // the launch's start: the first warp's clock, shared through t_start
            const unsigned long long now = now_ns();
            const unsigned long long prev = atomicCAS(&P.ctl->t_start, 0ull, now);
            sm->deadline = (prev ? prev : now) + P.time_limit_ns;
        }
    }
    for (int c = lane; c < kArenaClasses; c += 32) {
        sm->fhead[c] = 0;
        sm->fcount[c] = 0;
    }
    if (lane == 0) {
        sm->nsfree = 0;
        sm->hot_rec = ~0ull;
    }
    __syncwarp();
#ifndef QC_EMULATION
    if (stage) stage_bar_init(sm);
#endif
    for (;;) {
        WorkItem it;
        TaskHdr hv{};
        int r = 0;
        int local = 0;
        if (lane == 0) local = sm->lcount > 0;
        if (__shfl_sync(QC_FULL, local, 0)) {
            donate(P, ws);
            if (lane == 0) {
                const LocalTask lt = sm->lstack[--sm->lcount];
                it.rec = lt.rec;
                it.q_lo = -1;
                it.q_hi = -1;
                r = 1;
                if (lt.t > 0) {
                    // a child this warp wrote: its header is known
                    hv.t = lt.t;
                    hv.m = lt.m;
                    hv.cov = 0;
                    hv.W = lt.W;
                    hv.cls = lt.cls;
                    hv.inst = lt.inst;
                    hv.flags = lt.flags;
                    hv.refs = 1;
                    r = 2;
                }
            }
        } else {
            r = pop_item(P, ws, it);
        }
        if (lane == 0 && r == 1 && !item_ok(P, it, hv)) r = -1;
        r = __shfl_sync(QC_FULL, r, 0);
        if (r <= 0) break;
        it.rec = __shfl_sync(QC_FULL, it.rec, 0);
        it.q_lo = __shfl_sync(QC_FULL, it.q_lo, 0);
        it.q_hi = __shfl_sync(QC_FULL, it.q_hi, 0);
        hv.t = __shfl_sync(QC_FULL, hv.t, 0);
        hv.m = __shfl_sync(QC_FULL, hv.m, 0);
        hv.cov = __shfl_sync(QC_FULL, hv.cov, 0);
        hv.W = __shfl_sync(QC_FULL, hv.W, 0);
        hv.inst = __shfl_sync(QC_FULL, hv.inst, 0);
        hv.flags = __shfl_sync(QC_FULL, hv.flags, 0);
        // idle warps and run status, read now and looked at while the next
        // item is taken and run, so the reads overlap this item's work
        int idle_now = 0, stat_now = 0;
        if (lane == 0) {
            idle_now = *(volatile int*)&P.ctl->idle_warps;
            stat_now = *(volatile int*)&P.ctl->status;
        }
        // a child this warp wrote last is read from its copy in shared memory
        const bool hot = r == 2 && sm->hot_rec == it.rec;
        bool shared = process_item(P, ws, wss, stage, it, hv, hot);
        __syncwarp();
        if (lane == 0) {
            sm->hungry = idle_now;
            sm->stat = stat_now;
            release_record(P, ws, it.rec, !shared, hv);
            // the warp stays counted in `pending` while its own stack holds work
            if (sm->lcount == 0) atomicSub(&P.ctl->pending, 1);
        }
    }
    emit_flush(P, ws);
    if (lane == 0) {
        const WarpCount& c = sm->cnt;
        if (c.tasks) atomicAdd(&P.ctl->tasks, c.tasks);
        if (c.branches) atomicAdd(&P.ctl->branches, c.branches);
        if (c.children) atomicAdd(&P.ctl->children, c.children);
        if (c.lookahead_hits) atomicAdd(&P.ctl->lookahead_hits, c.lookahead_hits);
        if (c.parent_vertices) atomicAdd(&P.ctl->parent_vertices, c.parent_vertices);
        if (c.p_rows) atomicAdd(&P.ctl->p_rows, c.p_rows);
        if (c.child_vertices) atomicAdd(&P.ctl->child_vertices, c.child_vertices);
        if (c.max_task) atomicMax(&P.ctl->max_task, (int)c.max_task);
    }
}

} // namespace qcb
