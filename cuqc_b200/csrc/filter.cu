// filter.cu -- non-maximal removal on the GPU (replaces the reference's host
// prefix-tree pass RemoveNonMax, Mike12041204/cuQC main.cu:4571-4960).
//
// Input: the emitted sets in the device result buffer, [k, id_1..id_k] each,
// and the start offset of every set (written by the expansion kernel).
//   1. one warp per set: sort its ids ascending into the sorted buffer, build
//      its 256-bit signature and its order-free 64-bit hash (the sum of a
//      mix of each id);
//   2. the one-less pass: every set is entered in an open-addressing table
//      by its hash; every set T looks up T minus each of its ids (hash
//      H(T) - mix(x)) and marks the sets equal to it, and looks up its own
//      hash for an exact copy of smaller index, which marks T;
//   3. the residual -- the unmarked sets -- holds every maximal set (a set
//      inside any emitted set is inside a maximal one, and a maximal set is
//      never marked), so only the residual is tested for supersets, against
//      itself: pairwise (signature first, then an exact warp check) when it
//      has at most 4,096 sets, else through an inverted index (incidences
//      radix-sorted by vertex and set size, one warp per set scanning the
//      posting list of its rarest vertex for larger sets);
//   4. each maximal set is appended to the output at a slot reserved with an
//      atomic add, with an entry for the ordering.  The entries are put in the
//      order the reference's prefix tree writes (lexicographic): by 256-bit
//      vectors over the survivors' ranked ids when there are at most 256
//      distinct ids (few survivors ranked by counting, many by a merge sort),
//      else by a merge sort comparing the sets; the host only gathers.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <cub/device/device_merge_sort.cuh>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "filter.h"

namespace qcb {

namespace {

// signature bit of an id: the top 8 bits of a multiplicative (Fibonacci) hash
__device__ __forceinline__ unsigned sig_bit(int32_t v) { return ((unsigned)v * 0x9E3779B1u) >> 24; }

// 1. per-set sort + signature (one warp per set)
// id -> 64-bit word: the finalizer of SplitMix64 (Steele, Lea and Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014)
__device__ __forceinline__ unsigned long long id_mix(int32_t v)
{
    unsigned long long z = (unsigned long long)(unsigned)v + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void sort_sig_kernel(const int32_t* res, const unsigned long long* starts, int64_t nsets,
                                int32_t* sorted, uint4* sig, unsigned long long* hsh)
{
    int lane = threadIdx.x & 31;
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < nsets; s += nw) {
        unsigned long long a = starts[s];
        int k = res[a];
        const int32_t* in = res + a + 1;
        int32_t* out = sorted + a + 1;
        unsigned sg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        unsigned long long h = 0;
        for (int i = lane; i < k; i += 32) {
            const int32_t v = in[i];
            if (k > 32) out[i] = v;
            h += id_mix(v);
            const unsigned b = sig_bit(v);
#pragma unroll
            for (int w = 0; w < 8; w++)
                if ((int)(b >> 5) == w) sg[w] |= 1u << (b & 31);
        }
#pragma unroll
        for (int w = 0; w < 8; w++) sg[w] = __reduce_or_sync(0xffffffffu, sg[w]);
        for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
        if (k <= 32) {
            // one id per lane, bitonic sort in registers (ids are >= 0, the
            // padding lanes hold INT_MAX and sort to the end)
            int x = lane < k ? in[lane] : INT_MAX;
            for (int sz = 2; sz <= 32; sz <<= 1)
                for (int j = sz >> 1; j > 0; j >>= 1) {
                    const int o = __shfl_xor_sync(0xffffffffu, x, j);
                    const bool up = (lane & sz) == 0;
                    const bool lower = (lane & j) == 0;
                    if ((lower == up) != (x < o)) x = o;
                }
            if (lane < k) out[lane] = x;
        } else {
            __syncwarp();
            // bitonic sort of out[0..k) in place, all compare-exchanges
            // ascending (mirror step, then half-cleaners), so virtual +inf
            // padding at [k, N) never moves into the real range
            int N = 1;
            while (N < k) N <<= 1;
            for (int sz = 2; sz <= N; sz <<= 1) {
                for (int j = sz >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < N; i += 32) {
                        int p = (j == (sz >> 1)) ? (i ^ (sz - 1)) : (i ^ j);
                        if (p > i && p < k) {
                            int x = out[i], y = out[p];
                            if (x > y) {
                                out[i] = y;
                                out[p] = x;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
        }
        if (lane == 0) {
            sorted[a] = k;
            hsh[s] = h;
            sig[2 * s] = make_uint4(sg[0], sg[1], sg[2], sg[3]);
            sig[2 * s + 1] = make_uint4(sg[4], sg[5], sg[6], sg[7]);
        }
    }
}

// incidence key: vertex in the high bits, then the set's size descending
__device__ __forceinline__ unsigned long long inc_key(int v, int k)
{
    return ((unsigned long long)(unsigned)v << 16) | (unsigned long long)(0xffff - (k < 0xffff ? k : 0xffff));
}
__device__ __forceinline__ int inc_size(unsigned long long key) { return 0xffff - (int)(key & 0xffffull); }

// 2. every set writes its (vertex, size) keys and set id at slots reserved
// with one atomic add on `inc_top` (one warp per set; the order does not
// matter, the keys are sorted next)
__global__ void emit_incidences_kernel(const int32_t* srt, const unsigned long long* starts,
                                       int64_t nsets, unsigned long long* inc_top,
                                       unsigned long long* key, int32_t* val)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < nsets; s += nw) {
        const unsigned long long a = starts[s];
        const int k = srt[a];
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(inc_top, (unsigned long long)k);
        at = __shfl_sync(0xffffffffu, at, 0);
        for (int x = lane; x < k; x += 32) {
            key[at + x] = inc_key(srt[a + 1 + x], k);
            val[at + x] = (int32_t)s;
        }
    }
}

// 3c. start of every vertex's posting list in the sorted incidences
__global__ void inc_offsets_kernel(const unsigned long long* key, int64_t total, int64_t nv,
                                   int64_t* poff)
{
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v > nv) return;
    unsigned long long want = (unsigned long long)v << 16;
    int64_t lo = 0, hi = total; // first index with key >= want
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (key[mid] < want) lo = mid + 1;
        else hi = mid;
    }
    poff[v] = lo;
}

// does signature T have every bit of signature S?
__device__ __forceinline__ bool sig_covers(const uint4& s0, const uint4& s1, const uint4& t0,
                                           const uint4& t1)
{
    return ((s0.x & ~t0.x) | (s0.y & ~t0.y) | (s0.z & ~t0.z) | (s0.w & ~t0.w) | (s1.x & ~t1.x) |
            (s1.y & ~t1.y) | (s1.z & ~t1.z) | (s1.w & ~t1.w)) == 0;
}

// Is sorted set S (k ids at srt[a+1..]) contained in sorted set T (at bt)?
// Warp-wide: every lane looks its share of S's ids up in T by binary search.
__device__ __forceinline__ bool warp_subset(const int32_t* srt, unsigned long long a, int k,
                                            unsigned long long bt, int lane)
{
    const int kt = srt[bt];
    const int32_t* T = srt + bt + 1;
    bool all = true;
    for (int i = lane; i < k; i += 32) {
        const int x = srt[a + 1 + i];
        int l = 0, r = kt - 1;
        while (l < r) {
            const int mid = (l + r) >> 1;
            if (T[mid] < x) l = mid + 1;
            else r = mid;
        }
        if (T[l] != x) all = false;
    }
    return __all_sync(0xffffffffu, all);
}

constexpr int MAX_ROUND = 4; // candidate groups of 32 fetched per round

// 4. superset test, one warp per kept set
// a surviving set: key of its first two ids (see set_key) and its offset in
// the output
struct SetEnt {
    unsigned long long key;
    long long at;
};

// The maximal sets form an antichain: no set is a subset, so none is a
// prefix, of another.  For such sets with ids sorted ascending, the
// lexicographic order is the descending order of the bit vectors that set bit
// 255 - r for every id of rank r in the survivors' universe (the smallest id
// is the most significant bit): at the first position where two sets differ,
// the smaller id is in one set only and every smaller id is in both or
// neither.  With at most 256 distinct ids, four words order every pair.
constexpr int kBitUniverse = 256;
struct BitEnt {
    unsigned long long w[4]; // w[0] most significant
    long long at;
};
struct BitMore {
    __device__ bool operator()(const BitEnt& x, const BitEnt& y) const
    {
        for (int i = 0; i < 4; i++)
            if (x.w[i] != y.w[i]) return x.w[i] > y.w[i];
        return false;
    }
};

// survivors' ids into a presence bitmap over the vertex range (one warp per
// survivor; the count of survivors is read on the device)
__global__ void uni_mark_kernel(const int32_t* out, const SetEnt* ents, const unsigned long long* ctr,
                                uint32_t* bitmap)
{
    const int lane = threadIdx.x & 31;
    const long long nsurv = (long long)ctr[2];
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long j = warp; j < nsurv; j += nw) {
        const long long at = ents[j].at;
        const int k = out[at];
        for (int i = lane; i < k; i += 32) {
            const int v = out[at + 1 + i];
            atomicOr(&bitmap[v >> 5], 1u << (v & 31));
        }
    }
}

// one block: rank_base[w] = ids present in bitmap words before w; ctr[3] =
// the universe size
__global__ void __launch_bounds__(1024) uni_rank_kernel(const uint32_t* bitmap, int nwords,
                                                        uint32_t* rank_base, unsigned long long* ctr)
{
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nwords; base += blockDim.x) {
        const int w = base + threadIdx.x;
        const uint32_t c = w < nwords ? (uint32_t)__popc(bitmap[w]) : 0u;
        uint32_t x = c; // inclusive scan within the warp
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint32_t t = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (lane >= o) t += y;
            }
            warp_tot[lane] = t; // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = (wid ? warp_tot[wid - 1] : 0u) + x - c;
        if (w < nwords) rank_base[w] = carry + before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[(blockDim.x >> 5) - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) ctr[3] = carry;
}

// bit-vector key of every survivor (universe of at most kBitUniverse ids)
__global__ void bit_key_kernel(const int32_t* out, const SetEnt* ents, long long nsurv,
                               const uint32_t* bitmap, const uint32_t* rank_base, BitEnt* bents)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long j = warp; j < nsurv; j += nw) {
        const long long at = ents[j].at;
        const int k = out[at];
        unsigned h[8] = {0, 0, 0, 0, 0, 0, 0, 0}; // 32-bit halves, h[0] most significant
        for (int i = lane; i < k; i += 32) {
            const int v = out[at + 1 + i];
            const unsigned r = rank_base[v >> 5] + (unsigned)__popc(bitmap[v >> 5] & ((1u << (v & 31)) - 1u));
            const unsigned p = 255u - (r < 256u ? r : 255u); // bit position, 255 = most significant
#pragma unroll
            for (int q = 0; q < 8; q++)
                if ((int)(p >> 5) == 7 - q) h[q] |= 1u << (p & 31);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) h[q] = __reduce_or_sync(0xffffffffu, h[q]);
        if (lane == 0) {
            BitEnt e;
            for (int i = 0; i < 4; i++)
                e.w[i] = ((unsigned long long)h[2 * i] << 32) | (unsigned long long)h[2 * i + 1];
            e.at = at;
            bents[j] = e;
        }
    }
}

// ids (sorted ascending) of a set at p: the first id in the high half, the
// second + 1 in the low half (0 for a set of one id), so that comparing keys
// compares the first two ids lexicographically
__device__ __forceinline__ unsigned long long set_key(const int32_t* d, long long p)
{
    const int k = d[p];
    unsigned long long key = k >= 1 ? (unsigned long long)(unsigned)d[p + 1] << 32 : 0ull;
    if (k >= 2) key |= (unsigned long long)((unsigned)d[p + 2] + 1u);
    return key;
}

// lexicographic order of two sets of the output (ids sorted ascending; a
// prefix orders first)
struct SetLess {
    const int32_t* d;
    __device__ bool operator()(const SetEnt& x, const SetEnt& y) const
    {
        if (x.key != y.key) return x.key < y.key;
        const int kx = d[x.at], ky = d[y.at];
        const int n = kx < ky ? kx : ky;
        for (int i = 2; i < n; i++) {
            const int a = d[x.at + 1 + i], b = d[y.at + 1 + i];
            if (a != b) return a < b;
        }
        return kx < ky;
    }
};

__global__ void maximal_kernel(const int32_t* srt, const unsigned long long* starts, int64_t nsets,
                               const int64_t* poff, const int32_t* post,
                               const unsigned long long* pkey, const uint4* sig,
                               unsigned long long* ctr, int32_t* out, SetEnt* ents)
{
    int lane = threadIdx.x & 31;
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < nsets; s += nw) {
        unsigned long long a = starts[s];
        int k = srt[a];
        // rarest vertex of S
        int64_t best_len = INT64_MAX;
        int best_v = -1;
        for (int i = lane; i < k; i += 32) {
            int v = srt[a + 1 + i];
            int64_t len = poff[v + 1] - poff[v];
            if (len < best_len || (len == best_len && v < best_v)) {
                best_len = len;
                best_v = v;
            }
        }
        for (int o = 16; o; o >>= 1) {
            int64_t ol = __shfl_xor_sync(0xffffffffu, best_len, o);
            int ov = __shfl_xor_sync(0xffffffffu, best_v, o);
            if (ol < best_len || (ol == best_len && ov < best_v)) {
                best_len = ol;
                best_v = ov;
            }
        }
        bool covered = false;
        if (k > 0 && best_v >= 0) {
            const uint4 s0 = sig[2 * s], s1 = sig[2 * s + 1];
            const int64_t lo = poff[best_v], hi = poff[best_v + 1];
            int64_t eq = hi; // first entry not larger than S
            // the list is ordered by size, largest first: past the sets larger
            // than S nothing can contain it
            for (int64_t base = lo; base < hi; base += 32 * MAX_ROUND) {
                bool larger[MAX_ROUND];
                int32_t t[MAX_ROUND];
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    const int64_t e = base + u * 32 + lane;
                    larger[u] = e < hi && inc_size(pkey[e]) > k;
                    t[u] = larger[u] ? post[e] : 0;
                }
                bool pass[MAX_ROUND];
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    pass[u] = false;
                    if (larger[u]) {
                        const uint4 t0 = sig[2 * (int64_t)t[u]], t1 = sig[2 * (int64_t)t[u] + 1];
                        pass[u] = sig_covers(s0, s1, t0, t1);
                    }
                }
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    unsigned pb = __ballot_sync(0xffffffffu, pass[u]);
                    while (pb && !covered) {
                        const int c = __ffs(pb) - 1;
                        pb &= pb - 1;
                        const int32_t tt = __shfl_sync(0xffffffffu, t[u], c);
                        covered = warp_subset(srt, a, k, starts[tt], lane);
                    }
                }
                if (covered) break;
                bool end = false;
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    const unsigned lb = __ballot_sync(0xffffffffu, larger[u]); // a prefix of lanes
                    if (!end && lb != 0xffffffffu) {
                        eq = base + u * 32 + __popc(lb);
                        end = true;
                    }
                }
                if (end) break;
            }
            // Exact copies of S (same size, after the larger sets in the
            // list): the copy of the smallest index stands for all of them.
            // Only sets no larger set contains get here.
            for (int64_t base = eq < hi ? eq : hi; !covered && base < hi;
                 base += 32 * MAX_ROUND) {
                bool same[MAX_ROUND];
                int32_t tt[MAX_ROUND];
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    const int64_t e = base + u * 32 + lane;
                    same[u] = e < hi && inc_size(pkey[e]) == k;
                    tt[u] = same[u] ? post[e] : 0;
                }
                bool pass[MAX_ROUND];
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    pass[u] = false;
                    if (same[u] && tt[u] < s) {
                        const uint4 t0 = sig[2 * (int64_t)tt[u]], t1 = sig[2 * (int64_t)tt[u] + 1];
                        pass[u] = s0.x == t0.x && s0.y == t0.y && s0.z == t0.z && s0.w == t0.w &&
                                  s1.x == t1.x && s1.y == t1.y && s1.z == t1.z && s1.w == t1.w;
                    }
                }
#pragma unroll
                for (int u = 0; u < MAX_ROUND; u++) {
                    unsigned pb = __ballot_sync(0xffffffffu, pass[u]);
                    while (pb && !covered) {
                        const int c = __ffs(pb) - 1;
                        pb &= pb - 1;
                        const int32_t t2 = __shfl_sync(0xffffffffu, tt[u], c);
                        covered = warp_subset(srt, a, k, starts[t2], lane); // equal sizes: equal sets
                    }
                }
                // sizes only fall along the list: a round that is not all of
                // S's size reached the end of the copies
                if (__ballot_sync(0xffffffffu, same[MAX_ROUND - 1]) != 0xffffffffu) break;
            }
        }
        if (covered) continue;
        // a maximal set: [k, ids..] to a reserved slot of the output, and
        // its entry for the ordering
        unsigned long long at = 0;
        if (lane == 0) {
            at = atomicAdd(&ctr[1], (unsigned long long)(k + 1));
            const unsigned long long j = atomicAdd(&ctr[2], 1ull);
            ents[j] = SetEnt{set_key(srt, (long long)a), (long long)at};
        }
        at = __shfl_sync(0xffffffffu, at, 0);
        for (int i = lane; i <= k; i += 32) out[at + i] = srt[a + i];
    }
}

// ---------------------------------------------------------------------------
// One-less pass: a set S that is T minus one id, for some emitted set T, is not
// maximal.  Every set carries an order-free 64-bit hash H(S) = sum over its ids
// of mix(id) (mod 2^64), so H(T \ {x}) = H(T) - mix(x); the sets are entered in
// an open-addressing table by hash, and every T looks up its |T| one-less sets
// there (an exact check confirms each hit).  The same lookup with H(T) itself
// finds exact copies of T, of which the one of the smallest index is kept.  On
// the emitted families of this miner almost every non-maximal set has a
// superset one larger (all of them on ER n = 1,000 + 5 planted groups of 30,
// gamma 0.9, min 20: 35,809 of 35,809), so the survivors -- the residual --
// are few, and only they go through the exact superset test against each
// other: a set contained in any emitted set is contained in a maximal one,
// and every maximal set is in the residual.
// ---------------------------------------------------------------------------

// A table entry: the set's index (low 32 bits), its size (capped at 255) and
// 24 more bits of its hash, so that a probe rejects most sets that are not a
// hit without reading them (all ones: an empty slot).
__device__ __forceinline__ unsigned long long slot_entry(unsigned long long h, int k, int64_t s)
{
    return (((h >> 32) & 0xffffffull) << 40) | ((unsigned long long)(k < 255 ? k : 255) << 32) |
           (unsigned long long)(uint32_t)s;
}
// does entry e stand for a set of hash h and size k (a candidate to check)?
__device__ __forceinline__ bool slot_may_be(unsigned long long e, unsigned long long h, int k)
{
    return (e >> 32) == ((((h >> 32) & 0xffffffull) << 8) | (unsigned long long)(k < 255 ? k : 255));
}
constexpr unsigned long long kSlotEmpty = ~0ull;

// every set into the table by its hash
__global__ void set_insert_kernel(const unsigned long long* hsh, const int32_t* srt,
                                  const unsigned long long* starts, int64_t nsets,
                                  unsigned long long* table, unsigned long long mask)
{
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nsets; s += nt) {
        const unsigned long long h = hsh[s];
        const unsigned long long e = slot_entry(h, srt[starts[s]], s);
        unsigned long long p = h & mask;
        for (unsigned long long it = 0; it <= mask; it++) { // the table is never full
            if (atomicCAS(&table[p], kSlotEmpty, e) == kSlotEmpty) break;
            p = (p + 1) & mask;
        }
    }
}

// is sorted set A (ka ids) contained in sorted set B (kb ids)?  one thread
__device__ __forceinline__ bool thread_subset(const int32_t* A, int ka, const int32_t* B, int kb)
{
    int j = 0;
    for (int i = 0; i < ka; i++) {
        const int x = A[i];
        while (j < kb && B[j] < x) j++;
        if (j == kb || B[j] != x) return false;
        j++;
    }
    return true;
}

// One warp per set T: the lanes look up T minus each of its ids (lane i takes
// ids i, i+32, ..) and mark every emitted set equal to it; lane 0 also looks
// up T's own hash for an exact copy of smaller index, which marks T.
__global__ void one_less_kernel(const int32_t* srt, const unsigned long long* starts, int64_t nsets,
                                const unsigned long long* hsh, const unsigned long long* table,
                                unsigned long long mask, int32_t* dead)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nsets; s += nw) {
        const unsigned long long a = starts[s];
        const int k = srt[a];
        const int32_t* T = srt + a + 1;
        const unsigned long long hT = hsh[s];
        if (k >= 32) {
            // sets of 32 ids or more: each lane checks its own hits
            for (int i = lane; i < k; i += 32) {
                const unsigned long long h = hT - id_mix(T[i]);
                unsigned long long p = h & mask;
                for (unsigned long long it = 0; it <= mask; it++) {
                    const unsigned long long e = table[p];
                    if (e == kSlotEmpty) break;
                    const int32_t c = (int32_t)(uint32_t)e;
                    if (slot_may_be(e, h, k - 1) && hsh[c] == h) {
                        const unsigned long long b = starts[c];
                        if (srt[b] == k - 1 && thread_subset(srt + b + 1, k - 1, T, k)) dead[c] = 1;
                    }
                    p = (p + 1) & mask;
                }
            }
            if (lane == 0) {
                unsigned long long p = hT & mask;
                for (unsigned long long it = 0; it <= mask; it++) {
                    const unsigned long long e = table[p];
                    if (e == kSlotEmpty) break;
                    const int32_t c = (int32_t)(uint32_t)e;
                    if (c < s && slot_may_be(e, hT, k) && hsh[c] == hT) {
                        const unsigned long long b = starts[c];
                        if (srt[b] == k && thread_subset(srt + b + 1, k, T, k)) {
                            dead[s] = 1;
                            break;
                        }
                    }
                    p = (p + 1) & mask;
                }
            }
            continue;
        }
        // sets of at most 31 ids: lane j holds T[j].  Lane i (< k) walks the
        // probe sequence of T minus T[i] and lane k that of T itself (for an
        // exact copy of smaller index); every hit -- a set of the right size
        // and hash -- is checked by the whole warp at once: id j of the hit
        // against T's id j (or j + 1 past the dropped one).
        const int my = lane < k ? T[lane] : 0;
        const bool prober = lane <= k;
        const unsigned long long h = lane < k ? hT - id_mix(my) : hT;
        const int want = lane < k ? k - 1 : k;
        unsigned long long p = h & mask;
        bool walking = prober;
        for (unsigned long long it = 0; it <= mask && __any_sync(0xffffffffu, walking); it++) {
            int32_t c = -1;
            bool may = false;
            if (walking) {
                const unsigned long long e = table[p];
                if (e == kSlotEmpty) walking = false;
                else {
                    c = (int32_t)(uint32_t)e;
                    may = slot_may_be(e, h, want);
                    p = (p + 1) & mask;
                }
            }
            const bool hit = may && (lane < k || c < s) && hsh[c] == h && srt[starts[c]] == want;
            unsigned pend = __ballot_sync(0xffffffffu, hit);
            while (pend) {
                const int i = __ffs(pend) - 1;
                pend &= pend - 1;
                const int32_t cc = __shfl_sync(0xffffffffu, c, i);
                const int n = i < k ? k - 1 : k; // ids of the hit
                const unsigned long long b = starts[cc];
                const int src = (i < k && lane >= i) ? lane + 1 : lane;
                const int tv = __shfl_sync(0xffffffffu, my, src & 31);
                const bool eq = lane >= n || srt[b + 1 + lane] == tv;
                if (__all_sync(0xffffffffu, eq) && lane == 0) dead[i < k ? cc : s] = 1;
            }
        }
    }
}

// the residual: starts and signatures of the sets not marked, compacted
// (ctr[0] counts them, ctr[1] their ints)
__global__ void residual_kernel(const int32_t* srt, const unsigned long long* starts, int64_t nsets,
                                const int32_t* dead, const uint4* sig, unsigned long long* rstarts,
                                uint4* rsig, int32_t* rsz, unsigned long long* ctr)
{
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nsets; s += nt) {
        if (dead[s]) continue;
        const unsigned long long j = atomicAdd(&ctr[0], 1ull);
        const int k = srt[starts[s]];
        atomicAdd(&ctr[1], (unsigned long long)(k + 1));
        rstarts[j] = starts[s];
        rsig[2 * j] = sig[2 * s];
        rsig[2 * j + 1] = sig[2 * s + 1];
        rsz[j] = k;
    }
}

// Residuals of at most this many sets are checked pairwise (every set
// against every larger one); larger residuals go through the inverted index.
constexpr int64_t kPairsMax = 4096;

// One warp per residual set S, when the residual is small (its size is read
// from ctr[4] on the device; above kPairsMax this does nothing): S is maximal
// unless a larger residual set contains it (signature test, then exact).
// Maximal sets are appended to the output with their ordering entry.
__global__ void residual_pairs_kernel(const int32_t* srt, const unsigned long long* rstarts,
                                      const uint4* rsig, const int32_t* rsz, unsigned long long* ctr,
                                      int32_t* out, SetEnt* ents)
{
    const int64_t nr = (int64_t)ctr[4];
    if (nr > kPairsMax) return;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nr; s += nw) {
        const unsigned long long a = rstarts[s];
        const int k = rsz[s];
        const uint4 s0 = rsig[2 * s], s1 = rsig[2 * s + 1];
        bool covered = false;
        // four chunks of 32 candidates per step, their sizes and signatures
        // loaded together
        for (int64_t base = 0; base < nr && !covered; base += 128) {
            bool pass[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int64_t t = base + 32 * u + lane;
                pass[u] = false;
                if (t < nr && t != s && rsz[t] > k) {
                    const uint4 t0 = rsig[2 * t], t1 = rsig[2 * t + 1];
                    pass[u] = sig_covers(s0, s1, t0, t1);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                unsigned pb = __ballot_sync(0xffffffffu, pass[u]);
                while (pb && !covered) {
                    const int c = __ffs(pb) - 1;
                    pb &= pb - 1;
                    covered = warp_subset(srt, a, k, rstarts[base + 32 * u + c], lane);
                }
            }
        }
        if (covered) continue;
        unsigned long long at = 0;
        if (lane == 0) {
            at = atomicAdd(&ctr[1], (unsigned long long)(k + 1));
            const unsigned long long j = atomicAdd(&ctr[2], 1ull);
            ents[j] = SetEnt{set_key(srt, (long long)a), (long long)at};
        }
        at = __shfl_sync(0xffffffffu, at, 0);
        for (int i = lane; i <= k; i += 32) out[at + i] = srt[a + i];
    }
}

// Up to kRankSortMax bit-vector entries put in descending order by rank:
// one warp per entry counts the entries above it and writes it at that
// position (the vectors are distinct: they stand for distinct maximal sets).
// n^2 comparisons, spread over the whole grid.
constexpr int kRankSortMax = 4096;
__global__ void bit_rank_kernel(const BitEnt* in, int n, BitEnt* out)
{
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    const BitMore more;
    for (long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const BitEnt x = in[i];
        int c = 0;
        for (int j = lane; j < n; j += 32) c += more(in[j], x) ? 1 : 0;
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) out[c] = x;
    }
}

} // namespace

#define FCK(call)                                                                \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return std::string(#call) + ": " + cudaGetErrorString(e_); \
    } while (0)

std::string FilterScratch::ensure(void** p, size_t* have, size_t need)
{
    if (need <= *have) return "";
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMalloc(p, need);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return std::string("filter scratch: ") + cudaGetErrorString(e);
    }
    *have = need;
    return "";
}

void FilterScratch::release()
{
    if (host) cudaFreeHost(host);
    host = nullptr;
    host_n = 0;
    for (auto* pp : {&sorted, &sig, &poff, &post, &ctr, &ents, &bents, &temp, &ikey, &ikey2,
                     &ival, &rsig, &hsh, &table, &dead, &rstarts, &ikey3, &bents2, &rsz}) {
        if (*pp) cudaFree(*pp);
        *pp = nullptr;
    }
    sorted_n = sig_n = poff_n = post_n = ctr_n = ents_n = bents_n = temp_n = ikey_n = ikey2_n =
        ival_n = rsig_n = hsh_n = table_n = dead_n = rstarts_n = ikey3_n = bents2_n = rsz_n = 0;
}

std::string filter_maximal(FilterScratch& F, const int32_t* d_res, int64_t nints,
                           const unsigned long long* d_starts, int64_t nsets, int32_t n_vertices,
                           cudaStream_t s, int sms, std::vector<int32_t>& host_out,
                           int64_t& host_nsets, int64_t* launches)
{
    host_out.clear();
    host_nsets = 0;
    if (nsets == 0) return "";
    if (nsets > INT32_MAX) return "filter: more than 2^31 emitted sets";
    std::string e;
    const int64_t nv = std::max<int64_t>(n_vertices, 1);
#define ENS(ptr, n, bytes)                                              \
    e = F.ensure((void**)&F.ptr, &F.ptr##_n, (size_t)(bytes));          \
    if (!e.empty()) return e;
    int64_t cap = 1;
    while (cap < 2 * nsets) cap <<= 1;
    ENS(sorted, sorted_n, sizeof(int32_t) * nints);
    ENS(sig, sig_n, 2 * sizeof(uint4) * nsets);
    ENS(rsig, rsig_n, 2 * sizeof(uint4) * nsets);
    ENS(hsh, hsh_n, sizeof(unsigned long long) * nsets);
    ENS(table, table_n, sizeof(unsigned long long) * cap);
    ENS(dead, dead_n, sizeof(int32_t) * nsets);
    ENS(rstarts, rstarts_n, sizeof(unsigned long long) * nsets);
    ENS(rsz, rsz_n, sizeof(int32_t) * nsets);
    ENS(poff, poff_n, sizeof(int64_t) * (nv + 1));
    ENS(ctr, ctr_n, 8 * sizeof(unsigned long long));
    ENS(ents, ents_n, sizeof(SetEnt) * nsets);
    // survivors' flat output: at most every emitted int
    ENS(ikey, ikey_n, sizeof(int32_t) * nints);
    unsigned long long* ctr = (unsigned long long*)F.ctr;
    // ctr: [0] incidences, [1] output ints, [2] output sets, [3] universe,
    //      [4] residual sets, [5] residual ints
    const int blocks = sms * 8;
    int64_t nlaunch = 0;
    sort_sig_kernel<<<blocks, 256, 0, s>>>(d_res, d_starts, nsets, (int32_t*)F.sorted,
                                           (uint4*)F.sig, (unsigned long long*)F.hsh);
    FCK(cudaMemsetAsync(F.table, 0xff, sizeof(unsigned long long) * cap, s));
    FCK(cudaMemsetAsync(F.dead, 0, sizeof(int32_t) * nsets, s));
    FCK(cudaMemsetAsync(ctr, 0, 8 * sizeof(unsigned long long), s));
    set_insert_kernel<<<blocks, 256, 0, s>>>((const unsigned long long*)F.hsh, (const int32_t*)F.sorted,
                                             d_starts, nsets, (unsigned long long*)F.table,
                                             (unsigned long long)(cap - 1));
    one_less_kernel<<<blocks, 256, 0, s>>>((const int32_t*)F.sorted, d_starts, nsets,
                                           (const unsigned long long*)F.hsh,
                                           (const unsigned long long*)F.table, (unsigned long long)(cap - 1),
                                           (int32_t*)F.dead);
    residual_kernel<<<blocks, 256, 0, s>>>((const int32_t*)F.sorted, d_starts, nsets,
                                           (const int32_t*)F.dead, (const uint4*)F.sig,
                                           (unsigned long long*)F.rstarts, (uint4*)F.rsig,
                                           (int32_t*)F.rsz, ctr + 4);
    int32_t* d_out = (int32_t*)F.ikey;
    residual_pairs_kernel<<<blocks, 256, 0, s>>>((const int32_t*)F.sorted,
                                                 (const unsigned long long*)F.rstarts,
                                                 (const uint4*)F.rsig, (const int32_t*)F.rsz, ctr,
                                                 d_out, (SetEnt*)F.ents);
    nlaunch += 5;
    // the survivors' universe: presence bitmap and ranks over the vertex range
    // (in the posting-list offsets' buffer)
    const int nwords = (int)((nv + 31) / 32);
    uint32_t* bitmap = (uint32_t*)F.poff;
    uint32_t* rank_base = bitmap + nwords;
    auto universe = [&]() -> std::string {
        FCK(cudaMemsetAsync(bitmap, 0, sizeof(uint32_t) * nwords, s));
        uni_mark_kernel<<<blocks, 256, 0, s>>>(d_out, (const SetEnt*)F.ents, ctr, bitmap);
        uni_rank_kernel<<<1, 1024, 0, s>>>(bitmap, nwords, rank_base, ctr);
        nlaunch += 2;
        return "";
    };
    e = universe();
    if (!e.empty()) return e;
    FCK(cudaGetLastError());
    if (!F.host || F.host_n < 16) {
        if (F.host) cudaFreeHost(F.host);
        F.host = nullptr;
        F.host_n = 0;
        FCK(cudaHostAlloc((void**)&F.host, 4096, cudaHostAllocDefault));
        F.host_n = 4096 / sizeof(int32_t);
    }
    int64_t c8[8];
    auto read_counts = [&]() -> std::string {
        FCK(cudaMemcpyAsync(F.host, ctr, 8 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        FCK(cudaStreamSynchronize(s));
        std::memcpy(c8, F.host, sizeof(c8));
        return "";
    };
    e = read_counts();
    if (!e.empty()) return e;
    const int64_t nres = c8[4], nres_ints = c8[5];
    if (nres < 0 || nres > nsets || nres_ints < 0 || nres_ints > nints)
        return "filter: residual count out of range";
    if (nres > kPairsMax) {
        // a large residual: inverted index over its incidences, sorted by
        // (vertex, set size descending), then the superset test per set
        const int64_t total = std::max<int64_t>(nres_ints - nres, 1);
        if (total > INT32_MAX) return "filter: more than 2^31 vertex incidences in the residual";
        ENS(ikey2, ikey2_n, sizeof(unsigned long long) * total);
        ENS(ikey3, ikey3_n, sizeof(unsigned long long) * total);
        ENS(ival, ival_n, sizeof(int32_t) * total);
        ENS(post, post_n, sizeof(int32_t) * total);
        emit_incidences_kernel<<<blocks, 256, 0, s>>>((int32_t*)F.sorted,
                                                      (const unsigned long long*)F.rstarts, nres,
                                                      ctr, (unsigned long long*)F.ikey3,
                                                      (int32_t*)F.ival);
        int vbits = 1;
        while (vbits < 47 && ((int64_t)1 << vbits) <= nv) vbits++;
        size_t tb4 = 0;
        FCK(cub::DeviceRadixSort::SortPairs(nullptr, tb4, (unsigned long long*)F.ikey3,
                                            (unsigned long long*)F.ikey2, (int32_t*)F.ival,
                                            (int32_t*)F.post, (int)total, 0, 16 + vbits, s));
        ENS(temp, temp_n, tb4 + 256);
        tb4 = F.temp_n;
        FCK(cub::DeviceRadixSort::SortPairs(F.temp, tb4, (unsigned long long*)F.ikey3,
                                            (unsigned long long*)F.ikey2, (int32_t*)F.ival,
                                            (int32_t*)F.post, (int)total, 0, 16 + vbits, s));
        inc_offsets_kernel<<<(unsigned)((nv + 1 + 255) / 256), 256, 0, s>>>(
            (unsigned long long*)F.ikey2, total, nv, (int64_t*)F.poff);
        maximal_kernel<<<blocks, 256, 0, s>>>((int32_t*)F.sorted,
                                              (const unsigned long long*)F.rstarts, nres,
                                              (int64_t*)F.poff, (int32_t*)F.post,
                                              (unsigned long long*)F.ikey2, (const uint4*)F.rsig,
                                              ctr, d_out, (SetEnt*)F.ents);
        nlaunch += 3;
        e = universe();
        if (!e.empty()) return e;
        FCK(cudaGetLastError());
        e = read_counts();
        if (!e.empty()) return e;
    }
    const int64_t out_ints = c8[1], out_sets = c8[2], uni = c8[3];
    if (out_ints < 0 || out_ints > nints || out_sets < 0 || out_sets > nsets)
        return "filter: survivor count out of range";
    // lexicographic order of the survivors on the device: by bit vectors when
    // the universe is small (one block for a few thousand), else by comparing
    // the sets
    const bool bits = uni <= kBitUniverse && out_sets > 1;
    void* sorted_bents = nullptr; // where the ordered bit-vector entries end up
    if (bits) {
        ENS(bents, bents_n, sizeof(BitEnt) * out_sets);
        sorted_bents = F.bents;
        bit_key_kernel<<<blocks, 256, 0, s>>>(d_out, (const SetEnt*)F.ents, (long long)out_sets,
                                              bitmap, rank_base, (BitEnt*)F.bents);
        nlaunch += 1;
        if (out_sets <= kRankSortMax) {
            ENS(bents2, bents2_n, sizeof(BitEnt) * out_sets);
            bit_rank_kernel<<<blocks, 256, 0, s>>>((const BitEnt*)F.bents, (int)out_sets,
                                                   (BitEnt*)F.bents2);
            nlaunch += 1;
            sorted_bents = F.bents2;
        } else {
            size_t tbm = 0;
            FCK(cub::DeviceMergeSort::SortKeys(nullptr, tbm, (BitEnt*)F.bents, (int64_t)out_sets,
                                               BitMore{}, s));
            ENS(temp, temp_n, tbm + 256);
            tbm = F.temp_n;
            FCK(cub::DeviceMergeSort::SortKeys(F.temp, tbm, (BitEnt*)F.bents, (int64_t)out_sets,
                                               BitMore{}, s));
        }
    } else if (out_sets > 1) {
        size_t tbm = 0;
        FCK(cub::DeviceMergeSort::SortKeys(nullptr, tbm, (SetEnt*)F.ents, (int64_t)out_sets,
                                           SetLess{d_out}, s));
        ENS(temp, temp_n, tbm + 256);
        tbm = F.temp_n;
        FCK(cub::DeviceMergeSort::SortKeys(F.temp, tbm, (SetEnt*)F.ents, (int64_t)out_sets,
                                           SetLess{d_out}, s));
    }
    FCK(cudaGetLastError());
    if (launches) *launches += nlaunch;
    // read back: the sets as appended, then their entries in order
    const size_t ent_ints = (bits ? sizeof(BitEnt) : sizeof(SetEnt)) / sizeof(int32_t);
    const size_t want_ints = (size_t)out_ints + 4 + ent_ints * (size_t)out_sets;
    if (want_ints > F.host_n) {
        const size_t want = std::max<size_t>(want_ints, 2 * F.host_n);
        cudaFreeHost(F.host);
        F.host = nullptr;
        F.host_n = 0;
        FCK(cudaHostAlloc((void**)&F.host, sizeof(int32_t) * want, cudaHostAllocDefault));
        F.host_n = want;
    }
    const SetEnt* he = (const SetEnt*)(F.host + (size_t)out_ints + ((size_t)out_ints & 3u ? 4 - ((size_t)out_ints & 3u) : 0));
    if (out_ints) {
        FCK(cudaMemcpyAsync(F.host, d_out, sizeof(int32_t) * out_ints, cudaMemcpyDeviceToHost, s));
        if (bits)
            FCK(cudaMemcpyAsync((void*)he, sorted_bents, sizeof(BitEnt) * out_sets,
                                cudaMemcpyDeviceToHost, s));
        else
            FCK(cudaMemcpyAsync((void*)he, F.ents, sizeof(SetEnt) * out_sets, cudaMemcpyDeviceToHost, s));
        FCK(cudaStreamSynchronize(s));
    }
#undef ENS
    const int32_t* F0 = F.host;
    host_out.resize((size_t)out_ints);
    int32_t* o = host_out.data();
    int64_t done = 0;
    for (int64_t j = 0; j < out_sets; j++) {
        const long long at = bits ? ((const BitEnt*)he)[j].at : he[j].at;
        const int32_t k = at >= 0 && at < out_ints ? F0[at] : -1;
        if (k < 0 || at + 1 + k > out_ints || done + 1 + k > out_ints)
            return "filter: malformed survivor record";
        std::memcpy(o, F0 + at, sizeof(int32_t) * (size_t)(k + 1));
        o += k + 1;
        done += k + 1;
    }
    if (done != out_ints) return "filter: survivor records do not cover the output";
    host_nsets = out_sets;
    return "";
}

} // namespace qcb
