// level0_grid.cuh -- level 0 of the search (the root task) over the whole
// grid, for graphs above the one-block limit of level0_kernel.cuh.  Included
// by qc.cu and, for the CPU test suite, by the warp emulator (tests/emu), which
// runs it as a grid of one block.
//
// Same rules as the one-block form (initialize_tasks, main.cu:846-998; the
// host form is build_root in host.cpp): keep the vertices with deg >= need and
// |N2| >= min_size-1, peel to the subgraph where every kept vertex has >= need
// kept neighbours (the k-core of the kept vertices is unique, so peeling in
// rounds keeps the same vertices as the reference's order), mark the cover
// vertex (largest exdeg, smallest id on ties) and its surviving neighbours,
// and write the survivors in Q order: covered, candidates, cover, then
// exdeg, 2-hop size and id, all descending.
//
// One cooperative launch: the phases are separated by grid-wide barriers
// (every block is resident, so a barrier always completes).  Arrays that
// other blocks write are read through L2 (ld.global.cg), never from a stale
// L1 line.  The survivors are ordered by a bitonic network over 128-bit keys
// (rank, exdeg, 2-hop size | id), one compare-exchange stage per barrier.
#pragma once
#include <stdint.h>

#ifndef QC_EMULATION
#include <cooperative_groups.h>
#endif

// Largest vertex count of the grid form (ids, degrees and 2-hop sizes are
// 31-bit key fields).
constexpr int64_t kLevel0GridMax = (int64_t)1 << 30;

struct L0Key {
    unsigned long long hi, lo;
};

// Scratch of one grid level-0 run over n vertices: int32 exdeg, label, 2-hop
// size; 128-bit keys for up to n survivors padded to a power of two; a
// control block of 8 words (round flags, best cover key, counts).
__host__ __device__ inline int64_t level0_grid_scratch_bytes(int64_t n)
{
    int64_t P = 1;
    while (P < n) P <<= 1;
    const int64_t a = ((n * 4 + 15) / 16) * 16;
    return 3 * a + 16 * P + 64;
}

__device__ __forceinline__ void l0_grid_sync()
{
#ifdef QC_EMULATION
    __syncthreads(); // the emulator runs the grid as one block
#else
    cooperative_groups::this_grid().sync();
#endif
}

// a word other blocks may have written since the last barrier (through L2)
__device__ __forceinline__ int l0_ld(const int32_t* p) { return __ldcg(p); }

__device__ __forceinline__ bool key_gt(const L0Key& a, const L0Key& b)
{
    return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo);
}

// info = {root size, covered count}; ids receives the root in Q order.
__global__ void __launch_bounds__(256) level0_grid_kernel(const int64_t* off, const int32_t* adj,
                                                          const int64_t* off2, int64_t n, int need,
                                                          int min_size, char* scratch, int32_t* ids,
                                                          int32_t* info)
{
    const int64_t a = ((n * 4 + 15) / 16) * 16;
    int32_t* exdeg = (int32_t*)scratch;
    int32_t* label = (int32_t*)(scratch + a);
    int32_t* l2 = (int32_t*)(scratch + 2 * a);
    int64_t P = 1;
    while (P < n) P <<= 1;
    L0Key* keys = (L0Key*)(scratch + 3 * a);
    unsigned long long* ctl = (unsigned long long*)(scratch + 3 * a + 16 * P);
    // ctl[0], ctl[1]: "a vertex left" flags of even and odd rounds; ctl[2]: best
    // cover key; ctl[3]: survivors; ctl[4]: covered (all zero at launch)
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * blockDim.x;
    for (int64_t v = tid; v < n; v += nt) {
        const int64_t d = off[v + 1] - off[v];
        const int64_t d2 = off2[v + 1] - off2[v];
        l2[v] = (int32_t)d2;
        label[v] = (d >= need && d2 >= min_size - 1) ? 0 : -1;
    }
    l0_grid_sync();
    for (int64_t v = tid; v < n; v += nt) {
        if (l0_ld(label + v) != 0) continue;
        int c = 0;
        for (int64_t e = off[v]; e < off[v + 1]; e++) c += l0_ld(label + adj[e]) == 0;
        exdeg[v] = c;
    }
    l0_grid_sync();
    for (int r = 0;; r++) {
        unsigned long long* flag = ctl + (r & 1);
        bool any = false;
        for (int64_t v = tid; v < n; v += nt)
            if (l0_ld(label + v) == 0 && l0_ld(exdeg + v) < need) {
                label[v] = -2;
                any = true;
            }
        if (any) atomicOr(flag, 1ull);
        l0_grid_sync();
        if (*(volatile unsigned long long*)flag == 0) break;
        if (tid == 0) ctl[(r + 1) & 1] = 0; // the next round's flag, read last a round ago
        for (int64_t v = tid; v < n; v += nt)
            if (l0_ld(label + v) == -2)
                for (int64_t e = off[v]; e < off[v + 1]; e++) {
                    const int64_t w = adj[e];
                    if (l0_ld(label + w) == 0) atomicSub(&exdeg[w], 1);
                }
        l0_grid_sync();
        for (int64_t v = tid; v < n; v += nt)
            if (l0_ld(label + v) == -2) label[v] = -1;
        l0_grid_sync();
    }
    for (int64_t v = tid; v < n; v += nt)
        if (l0_ld(label + v) == 0) {
            const int ex = l0_ld(exdeg + v);
            if (ex > 0)
                atomicMax(ctl + 2, ((unsigned long long)(unsigned)ex << 32) |
                                       (unsigned long long)(0xffffffffu - (unsigned)v));
        }
    l0_grid_sync();
    const unsigned long long best = *(volatile unsigned long long*)(ctl + 2);
    if (best) {
        const int64_t bv = (int64_t)(0xffffffffu - (unsigned)(best & 0xffffffffull));
        for (int64_t e = off[bv] + tid; e < off[bv + 1]; e += nt) {
            const int64_t w = adj[e];
            if (l0_ld(label + w) == 0) label[w] = 2;
        }
        l0_grid_sync();
        if (tid == 0) label[bv] = 3;
    }
    l0_grid_sync();
    for (int64_t v = tid; v < n; v += nt) {
        const int lb = l0_ld(label + v);
        if (lb < 0) continue;
        const unsigned long long rank = lb == 2 ? 0ull : (lb == 0 ? 1ull : 2ull);
        L0Key k;
        k.hi = (rank << 62) | ((unsigned long long)(0x7fffffff - l0_ld(exdeg + v)) << 31) |
               (unsigned long long)(0x7fffffff - l2[v]);
        k.lo = (unsigned long long)(0x7fffffffll - v);
        keys[atomicAdd(ctl + 3, 1ull)] = k;
        if (lb == 2) atomicAdd(ctl + 4, 1ull);
    }
    l0_grid_sync();
    const int64_t t = (int64_t)*(volatile unsigned long long*)(ctl + 3);
    int64_t N = 1;
    while (N < t) N <<= 1;
    for (int64_t i = t + tid; i < N; i += nt) keys[i] = L0Key{~0ull, ~0ull};
    l0_grid_sync();
    for (int64_t k = 2; k <= N; k <<= 1)
        for (int64_t j = k >> 1; j > 0; j >>= 1) {
            for (int64_t i = tid; i < N; i += nt) {
                const int64_t p = i ^ j;
                if (p > i) {
                    volatile L0Key* vk = (volatile L0Key*)keys;
                    const L0Key x{vk[i].hi, vk[i].lo}, y{vk[p].hi, vk[p].lo};
                    if (key_gt(x, y) == ((i & k) == 0)) {
                        keys[i] = y;
                        keys[p] = x;
                    }
                }
            }
            l0_grid_sync();
        }
    for (int64_t i = tid; i < t; i += nt) {
        const volatile L0Key* vk = (const volatile L0Key*)keys;
        ids[i] = (int32_t)(0x7fffffffll - (long long)vk[i].lo);
    }
    if (tid == 0) {
        info[0] = (int32_t)t;
        info[1] = (int32_t)*(volatile unsigned long long*)(ctl + 4);
    }
}
