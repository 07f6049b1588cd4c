// level0_kernel.cuh -- level 0 of the search on the device (the root task),
// for graphs of at most kLevel0DeviceMax vertices.  Included by qc.cu and, for
// the CPU test suite, by the warp emulator (tests/emu).
#pragma once
#include <stdint.h>

// Level 0 on the device for graphs of at most kLevel0DeviceMax vertices
// (initialize_tasks, main.cu:846-998; the host form is build_root in
// host.cpp): one block keeps the vertices with deg >= need and
// |N2| >= min_size-1, peels to the subgraph where every vertex keeps >= need
// neighbours (the k-core of the kept vertices is unique, so removing the
// vertices in rounds instead of the reference's order keeps the same ones),
// marks the cover vertex (largest exdeg, smallest id on ties) and its
// surviving neighbours, and writes the survivors in Q order: covered,
// candidates, cover, then exdeg, 2-hop size and id, all descending.
// info = {root size, covered count}.
constexpr int kLevel0DeviceMax = 65536;

// Scratch of one level-0 run over n vertices: int32 exdeg, label and 2-hop
// size arrays, then the 64-bit sort keys (padded to a power of two); every
// array starts 16-byte aligned.
__host__ __device__ inline int64_t level0_array_bytes(int n) { return ((int64_t)n * 4 + 15) & ~(int64_t)15; }
__host__ __device__ inline int64_t level0_scratch_bytes(int n)
{
    int64_t P = 1;
    while (P < n) P <<= 1;
    return 3 * level0_array_bytes(n) + 8 * P;
}

// One instance of a batched launch: its graph, rules and where its scratch
// and root ids go.
struct Level0Job {
    const int64_t* off;
    const int32_t* adj;
    const int64_t* off2;
    int32_t n, need, min_size, pad;
    int64_t scratch_at; // byte offset of the instance's scratch
    int64_t ids_at;     // first entry of its root ids in the shared id array
};

// The work of one block (all of its threads take part).
__device__ void level0_block(const int64_t* off, const int32_t* adj, const int64_t* off2, int n,
                             int need, int min_size, int32_t* exdeg, int32_t* label, int32_t* l2,
                             unsigned long long* keys, int32_t* ids, int32_t* info)
{
    __shared__ int changed, cnt, ncov;
    __shared__ unsigned long long best;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int v = tid; v < n; v += nt) {
        const int d = (int)(off[v + 1] - off[v]);
        const int d2 = (int)(off2[v + 1] - off2[v]);
        l2[v] = d2;
        label[v] = (d >= need && d2 >= min_size - 1) ? 0 : -1;
    }
    __syncthreads();
    for (int v = tid; v < n; v += nt) {
        if (label[v] != 0) continue;
        int c = 0;
        for (int64_t e = off[v]; e < off[v + 1]; e++) c += label[adj[e]] == 0;
        exdeg[v] = c;
    }
    __syncthreads();
    for (;;) {
        if (tid == 0) changed = 0;
        __syncthreads();
        for (int v = tid; v < n; v += nt)
            if (label[v] == 0 && exdeg[v] < need) {
                label[v] = -2;
                changed = 1;
            }
        __syncthreads();
        if (!changed) break;
        for (int v = tid; v < n; v += nt)
            if (label[v] == -2)
                for (int64_t e = off[v]; e < off[v + 1]; e++) {
                    const int w = adj[e];
                    if (label[w] == 0) atomicSub(&exdeg[w], 1);
                }
        __syncthreads();
        for (int v = tid; v < n; v += nt)
            if (label[v] == -2) label[v] = -1;
        __syncthreads();
    }
    if (tid == 0) {
        best = 0;
        cnt = 0;
        ncov = 0;
    }
    __syncthreads();
    for (int v = tid; v < n; v += nt)
        if (label[v] == 0 && exdeg[v] > 0)
            atomicMax(&best, ((unsigned long long)(unsigned)exdeg[v] << 32) |
                                 (unsigned long long)(0xffffffffu - (unsigned)v));
    __syncthreads();
    if (best) {
        const int bv = (int)(0xffffffffu - (unsigned)(best & 0xffffffffull));
        for (int64_t e = off[bv] + tid; e < off[bv + 1]; e += nt) {
            const int w = adj[e];
            if (label[w] == 0) label[w] = 2;
        }
        __syncthreads();
        if (tid == 0) label[bv] = 3;
    }
    __syncthreads();
    for (int v = tid; v < n; v += nt) {
        const int lb = label[v];
        if (lb < 0) continue;
        const unsigned long long rank = lb == 2 ? 0ull : (lb == 0 ? 1ull : 2ull);
        const unsigned long long key = (rank << 51) |
                                       ((unsigned long long)(0x1ffff - exdeg[v]) << 34) |
                                       ((unsigned long long)(0x1ffff - l2[v]) << 17) |
                                       (unsigned long long)(0x1ffff - v);
        keys[atomicAdd(&cnt, 1)] = key;
        if (lb == 2) atomicAdd(&ncov, 1);
    }
    __syncthreads();
    const int t = cnt;
    if ((int64_t)t * t <= 4096ll * nt) {
        // few survivors: each key's place is the number of smaller keys (the
        // keys are distinct: they end in the vertex id)
        for (int i = tid; i < t; i += nt) {
            const unsigned long long k = keys[i];
            int r = 0;
            for (int j = 0; j < t; j++) r += keys[j] < k ? 1 : 0;
            ids[r] = 0x1ffff - (int)(k & 0x1ffffull);
        }
        if (tid == 0) {
            info[0] = t;
            info[1] = ncov;
        }
        return;
    }
    int N = 1;
    while (N < t) N <<= 1;
    for (int i = t + tid; i < N; i += nt) keys[i] = ~0ull;
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < N; i += nt) {
                const int p = i ^ j;
                if (p > i) {
                    const unsigned long long x = keys[i], y = keys[p];
                    if ((x > y) == ((i & k) == 0)) {
                        keys[i] = y;
                        keys[p] = x;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = tid; i < t; i += nt) ids[i] = 0x1ffff - (int)(keys[i] & 0x1ffffull);
    if (tid == 0) {
        info[0] = t;
        info[1] = ncov;
    }
}

__global__ void __launch_bounds__(1024) level0_kernel(const int64_t* off, const int32_t* adj,
                                                      const int64_t* off2, int n, int need,
                                                      int min_size, int32_t* exdeg, int32_t* label,
                                                      int32_t* l2, unsigned long long* keys,
                                                      int32_t* ids, int32_t* info)
{
    level0_block(off, adj, off2, n, need, min_size, exdeg, label, l2, keys, ids, info);
}

// Graphs of at most this many vertices keep level 0's arrays (exdeg, label,
// 2-hop sizes, sort keys: level0_scratch_bytes, 40 KB at this size) in the
// block's shared memory instead of global scratch.
constexpr int kLevel0SmemMax = 2048;

#ifndef QC_EMULATION
extern __shared__ __align__(16) unsigned char qc_l0_smem[];
__global__ void __launch_bounds__(1024) level0_smem_kernel(const int64_t* off, const int32_t* adj,
                                                           const int64_t* off2, int n, int need,
                                                           int min_size, int32_t* ids, int32_t* info)
{
    char* z = (char*)qc_l0_smem;
    const int64_t nb = level0_array_bytes(n);
    level0_block(off, adj, off2, n, need, min_size, (int32_t*)z, (int32_t*)(z + nb),
                 (int32_t*)(z + 2 * nb), (unsigned long long*)(z + 3 * nb), ids, info);
}
#endif

// Level 0 of many instances at once, one block per instance (batched mining):
// info[2i], info[2i+1] = root size and covered count of instance i.
__global__ void __launch_bounds__(256) level0_batch_kernel(const Level0Job* jobs, char* scratch,
                                                           int32_t* ids_all, int32_t* info)
{
    const Level0Job J = jobs[blockIdx.x];
    char* z = scratch + J.scratch_at;
    const int64_t nb = level0_array_bytes(J.n);
    level0_block(J.off, J.adj, J.off2, J.n, J.need, J.min_size, (int32_t*)z, (int32_t*)(z + nb),
                 (int32_t*)(z + 2 * nb), (unsigned long long*)(z + 3 * nb), ids_all + J.ids_at,
                 info + 2 * (int64_t)blockIdx.x);
}
