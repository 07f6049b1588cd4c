// cuda_emu.h -- TEST INFRASTRUCTURE: runs warp-synchronous CUDA device code
// on the CPU so the expansion kernel's logic can be checked without a GPU.
//
// Every emulated lane is a std::thread; a warp is 32 of them sharing a
// barrier.  Warp collectives (__shfl*_sync, __ballot_sync, __any_sync,
// __syncwarp) exchange through per-warp slots between two barrier phases, so
// the code must call them uniformly across the warp -- the same requirement
// CUDA places on full-mask collectives.  Global-memory atomics map to GCC
// __atomic builtins.  This file is never part of the product library.
#pragma once
#include <atomic>
#include <barrier>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#define QC_EMULATION 1
#define __device__
#define __global__
#define __host__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
// block-shared variables of a kernel: one copy per process, so an emulated
// kernel that declares them runs as a single block, one launch at a time
#define __shared__ static

struct emu_dim3 {
    unsigned x = 0, y = 0, z = 0;
};
inline thread_local emu_dim3 threadIdx, blockIdx, blockDim, gridDim;

// Sense-reversing barrier of the 32 emulated lanes: lanes spin briefly, then
// yield the core (the futex-based std::barrier spent most of its time in the
// kernel with 32 threads per warp on a few cores).
struct EmuBarrier {
    std::atomic<int> count{0};
    std::atomic<int> phase{0};
    int parties = 32;
    void arrive_and_wait()
    {
        int ph = phase.load(std::memory_order_acquire);
        if (count.fetch_add(1, std::memory_order_acq_rel) == parties - 1) {
            count.store(0, std::memory_order_relaxed);
            phase.store(ph + 1, std::memory_order_release);
            return;
        }
        for (int spin = 0; phase.load(std::memory_order_acquire) == ph; spin++)
            if (spin > 64) std::this_thread::yield();
    }
};

struct EmuWarp {
    EmuBarrier bar;
    uint64_t slot[32];
};
inline thread_local EmuWarp* emu_w = nullptr;
inline thread_local EmuBarrier* emu_blk = nullptr; // every thread of this block
inline thread_local int emu_lane = 0;
inline thread_local unsigned char* emu_smem = nullptr; // this block's dynamic shared memory
inline unsigned char* emu_dyn_smem() { return emu_smem; }

inline uint64_t emu_xchg(uint64_t v, int src)
{
    emu_w->slot[emu_lane] = v;
    emu_w->bar.arrive_and_wait();
    uint64_t r = emu_w->slot[src & 31];
    emu_w->bar.arrive_and_wait();
    return r;
}

template <class T> inline uint64_t emu_bits(T v)
{
    uint64_t b = 0;
    std::memcpy(&b, &v, sizeof(T));
    return b;
}
template <class T> inline T emu_from(uint64_t b)
{
    T v;
    std::memcpy(&v, &b, sizeof(T));
    return v;
}

template <class T> inline T __shfl_sync(unsigned, T v, int src)
{
    return emu_from<T>(emu_xchg(emu_bits(v), src));
}
template <class T> inline T __shfl_xor_sync(unsigned, T v, int x)
{
    return emu_from<T>(emu_xchg(emu_bits(v), emu_lane ^ x));
}
template <class T> inline T __shfl_up_sync(unsigned, T v, int d)
{
    int src = emu_lane - d;
    T r = emu_from<T>(emu_xchg(emu_bits(v), src < 0 ? emu_lane : src));
    return r;
}
inline unsigned __ballot_sync(unsigned, int pred)
{
    emu_w->slot[emu_lane] = pred ? 1 : 0;
    emu_w->bar.arrive_and_wait();
    unsigned r = 0;
    for (int i = 0; i < 32; i++)
        if (emu_w->slot[i]) r |= 1u << i;
    emu_w->bar.arrive_and_wait();
    return r;
}
// lanes whose value equals this lane's
inline unsigned __match_any_sync(unsigned, int v)
{
    emu_w->slot[emu_lane] = (uint64_t)(uint32_t)v;
    emu_w->bar.arrive_and_wait();
    unsigned r = 0;
    for (int i = 0; i < 32; i++)
        if (emu_w->slot[i] == (uint64_t)(uint32_t)v) r |= 1u << i;
    emu_w->bar.arrive_and_wait();
    return r;
}
inline int __any_sync(unsigned m, int pred) { return __ballot_sync(m, pred) != 0; }
inline int __all_sync(unsigned m, int pred) { return __ballot_sync(m, pred) == 0xffffffffu; }
inline void __syncwarp(unsigned = 0xffffffffu) { emu_w->bar.arrive_and_wait(); }
inline void __syncthreads()
{
    std::atomic_thread_fence(std::memory_order_seq_cst);
    emu_blk->arrive_and_wait();
    std::atomic_thread_fence(std::memory_order_seq_cst);
}
inline int __popc(unsigned x) { return __builtin_popcount(x); }
template <class T> inline T __ldcg(const T* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
template <class T> inline T __ldg(const T* p) { return *p; }
struct uint4 {
    unsigned x, y, z, w;
};
inline uint4 __ldcg(const uint4* p) { return *p; }
// every emulated address is host memory; the kernel's global-only loads work on all of it
inline unsigned __isGlobal(const void*) { return 1; }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __ffs(unsigned x) { return x ? __builtin_ctz(x) + 1 : 0; }
inline int __clz(unsigned x) { return x ? __builtin_clz(x) : 32; }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
// an idle emulated warp sleeps instead of spinning, so busy warps get the host cores
inline void __nanosleep(unsigned ns) { std::this_thread::sleep_for(std::chrono::microseconds(20 + ns / 100)); }

inline int atomicAdd(int* a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicAdd(unsigned long long* a, unsigned long long v)
{
    return __atomic_fetch_add(a, v, __ATOMIC_SEQ_CST);
}
inline int atomicSub(int* a, int v) { return __atomic_fetch_sub(a, v, __ATOMIC_SEQ_CST); }
inline int atomicOr(int* a, int v) { return __atomic_fetch_or(a, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicOr(unsigned* a, unsigned v) { return __atomic_fetch_or(a, v, __ATOMIC_SEQ_CST); }
inline unsigned long long atomicOr(unsigned long long* a, unsigned long long v)
{
    return __atomic_fetch_or(a, v, __ATOMIC_SEQ_CST);
}
inline int atomicExch(int* a, int v) { return __atomic_exchange_n(a, v, __ATOMIC_SEQ_CST); }
inline int atomicCAS(int* a, int cmp, int v)
{
    __atomic_compare_exchange_n(a, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
inline unsigned long long atomicCAS(unsigned long long* a, unsigned long long cmp,
                                    unsigned long long v)
{
    __atomic_compare_exchange_n(a, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
inline unsigned long long atomicMax(unsigned long long* a, unsigned long long v)
{
    unsigned long long cur = __atomic_load_n(a, __ATOMIC_SEQ_CST);
    while (cur < v && !__atomic_compare_exchange_n(a, &cur, v, false, __ATOMIC_SEQ_CST,
                                                   __ATOMIC_SEQ_CST)) {
    }
    return cur;
}
inline int atomicMax(int* a, int v)
{
    int cur = __atomic_load_n(a, __ATOMIC_SEQ_CST);
    while (cur < v && !__atomic_compare_exchange_n(a, &cur, v, false, __ATOMIC_SEQ_CST,
                                                   __ATOMIC_SEQ_CST)) {
    }
    return cur;
}

inline unsigned long long emu_globaltimer()
{
    return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Run `fn` as a grid of `blocks` x `threads` (threads a multiple of 32) with
// `smem_bytes` of dynamic shared memory per block.
inline void emu_launch(int blocks, int threads, const std::function<void()>& fn,
                       size_t smem_bytes = 0)
{
    int nwarps_per_block = threads / 32;
    std::vector<EmuWarp*> warps;
    std::vector<std::thread> th;
    std::vector<std::vector<unsigned char>> smem((size_t)blocks,
                                                 std::vector<unsigned char>(smem_bytes + 16));
    std::vector<EmuBarrier> blk((size_t)blocks);
    for (auto& bb : blk) bb.parties = threads;
    for (int b = 0; b < blocks; b++)
        for (int w = 0; w < nwarps_per_block; w++) {
            EmuWarp* ew = new EmuWarp();
            warps.push_back(ew);
            unsigned char* sb = smem[(size_t)b].data();
            EmuBarrier* bbar = &blk[(size_t)b];
            for (int l = 0; l < 32; l++) {
                th.emplace_back([=, &fn] {
                    emu_w = ew;
                    emu_blk = bbar;
                    emu_lane = l;
                    emu_smem = sb;
                    threadIdx.x = w * 32 + l;
                    blockIdx.x = b;
                    blockDim.x = threads;
                    gridDim.x = blocks;
                    fn();
                });
            }
        }
    for (auto& t : th) t.join();
    for (auto* w : warps) delete w;
}
