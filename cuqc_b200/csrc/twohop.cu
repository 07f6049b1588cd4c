// twohop.cu -- 2-hop lists on the GPU (replaces the offline preprocessing of
// Mike12041204/cuQC adjToSer.cpp:115-156):
//     N2(v) = sorted(N(v) u N(N(v)) minus {v})
//
// One warp per vertex.  Each warp owns a bitmap of n bits in global memory
// (L2-resident for moderate n) and a list of the bitmap words it touched.
// Lanes stream N(v) and every N(u), u in N(v), with coalesced loads and set
// bits with atomicOr; a word seen for the first time is appended to the
// touched list.  Pass 1 counts set bits per vertex, a scan gives the offsets,
// pass 2 repeats the marking, sorts the touched word indices (warp bitonic)
// and writes each word's set bits in order -- ascending ids -- then clears
// the touched words.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qc.h"
#include "host.h"

using namespace qcb;

namespace {

constexpr int kTwohopWarpsPerBlock = 8;

// Marks N(v) u N(N(v)) minus {v} in the warp's bitmap.  With `err` set (the
// no-allocation form, whose CSR was not checked on the host) an id outside
// [0, n) is skipped and recorded instead of being used as an index.
__device__ void mark_row(int n, const int64_t* off, const int32_t* adj, int v, uint32_t* bm,
                         int32_t* touched, int* ntouched, int lane, int* err)
{
    auto mark = [&](int w) {
        if (err && (unsigned)w >= (unsigned)n) {
            atomicOr(err, 2);
            return;
        }
        uint32_t b = 1u << (w & 31);
        uint32_t old = atomicOr(&bm[w >> 5], b);
        if (old == 0) {
            int k = atomicAdd(ntouched, 1);
            touched[k] = w >> 5;
        }
    };
    for (int64_t e = off[v] + lane; e < off[v + 1]; e += 32) mark(adj[e]);
    for (int64_t e = off[v]; e < off[v + 1]; e++) {
        int u = adj[e];
        if (err && (unsigned)u >= (unsigned)n) continue; // recorded by mark(u) above
        for (int64_t f = off[u] + lane; f < off[u + 1]; f += 32) {
            int w = adj[f];
            if (w != v) mark(w);
        }
    }
    __syncwarp();
}

// pass 1: counts; pass 2: write rows (off2 known)
__global__ void twohop_kernel(int n, const int64_t* off, const int32_t* adj, uint32_t* bitmaps,
                              int64_t bm_words, int32_t* touched_all, int64_t touched_cap,
                              int* ntouched_all, int64_t* count_out, const int64_t* off2,
                              int32_t* adj2, int* err)
{
    if (err && *(volatile int*)err) return; // the CSR check failed: write nothing
    int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int nw = (gridDim.x * blockDim.x) >> 5;
    uint32_t* bm = bitmaps + (int64_t)warp * bm_words;
    int32_t* touched = touched_all + (int64_t)warp * touched_cap;
    int* nt = ntouched_all + warp;
    for (int v = warp; v < n; v += nw) {
        if (lane == 0) *nt = 0;
        __syncwarp();
        mark_row(n, off, adj, v, bm, touched, nt, lane, err);
        // a self loop in N(v) keeps v (as the reference keeps it); v is never
        // added through N(N(v))
        int k = *(volatile int*)nt;
        if (!off2) {
            int c = 0;
            for (int i = lane; i < k; i += 32) c += __popc(bm[touched[i]]);
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0) count_out[v] = c;
        } else {
            // sort touched word indices ascending (bitonic, padded with INT_MAX)
            int N = 1;
            while (N < k) N <<= 1;
            for (int i = k + lane; i < N; i += 32) touched[i] = 0x7fffffff;
            __syncwarp();
            for (int s = 2; s <= N; s <<= 1)
                for (int j = s >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < N; i += 32) {
                        int p = i ^ j;
                        if (p > i) {
                            int a = touched[i], b = touched[p];
                            bool up = (i & s) == 0;
                            if ((a > b) == up) {
                                touched[i] = b;
                                touched[p] = a;
                            }
                        }
                    }
                    __syncwarp();
                }
            // write ids in ascending order
            int64_t base = off2[v];
            int carry = 0;
            for (int c0 = 0; c0 < k; c0 += 32) {
                int i = c0 + lane;
                uint32_t word = i < k ? bm[touched[i]] : 0u;
                int cnt = __popc(word);
                int inc = cnt;
                for (int o = 1; o < 32; o <<= 1) {
                    int y = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += y;
                }
                int at = carry + inc - cnt;
                int wbase = i < k ? touched[i] * 32 : 0;
                while (word) {
                    int b = __ffs(word) - 1;
                    word &= word - 1;
                    adj2[base + at++] = wbase + b;
                }
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
        }
        __syncwarp();
        for (int i = lane; i < k; i += 32) bm[touched[i]] = 0;
        __syncwarp();
    }
}

std::string g_th_err;

} // namespace

#define TCK(call)                                                              \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            g_th_err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
            goto done;                                                         \
        }                                                                      \
    } while (0)

// Build 2-hop lists on device 0.  Returns "" or an error message.
std::string qcb_twohop_device(const HostGraph& h, std::vector<int64_t>& off2,
                              std::vector<int32_t>& adj2)
{
    const int n = h.n;
    off2.assign((size_t)n + 1, 0);
    adj2.clear();
    if (n == 0) return "";
    int64_t *d_off = nullptr, *d_cnt = nullptr, *d_off2 = nullptr;
    int32_t *d_adj = nullptr, *d_touched = nullptr, *d_adj2 = nullptr;
    uint32_t* d_bm = nullptr;
    int* d_nt = nullptr;
    int sms = 0;
    int64_t bm_words = ((int64_t)n + 31) / 32;
    int64_t touched_cap = 1;
    int blocks = 0, nwarps = 0;
    std::vector<int64_t> cnt;
    g_th_err.clear();
    while (touched_cap < bm_words) touched_cap <<= 1;
    TCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    blocks = sms * 2;
    nwarps = blocks * kTwohopWarpsPerBlock;
    TCK(cudaMalloc(&d_off, sizeof(int64_t) * (n + 1)));
    TCK(cudaMalloc(&d_adj, sizeof(int32_t) * std::max<size_t>(h.adj.size(), 1)));
    TCK(cudaMalloc(&d_cnt, sizeof(int64_t) * n));
    TCK(cudaMalloc(&d_bm, sizeof(uint32_t) * bm_words * nwarps));
    TCK(cudaMalloc(&d_touched, sizeof(int32_t) * touched_cap * nwarps));
    TCK(cudaMalloc(&d_nt, sizeof(int) * nwarps));
    TCK(cudaMemset(d_bm, 0, sizeof(uint32_t) * bm_words * nwarps));
    TCK(cudaMemcpy(d_off, h.off.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
    if (!h.adj.empty())
        TCK(cudaMemcpy(d_adj, h.adj.data(), sizeof(int32_t) * h.adj.size(), cudaMemcpyHostToDevice));
    twohop_kernel<<<blocks, kTwohopWarpsPerBlock * 32>>>(n, d_off, d_adj, d_bm, bm_words, d_touched,
                                                         touched_cap, d_nt, d_cnt, nullptr, nullptr,
                                                         nullptr);
    TCK(cudaGetLastError());
    cnt.resize((size_t)n);
    TCK(cudaMemcpy(cnt.data(), d_cnt, sizeof(int64_t) * n, cudaMemcpyDeviceToHost));
    for (int v = 0; v < n; v++) off2[(size_t)v + 1] = off2[(size_t)v] + cnt[(size_t)v];
    adj2.resize((size_t)off2[(size_t)n]);
    TCK(cudaMalloc(&d_off2, sizeof(int64_t) * (n + 1)));
    TCK(cudaMalloc(&d_adj2, sizeof(int32_t) * std::max<size_t>(adj2.size(), 1)));
    TCK(cudaMemcpy(d_off2, off2.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
    twohop_kernel<<<blocks, kTwohopWarpsPerBlock * 32>>>(n, d_off, d_adj, d_bm, bm_words, d_touched,
                                                         touched_cap, d_nt, nullptr, d_off2, d_adj2,
                                                         nullptr);
    TCK(cudaGetLastError());
    if (!adj2.empty())
        TCK(cudaMemcpy(adj2.data(), d_adj2, sizeof(int32_t) * adj2.size(), cudaMemcpyDeviceToHost));
done:
    cudaFree(d_off);
    cudaFree(d_adj);
    cudaFree(d_cnt);
    cudaFree(d_bm);
    cudaFree(d_touched);
    cudaFree(d_nt);
    cudaFree(d_off2);
    cudaFree(d_adj2);
    return g_th_err;
}

// ------------------------------------------------------------------
// Two-hop lists without any device allocation (qc_twohop_noalloc).
//
// For callers that cannot call cudaMalloc: an application whose device
// memory is owned by its own pool or fixed memory plan, or that must not
// allocate while it is serving requests.  Inputs and outputs are the
// caller's device buffers; the working memory lives in one file-scope
// __device__ array that every GPU which loads this library holds until the
// process exits:
//   [0, 256)        status: the two-hop entry count and the CSR-check flags
//   [256, ...)      per-warp bitmaps of n bits, touched-word lists, counters
// The caller's CSR is in device memory, so it is checked on the device
// (csr_check_kernel) before any of it is used as an index.
// ------------------------------------------------------------------

namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB per device
constexpr size_t kNoAllocHeaderBytes = 256;          // status words ahead of the warps' memory
constexpr int kNoAllocMinWarps = 32;                 // fewest warps a call may run on
constexpr int kNoAllocMaxDevices = 64;

// CSR-check flags (NoAllocStatus::err)
constexpr int kErrOffsets = 1;   // off[0] != 0 or off[v] > off[v+1]
constexpr int kErrIds = 2;       // a neighbour id outside [0, n)
constexpr int kErrNullAdj = 4;   // entries but no adjacency array

struct NoAllocStatus {
    int64_t total; // two-hop entries (off2[n]) after the scan
    int32_t err;   // CSR-check flags
};

__device__ __align__(256) unsigned char g_twohop_scratch[kNoAllocScratchBytes];

// Device address of g_twohop_scratch, looked up once per device (the host
// symbol is only a stand-in: a kernel handed it would fault or read the
// wrong memory).  The cached address belongs to the device's primary
// context, which is assumed to live as long as the process: after a
// cudaDeviceReset on that device the cache is stale.
struct ScratchAddr {
    std::mutex mu;
    void* ptr[kNoAllocMaxDevices] = {};
};
ScratchAddr g_scratch_addr;

cudaError_t scratch_for_device(int dev, unsigned char** out)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_addr.mu);
    if (!g_scratch_addr.ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_twohop_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr.ptr[dev] = p;
    }
    *out = (unsigned char*)g_scratch_addr.ptr[dev];
    return cudaSuccess;
}

// Checks the caller's device CSR before the two-hop passes read it: off[0] =
// 0, offsets non-decreasing, off[n] >= 0, an adjacency array when off[n] > 0,
// and every neighbour id in [0, n).  Only off[0..n] and adj[0..off[n]) are
// read -- the extents the caller's contract gives.  Failures are or-ed into
// st->err, which the two-hop passes read first.
__global__ void csr_check_kernel(int n, const int64_t* off, const int32_t* adj, NoAllocStatus* st)
{
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int bad = 0;
    const int64_t m = off[n];
    if (tid == 0 && (off[0] != 0 || m < 0)) bad |= kErrOffsets;
    for (int64_t v = tid; v < n; v += stride)
        if (off[v] > off[v + 1]) bad |= kErrOffsets;
    if (m > 0 && !adj) {
        bad |= kErrNullAdj;
    } else {
        for (int64_t e = tid; e < m; e += stride)
            if ((unsigned)adj[e] >= (unsigned)n) bad |= kErrIds;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && (threadIdx.x & 31) == 0) atomicOr(&st->err, bad);
}

// In-place scan of off2[1..n] (per-vertex counts) into CSR offsets, off2[0] = 0;
// the total goes to st->total.  One block walks the array in chunks of its
// size, carrying the running total.  Skipped (total 0) when the CSR check failed.
__global__ void twohop_scan_kernel(int64_t* off2, int n, NoAllocStatus* st)
{
    __shared__ int64_t warp_tot[32];
    __shared__ int64_t carry;
    if (*(volatile int32_t*)&st->err) {
        if (threadIdx.x == 0) st->total = 0;
        return;
    }
    int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) {
        carry = 0;
        off2[0] = 0;
    }
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + tid;
        int64_t x = i < n ? off2[(int64_t)i + 1] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_tot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int nw = blockDim.x >> 5;
            int64_t w = lane < nw ? warp_tot[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int64_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < nw) warp_tot[lane] = w;
        }
        __syncthreads();
        int64_t before = (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
        if (i < n) off2[(int64_t)i + 1] = before + x;
        __syncthreads();
        if (tid == blockDim.x - 1) carry = before + x;
        __syncthreads();
    }
    if (tid == 0) st->total = carry;
}

std::string csr_error_text(int err)
{
    std::string t;
    if (err & kErrOffsets) t += "offsets do not start at 0 or decrease";
    if (err & kErrIds) t += std::string(t.empty() ? "" : "; ") + "a neighbour id is outside [0, n)";
    if (err & kErrNullAdj) t += std::string(t.empty() ? "" : "; ") + "d_adj is NULL but off[n] > 0";
    return "malformed device CSR: " + t;
}

// Per-warp working memory for n vertices: bitmap words, touched-word list
// (padded to a power of two for the warp sort), touched counter.
int64_t noalloc_bytes_per_warp(int64_t n, int64_t* bm_words, int64_t* touched_cap)
{
    int64_t w = (n + 31) / 32, tc = 1;
    while (tc < w) tc <<= 1;
    if (bm_words) *bm_words = w;
    if (touched_cap) *touched_cap = tc;
    return 4 * w + 4 * tc + 4;
}

constexpr int64_t kNoAllocWarpBytes = (int64_t)(kNoAllocScratchBytes - kNoAllocHeaderBytes);

} // namespace

std::string qcb_twohop_noalloc(int32_t n, const int64_t* d_off, const int32_t* d_adj,
                               int64_t* d_off2, int32_t* d_adj2, int64_t adj2_cap,
                               int64_t* total_out, cudaStream_t s, int* too_large, int* too_small,
                               int* bad_csr)
{
    *too_large = 0;
    *too_small = 0;
    *bad_csr = 0;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    unsigned char* scratch = nullptr;
    e = scratch_for_device(dev, &scratch);
    if (e != cudaSuccess) return std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
    if (n == 0) {
        e = cudaMemsetAsync(d_off2, 0, sizeof(int64_t), s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (total_out) *total_out = 0;
        return e == cudaSuccess ? "" : std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
    }
    int64_t bm_words = 0, touched_cap = 0;
    const int64_t per_warp = noalloc_bytes_per_warp(n, &bm_words, &touched_cap);
    const int64_t fit = kNoAllocWarpBytes / per_warp;
    if (fit < kNoAllocMinWarps) {
        *too_large = 1;
        return "graph has " + std::to_string(n) + " vertices; qc_twohop_noalloc supports at most " +
               std::to_string(qc_twohop_noalloc_max_vertices());
    }
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e);
    int64_t nwarps = std::min<int64_t>(fit, (int64_t)sms * 2 * kTwohopWarpsPerBlock);
    nwarps -= nwarps % kTwohopWarpsPerBlock;
    const int blocks = (int)(nwarps / kTwohopWarpsPerBlock);
    NoAllocStatus* st = (NoAllocStatus*)scratch;
    unsigned char* warp_mem = scratch + kNoAllocHeaderBytes;
    uint32_t* bm = (uint32_t*)warp_mem;
    int32_t* touched = (int32_t*)(warp_mem + 4 * bm_words * nwarps);
    int* nt = (int*)(warp_mem + 4 * bm_words * nwarps + 4 * touched_cap * nwarps);
    // the array keeps the last call's contents: the status words and the
    // bitmaps (contiguous) must start at zero
    e = cudaMemsetAsync(scratch, 0, kNoAllocHeaderBytes + sizeof(uint32_t) * bm_words * nwarps, s);
    if (e != cudaSuccess) return std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
    csr_check_kernel<<<sms * 4, 256, 0, s>>>(n, d_off, d_adj, st);
    // pass 1: per-vertex counts into off2[1..n], then the scan
    twohop_kernel<<<blocks, kTwohopWarpsPerBlock * 32, 0, s>>>(
        n, d_off, d_adj, bm, bm_words, touched, touched_cap, nt, d_off2 + 1, nullptr, nullptr,
        &st->err);
    twohop_scan_kernel<<<1, 1024, 0, s>>>(d_off2, n, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return std::string("launch: ") + cudaGetErrorString(e);
    NoAllocStatus hs{};
    e = cudaMemcpyAsync(&hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return std::string("two-hop count: ") + cudaGetErrorString(e);
    if (hs.err) {
        *bad_csr = 1;
        return csr_error_text(hs.err);
    }
    if (total_out) *total_out = hs.total;
    if (!d_adj2) return ""; // size query
    if (hs.total > adj2_cap) {
        *too_small = 1;
        return "adj2 holds " + std::to_string(adj2_cap) + " entries; the two-hop lists need " +
               std::to_string(hs.total);
    }
    // pass 2: sorted rows
    twohop_kernel<<<blocks, kTwohopWarpsPerBlock * 32, 0, s>>>(
        n, d_off, d_adj, bm, bm_words, touched, touched_cap, nt, nullptr, d_off2, d_adj2,
        &st->err);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return std::string("two-hop rows: ") + cudaGetErrorString(e);
    return "";
}

extern "C" int32_t qc_twohop_noalloc_max_vertices(void)
{
    // largest n (a multiple of 32) whose per-warp working memory still leaves
    // room for kNoAllocMinWarps warps; the need grows with n
    auto fits = [](int64_t n) {
        return kNoAllocWarpBytes / noalloc_bytes_per_warp(n, nullptr, nullptr) >= kNoAllocMinWarps;
    };
    int64_t lo = 32, hi = (int64_t)1 << 30; // fits(lo), !fits(hi)
    while (hi - lo > 32) {
        int64_t mid = ((lo + hi) / 2) & ~int64_t(31);
        if (mid <= lo) mid = lo + 32;
        if (fits(mid)) lo = mid;
        else hi = mid;
    }
    return (int32_t)lo;
}
