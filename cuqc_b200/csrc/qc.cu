// qc.cu -- libqc.so: C ABI (include/qc.h) over the B200 expansion kernel.
//
// Flow of qc_mine (replaces Mike12041204/cuQC search() + RemoveNonMax(),
// main.cu:535-692 and 4939-4960):
//   1. gamma tables (md, ubt) on the host, exactly as the reference computes
//      them in double, uploaded once per call;
//   2. level 0 on the host (main.cu:846-998) -> root ids + covered count;
//   3. root task record built on the device from the CSR (one warp per root
//      vertex scans its 1-hop and 2-hop rows, 128-bit coalesced by lanes);
//   4. one persistent launch of expand_kernel drains the device work stack;
//   5. emitted sets copied back, maximal filter, lexicographic order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/qc.h"
#include "expand_kernel.cuh"
#include "level0_kernel.cuh"
#include "level0_grid.cuh"
#include "filter.h"
#include "host.h"

using namespace qcb;

// ------------------------------------------------------------------
// errors
// ------------------------------------------------------------------

static thread_local std::string g_err;

static qc_status fail(qc_status s, const std::string& msg)
{
    g_err = msg;
    return s;
}

#define CK(call)                                                                      \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return fail(e_ == cudaErrorMemoryAllocation ? QC_ERR_NOMEM : QC_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));          \
    } while (0)

extern "C" const char* qc_status_str(qc_status s)
{
    switch (s) {
    case QC_OK: return "ok";
    case QC_ERR_ARGS: return "invalid argument";
    case QC_ERR_IO: return "file error";
    case QC_ERR_FORMAT: return "malformed graph";
    case QC_ERR_CUDA: return "CUDA error";
    case QC_ERR_NOMEM: return "out of memory";
    case QC_ERR_TASK_OVERFLOW: return "task stack or record arena exhausted";
    case QC_ERR_RESULT_OVERFLOW: return "result buffer exhausted";
    case QC_ERR_ITER_LIMIT: return "bounded device wait gave up";
    case QC_ERR_TOO_LARGE: return "task too large";
    case QC_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char* qc_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------------
// objects
// ------------------------------------------------------------------

static std::atomic<unsigned long long> g_graph_serial{1};

struct qc_graph {
    HostGraph h;
    unsigned long long serial = g_graph_serial.fetch_add(1); // identity for device caches
    mutable std::atomic<int> resident_in{0}; // contexts holding a device copy
};

// Graphs freed while contexts still hold their device copies: serial ->
// contexts yet to notice.  A context reuses such a copy's buffers for the
// next graph it uploads instead of allocating new ones.
static std::mutex g_dead_mu;
static std::unordered_map<unsigned long long, int> g_dead;

struct qc_result {
    std::vector<int32_t> sets;
    int64_t nsets = 0;
    std::vector<int32_t> emitted;
    int64_t emitted_sets = 0;
    qc_stats st{};
};

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) n = bytes;
        else cudaGetLastError(); // a failed allocation must not surface at a later check
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    template <class T> T* as() const { return (T*)p; }
};

} // namespace

struct BatchBufs {
    DevBuf md, ubt, rules, meta, ids, pos, jobs, l0scratch, l0info;
    void release()
    {
        for (DevBuf* b : {&md, &ubt, &rules, &meta, &ids, &pos, &jobs, &l0scratch, &l0info})
            b->release();
    }
};

// A graph's CSR and two-hop CSR on the device.
struct ResidentGraph {
    DevBuf off, adj, off2, adj2;
    size_t bytes = 0;
    uint64_t last_use = 0;
    void release()
    {
        for (DevBuf* b : {&off, &adj, &off2, &adj2}) b->release();
    }
};

struct qc_context {
    qc_config cfg{};
    BatchBufs batch;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    DevBuf pos, ids, md, ubt, ctl, arena, stack, slot, results, ws, starts, rules, lvl0;
    FilterScratch filt;
    int32_t pos_n = 0;
    // graphs kept on the device, by graph serial; least recently used ones are
    // dropped when their bytes exceed res_budget
    std::unordered_map<unsigned long long, std::unique_ptr<ResidentGraph>> res;
    size_t res_bytes = 0, res_budget = 0;
    uint64_t use_clock = 0;
    int64_t arena_bytes = 0, stack_slots = 0, result_ints = 0;
    int64_t launches = 0;
    qc_stats last{}; // counters of the most recent expansion, also of one that stopped
    // page-locked staging for the small copies of a call (the Control head,
    // the root's header, stack entry and slot, the rules): copies from it are
    // plain DMA, with no staging by the driver
    char* pin = nullptr;
    size_t pin_n = 0, pin_at = 0;
    // md / ubt as last uploaded: the same tables are not copied again
    std::vector<int32_t> md_up, ubt_up;
};

// The Control fields up to the free-list heads; the heads (most of the
// block) start at zero on every launch and are cleared on the device.
static constexpr size_t kControlHead = offsetof(Control, free_head);

// A page-locked copy of `bytes` bytes for this call's host-to-device copies
// (the buffer is reused once the call has synchronised).
static void* pin_stage(qc_context* c, const void* src, size_t bytes)
{
    const size_t at = (c->pin_at + 15) & ~(size_t)15;
    if (!c->pin || at + bytes > c->pin_n) return nullptr;
    std::memcpy(c->pin + at, src, bytes);
    c->pin_at = at + bytes;
    return c->pin + at;
}

// host-to-device copy of a small host object through the staging buffer
// (a plain copy when it does not fit)
static cudaError_t put_small(qc_context* c, void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    const void* p = pin_stage(c, src, bytes);
    return cudaMemcpyAsync(dst, p ? p : src, bytes, cudaMemcpyHostToDevice, s);
}

// The Control block for a launch: the head from `ctl`, the free lists zeroed
static cudaError_t put_control(qc_context* c, const Control& ctl, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(c->ctl.as<char>() + kControlHead, 0, sizeof(Control) - kControlHead, s);
    if (e != cudaSuccess) return e;
    return put_small(c, c->ctl.p, &ctl, kControlHead, s);
}

// The launch's Control head back into `ctl` (free lists left out); the
// caller synchronises before reading it
static cudaError_t get_control(qc_context* c, Control& ctl, cudaStream_t s)
{
    std::memset(&ctl, 0, sizeof(ctl));
    return cudaMemcpyAsync(&ctl, c->ctl.p, kControlHead, cudaMemcpyDeviceToHost, s);
}

extern "C" void qc_config_default(qc_config* c)
{
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->wait_limit_ms = 10000;
}

static qc_status warm_kernels(qc_context* c);

extern "C" qc_status qc_context_create(const qc_config* cfg, qc_context** out)
{
    if (!out) return fail(QC_ERR_ARGS, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QC_ERR_NO_DEVICE, "no CUDA device visible");
    std::unique_ptr<qc_context> c(new qc_context());
    if (cfg) c->cfg = *cfg;
    else qc_config_default(&c->cfg);
    if (c->cfg.device < 0 || c->cfg.device >= ndev) return fail(QC_ERR_ARGS, "bad device ordinal");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (auto& e : c->ev) CK(cudaEventCreate(&e));
    CK(cudaHostAlloc((void**)&c->pin, 64 << 10, cudaHostAllocDefault));
    c->pin_n = 64 << 10;
    c->arena_bytes = c->cfg.arena_bytes > 0 ? c->cfg.arena_bytes : (256ll << 20);
    c->stack_slots = c->cfg.stack_slots > 0 ? c->cfg.stack_slots : (1ll << 20);
    c->result_ints = c->cfg.result_ints > 0 ? c->cfg.result_ints : (16ll << 20);
    if (c->cfg.wait_limit_ms <= 0) c->cfg.wait_limit_ms = 10000;
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b));
    c->res_budget = total_b / 4;
    qc_status ws = warm_kernels(c.get());
    if (ws != QC_OK) return ws;
    *out = c.release();
    return QC_OK;
}

extern "C" void qc_context_free(qc_context* c)
{
    if (!c) return;
    cudaSetDevice(c->cfg.device);
    {
        std::lock_guard<std::mutex> lk(g_dead_mu);
        for (auto& kv : c->res) {
            auto d = g_dead.find(kv.first);
            if (d != g_dead.end() && --d->second <= 0) g_dead.erase(d);
        }
    }
    for (auto& kv : c->res) kv.second->release();
    c->res.clear();
    for (DevBuf* b : {&c->pos, &c->ids, &c->md, &c->ubt, &c->ctl, &c->arena, &c->stack, &c->slot, &c->results, &c->ws, &c->starts, &c->lvl0,
                      &c->rules})
        b->release();
    c->filt.release();
    c->batch.release();
    if (c->pin) cudaFreeHost(c->pin);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// ------------------------------------------------------------------
// graphs
// ------------------------------------------------------------------

extern "C" qc_status qc_graph_read_serialized(const char* path, qc_graph** out)
{
    if (!path || !out) return fail(QC_ERR_ARGS, "NULL argument");
    *out = nullptr;
    std::unique_ptr<qc_graph> g(new qc_graph());
    std::string e = read_serialized(path, g->h);
    if (!e.empty()) {
        if (e.rfind("cannot open", 0) == 0) return fail(QC_ERR_IO, e);
        return fail(QC_ERR_FORMAT, e);
    }
    e = validate(g->h, true);
    if (!e.empty()) return fail(QC_ERR_FORMAT, e);
    *out = g.release();
    return QC_OK;
}

// Copy one caller CSR (n + 1 offsets, then off[n] ids) into the graph.  The
// offsets' ends are checked before anything is copied: a negative or
// impossible entry count would otherwise size the copy itself.  With n = 0
// the offsets may be NULL (one offset, 0).
static qc_status adopt_rows(int32_t n, const int64_t* off, const int32_t* adj, const char* what,
                            const char* adj_name, std::vector<int64_t>& o, std::vector<int32_t>& a)
{
    static const int64_t zero = 0;
    if (n == 0 && !off) off = &zero;
    if (off[0] != 0 || off[n] < 0 || off[n] > (int64_t)(PTRDIFF_MAX / sizeof(int32_t)))
        return fail(QC_ERR_FORMAT, std::string(what) + " offsets must start at 0 and end at the entry count");
    if (off[n] > 0 && !adj) return fail(QC_ERR_ARGS, std::string(adj_name) + " is NULL");
    try {
        o.assign(off, off + n + 1);
        a.assign(adj, adj + off[n]);
    } catch (const std::bad_alloc&) {
        return fail(QC_ERR_NOMEM, std::string("host copy of the ") + what + " lists");
    }
    return QC_OK;
}

extern "C" qc_status qc_graph_from_csr2(int32_t n, const int64_t* off, const int32_t* adj,
                                        const int64_t* off2, const int32_t* adj2, qc_graph** out)
{
    if (!out || n < 0 || (n > 0 && (!off || !off2))) return fail(QC_ERR_ARGS, "bad CSR arguments");
    *out = nullptr;
    std::unique_ptr<qc_graph> g(new qc_graph());
    g->h.n = n;
    qc_status as = adopt_rows(n, off, adj, "1-hop", "adj", g->h.off, g->h.adj);
    if (as != QC_OK) return as;
    as = adopt_rows(n, off2, adj2, "2-hop", "adj2", g->h.off2, g->h.adj2);
    if (as != QC_OK) return as;
    std::string e = validate(g->h, true);
    if (!e.empty()) return fail(QC_ERR_FORMAT, e);
    *out = g.release();
    return QC_OK;
}

std::string qcb_twohop_device(const HostGraph& h, std::vector<int64_t>& off2,
                              std::vector<int32_t>& adj2);

extern "C" qc_status qc_graph_read_binary(const char* path, qc_graph** out)
{
    if (!path || !out) return fail(QC_ERR_ARGS, "NULL argument");
    *out = nullptr;
    std::unique_ptr<qc_graph> g(new qc_graph());
    bool two = false;
    std::string e = read_binary(path, g->h, two);
    if (!e.empty()) {
        if (e.rfind("cannot open", 0) == 0) return fail(QC_ERR_IO, e);
        return fail(QC_ERR_FORMAT, e);
    }
    e = validate(g->h, two);
    if (!e.empty()) return fail(QC_ERR_FORMAT, e);
    if (!two) {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
            return fail(QC_ERR_NO_DEVICE, "no CUDA device to build the two-hop lists");
        e = qcb_twohop_device(g->h, g->h.off2, g->h.adj2);
        if (!e.empty()) return fail(QC_ERR_CUDA, e);
    }
    *out = g.release();
    return QC_OK;
}

extern "C" qc_status qc_graph_write_binary(const qc_graph* g, const char* path)
{
    if (!g || !path) return fail(QC_ERR_ARGS, "NULL argument");
    std::string e = write_binary(g->h, path);
    return e.empty() ? QC_OK : fail(QC_ERR_IO, e);
}

extern "C" qc_status qc_graph_read(const char* path, qc_graph** out)
{
    if (path && is_binary_graph(path)) return qc_graph_read_binary(path, out);
    return qc_graph_read_serialized(path, out);
}

extern "C" qc_status qc_graph_write_serialized(const qc_graph* g, const char* path)
{
    if (!g || !path) return fail(QC_ERR_ARGS, "NULL argument");
    std::string e = write_serialized(g->h, path);
    return e.empty() ? QC_OK : fail(QC_ERR_IO, e);
}

extern "C" int32_t qc_graph_num_vertices(const qc_graph* g) { return g ? g->h.n : 0; }
extern "C" int64_t qc_graph_num_entries(const qc_graph* g) { return g ? (int64_t)g->h.adj.size() : 0; }
extern "C" int64_t qc_graph_num_twohop(const qc_graph* g) { return g ? (int64_t)g->h.adj2.size() : 0; }
extern "C" const int64_t* qc_graph_offsets(const qc_graph* g) { return g ? g->h.off.data() : nullptr; }
extern "C" const int32_t* qc_graph_neighbors(const qc_graph* g) { return g ? g->h.adj.data() : nullptr; }
extern "C" const int64_t* qc_graph_twohop_offsets(const qc_graph* g) { return g ? g->h.off2.data() : nullptr; }
extern "C" const int32_t* qc_graph_twohop_neighbors(const qc_graph* g) { return g ? g->h.adj2.data() : nullptr; }
extern "C" void qc_graph_free(qc_graph* g)
{
    if (!g) return;
    int held = g->resident_in.load();
    if (held > 0) {
        std::lock_guard<std::mutex> lk(g_dead_mu);
        g_dead[g->serial] += held;
    }
    delete g;
}

// ------------------------------------------------------------------
// device kernels: root task record
// ------------------------------------------------------------------

__global__ void root_pos_kernel(const int32_t* ids, int t, int32_t* pos, int set)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < t) pos[ids[i]] = set ? i : -1;
}

// The root's set-up when level 0 ran on the device and its size stays there
// (info = {root size t, covered count}): one block writes the Control block
// (the head as the host prepared it, free-list heads zeroed, then the root's
// arena use, stack entry and size), the root record's header and ids with its
// rows zeroed, the shared stack's root entry, the rules, and each root
// vertex's position.  A root whose block exceeds the arena is not written: the
// launch then ends at once with ST_TASK_OVERFLOW and the host grows the arena.
struct RootSetup {
    unsigned long long head[offsetof(Control, free_head) / 8];
    Rules rule;
    int32_t flags, pad;
};
__global__ void __launch_bounds__(256) root_setup_kernel(RootSetup S, const int32_t* info,
                                                         const int32_t* ids, char* arena,
                                                         unsigned long long arena_cap, Control* ctl,
                                                         StackEntry* stack, int32_t* slot,
                                                         Rules* rules, int32_t* pos)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    const int t = info[0], cov = info[1];
    const int W = words_for(t);
    const unsigned long long block = t > 0 ? arena_class_bytes(arena_class(rec_block_bytes(t, W))) : 0;
    const bool fits = t > 0 && block <= arena_cap;
    unsigned long long* c8 = (unsigned long long*)ctl;
    constexpr int kHead = (int)(offsetof(Control, free_head) / 8);
    for (int i = tid; i < (int)(sizeof(Control) / 8); i += nt) c8[i] = i < kHead ? S.head[i] : 0ull;
    if (fits) {
        uint4* z = (uint4*)arena;
        const int64_t n16 = (int64_t)(rec_bytes(t, W) / 16);
        for (int64_t i = tid; i < n16; i += nt) z[i] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();
    for (int i = tid; i < t; i += nt) {
        const int v = ids[i];
        pos[v] = i;
        if (fits) ((int32_t*)(arena + rec_ids_off()))[i] = v;
    }
    if (tid == 0) {
        if (fits) {
            TaskHdr* h = (TaskHdr*)arena;
            h->t = t;
            h->m = 0;
            h->cov = cov;
            h->W = W;
            h->refs = 1;
            h->cls = arena_class(rec_block_bytes(t, W));
            h->inst = 0;
            h->flags = S.flags;
            StackEntry e{};
            e.rec[0] = 0;
            e.n = 1;
            e.q_lo = -1;
            e.q_hi = -1;
            stack[0] = e;
            slot[0] = 1;
        }
        ctl->arena_top = block;
        ctl->stack_top[0] = fits ? 1 : 0;
        ctl->pending = fits ? 1 : 0;
        if (t > 0 && !fits) ctl->status = ST_TASK_OVERFLOW;
        ctl->root_t = t;
        ctl->root_cov = cov;
        *rules = S.rule;
    }
}

// root_rows_kernel and the positions' reset for a root whose size is on the
// device (root_setup_kernel wrote the record when it fits the arena).  A
// block per root vertex (blocks beyond the root's size return at once): its
// threads share the vertex's 1-hop and 2-hop rows, so the long 2-hop rows
// are read by many loads in flight.
__global__ void __launch_bounds__(256) root_rows_dev_kernel(const int64_t* off, const int32_t* adj,
                                                            const int64_t* off2, const int32_t* adj2,
                                                            const int32_t* ids, const int32_t* info,
                                                            const int32_t* pos, char* arena,
                                                            unsigned long long arena_cap)
{
    const int t = info[0], W = words_for(t);
    if (t <= 0 || arena_class_bytes(arena_class(rec_block_bytes(t, W))) > arena_cap) return;
    uint32_t* A1 = (uint32_t*)(arena + rec_a1_off(t));
    uint32_t* A2 = (uint32_t*)(arena + rec_a2_off(t, W));
    for (int i = blockIdx.x; i < t; i += gridDim.x) {
        const int u = ids[i];
        uint32_t* r1 = A1 + (int64_t)i * W;
        uint32_t* r2 = A2 + (int64_t)i * W;
        for (int64_t e = off[u] + threadIdx.x; e < off[u + 1]; e += blockDim.x) {
            const int p = pos[adj[e]];
            if (p >= 0) atomicOr(&r1[p >> 5], 1u << (p & 31));
        }
        for (int64_t e = off2[u] + threadIdx.x; e < off2[u + 1]; e += blockDim.x) {
            const int p = pos[adj2[e]];
            if (p >= 0) atomicOr(&r2[p >> 5], 1u << (p & 31));
        }
    }
}
__global__ void root_unpos_dev_kernel(const int32_t* ids, const int32_t* info, int32_t* pos)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < info[0]) pos[ids[i]] = -1;
}

// one warp per root vertex: mark its 1-hop and 2-hop neighbours inside the root
__global__ void root_rows_kernel(const int64_t* off, const int32_t* adj, const int64_t* off2,
                                 const int32_t* adj2, const int32_t* ids, int t, int W,
                                 const int32_t* pos, uint32_t* A1, uint32_t* A2)
{
    int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < t; i += nw) {
        int u = ids[i];
        uint32_t* r1 = A1 + (int64_t)i * W;
        uint32_t* r2 = A2 + (int64_t)i * W;
        for (int64_t e = off[u] + lane; e < off[u + 1]; e += 32) {
            int p = pos[adj[e]];
            if (p >= 0) atomicOr(&r1[p >> 5], 1u << (p & 31));
        }
        for (int64_t e = off2[u] + lane; e < off2[u + 1]; e += 32) {
            int p = pos[adj2[e]];
            if (p >= 0) atomicOr(&r2[p >> 5], 1u << (p & 31));
        }
    }
}

// ------------------------------------------------------------------
// mining
// ------------------------------------------------------------------

namespace {

using clk = std::chrono::steady_clock;

double ms_since(clk::time_point t0)
{
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

template <class T> cudaError_t upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s)
{
    cudaError_t e = b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

} // namespace

// A table upload that is skipped when the device buffer still holds the
// values it was last given (`last`); a reallocated buffer is filled again.
template <class T>
static cudaError_t upload_cached(qc_context* c, DevBuf& b, std::vector<T>& last, const std::vector<T>& v,
                                 cudaStream_t s)
{
    void* before = b.p;
    cudaError_t e = b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (e != cudaSuccess) return e;
    if (b.p == before && last == v) return cudaSuccess;
    last = v;
    if (v.empty()) return cudaSuccess;
    return put_small(c, b.p, v.data(), v.size() * sizeof(T), s);
}

// stack slots rounded up so that every shard's capacity is a power of two
// (the FIFO form of the shards indexes its ring by a wrapping count)
static int64_t shard_slots(int64_t want)
{
    int64_t per = 2;
    while (per * kStackShards < want) per <<= 1;
    return per * kStackShards;
}

// entries on the fullest shard of the shared stack
static int max_top(const Control& ctl)
{
    int m = 0;
    for (int i = 0; i < kStackShards; i++)
        m = std::max(m, (int)((unsigned)ctl.stack_top[i] - (unsigned)ctl.stack_bot[i]));
    return m;
}

// Launch shape of expand_kernel for tasks of up to max_t vertices: warps per
// block, blocks, and the largest task staged in shared memory (the biggest
// candidate whose per-warp buffers fit the blocks resident on one SM).
struct Shape {
    int wpb = 4, blocks = 0, smem_t = 0;
    size_t smem_bytes = 0;
};

static qc_status launch_shape(qc_context* c, int max_t, Shape& sh)
{
    // expand_kernel is compiled with __launch_bounds__(256, 2): at most 8 warps a
    // block.  The default is one block of 8 warps per SM (two warps per SM
    // sub-partition, so one hides the other's latency).
    sh.wpb = c->cfg.warps_per_block > 0 ? std::min(c->cfg.warps_per_block, 8) : 8;
    const int want_bps = c->cfg.blocks_per_sm > 0 ? c->cfg.blocks_per_sm : 1;
    // Of the SM's 256 KB of L1 and shared memory, the 196 KB carve-out (195
    // KB for the blocks plus 1 KB each reserved) leaves 60 KB of L1; the
    // next, 228 KB, leaves 28 KB.
    const size_t sm_budget = 195u << 10;
    sh.smem_t = 0;
    if (max_t > 32 && c->cfg.stage_max >= 0) {
        // the first of these sizes whose buffers fit; no finer: the shared
        // memory staging takes is the L1 cache's loss, and tasks too large to
        // stage keep their workspace in global memory, read through L1 (a
        // stage fitted to the last vertex, 156 for 8 warps in the 228 KB
        // carve-out, left config 2's large tasks 26 times slower).  Eight
        // warps stage 160 vertices: config 1's 150-vertex root among them.
        for (int cand : {256, 192, 160, 128, 96, 64}) {
            int tt = std::min(cand, max_t);
            if (c->cfg.stage_max > 0) tt = std::min(tt, c->cfg.stage_max);
            if (tt <= 32) break;
            if (warp_smem_bytes(tt) * sh.wpb * want_bps <= sm_budget) {
                sh.smem_t = tt;
                break;
            }
        }
    }
    sh.smem_bytes = expand_smem_bytes(sh.wpb, sh.smem_t);
    {
        // raised once per device to the opt-in maximum and never lowered:
        // contexts on other threads launch with their own sizes meanwhile
        static std::mutex mu;
        static bool raised[64] = {};
        std::lock_guard<std::mutex> lk(mu);
        int dev = c->cfg.device;
        if (dev < 0 || dev >= 64) return fail(QC_ERR_ARGS, "device ordinal above 63");
        if (!raised[dev]) {
            int optin = 0;
            CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            CK(cudaFuncSetAttribute(expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    optin));
            raised[dev] = true;
        }
    }
    int resident = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, expand_kernel, sh.wpb * 32,
                                                     sh.smem_bytes));
    if (resident < 1) return fail(QC_ERR_CUDA, "expand_kernel cannot be resident");
    // a persistent launch: never more blocks than can be resident at once
    const int bps = std::min(want_bps, resident);
    sh.blocks = c->sms * bps;
    if (c->cfg.max_blocks > 0) sh.blocks = std::min(sh.blocks, c->cfg.max_blocks);
    return QC_OK;
}

// Device copy of graph g, uploaded on first use and kept for later calls.
// When the resident graphs exceed the context's budget, the least recently
// used ones (other than g and those in `keep`) are dropped.  Also sizes the
// vertex-position scratch for g.
static qc_status make_resident(qc_context* c, const qc_graph* g,
                               const std::unordered_set<unsigned long long>* keep,
                               ResidentGraph** out)
{
    const HostGraph& h = g->h;
    cudaStream_t s = c->stream;
    auto it = c->res.find(g->serial);
    if (it == c->res.end()) {
        std::unique_ptr<ResidentGraph> rg;
        {
            // reuse the buffers of a copy whose graph has been freed
            std::lock_guard<std::mutex> lk(g_dead_mu);
            if (!g_dead.empty()) {
                for (auto j = c->res.begin(); j != c->res.end(); ++j) {
                    auto d = g_dead.find(j->first);
                    if (d == g_dead.end()) continue;
                    if (--d->second <= 0) g_dead.erase(d);
                    CK(cudaStreamSynchronize(s)); // queued work may still read it
                    rg = std::move(j->second);
                    c->res_bytes -= rg->bytes;
                    c->res.erase(j);
                    break;
                }
            }
        }
        if (!rg) rg.reset(new ResidentGraph());
        CK(upload(rg->off, h.off, s));
        CK(upload(rg->adj, h.adj, s));
        CK(upload(rg->off2, h.off2, s));
        CK(upload(rg->adj2, h.adj2, s));
        rg->bytes = rg->off.n + rg->adj.n + rg->off2.n + rg->adj2.n;
        c->res_bytes += rg->bytes;
        it = c->res.emplace(g->serial, std::move(rg)).first;
        g->resident_in.fetch_add(1);
        while (c->res_bytes > c->res_budget && c->res.size() > 1) {
            auto victim = c->res.end();
            for (auto j = c->res.begin(); j != c->res.end(); ++j) {
                if (j->first == g->serial || (keep && keep->count(j->first))) continue;
                if (victim == c->res.end() || j->second->last_use < victim->second->last_use)
                    victim = j;
            }
            if (victim == c->res.end()) break;
            CK(cudaStreamSynchronize(s)); // its buffers may still be read by queued work
            c->res_bytes -= victim->second->bytes;
            victim->second->release();
            c->res.erase(victim);
        }
    }
    it->second->last_use = ++c->use_clock;
    if (c->pos_n < h.n || !c->pos.p) {
        CK(c->pos.ensure(sizeof(int32_t) * (size_t)std::max(h.n, 1)));
        CK(cudaMemsetAsync(c->pos.p, 0xff, sizeof(int32_t) * (size_t)std::max(h.n, 1), s));
        c->pos_n = h.n;
    }
    *out = it->second.get();
    return QC_OK;
}

// The work counters of the launch that just ended, kept in the context so a
// caller can read them after a run that stopped at its time limit.
static void record_last(qc_context* c, const Control& ctl, float kms, int root_size)
{
    qc_stats& l = c->last;
    l = qc_stats{};
    l.tasks = (int64_t)ctl.tasks;
    l.branches = (int64_t)ctl.branches;
    l.children = (int64_t)ctl.children;
    l.emitted = (int64_t)ctl.emitted;
    l.emitted_ints = (int64_t)ctl.result_top;
    l.root_size = root_size;
    l.max_task = ctl.max_task;
    l.arena_peak = (int64_t)std::min(ctl.arena_top, ctl.arena_cap);
    l.kernel_launches = c->launches;
    l.kernel_ms = kms;
    l.parent_vertices = (int64_t)ctl.parent_vertices;
    l.p_rows = (int64_t)ctl.p_rows;
    l.child_vertices = (int64_t)ctl.child_vertices;
}

// Level 0 of graph h (resident as rg): the root task's vertex ids in Q order
// land in c->ids on the device; t = root size, cov = covered count.  On the
// device for graphs of up to kLevel0DeviceMax vertices (one block) and up to
// kLevel0GridMax (the whole grid, one cooperative launch); on the host above.
// *on_device tells which.
// Level 0 of a graph of at most kLevel0DeviceMax vertices on one block, with
// nothing read back: the root's ids go to c->ids and {size, covered count} to
// *info (device memory).
static qc_status launch_level0(qc_context* c, const HostGraph& h, ResidentGraph* rg,
                               const std::vector<int32_t>& md, int32_t min_size, int32_t** info_out)
{
    cudaStream_t s = c->stream;
    int P = 1;
    while (P < h.n) P <<= 1;
    // int32 arrays of n (exdeg, label, 2-hop size), then the 64-bit sort keys,
    // then two ints of results: every array starts 16-byte aligned
    const size_t nb = ((size_t)h.n * 4 + 15) & ~(size_t)15;
    CK(c->lvl0.ensure(3 * nb + 8 * (size_t)P + 64));
    CK(c->ids.ensure(std::max<size_t>((size_t)h.n * 4, 16)));
    char* z = c->lvl0.as<char>();
    int32_t* info = (int32_t*)(z + 3 * nb + 8 * (size_t)P);
    if (h.n <= kLevel0SmemMax)
        level0_smem_kernel<<<1, 1024, (size_t)level0_scratch_bytes(h.n), s>>>(
            rg->off.as<int64_t>(), rg->adj.as<int32_t>(), rg->off2.as<int64_t>(), h.n,
            md[(size_t)min_size], min_size, c->ids.as<int32_t>(), info);
    else
        level0_kernel<<<1, 1024, 0, s>>>(rg->off.as<int64_t>(), rg->adj.as<int32_t>(),
                                         rg->off2.as<int64_t>(), h.n, md[(size_t)min_size],
                                         min_size, (int32_t*)z, (int32_t*)(z + nb),
                                         (int32_t*)(z + 2 * nb), (unsigned long long*)(z + 3 * nb),
                                         c->ids.as<int32_t>(), info);
    CK(cudaGetLastError());
    c->launches += 1;
    *info_out = info;
    return QC_OK;
}

// The vertices level 0 keeps at first (deg >= need, |N2| >= min_size - 1): the
// root is a subset of them (initialize_tasks, main.cu:846-998)
static int root_bound(const HostGraph& h, int need, int32_t min_size)
{
    int k = 0;
    for (int32_t v = 0; v < h.n; v++)
        if (h.off[(size_t)v + 1] - h.off[(size_t)v] >= need &&
            h.off2[(size_t)v + 1] - h.off2[(size_t)v] >= min_size - 1)
            k++;
    return k;
}

static qc_status compute_root(qc_context* c, const HostGraph& h, ResidentGraph* rg,
                              const std::vector<int32_t>& md, int32_t min_size, int& t, int& cov,
                              bool* on_device)
{
    cudaStream_t s = c->stream;
    std::vector<int32_t> ids;
    t = 0;
    cov = 0;
    const bool l0_dev = h.n > 0 && h.n <= kLevel0DeviceMax;
    const bool l0_grid = h.n > kLevel0DeviceMax && (int64_t)h.n <= kLevel0GridMax;
    if (l0_dev) {
        // root ids straight into c->ids; only the root size and the covered
        // count come back
        int32_t* info = nullptr;
        {
            qc_status ls = launch_level0(c, h, rg, md, min_size, &info);
            if (ls != QC_OK) return ls;
        }
        int32_t hinfo[2] = {0, 0};
        CK(cudaMemcpyAsync(hinfo, info, sizeof(hinfo), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        t = hinfo[0];
        cov = hinfo[1];
        if (t < 0 || t > h.n || cov < 0 || cov > t) return fail(QC_ERR_CUDA, "level 0 size out of range");
    } else if (l0_grid) {
        // above one block's reach: the whole grid in one cooperative launch
        const size_t sb = (size_t)level0_grid_scratch_bytes(h.n);
        CK(c->lvl0.ensure(sb + 16));
        CK(c->ids.ensure(std::max<size_t>((size_t)h.n * 4, 16)));
        char* z = c->lvl0.as<char>();
        int32_t* info = (int32_t*)(z + sb);
        CK(cudaMemsetAsync(z + sb - 64, 0, 64, s)); // round flags, cover key, counts
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, level0_grid_kernel, 256, 0));
        if (per_sm < 1) return fail(QC_ERR_CUDA, "level 0 grid kernel cannot be resident");
        const int64_t* a_off = rg->off.as<int64_t>();
        const int32_t* a_adj = rg->adj.as<int32_t>();
        const int64_t* a_off2 = rg->off2.as<int64_t>();
        int64_t a_n = h.n;
        int a_need = md[(size_t)min_size], a_ms = min_size;
        int32_t* a_ids = c->ids.as<int32_t>();
        void* args[] = {(void*)&a_off, (void*)&a_adj, (void*)&a_off2, (void*)&a_n, (void*)&a_need,
                        (void*)&a_ms, (void*)&z, (void*)&a_ids, (void*)&info};
        CK(cudaLaunchCooperativeKernel((const void*)level0_grid_kernel, dim3(c->sms * per_sm),
                                       dim3(256), args, 0, s));
        c->launches += 1;
        int32_t hinfo[2] = {0, 0};
        CK(cudaMemcpyAsync(hinfo, info, sizeof(hinfo), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        t = hinfo[0];
        cov = hinfo[1];
        if (t < 0 || t > h.n || cov < 0 || cov > t) return fail(QC_ERR_CUDA, "level 0 size out of range");
    } else {
        build_root(h, md.data(), min_size, ids, cov);
        t = (int)ids.size();
    }
    if (!l0_dev && !l0_grid) CK(upload(c->ids, ids, s));
    if (on_device) *on_device = l0_dev || l0_grid;
    return QC_OK;
}

static qc_status mine_one(qc_context* c, const qc_graph* g, double gamma, int32_t min_size,
                          qc_result* r, int32_t shard = 0, int32_t nshards = 1)
{
    auto t_all = clk::now();
    const HostGraph& h = g->h;
    cudaStream_t s = c->stream;
    CK(cudaSetDevice(c->cfg.device));

    // graph -> device (timed as load; skipped when already resident)
    auto t_load = clk::now();
    ResidentGraph* rg = nullptr;
    {
        qc_status us = make_resident(c, g, nullptr, &rg);
        if (us != QC_OK) return us;
    }
    r->st.load_ms = ms_since(t_load);

    // enumeration: level 0 + device expansion
    auto t_enum = clk::now();
    std::vector<int32_t> md, ubt;
    gamma_tables(gamma, h.n, min_size, md, ubt);
    int cov = 0, t = 0;
    bool l0_on_device = false;
    // A graph level 0 handles in one block keeps its root on the device: the
    // root's size comes back with the expansion's counters, and the launches
    // are sized for the vertices level 0 keeps at first (tmax), so the host
    // does not wait for level 0 before setting up the expansion.
    const bool root_dev = h.n > 0 && h.n <= kLevel0DeviceMax && h.off2.size() == (size_t)h.n + 1;
    int tmax = 0;
    int32_t* d_info = nullptr;
    if (root_dev) {
        tmax = root_bound(h, md[(size_t)min_size], min_size);
        l0_on_device = true;
        if (tmax > 0) {
            qc_status ls = launch_level0(c, h, rg, md, min_size, &d_info);
            if (ls != QC_OK) return ls;
        }
    } else {
        qc_status ls = compute_root(c, h, rg, md, min_size, t, cov, &l0_on_device);
        if (ls != QC_OK) return ls;
        tmax = t;
    }
    r->st.level0_on_device = l0_on_device ? 1 : 0;
    r->st.root_size = (int64_t)t;
    if (tmax == 0) {
        r->st.enum_ms = ms_since(t_enum);
        r->st.total_ms = ms_since(t_all);
        return QC_OK;
    }
    const int W = words_for(t);
    c->pin_at = 0;
    CK(upload_cached(c, c->md, c->md_up, md, s));
    CK(upload_cached(c, c->ubt, c->ubt_up, ubt, s));

    Shape sh;
    {
        qc_status ss = launch_shape(c, tmax, sh);
        if (ss != QC_OK) return ss;
    }
    const int wpb = sh.wpb, blocks = sh.blocks;
    int nwarps = blocks * wpb;
    WsLayout L = ws_layout(tmax);
    CK(c->ws.ensure((size_t)L.total * nwarps));
    CK(c->ctl.ensure(sizeof(Control)));

    std::vector<int32_t> flat;
    for (int attempt = 0;; attempt++) {
        if (attempt > 0) c->pin_at = 0; // the previous attempt synchronised
        CK(c->arena.ensure((size_t)c->arena_bytes));
        c->stack_slots = shard_slots(std::max<int64_t>(c->stack_slots, 2 * kStackShards));
        CK(c->stack.ensure(sizeof(StackEntry) * (size_t)c->stack_slots));
        CK(c->slot.ensure(sizeof(int32_t) * (size_t)c->stack_slots));
        CK(c->results.ensure(sizeof(int32_t) * (size_t)c->result_ints));
        const int64_t set_cap = std::max<int64_t>(c->result_ints / 4, 1024);
        CK(c->starts.ensure(sizeof(unsigned long long) * (size_t)set_cap));
        CK(cudaMemsetAsync(c->slot.p, 0, sizeof(int32_t) * (size_t)c->stack_slots, s));

        Rules rule{};
        rule.off = rg->off.as<int64_t>();
        rule.off2 = rg->off2.as<int64_t>();
        rule.adj = rg->adj.as<int32_t>();
        rule.adj2 = rg->adj2.as<int32_t>();
        rule.md = c->md.as<int32_t>();
        rule.ubt = c->ubt.as<int32_t>();
        rule.mdlen = (int32_t)md.size();
        rule.min_size = min_size;
        rule.vbase = 0;
        rule.n = h.n;
        CK(c->rules.ensure(sizeof(Rules)));
        Control ctl{};
        ctl.arena_cap = (unsigned long long)c->arena_bytes;
        ctl.result_cap = (unsigned long long)c->result_ints;
        ctl.set_cap = (unsigned long long)set_cap;
        ctl.stack_cap = (int)std::min<int64_t>(c->stack_slots / kStackShards, INT32_MAX);
        if (root_dev) {
            CK(cudaEventRecord(c->ev[0], s));
            RootSetup S{};
            std::memcpy(S.head, &ctl, sizeof(S.head));
            S.rule = rule;
            S.flags = nshards > 1 ? kFlagShardRoot : 0;
            root_setup_kernel<<<1, 256, 0, s>>>(S, d_info, c->ids.as<int32_t>(), c->arena.as<char>(),
                                                (unsigned long long)c->arena_bytes, c->ctl.as<Control>(),
                                                c->stack.as<StackEntry>(), c->slot.as<int32_t>(),
                                                c->rules.as<Rules>(), c->pos.as<int32_t>());
            root_rows_dev_kernel<<<std::max(1, std::min(tmax, c->sms * 8)), 256, 0, s>>>(
                rg->off.as<int64_t>(), rg->adj.as<int32_t>(), rg->off2.as<int64_t>(),
                rg->adj2.as<int32_t>(), c->ids.as<int32_t>(), d_info, c->pos.as<int32_t>(),
                c->arena.as<char>(), (unsigned long long)c->arena_bytes);
            root_unpos_dev_kernel<<<(tmax + 255) / 256, 256, 0, s>>>(c->ids.as<int32_t>(), d_info,
                                                                    c->pos.as<int32_t>());
            CK(cudaGetLastError());
            c->launches += 3;
        } else {
        uint64_t rb = rec_bytes(t, W);
        const int root_cls = arena_class(rec_block_bytes(t, W));
        const uint64_t root_block = arena_class_bytes(root_cls);
        if ((int64_t)root_block > c->arena_bytes) {
            c->arena_bytes = (int64_t)root_block * 4;
            continue;
        }
        CK(cudaEventRecord(c->ev[0], s));
        // root record: header, ids, zero l2 and matrices, then rows
        char* rec = c->arena.as<char>();
        CK(cudaMemsetAsync(rec, 0, rb, s));
        TaskHdr hd{};
        hd.t = t;
        hd.m = 0;
        hd.cov = cov;
        hd.W = W;
        hd.refs = 1;
        hd.cls = root_cls;
        hd.inst = 0;
        hd.flags = nshards > 1 ? kFlagShardRoot : 0;
        CK(put_small(c, rec, &hd, sizeof(hd), s));
        CK(cudaMemcpyAsync(rec + rec_ids_off(), c->ids.p, sizeof(int32_t) * t,
                           cudaMemcpyDeviceToDevice, s));
        root_pos_kernel<<<(t + 255) / 256, 256, 0, s>>>(c->ids.as<int32_t>(), t,
                                                        c->pos.as<int32_t>(), 1);
        root_rows_kernel<<<std::min(blocks * 4, (t + 7) / 8), 256, 0, s>>>(
            rg->off.as<int64_t>(), rg->adj.as<int32_t>(), rg->off2.as<int64_t>(),
            rg->adj2.as<int32_t>(), c->ids.as<int32_t>(), t, W, c->pos.as<int32_t>(),
            (uint32_t*)(rec + rec_a1_off(t)), (uint32_t*)(rec + rec_a2_off(t, W)));
        root_pos_kernel<<<(t + 255) / 256, 256, 0, s>>>(c->ids.as<int32_t>(), t,
                                                        c->pos.as<int32_t>(), 0);
        CK(cudaGetLastError());
        c->launches += 3;

        ctl.arena_top = root_block;
        ctl.stack_top[0] = 1;
        ctl.pending = 1;
        CK(put_control(c, ctl, s));
        StackEntry root{};
        root.rec[0] = 0;
        root.n = 1;
        root.q_lo = -1;
        root.q_hi = -1;
        CK(put_small(c, c->stack.p, &root, sizeof(root), s));
        int one = 1;
        CK(put_small(c, c->slot.p, &one, sizeof(one), s));
        CK(put_small(c, c->rules.p, &rule, sizeof(rule), s));
        }
        ExpandParams P{};
        P.rules = c->rules.as<Rules>();
        P.nrules = 1;
        P.ctl = c->ctl.as<Control>();
        P.arena = c->arena.as<char>();
        P.stack = c->stack.as<StackEntry>();
        P.slot = c->slot.as<int32_t>();
        P.results = c->results.as<int32_t>();
        P.set_starts = c->starts.as<unsigned long long>();
        P.ws = c->ws.as<char>();
        P.ws_stride = L.total;
        P.arena_cap = (unsigned long long)c->arena_bytes;
        P.max_t = tmax;
        P.smem_t = sh.smem_t;
        // single instance: 0 lets the kernel choose by task size (one branch
        // an item up to 256 vertices, two above); the batched form keeps 2,
        // since there the work, not the start, bounds the run
        P.split = c->cfg.split > 0 ? c->cfg.split : 0;
        P.small_path = 1;
        P.shard = shard;
        P.nshards = nshards;
        P.shared_fifo = c->cfg.shared_order == 2 ? 1 : 0;
        P.wait_ns = (int64_t)c->cfg.wait_limit_ms * 1000000ll;
        P.time_limit_ns = c->cfg.time_limit_ms > 0
                              ? (unsigned long long)c->cfg.time_limit_ms * 1000000ull : 0ull;
        CK(cudaEventRecord(c->ev[1], s));
        expand_kernel<<<blocks, wpb * 32, sh.smem_bytes, s>>>(P);
        CK(cudaGetLastError());
        c->launches += 1;
        CK(cudaEventRecord(c->ev[2], s));
        CK(get_control(c, ctl, s));
        CK(cudaStreamSynchronize(s));
        float kms = 0;
        cudaEventElapsedTime(&kms, c->ev[1], c->ev[2]);
        if (root_dev) {
            t = ctl.root_t;
            cov = ctl.root_cov;
            if (t < 0 || t > tmax || cov < 0 || cov > t)
                return fail(QC_ERR_CUDA, "level 0 size out of range");
            r->st.root_size = (int64_t)t;
        }
        record_last(c, ctl, kms, t);

        if (ctl.status & ST_TASK_OVERFLOW) {
            if (ctl.arena_top > ctl.arena_cap) c->arena_bytes *= 4;
            const bool stack_full = max_top(ctl) >= ctl.stack_cap;
            if (stack_full) c->stack_slots *= 4;
            if (ctl.arena_top <= ctl.arena_cap && !stack_full) {
                c->arena_bytes *= 2;
                c->stack_slots *= 2;
            }
            if (attempt < 6) continue;
            return fail(QC_ERR_TASK_OVERFLOW, "task arena/stack exhausted after growing");
        }
        if (ctl.status & ST_RESULT_OVERFLOW) {
            c->result_ints = std::max<int64_t>({c->result_ints * 4, (int64_t)ctl.result_top * 2,
                                                (int64_t)ctl.emitted * 8});
            if (attempt < 6) continue;
            return fail(QC_ERR_RESULT_OVERFLOW, "result buffer exhausted after growing");
        }
        if (ctl.status & ST_CHECK)
            return fail(QC_ERR_CUDA, "device self-check failed at site " +
                                         std::to_string(ctl.check_site) + " value " +
                                         std::to_string(ctl.check_value));
        if (ctl.status & ST_TOO_LARGE) return fail(QC_ERR_TOO_LARGE, "task larger than workspace");
        if (ctl.status & ST_DEADLINE)
            return fail(QC_ERR_ITER_LIMIT,
                        "time limit reached after " + std::to_string(ctl.tasks) + " tasks, " +
                            std::to_string(ctl.branches) + " branches, " +
                            std::to_string(ctl.emitted) + " emitted sets, " +
                            std::to_string(ctl.result_top) + " result ints, " +
                            std::to_string(ctl.arena_top) + " arena bytes, stack " +
                            std::to_string(max_top(ctl)) + " on the fullest stack shard, max task " +
                            std::to_string(ctl.max_task));
        if (ctl.status & ST_ITER_LIMIT)
            return fail(QC_ERR_ITER_LIMIT, "device wait gave up (site " +
                                               std::to_string(ctl.wait_fail_where) + ")");
        r->st.tasks = (int64_t)ctl.tasks;
        r->st.branches = (int64_t)ctl.branches;
        r->st.children = (int64_t)ctl.children;
        r->st.emitted = (int64_t)ctl.emitted;
        r->st.emitted_ints = (int64_t)ctl.result_top;
        r->st.max_task = ctl.max_task;
        r->st.parent_vertices = (int64_t)ctl.parent_vertices;
        r->st.p_rows = (int64_t)ctl.p_rows;
        r->st.child_vertices = (int64_t)ctl.child_vertices;
        r->st.kernel_ms = kms;
        r->st.arena_peak = (int64_t)std::min(ctl.arena_top, ctl.arena_cap);
        r->st.kernel_launches = c->launches;
        if (c->cfg.keep_emitted) {
            flat.resize((size_t)ctl.result_top);
            if (!flat.empty())
                CK(cudaMemcpyAsync(flat.data(), c->results.p, sizeof(int32_t) * flat.size(),
                                   cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        r->st.enum_ms = ms_since(t_enum);
        break;
    }

    // non-maximal removal on the device
    auto t_filter = clk::now();
    std::string fe = filter_maximal(c->filt, c->results.as<int32_t>(), r->st.emitted_ints,
                                    c->starts.as<unsigned long long>(), r->st.emitted, h.n, s,
                                    c->sms, r->sets, r->nsets, &c->launches);
    if (!fe.empty()) return fail(QC_ERR_CUDA, fe);
    r->st.filter_ms = ms_since(t_filter);
    r->st.maximal = r->nsets;
    r->st.kernel_launches = c->launches;
    if (c->cfg.keep_emitted) {
        r->emitted.swap(flat);
        r->emitted_sets = r->st.emitted;
    }
    r->st.total_ms = ms_since(t_all);
    return QC_OK;
}

extern "C" qc_status qc_maximal_sets(qc_context* c, const int32_t* flat, int64_t n_ints,
                                     int32_t n_vertices, qc_result** out)
{
    if (!c || !out || n_ints < 0 || (n_ints > 0 && !flat) || n_vertices < 0)
        return fail(QC_ERR_ARGS, "bad arguments");
    *out = nullptr;
    // set starts, with the checks the device filter relies on
    std::vector<unsigned long long> starts;
    std::vector<uint8_t> seen((size_t)n_vertices, 0);
    for (int64_t p = 0; p < n_ints;) {
        const int32_t k = flat[p];
        if (k < 1 || p + 1 + k > n_ints) return fail(QC_ERR_FORMAT, "malformed set record");
        for (int32_t i = 0; i < k; i++) {
            const int32_t v = flat[p + 1 + i];
            if (v < 0 || v >= n_vertices) return fail(QC_ERR_FORMAT, "vertex id out of range");
            if (seen[(size_t)v]) return fail(QC_ERR_FORMAT, "repeated id within a set");
            seen[(size_t)v] = 1;
        }
        for (int32_t i = 0; i < k; i++) seen[(size_t)flat[p + 1 + i]] = 0;
        starts.push_back((unsigned long long)p);
        p += 1 + k;
    }
    CK(cudaSetDevice(c->cfg.device));
    std::unique_ptr<qc_result> r(new qc_result());
    auto t0 = clk::now();
    const int64_t nsets = (int64_t)starts.size();
    if (nsets > 0) {
        cudaStream_t s = c->stream;
        CK(c->results.ensure(sizeof(int32_t) * (size_t)n_ints));
        CK(c->starts.ensure(sizeof(unsigned long long) * (size_t)nsets));
        CK(cudaMemcpyAsync(c->results.p, flat, sizeof(int32_t) * (size_t)n_ints,
                           cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(c->starts.p, starts.data(), sizeof(unsigned long long) * (size_t)nsets,
                           cudaMemcpyHostToDevice, s));
        std::string fe = filter_maximal(c->filt, c->results.as<int32_t>(), n_ints,
                                        c->starts.as<unsigned long long>(), nsets,
                                        std::max<int32_t>(n_vertices, 1), s, c->sms, r->sets,
                                        r->nsets, &c->launches);
        if (!fe.empty()) return fail(QC_ERR_CUDA, fe);
    }
    r->st.emitted = nsets;
    r->st.emitted_ints = n_ints;
    r->st.maximal = r->nsets;
    r->st.filter_ms = ms_since(t0);
    r->st.total_ms = r->st.filter_ms;
    *out = r.release();
    return QC_OK;
}

extern "C" qc_status qc_context_upload(qc_context* c, const qc_graph* g)
{
    if (!c || !g) return fail(QC_ERR_ARGS, "NULL argument");
    CK(cudaSetDevice(c->cfg.device));
    ResidentGraph* rg = nullptr;
    return make_resident(c, g, nullptr, &rg);
}

extern "C" void* qc_context_stream(qc_context* c) { return c ? (void*)c->stream : nullptr; }

extern "C" qc_status qc_context_last_stats(const qc_context* c, qc_stats* out)
{
    if (!c || !out) return fail(QC_ERR_ARGS, "NULL argument");
    *out = c->last;
    return QC_OK;
}

// Load the mining path's kernels now, at context creation, by mining a
// 6-vertex clique once: with lazy module loading each kernel would otherwise
// be loaded at its first launch, inside the first mining call.
static qc_status warm_kernels(qc_context* c)
{
    qc_graph* g = new qc_graph();
    const int n = 6;
    g->h.n = n;
    for (int v = 0; v <= n; v++) g->h.off.push_back((int64_t)v * (n - 1));
    for (int v = 0; v < n; v++)
        for (int w = 0; w < n; w++)
            if (w != v) g->h.adj.push_back(w);
    g->h.off2 = g->h.off;
    g->h.adj2 = g->h.adj;
    qc_result r;
    const int64_t launches = c->launches;
    qc_status st = mine_one(c, g, 0.9, 3, &r);
    qc_graph_free(g); // its device copy's buffers go to the next graph
    c->launches = launches;
    return st;
}

extern "C" qc_status qc_mine(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                             int32_t sched, qc_result** out)
{
    (void)sched;
    if (!ctx || !g || !out) return fail(QC_ERR_ARGS, "NULL argument");
    *out = nullptr;
    if (!(gamma >= 0.5 && gamma <= 1.0))
        return fail(QC_ERR_ARGS, "minimum degree ratio must be between .5 and 1 inclusive");
    if (min_size <= 1) return fail(QC_ERR_ARGS, "minimum size must be greater than 1");
    if (g->h.off2.size() != g->h.off.size()) return fail(QC_ERR_FORMAT, "graph has no 2-hop lists");
    std::unique_ptr<qc_result> r(new qc_result());
    qc_status st = mine_one(ctx, g, gamma, min_size, r.get());
    if (st != QC_OK) return st;
    *out = r.release();
    return QC_OK;
}

static qc_status check_mine_args(const qc_graph* g, double gamma, int32_t min_size)
{
    if (!(gamma >= 0.5 && gamma <= 1.0))
        return fail(QC_ERR_ARGS, "minimum degree ratio must be between .5 and 1 inclusive");
    if (min_size <= 1) return fail(QC_ERR_ARGS, "minimum size must be greater than 1");
    if (g->h.off2.size() != g->h.off.size()) return fail(QC_ERR_FORMAT, "graph has no 2-hop lists");
    return QC_OK;
}

extern "C" qc_status qc_mine_shard(qc_context* ctx, const qc_graph* g, double gamma,
                                   int32_t min_size, int32_t shard, int32_t nshards,
                                   qc_result** out)
{
    if (!ctx || !g || !out) return fail(QC_ERR_ARGS, "NULL argument");
    *out = nullptr;
    if (nshards < 1 || shard < 0 || shard >= nshards) return fail(QC_ERR_ARGS, "bad shard");
    qc_status st = check_mine_args(g, gamma, min_size);
    if (st != QC_OK) return st;
    std::unique_ptr<qc_result> r(new qc_result());
    st = mine_one(ctx, g, gamma, min_size, r.get(), shard, nshards);
    if (st != QC_OK) return st;
    *out = r.release();
    return QC_OK;
}

extern "C" qc_status qc_root(qc_context* c, const qc_graph* g, double gamma, int32_t min_size,
                             int32_t* ids_out, int64_t cap, int32_t* t_out, int32_t* cov_out)
{
    if (!c || !g || !t_out || !cov_out || cap < 0 || (cap > 0 && !ids_out))
        return fail(QC_ERR_ARGS, "bad arguments");
    qc_status st = check_mine_args(g, gamma, min_size);
    if (st != QC_OK) return st;
    CK(cudaSetDevice(c->cfg.device));
    ResidentGraph* rg = nullptr;
    st = make_resident(c, g, nullptr, &rg);
    if (st != QC_OK) return st;
    std::vector<int32_t> md, ubt;
    gamma_tables(gamma, g->h.n, min_size, md, ubt);
    int t = 0, cov = 0;
    st = compute_root(c, g->h, rg, md, min_size, t, cov, nullptr);
    if (st != QC_OK) return st;
    const int64_t k = std::min<int64_t>(cap, t);
    if (k > 0) {
        CK(cudaMemcpyAsync(ids_out, c->ids.p, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    *t_out = t;
    *cov_out = cov;
    return QC_OK;
}

// ------------------------------------------------------------------
// autotuning of the launch shape (in place of the reference's compile-time
// BLOCK_SIZE / NUM_OF_BLOCKS / TASKS_PER_WARP / EXPAND_THRESHOLD #defines,
// main.cu:21-55)
// ------------------------------------------------------------------

// The search behind qc_tune and qc_tune_batch.  `run(kernel_ms, nsets)` mines
// the sample workload once with ctx->cfg.  First the launch shape (warps per
// block, blocks per SM, branches per work item of a large task), then, from
// the best shape, the largest task staged in shared memory (beyond it task
// records are read through L2) and the order idle warps take donated tasks
// in, one knob at a time.  Every run must give the same number of sets.
template <class Run>
static qc_status tune_search(qc_context* ctx, int32_t repeats, Run run, qc_config* best)
{
    if (repeats < 1) repeats = 2;
    const qc_config keep = ctx->cfg;
    qc_config chosen = keep;
    double best_ms = 1e300;
    int64_t want_sets = -1;
    auto time_cfg = [&](const qc_config& cfg, double& t) -> qc_status {
        ctx->cfg = cfg;
        t = 1e300;
        for (int32_t rep = 0; rep <= repeats; rep++) { // the first run warms up
            double ms = 0;
            int64_t nsets = 0;
            qc_status st = run(ms, nsets);
            if (st != QC_OK) return st;
            if (want_sets < 0) want_sets = nsets;
            if (nsets != want_sets) return fail(QC_ERR_CUDA, "tuning runs disagree on the result");
            if (rep > 0) t = std::min(t, ms);
        }
        return QC_OK;
    };
    auto consider = [&](const qc_config& cfg) -> qc_status {
        double t = 0;
        qc_status st = time_cfg(cfg, t);
        if (st != QC_OK) return st;
        if (t < best_ms) {
            best_ms = t;
            chosen = cfg;
        }
        return QC_OK;
    };
    static const int32_t kWpb[] = {4, 8};
    static const int32_t kBps[] = {1, 2};
    static const int32_t kSplit[] = {1, 2, 4};
    for (int32_t wpb : kWpb)
        for (int32_t bps : kBps)
            for (int32_t split : kSplit) {
                qc_config cfg = keep;
                cfg.warps_per_block = wpb;
                cfg.blocks_per_sm = bps;
                cfg.split = split;
                qc_status st = consider(cfg);
                if (st != QC_OK) {
                    ctx->cfg = keep;
                    return st;
                }
            }
    const qc_config shape = chosen;
    for (int32_t stage : {64, -1}) {
        qc_config cfg = shape;
        cfg.stage_max = stage;
        qc_status st = consider(cfg);
        if (st != QC_OK) {
            ctx->cfg = keep;
            return st;
        }
    }
    const qc_config staged = chosen;
    for (int32_t order : {1, 2}) {
        qc_config cfg = staged;
        cfg.shared_order = order;
        qc_status st = consider(cfg);
        if (st != QC_OK) {
            ctx->cfg = keep;
            return st;
        }
    }
    ctx->cfg = chosen;
    if (best) *best = chosen;
    return QC_OK;
}

extern "C" qc_status qc_tune(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                             int32_t repeats, qc_config* best)
{
    if (!ctx || !g) return fail(QC_ERR_ARGS, "NULL argument");
    qc_status st = check_mine_args(g, gamma, min_size);
    if (st != QC_OK) return st;
    return tune_search(ctx, repeats, [&](double& ms, int64_t& nsets) -> qc_status {
        qc_result r;
        qc_status s2 = mine_one(ctx, g, gamma, min_size, &r);
        ms = r.st.kernel_ms;
        nsets = r.nsets;
        return s2;
    }, best);
}

static qc_status mine_batch(qc_context* c, const qc_graph* const* graphs, const double* gammas,
                            const int32_t* min_sizes, int32_t count, std::vector<qc_result*>& res);

extern "C" qc_status qc_tune_batch(qc_context* ctx, const qc_graph* const* graphs,
                                   const double* gammas, const int32_t* min_sizes, int32_t count,
                                   int32_t repeats, qc_config* best)
{
    if (!ctx || !graphs || !gammas || !min_sizes || count < 1) return fail(QC_ERR_ARGS, "bad arguments");
    for (int32_t i = 0; i < count; i++) {
        if (!graphs[i]) return fail(QC_ERR_ARGS, "NULL graph in batch");
        qc_status st = check_mine_args(graphs[i], gammas[i], min_sizes[i]);
        if (st != QC_OK) return st;
    }
    return tune_search(ctx, repeats, [&](double& ms, int64_t& nsets) -> qc_status {
        std::vector<qc_result*> res;
        qc_status s2 = mine_batch(ctx, graphs, gammas, min_sizes, count, res);
        ms = 0;
        nsets = 0;
        if (s2 == QC_OK && !res.empty()) ms = res[0]->st.kernel_ms;
        for (auto* r : res) {
            if (r) nsets += r->nsets;
            delete r;
        }
        return s2;
    }, best);
}

// ------------------------------------------------------------------
// batched mining: many independent instances in one persistent launch
// ------------------------------------------------------------------

struct RootMeta {
    unsigned long long rec; // arena offset of the root record
    int32_t t, W, cov, inst, cls, vbase;
    int64_t id_at;          // first id in the concatenated root-id array
    int64_t row_at;         // first row in the flattened row index
};

// headers and ids of every root record (one thread per root id)
__global__ void batch_root_fill_kernel(const RootMeta* meta, int nroots, const int32_t* ids_all,
                                       int64_t total_rows, char* arena, int32_t* pos)
{
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= total_rows) return;
    int lo = 0, hi = nroots - 1; // root j with row_at <= r
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (meta[mid].row_at <= r) lo = mid;
        else hi = mid - 1;
    }
    const RootMeta& M = meta[lo];
    int i = (int)(r - M.row_at);
    char* rec = arena + M.rec;
    int32_t id = ids_all[M.id_at + i];
    ((int32_t*)(rec + rec_ids_off()))[i] = id;
    ((int32_t*)(rec + rec_l2_off(M.t)))[i] = 0;
    pos[M.vbase + id] = i;
    if (i == 0) {
        TaskHdr* h = (TaskHdr*)rec;
        h->t = M.t;
        h->m = 0;
        h->cov = M.cov;
        h->W = M.W;
        h->refs = 1;
        h->cls = M.cls;
        h->inst = M.inst;
        h->flags = 0;
    }
}

// one warp per root row: set the bits of its 1-hop and 2-hop neighbours
__global__ void batch_root_rows_kernel(const RootMeta* meta, int nroots, const int32_t* ids_all,
                                       int64_t total_rows, const Rules* rules,
                                       char* arena, const int32_t* pos)
{
    int lane = threadIdx.x & 31;
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < total_rows; r += nw) {
        int lo = 0, hi = nroots - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (meta[mid].row_at <= r) lo = mid;
            else hi = mid - 1;
        }
        const RootMeta& M = meta[lo];
        int i = (int)(r - M.row_at);
        const Rules& R = rules[M.inst];
        const int32_t* adj = R.adj;
        const int32_t* adj2 = R.adj2;
        int u = ids_all[M.id_at + i];
        char* rec = arena + M.rec;
        uint32_t* r1 = (uint32_t*)(rec + rec_a1_off(M.t)) + (int64_t)i * M.W;
        uint32_t* r2 = (uint32_t*)(rec + rec_a2_off(M.t, M.W)) + (int64_t)i * M.W;
        const int32_t* pv = pos + M.vbase;
        for (int64_t e = R.off[u] + lane; e < R.off[u + 1]; e += 32) {
            int p = pv[adj[e]];
            if (p >= 0) atomicOr(&r1[p >> 5], 1u << (p & 31));
        }
        for (int64_t e = R.off2[u] + lane; e < R.off2[u + 1]; e += 32) {
            int p = pv[adj2[e]];
            if (p >= 0) atomicOr(&r2[p >> 5], 1u << (p & 31));
        }
    }
}

__global__ void batch_root_unpos_kernel(const RootMeta* meta, int nroots, const int32_t* ids_all,
                                        int64_t total_rows, int32_t* pos)
{
    int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= total_rows) return;
    int lo = 0, hi = nroots - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (meta[mid].row_at <= r) lo = mid;
        else hi = mid - 1;
    }
    const RootMeta& M = meta[lo];
    pos[M.vbase + ids_all[M.id_at + (r - M.row_at)]] = -1;
}


static qc_status mine_batch(qc_context* c, const qc_graph* const* graphs, const double* gammas,
                            const int32_t* min_sizes, int32_t count, std::vector<qc_result*>& res)
{
    auto t_all = clk::now();
    cudaStream_t s = c->stream;
    CK(cudaSetDevice(c->cfg.device));
    BatchBufs& B = c->batch; // reused across calls on this context
    // every instance's graph resident on the device (uploaded on first use);
    // the rules of instance i point at its own arrays, nothing is concatenated
    std::vector<int32_t> h_md, h_ubt;
    std::vector<Rules> rules(count);
    std::vector<int64_t> md_at_(count);
    std::vector<RootMeta> meta;
    int64_t vtotal = 0;
    int max_t = 1;
    auto t_load = clk::now();
    std::unordered_set<unsigned long long> batch_serials;
    for (int i = 0; i < count; i++) batch_serials.insert(graphs[i]->serial);
    for (int i = 0; i < count; i++) {
        const HostGraph& h = graphs[i]->h;
        ResidentGraph* rg = nullptr;
        qc_status us = make_resident(c, graphs[i], &batch_serials, &rg);
        if (us != QC_OK) return us;
        rules[i].off = rg->off.as<int64_t>();
        rules[i].off2 = rg->off2.as<int64_t>();
        rules[i].adj = rg->adj.as<int32_t>();
        rules[i].adj2 = rg->adj2.as<int32_t>();
        rules[i].vbase = (int32_t)vtotal;
        rules[i].n = h.n;
        vtotal += h.n;
    }
    if (vtotal > INT32_MAX) return fail(QC_ERR_TOO_LARGE, "batch has more than 2^31 vertices");
    double load_ms = ms_since(t_load);

    auto t_enum = clk::now();
    // level 0 of every instance: on the device, one block per instance, for
    // instances of up to kLevel0DeviceMax vertices (their root ids land in the
    // shared id array at the instance's vertex base); larger ones on the host
    std::vector<Level0Job> jobs;
    std::vector<int32_t> job_inst;
    std::vector<std::vector<int32_t>> host_ids(count);
    std::vector<int32_t> root_t(count, 0), root_cov(count, 0);
    int64_t l0_bytes = 0;
    for (int i = 0; i < count; i++) {
        const HostGraph& h = graphs[i]->h;
        std::vector<int32_t> md, ubt;
        gamma_tables(gammas[i], h.n, min_sizes[i], md, ubt);
        md_at_[i] = (int64_t)h_md.size();
        rules[i].mdlen = (int32_t)md.size();
        rules[i].min_size = min_sizes[i];
        h_md.insert(h_md.end(), md.begin(), md.end());
        h_ubt.insert(h_ubt.end(), ubt.begin(), ubt.end());
        if (h.n == 0) continue;
        if (h.n <= kLevel0DeviceMax) {
            Level0Job J{};
            J.off = rules[i].off;
            J.adj = rules[i].adj;
            J.off2 = rules[i].off2;
            J.n = h.n;
            J.need = md[(size_t)min_sizes[i]];
            J.min_size = min_sizes[i];
            J.scratch_at = l0_bytes;
            J.ids_at = rules[i].vbase;
            l0_bytes += level0_scratch_bytes(h.n);
            jobs.push_back(J);
            job_inst.push_back(i);
        } else {
            int cov = 0;
            build_root(h, md.data(), min_sizes[i], host_ids[(size_t)i], cov);
            root_t[(size_t)i] = (int32_t)host_ids[(size_t)i].size();
            root_cov[(size_t)i] = cov;
        }
    }
    CK(B.ids.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(vtotal, 4)));
    for (int i = 0; i < count; i++)
        if (!host_ids[(size_t)i].empty())
            CK(cudaMemcpyAsync(B.ids.as<int32_t>() + rules[i].vbase, host_ids[(size_t)i].data(),
                               sizeof(int32_t) * host_ids[(size_t)i].size(), cudaMemcpyHostToDevice,
                               s));
    if (!jobs.empty()) {
        CK(upload(B.jobs, jobs, s));
        CK(B.l0scratch.ensure((size_t)std::max<int64_t>(l0_bytes, 16)));
        CK(B.l0info.ensure(sizeof(int32_t) * 2 * jobs.size()));
        level0_batch_kernel<<<(unsigned)jobs.size(), 256, 0, s>>>(
            B.jobs.as<Level0Job>(), B.l0scratch.as<char>(), B.ids.as<int32_t>(),
            B.l0info.as<int32_t>());
        CK(cudaGetLastError());
        c->launches += 1;
        std::vector<int32_t> info(2 * jobs.size());
        CK(cudaMemcpyAsync(info.data(), B.l0info.p, sizeof(int32_t) * info.size(),
                           cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (size_t j = 0; j < jobs.size(); j++) {
            const int i = job_inst[j];
            const int32_t t = info[2 * j], cov = info[2 * j + 1];
            if (t < 0 || t > graphs[i]->h.n || cov < 0 || cov > t)
                return fail(QC_ERR_CUDA, "level 0 size out of range");
            root_t[(size_t)i] = t;
            root_cov[(size_t)i] = cov;
        }
    }
    uint64_t arena_at = 0;
    int64_t rows_at = 0;
    for (int i = 0; i < count; i++) {
        if (root_t[(size_t)i] == 0) continue;
        RootMeta M{};
        M.t = root_t[(size_t)i];
        M.W = words_for(M.t);
        M.cov = root_cov[(size_t)i];
        M.inst = i;
        M.cls = arena_class(rec_block_bytes(M.t, M.W));
        M.vbase = rules[i].vbase;
        M.rec = arena_at;
        M.id_at = rules[i].vbase;
        M.row_at = rows_at;
        rows_at += M.t;
        arena_at += arena_class_bytes(M.cls);
        max_t = std::max(max_t, M.t);
        meta.push_back(M);
    }
    CK(upload(B.md, h_md, s));
    CK(upload(B.ubt, h_ubt, s));
    for (int i = 0; i < count; i++) {
        rules[i].md = B.md.as<int32_t>() + md_at_[i];
        rules[i].ubt = B.ubt.as<int32_t>() + md_at_[i];
    }
    CK(upload(B.rules, rules, s));
    const int nroots = (int)meta.size();
    const int64_t total_rows = rows_at;

    Shape sh;
    {
        qc_status ss = launch_shape(c, max_t, sh);
        if (ss != QC_OK) return ss;
    }
    const int wpb = sh.wpb, blocks = sh.blocks;
    int nwarps = blocks * wpb;
    WsLayout L = ws_layout(max_t);
    CK(c->ws.ensure((size_t)L.total * nwarps));
    CK(c->ctl.ensure(sizeof(Control)));
    if (nroots > 0) {
        CK(upload(B.meta, meta, s));
        if (B.pos.n < sizeof(int32_t) * (size_t)std::max<int64_t>(vtotal, 1)) {
            CK(B.pos.ensure(sizeof(int32_t) * (size_t)std::max<int64_t>(vtotal, 1)));
            CK(cudaMemsetAsync(B.pos.p, 0xff, B.pos.n, s));
        }
    }

    Control ctl{};
    float kms = 0;
    c->pin_at = 0;
    for (int attempt = 0;; attempt++) {
        if (attempt > 0) c->pin_at = 0; // the previous attempt synchronised
        if ((int64_t)arena_at * 2 > c->arena_bytes) c->arena_bytes = (int64_t)arena_at * 2;
        c->stack_slots = std::max<int64_t>(c->stack_slots, (int64_t)nroots * 2 + 64 * kStackShards);
        CK(c->arena.ensure((size_t)c->arena_bytes));
        c->stack_slots = shard_slots(std::max<int64_t>(c->stack_slots, 2 * kStackShards));
        CK(c->stack.ensure(sizeof(StackEntry) * (size_t)c->stack_slots));
        CK(c->slot.ensure(sizeof(int32_t) * (size_t)c->stack_slots));
        CK(c->results.ensure(sizeof(int32_t) * (size_t)c->result_ints));
        const int64_t set_cap = std::max<int64_t>(c->result_ints / 4, 1024);
        CK(c->starts.ensure(sizeof(unsigned long long) * (size_t)set_cap));
        CK(cudaMemsetAsync(c->slot.p, 0, sizeof(int32_t) * (size_t)c->stack_slots, s));
        if (nroots == 0) break;
        CK(cudaEventRecord(c->ev[0], s));
        CK(cudaMemsetAsync(c->arena.p, 0, arena_at, s));
        int64_t rb = (total_rows + 255) / 256;
        batch_root_fill_kernel<<<(unsigned)rb, 256, 0, s>>>(B.meta.as<RootMeta>(), nroots,
                                                            B.ids.as<int32_t>(), total_rows,
                                                            c->arena.as<char>(), B.pos.as<int32_t>());
        batch_root_rows_kernel<<<std::max(1, blocks * 4), 256, 0, s>>>(
            B.meta.as<RootMeta>(), nroots, B.ids.as<int32_t>(), total_rows, B.rules.as<Rules>(),
            c->arena.as<char>(), B.pos.as<int32_t>());
        batch_root_unpos_kernel<<<(unsigned)rb, 256, 0, s>>>(B.meta.as<RootMeta>(), nroots,
                                                             B.ids.as<int32_t>(), total_rows,
                                                             B.pos.as<int32_t>());
        CK(cudaGetLastError());
        c->launches += 3;
        ctl = Control{};
        ctl.arena_top = arena_at;
        ctl.arena_cap = (unsigned long long)c->arena_bytes;
        ctl.result_cap = (unsigned long long)c->result_ints;
        ctl.set_cap = (unsigned long long)set_cap;
        // roots dealt round-robin over the stack shards: root j is entry j / S
        // of shard j % S, so every shard's entries are contiguous
        const int64_t per_shard = c->stack_slots / kStackShards;
        ctl.stack_cap = (int)std::min<int64_t>(per_shard, INT32_MAX);
        ctl.pending = nroots;
        std::vector<StackEntry> items((size_t)nroots);
        std::vector<int32_t> ones((size_t)nroots, 1);
        int64_t filled = 0;
        for (int shard = 0; shard < kStackShards; shard++) {
            int cnt = 0;
            for (int j = shard; j < nroots; j += kStackShards) {
                StackEntry e{};
                e.rec[0] = meta[(size_t)j].rec;
                e.n = 1;
                e.q_lo = -1;
                e.q_hi = -1;
                items[(size_t)(filled + cnt)] = e;
                cnt++;
            }
            ctl.stack_top[shard] = cnt;
            if (cnt > 0) {
                CK(cudaMemcpyAsync(c->stack.as<StackEntry>() + (size_t)shard * per_shard,
                                   items.data() + filled, sizeof(StackEntry) * cnt,
                                   cudaMemcpyHostToDevice, s));
                CK(cudaMemcpyAsync(c->slot.as<int32_t>() + (size_t)shard * per_shard, ones.data(),
                                   sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, s));
            }
            filled += cnt;
        }
        CK(put_control(c, ctl, s));
        ExpandParams P{};
        P.rules = B.rules.as<Rules>();
        P.nrules = count;
        P.ctl = c->ctl.as<Control>();
        P.arena = c->arena.as<char>();
        P.stack = c->stack.as<StackEntry>();
        P.slot = c->slot.as<int32_t>();
        P.results = c->results.as<int32_t>();
        P.set_starts = c->starts.as<unsigned long long>();
        P.ws = c->ws.as<char>();
        P.ws_stride = L.total;
        P.arena_cap = (unsigned long long)c->arena_bytes;
        P.max_t = max_t;
        P.smem_t = sh.smem_t;
        P.split = c->cfg.split > 0 ? c->cfg.split : 2;
        P.small_path = 1;
        P.shared_fifo = c->cfg.shared_order == 1 ? 0 : 1;
        P.wait_ns = (int64_t)c->cfg.wait_limit_ms * 1000000ll;
        P.time_limit_ns = c->cfg.time_limit_ms > 0
                              ? (unsigned long long)c->cfg.time_limit_ms * 1000000ull : 0ull;
        CK(cudaEventRecord(c->ev[1], s));
        expand_kernel<<<blocks, wpb * 32, sh.smem_bytes, s>>>(P);
        CK(cudaGetLastError());
        c->launches += 1;
        CK(cudaEventRecord(c->ev[2], s));
        CK(get_control(c, ctl, s));
        CK(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&kms, c->ev[1], c->ev[2]);
        record_last(c, ctl, kms, 0);
        if (ctl.status & ST_TASK_OVERFLOW) {
            if (ctl.arena_top > ctl.arena_cap) c->arena_bytes *= 4;
            const bool stack_full = max_top(ctl) >= ctl.stack_cap;
            if (stack_full) c->stack_slots *= 4;
            if (ctl.arena_top <= ctl.arena_cap && !stack_full) {
                c->arena_bytes *= 2;
                c->stack_slots *= 2;
            }
            if (attempt < 6) continue;
            return fail(QC_ERR_TASK_OVERFLOW, "task arena/stack exhausted after growing");
        }
        if (ctl.status & ST_RESULT_OVERFLOW) {
            c->result_ints = std::max<int64_t>({c->result_ints * 4, (int64_t)ctl.result_top * 2,
                                                (int64_t)ctl.emitted * 8});
            if (attempt < 6) continue;
            return fail(QC_ERR_RESULT_OVERFLOW, "result buffer exhausted after growing");
        }
        if (ctl.status & ST_CHECK)
            return fail(QC_ERR_CUDA, "device self-check failed at site " +
                                         std::to_string(ctl.check_site) + " value " +
                                         std::to_string(ctl.check_value));
        if (ctl.status & ST_TOO_LARGE) return fail(QC_ERR_TOO_LARGE, "task larger than workspace");
        if (ctl.status & ST_DEADLINE) return fail(QC_ERR_ITER_LIMIT, "time limit reached");
        if (ctl.status & ST_ITER_LIMIT)
            return fail(QC_ERR_ITER_LIMIT, "device wait gave up (site " +
                                               std::to_string(ctl.wait_fail_where) + ")");
        break;
    }
    double enum_ms = ms_since(t_enum);

    // one filter over all instances: ids are global (vbase + id), so sets of
    // different instances never contain one another
    auto t_filter = clk::now();
    std::vector<int32_t> flat;
    int64_t nsets = 0;
    std::string fe = filter_maximal(c->filt, c->results.as<int32_t>(), (int64_t)ctl.result_top,
                                    c->starts.as<unsigned long long>(), (int64_t)ctl.emitted,
                                    (int32_t)std::max<int64_t>(vtotal, 1), s, c->sms, flat, nsets,
                                    &c->launches);
    if (!fe.empty()) return fail(QC_ERR_CUDA, fe);
    double filter_ms = ms_since(t_filter);
    res.assign((size_t)count, nullptr);
    for (int i = 0; i < count; i++) res[(size_t)i] = new qc_result();
    std::vector<int32_t> vb(count);
    for (int i = 0; i < count; i++) vb[i] = rules[i].vbase;
    for (int64_t p = 0; p < (int64_t)flat.size();) {
        int32_t k = flat[(size_t)p];
        int32_t first = flat[(size_t)p + 1];
        int i = (int)(std::upper_bound(vb.begin(), vb.end(), first) - vb.begin()) - 1;
        qc_result* r = res[(size_t)i];
        r->sets.push_back(k);
        for (int32_t j = 0; j < k; j++) r->sets.push_back(flat[(size_t)(p + 1 + j)] - vb[i]);
        r->nsets++;
        p += 1 + k;
    }
    double total_ms = ms_since(t_all);
    for (int i = 0; i < count; i++) {
        qc_stats& st = res[(size_t)i]->st;
        st.load_ms = load_ms;
        st.enum_ms = enum_ms;
        st.filter_ms = filter_ms;
        st.total_ms = total_ms;
        st.kernel_ms = kms;
        st.tasks = (int64_t)ctl.tasks;
        st.branches = (int64_t)ctl.branches;
        st.children = (int64_t)ctl.children;
        st.emitted = (int64_t)ctl.emitted;
        st.emitted_ints = (int64_t)ctl.result_top;
        st.maximal = res[(size_t)i]->nsets;
        st.max_task = ctl.max_task;
        st.arena_peak = (int64_t)std::min(ctl.arena_top, ctl.arena_cap);
        st.kernel_launches = c->launches;
        st.parent_vertices = (int64_t)ctl.parent_vertices;
        st.p_rows = (int64_t)ctl.p_rows;
        st.child_vertices = (int64_t)ctl.child_vertices;
    }
    return QC_OK;
}

extern "C" qc_status qc_mine_batch(qc_context* ctx, const qc_graph* const* graphs,
                                   const double* gammas, const int32_t* min_sizes, int32_t count,
                                   qc_result** outs)
{
    if (!ctx || !graphs || !gammas || !min_sizes || !outs || count < 0)
        return fail(QC_ERR_ARGS, "NULL argument");
    for (int32_t i = 0; i < count; i++) outs[i] = nullptr;
    for (int32_t i = 0; i < count; i++) {
        if (!graphs[i]) return fail(QC_ERR_ARGS, "NULL graph in batch");
        if (!(gammas[i] >= 0.5 && gammas[i] <= 1.0))
            return fail(QC_ERR_ARGS, "minimum degree ratio must be between .5 and 1 inclusive");
        if (min_sizes[i] <= 1) return fail(QC_ERR_ARGS, "minimum size must be greater than 1");
        if (graphs[i]->h.off2.size() != graphs[i]->h.off.size())
            return fail(QC_ERR_FORMAT, "graph has no 2-hop lists");
    }
    if (count == 0) return QC_OK;
    std::vector<qc_result*> res;
    qc_status st = mine_batch(ctx, graphs, gammas, min_sizes, count, res);
    if (st != QC_OK) {
        for (auto* r : res) delete r;
        return st;
    }
    for (int32_t i = 0; i < count; i++) outs[i] = res[(size_t)i];
    return QC_OK;
}

// ------------------------------------------------------------------
// results
// ------------------------------------------------------------------

extern "C" int64_t qc_result_count(const qc_result* r) { return r ? r->nsets : 0; }
extern "C" const int32_t* qc_result_sets(const qc_result* r, int64_t* n_ints)
{
    if (!r) return nullptr;
    if (n_ints) *n_ints = (int64_t)r->sets.size();
    return r->sets.data();
}
extern "C" const int32_t* qc_result_emitted(const qc_result* r, int64_t* n_sets, int64_t* n_ints)
{
    if (!r) return nullptr;
    if (n_sets) *n_sets = r->emitted_sets;
    if (n_ints) *n_ints = (int64_t)r->emitted.size();
    return r->emitted.data();
}
extern "C" const qc_stats* qc_result_stats(const qc_result* r) { return r ? &r->st : nullptr; }
extern "C" qc_status qc_result_write(const qc_result* r, const char* path)
{
    if (!r || !path) return fail(QC_ERR_ARGS, "NULL argument");
    std::string e = write_result(r->sets.data(), (int64_t)r->sets.size(), path);
    return e.empty() ? QC_OK : fail(QC_ERR_IO, e);
}
extern "C" void qc_result_free(qc_result* r) { delete r; }

struct qc_writer {
    std::thread th;
    std::string err;
};

extern "C" qc_status qc_sets_write_async(const int32_t* flat, int64_t n_ints, const char* path,
                                         qc_writer** out)
{
    if (!path || !out || n_ints < 0 || (n_ints > 0 && !flat)) return fail(QC_ERR_ARGS, "bad arguments");
    qc_writer* w = new qc_writer;
    const std::string p(path);
    w->th = std::thread([w, flat, n_ints, p] { w->err = write_result(flat, n_ints, p.c_str()); });
    *out = w;
    return QC_OK;
}

extern "C" qc_status qc_result_write_async(const qc_result* r, const char* path, qc_writer** out)
{
    if (!r) return fail(QC_ERR_ARGS, "NULL result");
    return qc_sets_write_async(r->sets.data(), (int64_t)r->sets.size(), path, out);
}

extern "C" qc_status qc_writer_wait(qc_writer* w)
{
    if (!w) return fail(QC_ERR_ARGS, "NULL writer");
    w->th.join();
    const std::string e = w->err;
    delete w;
    if (e.empty()) return QC_OK;
    return fail(e == "malformed result record" ? QC_ERR_FORMAT : QC_ERR_IO, e);
}

// qc_graph_from_csr (device 2-hop builder) lives in twohop.cu

std::string qcb_twohop_device(const HostGraph& h, std::vector<int64_t>& off2,
                              std::vector<int32_t>& adj2);

std::string qcb_twohop_noalloc(int32_t n, const int64_t* d_off, const int32_t* d_adj,
                               int64_t* d_off2, int32_t* d_adj2, int64_t adj2_cap,
                               int64_t* total_out, cudaStream_t s, int* too_large, int* too_small,
                               int* bad_csr);

extern "C" qc_status qc_twohop_noalloc(int32_t n, const int64_t* d_off, const int32_t* d_adj,
                                       int64_t* d_off2, int32_t* d_adj2, int64_t adj2_cap,
                                       int64_t* total_out, void* stream)
{
    if (n < 0 || !d_off2 || (n > 0 && !d_off)) return fail(QC_ERR_ARGS, "bad CSR arguments");
    if (d_adj2 && adj2_cap < 0) return fail(QC_ERR_ARGS, "negative adj2 capacity");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QC_ERR_NO_DEVICE, "no CUDA device visible");
    int too_large = 0, too_small = 0, bad_csr = 0;
    std::string e = qcb_twohop_noalloc(n, d_off, d_adj, d_off2, d_adj2, adj2_cap, total_out,
                                       (cudaStream_t)stream, &too_large, &too_small, &bad_csr);
    if (e.empty()) return QC_OK;
    if (too_large) return fail(QC_ERR_TOO_LARGE, e);
    if (bad_csr) return fail(QC_ERR_FORMAT, e);
    if (too_small) return fail(QC_ERR_RESULT_OVERFLOW, e);
    return fail(QC_ERR_CUDA, e);
}

extern "C" qc_status qc_graph_from_csr(int32_t n, const int64_t* off, const int32_t* adj,
                                       qc_graph** out)
{
    if (!out || n < 0 || (n > 0 && !off)) return fail(QC_ERR_ARGS, "bad CSR arguments");
    *out = nullptr;
    std::unique_ptr<qc_graph> g(new qc_graph());
    g->h.n = n;
    qc_status as = adopt_rows(n, off, adj, "1-hop", "adj", g->h.off, g->h.adj);
    if (as != QC_OK) return as;
    std::string e = validate(g->h, false);
    if (!e.empty()) return fail(QC_ERR_FORMAT, e);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(QC_ERR_NO_DEVICE, "no CUDA device visible");
    e = qcb_twohop_device(g->h, g->h.off2, g->h.adj2);
    if (!e.empty()) return fail(QC_ERR_CUDA, e);
    *out = g.release();
    return QC_OK;
}
