// emu_expand.cpp -- TEST INFRASTRUCTURE: runs the product's expansion kernel
// source (cuqc_b200/csrc/expand_kernel.cuh) on the CPU under cuda_emu.h, with
// the product's host-side level 0 (cuqc_b200/csrc/host.cpp), so the kernel's
// branch-and-bound logic can be compared with the oracle on machines without a
// GPU.  The root record is built here on the host; on the GPU a kernel builds it.
#include "cuda_emu.h"

#include "../../cuqc_b200/csrc/expand_kernel.cuh"
#include "../../cuqc_b200/csrc/host.h"
#include "../../cuqc_b200/csrc/level0_kernel.cuh"
#include "../../cuqc_b200/csrc/level0_grid.cuh"

#include <algorithm>
#include <cstdlib>
#include <vector>

using namespace qcb;

// optional stop time for the next emulated launches (0: none), to exercise the
// kernel's deadline drain
static long long g_emu_time_limit_ms = 0;
extern "C" void emu_set_time_limit_ms(long long ms) { g_emu_time_limit_ms = ms; }
static StackEntry one_entry(unsigned long long rec)
{
    StackEntry e{};
    e.rec[0] = rec;
    e.n = 1;
    e.q_lo = -1;
    e.q_hi = -1;
    return e;
}
static unsigned long long emu_time_limit_ns()
{
    return g_emu_time_limit_ms > 0 ? (unsigned long long)g_emu_time_limit_ms * 1000000ull : 0ull;
}

extern "C" int emu_mine(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
                        const int32_t* adj2, double gamma, int min_size, int warps, int split,
                        int small_path,
                        long long arena_bytes, int64_t* out_nints, int32_t** out_buf,
                        int64_t* counters, int stack_cap, long long result_cap,
                        int shared_fifo)
{
    HostGraph g;
    g.n = n;
    g.off.assign(off, off + n + 1);
    g.adj.assign(adj, adj + off[n]);
    g.off2.assign(off2, off2 + n + 1);
    g.adj2.assign(adj2, adj2 + off2[n]);
    std::vector<int32_t> md, ubt;
    gamma_tables(gamma, n, min_size, md, ubt);
    std::vector<int32_t> ids;
    int cov = 0;
    build_root(g, md.data(), min_size, ids, cov);
    *out_nints = 0;
    *out_buf = nullptr;
    for (int i = 0; i < 11; i++) counters[i] = 0;
    if (ids.empty()) return 0;
    int t = (int)ids.size();
    int W = words_for(t);

    std::vector<char> arena((size_t)arena_bytes, 0);
    TaskHdr* h = (TaskHdr*)arena.data();
    h->t = t;
    h->m = 0;
    h->cov = cov;
    h->W = W;
    h->refs = 1;
    h->cls = arena_class(rec_bytes(t, W));
    h->inst = 0;
    int32_t* rid = (int32_t*)(arena.data() + rec_ids_off());
    uint32_t* A1 = (uint32_t*)(arena.data() + rec_a1_off(t));
    uint32_t* A2 = (uint32_t*)(arena.data() + rec_a2_off(t, W));
    std::vector<int32_t> pos((size_t)n, -1);
    for (int i = 0; i < t; i++) {
        rid[i] = ids[(size_t)i];
        pos[(size_t)ids[(size_t)i]] = i;
    }
    for (int i = 0; i < t; i++) {
        int u = ids[(size_t)i];
        for (int64_t e = off[u]; e < off[u + 1]; e++) {
            int p = pos[(size_t)adj[e]];
            if (p >= 0) A1[(int64_t)i * W + (p >> 5)] |= 1u << (p & 31);
        }
        for (int64_t e = off2[u]; e < off2[u + 1]; e++) {
            int p = pos[(size_t)adj2[e]];
            if (p >= 0) A2[(int64_t)i * W + (p >> 5)] |= 1u << (p & 31);
        }
    }
    Control ctl{};
    ctl.arena_top = arena_class_bytes(h->cls);
    ctl.arena_cap = (unsigned long long)arena_bytes;
    ctl.result_cap = result_cap > 0 ? (unsigned long long)result_cap : (1ull << 24);
    ctl.set_cap = ctl.result_cap / 2 + 1;
    const int want_slots = std::max(stack_cap > 0 ? stack_cap : (1 << 20), 2 * kStackShards);
    int per_shard = 2; // a power of two, as the library sizes it
    while (per_shard * kStackShards < want_slots) per_shard <<= 1;
    const int total_slots = per_shard * kStackShards;
    ctl.stack_cap = per_shard;
    ctl.stack_top[0] = 1;
    ctl.pending = 1;
    std::vector<StackEntry> stack((size_t)total_slots);
    std::vector<int32_t> slot((size_t)total_slots, 0);
    stack[0] = one_entry(0);
    slot[0] = 1;
    std::vector<int32_t> results((size_t)ctl.result_cap);
    std::vector<unsigned long long> set_starts((size_t)ctl.set_cap);
    WsLayout L = ws_layout(t);
    std::vector<char> ws((size_t)(L.total * warps));

    Rules rule{};
    rule.off = off;
    rule.off2 = off2;
    rule.md = md.data();
    rule.ubt = ubt.data();
    rule.mdlen = (int32_t)md.size();
    rule.min_size = min_size;
    rule.vbase = 0;
    rule.n = n;
    ExpandParams P{};
    P.rules = &rule;
    P.nrules = 1;
    P.ctl = &ctl;
    P.arena = arena.data();
    P.stack = stack.data();
    P.slot = slot.data();
    P.results = results.data();
    P.set_starts = set_starts.data();
    P.ws = ws.data();
    P.ws_stride = L.total;
    P.arena_cap = ctl.arena_cap;
    P.max_t = t;
    P.split = split;
    P.small_path = small_path;
    P.shared_fifo = shared_fifo;
    P.wait_ns = 20000000000ll;
    P.time_limit_ns = emu_time_limit_ns();
    // stage tasks of up to 96 vertices in (emulated) shared memory, as the
    // library does with its per-SM budget, so both task paths run here
    P.smem_t = t > 32 ? std::min(t, 96) : 0;
    emu_launch(1, warps * 32, [&] { expand_kernel(P); }, expand_smem_bytes(warps, P.smem_t));

    counters[0] = (int64_t)ctl.tasks;
    counters[1] = (int64_t)ctl.branches;
    counters[2] = (int64_t)ctl.children;
    counters[3] = (int64_t)ctl.emitted;
    counters[4] = (int64_t)ctl.lookahead_hits;
    counters[5] = ctl.status;
    counters[6] = ctl.max_task;
    counters[7] = (int64_t)std::min(ctl.arena_top, ctl.arena_cap);
    counters[8] = (int64_t)ctl.parent_vertices;
    counters[9] = (int64_t)ctl.p_rows;
    counters[10] = (int64_t)ctl.child_vertices;
    int64_t k = std::min<int64_t>((int64_t)ctl.result_top, (int64_t)ctl.result_cap);
    if (ctl.status) k = 0;
    int32_t* out = (int32_t*)malloc(sizeof(int32_t) * (size_t)(k > 0 ? k : 1));
    for (int64_t i = 0; i < k; i++) out[i] = results[(size_t)i];
    *out_nints = k;
    *out_buf = out;
    return ctl.status;
}

extern "C" void emu_free(void* p) { free(p); }

// Several instances in one emulated launch: graph i is given by its slices of
// the concatenated arrays (offsets local to the instance).  Emitted ids are
// global (instance vertex base + id).
extern "C" int emu_mine_batch(int count, const int32_t* ns, const int64_t* off_all,
                              const int32_t* adj_all, const int64_t* off2_all,
                              const int32_t* adj2_all, const double* gammas,
                              const int32_t* min_sizes, int warps, int split,
                              int64_t* out_nints, int32_t** out_buf, int64_t* counters)
{
    std::vector<Rules> rules((size_t)count);
    std::vector<std::vector<int32_t>> mds((size_t)count), ubts((size_t)count);
    std::vector<int64_t> off_at((size_t)count), adj_at((size_t)count), adj2_at((size_t)count);
    std::vector<char> arena((size_t)1 << 27, 0);
    uint64_t arena_at = 0;
    std::vector<StackEntry> items;
    int64_t oa = 0, aa = 0, a2 = 0, vb = 0;
    int max_t = 1;
    for (int i = 0; i < count; i++) {
        int n = ns[i];
        const int64_t* off = off_all + oa;
        const int64_t* off2 = off2_all + oa;
        const int32_t* adj = adj_all + aa;
        const int32_t* adj2 = adj2_all + a2;
        HostGraph g;
        g.n = n;
        g.off.assign(off, off + n + 1);
        g.adj.assign(adj, adj + off[n]);
        g.off2.assign(off2, off2 + n + 1);
        g.adj2.assign(adj2, adj2 + off2[n]);
        gamma_tables(gammas[i], n, min_sizes[i], mds[(size_t)i], ubts[(size_t)i]);
        Rules ru{};
        ru.md = mds[(size_t)i].data();
        ru.ubt = ubts[(size_t)i].data();
        ru.off = off;
        ru.off2 = off2;
        ru.adj = adj;
        ru.adj2 = adj2;
        ru.mdlen = (int32_t)mds[(size_t)i].size();
        ru.min_size = min_sizes[i];
        ru.vbase = (int32_t)vb;
        ru.n = n;
        rules[(size_t)i] = ru;
        std::vector<int32_t> ids;
        int cov = 0;
        build_root(g, mds[(size_t)i].data(), min_sizes[i], ids, cov);
        if (!ids.empty()) {
            int t = (int)ids.size(), W = words_for(t);
            int cls = arena_class(rec_bytes(t, W));
            char* rec = arena.data() + arena_at;
            TaskHdr* h = (TaskHdr*)rec;
            h->t = t; h->m = 0; h->cov = cov; h->W = W; h->refs = 1; h->cls = cls; h->inst = i;
            int32_t* rid = (int32_t*)(rec + rec_ids_off());
            uint32_t* A1 = (uint32_t*)(rec + rec_a1_off(t));
            uint32_t* A2 = (uint32_t*)(rec + rec_a2_off(t, W));
            std::vector<int32_t> pos((size_t)n, -1);
            for (int k = 0; k < t; k++) { rid[k] = ids[(size_t)k]; pos[(size_t)ids[(size_t)k]] = k; }
            for (int k = 0; k < t; k++) {
                int u = ids[(size_t)k];
                for (int64_t e = off[u]; e < off[u + 1]; e++) {
                    int p = pos[(size_t)adj[e]];
                    if (p >= 0) A1[(int64_t)k * W + (p >> 5)] |= 1u << (p & 31);
                }
                for (int64_t e = off2[u]; e < off2[u + 1]; e++) {
                    int p = pos[(size_t)adj2[e]];
                    if (p >= 0) A2[(int64_t)k * W + (p >> 5)] |= 1u << (p & 31);
                }
            }
            items.push_back(one_entry(arena_at));
            arena_at += arena_class_bytes(cls);
            max_t = std::max(max_t, t);
        }
        oa += n + 1;
        aa += off[n];
        a2 += off2[n];
        vb += n;
    }
    Control ctl{};
    ctl.arena_top = arena_at;
    ctl.arena_cap = arena.size();
    ctl.result_cap = 1ull << 24;
    ctl.set_cap = 1ull << 22;
    ctl.stack_cap = (1 << 20) / kStackShards;
    ctl.pending = (int)items.size();
    std::vector<StackEntry> stack((size_t)ctl.stack_cap * kStackShards);
    std::vector<int32_t> slot(stack.size(), 0);
    // item j is entry j / S of shard j % S, as the library seeds a batch
    for (size_t j = 0; j < items.size(); j++) {
        size_t at = (j % kStackShards) * (size_t)ctl.stack_cap + j / kStackShards;
        stack[at] = items[j];
        slot[at] = 1;
        ctl.stack_top[j % kStackShards]++;
    }
    std::vector<int32_t> results((size_t)ctl.result_cap);
    std::vector<unsigned long long> set_starts((size_t)ctl.set_cap);
    WsLayout L = ws_layout(max_t);
    std::vector<char> ws((size_t)(L.total * warps));
    ExpandParams P{};
    P.shared_fifo = 1; // oldest donated task first, as batched launches run
    P.rules = rules.data();
    P.nrules = count;
    P.ctl = &ctl;
    P.arena = arena.data();
    P.stack = stack.data();
    P.slot = slot.data();
    P.results = results.data();
    P.set_starts = set_starts.data();
    P.ws = ws.data();
    P.ws_stride = L.total;
    P.arena_cap = ctl.arena_cap;
    P.max_t = max_t;
    P.split = split;
    P.small_path = 1;
    P.wait_ns = 20000000000ll;
    P.time_limit_ns = emu_time_limit_ns();
    P.smem_t = max_t > 32 ? std::min(max_t, 96) : 0;
    if (!items.empty())
        emu_launch(1, warps * 32, [&] { expand_kernel(P); }, expand_smem_bytes(warps, P.smem_t));
    counters[0] = (int64_t)ctl.tasks;
    counters[1] = (int64_t)ctl.branches;
    counters[2] = ctl.status;
    int64_t k = ctl.status ? 0 : (int64_t)ctl.result_top;
    int32_t* out = (int32_t*)malloc(sizeof(int32_t) * (size_t)(k > 0 ? k : 1));
    for (int64_t i = 0; i < k; i++) out[i] = results[(size_t)i];
    *out_nints = k;
    *out_buf = out;
    return ctl.status;
}

// The product's device level 0 (level0_kernel.cuh) as one emulated block of
// `threads` threads; ids_out receives the root in Q order, info = {size,
// covered count}.
extern "C" int emu_level0(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
                          double gamma, int min_size, int threads, int32_t* ids_out,
                          int32_t* info)
{
    std::vector<int32_t> md, ubt;
    gamma_tables(gamma, n, min_size, md, ubt);
    int P = 1;
    while (P < n) P <<= 1;
    std::vector<int32_t> exdeg((size_t)n), label((size_t)n), l2((size_t)n);
    std::vector<unsigned long long> keys((size_t)P);
    emu_launch(1, threads, [&] {
        level0_kernel(off, adj, off2, n, md[(size_t)min_size], min_size, exdeg.data(),
                      label.data(), l2.data(), keys.data(), ids_out, info);
    });
    return 0;
}

// The product's grid-wide level 0 (level0_grid.cuh) as a grid of one emulated
// block of `threads` threads (its grid barriers become block barriers).
extern "C" int emu_level0_grid(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
                               double gamma, int min_size, int threads, int32_t* ids_out,
                               int32_t* info)
{
    std::vector<int32_t> md, ubt;
    gamma_tables(gamma, n, min_size, md, ubt);
    std::vector<char> scratch((size_t)level0_grid_scratch_bytes(n), 0);
    emu_launch(1, threads, [&] {
        level0_grid_kernel(off, adj, off2, (int64_t)n, md[(size_t)min_size], min_size,
                           scratch.data(), ids_out, info);
    });
    return 0;
}
