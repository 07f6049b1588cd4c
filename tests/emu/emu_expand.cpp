// emu_expand.cpp -- TEST INFRASTRUCTURE: runs the product's expansion kernel
// source (cuqc_b200/csrc/expand_kernel.cuh) on the CPU under cuda_emu.h, with
// the product's host-side level 0 (cuqc_b200/csrc/host.cpp), so the kernel's
// branch-and-bound logic can be compared with the oracle on machines without a
// GPU.  The root record is built here on the host; on the GPU a kernel builds it.
#include "cuda_emu.h"

#include "../../cuqc_b200/csrc/expand_kernel.cuh"
#include "../../cuqc_b200/csrc/host.h"

#include <algorithm>
#include <cstdlib>
#include <vector>

using namespace qcb;

extern "C" int emu_mine(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
                        const int32_t* adj2, double gamma, int min_size, int warps, int split,
                        int small_path,
                        long long arena_bytes, int64_t* out_nints, int32_t** out_buf,
                        int64_t* counters, int stack_cap, long long result_cap)
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
    for (int i = 0; i < 8; i++) counters[i] = 0;
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
    ctl.arena_live = ctl.arena_top;
    ctl.arena_cap = (unsigned long long)arena_bytes;
    ctl.result_cap = result_cap > 0 ? (unsigned long long)result_cap : (1ull << 24);
    ctl.set_cap = ctl.result_cap / 2 + 1;
    ctl.stack_cap = stack_cap > 0 ? stack_cap : (1 << 20);
    ctl.stack_top = 1;
    ctl.pending = 1;
    std::vector<WorkItem> stack((size_t)ctl.stack_cap);
    std::vector<int32_t> slot((size_t)ctl.stack_cap, 0);
    stack[0] = WorkItem{0, -1, -1};
    slot[0] = 1;
    std::vector<int32_t> results((size_t)ctl.result_cap);
    std::vector<unsigned long long> set_starts((size_t)ctl.set_cap);
    WsLayout L = ws_layout(t);
    std::vector<char> ws((size_t)(L.total * warps));

    ExpandParams P{};
    P.off = off;
    P.off2 = off2;
    P.md = md.data();
    P.ubt = ubt.data();
    P.mdlen = (int32_t)md.size();
    P.min_size = min_size;
    P.ctl = &ctl;
    P.arena = arena.data();
    P.stack = stack.data();
    P.slot = slot.data();
    P.results = results.data();
    P.set_starts = set_starts.data();
    P.ws = ws.data();
    P.ws_stride = L.total;
    P.max_t = t;
    P.split = split;
    P.small_path = small_path;
    P.wait_ns = 20000000000ll;
    emu_launch(1, warps * 32, [&] { expand_kernel(P); });

    counters[0] = (int64_t)ctl.tasks;
    counters[1] = (int64_t)ctl.branches;
    counters[2] = (int64_t)ctl.children;
    counters[3] = (int64_t)ctl.emitted;
    counters[4] = (int64_t)ctl.lookahead_hits;
    counters[5] = ctl.status;
    counters[6] = ctl.max_task;
    counters[7] = (int64_t)ctl.arena_live_peak;
    int64_t k = std::min<int64_t>((int64_t)ctl.result_top, (int64_t)ctl.result_cap);
    if (ctl.status) k = 0;
    int32_t* out = (int32_t*)malloc(sizeof(int32_t) * (size_t)(k > 0 ? k : 1));
    for (int64_t i = 0; i < k; i++) out[i] = results[(size_t)i];
    *out_nints = k;
    *out_buf = out;
    return ctl.status;
}

extern "C" void emu_free(void* p) { free(p); }
