// ref_cpu_driver.cu -- TEST INFRASTRUCTURE: runs the reference cuQC's own
// serial CPU enumeration (its host routines initialize_tasks, h_expand_level,
// flush_cliques, RemoveNonMax) without touching a GPU.
//
// The reference source is compiled from where it lies (the include path is
// given by oracle/Makefile); nothing of it is copied here.  The reference's
// `main` is renamed so this file can provide an extern "C" entry point.  Only
// the host-side allocation of the reference's allocate_memory (main.cu:695-843)
// is restated, with capacities chosen by the caller, because the reference's
// version also allocates ~35 GB of device memory.
//
// The loop mirrors the reference's host loop (main.cu:576-590) but keeps
// calling h_expand_level until the enumeration is complete, i.e. the
// reference's own CPU path with CPU_LEVELS raised to infinity.  Cliques are
// flushed to the temp file after every level (main.cu:580-582 flushes only
// above a threshold; flushing more often changes nothing but memory use).
#define main cuqc_reference_main
#include "main.cu"
#undef main

// Host-side buffers of the reference's CPU_Data / CPU_Cliques, with the
// capacities chosen by the caller (allocate_memory, main.cu:695-843, host part).
static void ref_alloc(CPU_Graph& hg, CPU_Data& hd, CPU_Cliques& hc, long long task_vertex_cap,
                      long long buffer_vertex_cap, long long buffer_task_cap, long long clique_cap)
{
    hd.tasks1_count = new uint64_t;
    hd.tasks1_offset = new uint64_t[EXPAND_THRESHOLD + 1];
    hd.tasks1_vertices = new Vertex[task_vertex_cap];
    hd.tasks1_offset[0] = 0;
    *hd.tasks1_count = 0;
    hd.tasks2_count = new uint64_t;
    hd.tasks2_offset = new uint64_t[EXPAND_THRESHOLD + 1];
    hd.tasks2_vertices = new Vertex[task_vertex_cap];
    hd.tasks2_offset[0] = 0;
    *hd.tasks2_count = 0;
    hd.buffer_count = new uint64_t;
    hd.buffer_offset = new uint64_t[buffer_task_cap];
    hd.buffer_vertices = new Vertex[buffer_vertex_cap];
    hd.buffer_offset[0] = 0;
    *hd.buffer_count = 0;
    hd.current_level = new uint64_t;
    hd.maximal_expansion = new bool;
    hd.dumping_cliques = new bool;
    *hd.current_level = 0;
    *hd.maximal_expansion = false;
    *hd.dumping_cliques = false;
    int nn = hg.number_of_vertices + 1;
    hd.vertex_order_map = new int[nn];
    hd.remaining_candidates = new int[2 * nn];
    hd.removed_candidates = new int[2 * nn];
    hd.remaining_count = new int;
    hd.removed_count = new int;
    hd.candidate_indegs = new int[2 * nn];
    memset(hd.vertex_order_map, -1, sizeof(int) * nn);
    hc.cliques_count = new uint64_t;
    hc.cliques_vertex = new int[clique_cap];
    hc.cliques_offset = new uint64_t[clique_cap];
    hc.cliques_offset[0] = 0;
    *hc.cliques_count = 0;
}

static void ref_release(CPU_Data& hd, CPU_Cliques& hc)
{
    delete hd.tasks1_count; delete[] hd.tasks1_offset; delete[] hd.tasks1_vertices;
    delete hd.tasks2_count; delete[] hd.tasks2_offset; delete[] hd.tasks2_vertices;
    delete hd.buffer_count; delete[] hd.buffer_offset; delete[] hd.buffer_vertices;
    delete hd.current_level; delete hd.maximal_expansion; delete hd.dumping_cliques;
    delete[] hd.vertex_order_map; delete[] hd.remaining_candidates;
    delete[] hd.removed_candidates; delete hd.remaining_count; delete hd.removed_count;
    delete[] hd.candidate_indegs;
    delete hc.cliques_count; delete[] hc.cliques_vertex; delete[] hc.cliques_offset;
    delete[] minimum_degrees;
}

extern "C" int refcpu_run(const char* graph_path, const char* gamma_str, int min_size,
                          const char* temp_path, const char* out_path,
                          long long task_vertex_cap, long long buffer_vertex_cap,
                          long long buffer_task_cap, long long clique_cap,
                          long long* levels_out, double* times_ms)
{
    auto t0 = std::chrono::steady_clock::now();
    ifstream gs(graph_path, ios::in);
    if (!gs.is_open()) return -1;
    CPU_Graph hg(gs);
    gs.close();
    minimum_degree_ratio = atof(gamma_str);
    minimum_clique_size = min_size;
    calculate_minimum_degrees(hg);

    CPU_Data hd;
    CPU_Cliques hc;
    ref_alloc(hg, hd, hc, task_vertex_cap, buffer_vertex_cap, buffer_task_cap, clique_cap);

    ofstream temp(temp_path);
    auto t1 = std::chrono::steady_clock::now();
    initialize_tasks(hg, hd);
    long long levels = 0;
    while (!*hd.maximal_expansion) {
        h_expand_level(hg, hd, hc);
        flush_cliques(hc, temp);
        levels++;
    }
    flush_cliques(hc, temp);
    temp.close();
    auto t2 = std::chrono::steady_clock::now();
    if (levels_out) *levels_out = levels;

    // RemoveNonMax dereferences an empty prefix tree (main.cu:4834); only
    // call it when the temp file holds at least one set.
    int rc = 0;
    {
        ifstream chk(temp_path);
        int first;
        if (chk >> first) {
            RemoveNonMax((char*)temp_path, (char*)out_path);
        } else {
            ofstream empty(out_path);
            rc = 1;
        }
    }
    auto t3 = std::chrono::steady_clock::now();
    if (times_ms) {
        times_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        times_ms[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
        times_ms[2] = std::chrono::duration<double, std::milli>(t3 - t2).count();
    }
    ref_release(hd, hc);
    return rc;
}

// The same enumeration under a wall-clock budget: levels run until the
// enumeration completes or `budget_ms` has passed (checked between levels).
// Counts the tasks the levels expanded (the size of each level's task array
// as h_expand_level reads it, main.cu:1034-1057) and the sets emitted; the
// sets themselves go to temp_path.  out[0] = tasks, out[1] = emitted sets,
// out[2] = levels, out[3] = 1 if the enumeration finished; *elapsed_ms is
// the time from initialize_tasks to the last level's end.
extern "C" int refcpu_budget(const char* graph_path, const char* gamma_str, int min_size,
                             const char* temp_path, double budget_ms,
                             long long task_vertex_cap, long long buffer_vertex_cap,
                             long long buffer_task_cap, long long clique_cap,
                             long long* out, double* elapsed_ms)
{
    ifstream gs(graph_path, ios::in);
    if (!gs.is_open()) return -1;
    CPU_Graph hg(gs);
    gs.close();
    minimum_degree_ratio = atof(gamma_str);
    minimum_clique_size = min_size;
    calculate_minimum_degrees(hg);

    CPU_Data hd;
    CPU_Cliques hc;
    ref_alloc(hg, hd, hc, task_vertex_cap, buffer_vertex_cap, buffer_task_cap, clique_cap);
    ofstream temp(temp_path);
    long long tasks = 0, emitted = 0, levels = 0;
    auto t1 = std::chrono::steady_clock::now();
    initialize_tasks(hg, hd);
    double el = 0;
    while (!*hd.maximal_expansion) {
        tasks += (long long)((*hd.current_level) % 2 == 0 ? *hd.tasks1_count : *hd.tasks2_count);
        h_expand_level(hg, hd, hc);
        emitted += (long long)*hc.cliques_count;
        flush_cliques(hc, temp);
        levels++;
        el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
        if (el >= budget_ms) break;
    }
    temp.close();
    out[0] = tasks;
    out[1] = emitted;
    out[2] = levels;
    out[3] = *hd.maximal_expansion ? 1 : 0;
    *elapsed_ms = el;
    ref_release(hd, hc);
    return 0;
}
