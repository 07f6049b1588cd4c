// cli.cpp -- `cuQC`, the drop-in command line of the B200 miner.
//
//   cuQC <graph_file> <gamma> <min_size> <output_file> <sched 0-dynamic/1-static>
//
// Same arguments, checks, messages and stdout lines as the reference
// (Mike12041204/cuQC main.cu:416-519): an invalid scheduling toggle is
// reported and the run continues; a CUDA or capacity error prints the
// library's message and exits with -1 as the reference's chkerr does
// (main.cu:2200-2207).  Differences: no temp.txt is written (the emitted sets
// stay on the device), and a run with no quasi-clique writes an empty result
// file instead of crashing (main.cu:4834).  One line is added after the
// ENUMERATION TIME line: the expansion kernel's own time, EXPANSION KERNEL TIME.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "../../include/qc.h"

using clk = std::chrono::steady_clock;

static long long ms_between(clk::time_point a, clk::time_point b)
{
    return (long long)std::chrono::duration_cast<std::chrono::milliseconds>(b - a).count();
}

int main(int argc, char* argv[])
{
    auto t_total = clk::now();
    if (argc != 6) {
        printf("Usage: ./main <graph_file> <gamma> <min_size> <output_file.txt> <scheduling toggle "
               "0-dyanmic/1-static>\n");
        return 1;
    }
    FILE* probe = fopen(argv[1], "r");
    if (!probe) {
        printf("invalid graph file\n");
        return 1;
    }
    fclose(probe);
    double gamma = atof(argv[2]);
    if (gamma < .5 || gamma > 1) {
        printf("minimum degree ratio must be between .5 and 1 inclusive\n");
        return 1;
    }
    int min_size = atoi(argv[3]);
    if (min_size <= 1) {
        printf("minimum size must be greater than 1\n");
        return 1;
    }
    int sched = atoi(argv[5]);
    if (!(sched == 0 || sched == 1)) std::cout << "scheduling toggle must be 0 or 1" << std::endl;

    auto t_load = clk::now();
    std::cout << ">:PRE-PROCESSING" << std::endl;
    qc_graph* g = nullptr;
    qc_status st = qc_graph_read(argv[1], &g); // serialized text, or binary CSR
    if (st != QC_OK) {
        std::cout << qc_status_str(st) << ": " << qc_last_error() << std::endl;
        return st == QC_ERR_IO ? 1 : -1;
    }
    std::cout << "--->:LOADING TIME: " << ms_between(t_load, clk::now()) << " ms" << std::endl;

    qc_context* ctx = nullptr;
    qc_config cfg;
    qc_config_default(&cfg);
    st = qc_context_create(&cfg, &ctx);
    if (st != QC_OK) {
        std::cout << qc_status_str(st) << ": " << qc_last_error() << std::endl;
        exit(-1);
    }
    // the graph goes to the device before the enumeration clock starts, as the
    // reference copies its CSR in allocate_memory ahead of its timer
    // (main.cu:545-551, 700-711)
    st = qc_context_upload(ctx, g);
    if (st != QC_OK) {
        std::cout << qc_status_str(st) << ": " << qc_last_error() << std::endl;
        exit(-1);
    }
    std::cout << ">:INITIALIZING TASKS" << std::endl;
    std::cout << ">:BEGINNING EXPANSION" << std::endl;
    qc_result* r = nullptr;
    st = qc_mine(ctx, g, gamma, min_size, sched, &r);
    if (st != QC_OK) {
        std::cout << qc_status_str(st) << ": " << qc_last_error() << std::endl;
        exit(-1);
    }
    const qc_stats* s = qc_result_stats(r);
    // the reference's span: level 0 through the last expansion level
    // (main.cu:551-685), without the graph copy; then the expansion kernel
    // alone (CUDA events), a line the reference does not print
    std::cout << "--->:ENUMERATION TIME: " << (long long)s->enum_ms << " ms" << std::endl;
    std::cout << "--->:EXPANSION KERNEL TIME: " << s->kernel_ms << " ms" << std::endl;
    auto t_rm = clk::now();
    std::cout << ">:REMOVING NON-MAXIMAL CLIQUES" << std::endl;
    st = qc_result_write(r, argv[4]);
    if (st != QC_OK) {
        printf("Error: cannot open file %s for write\n", argv[4]);
    }
    printf(">:NUMBER OF MAXIMAL CLIQUES: %lld\n", (long long)qc_result_count(r));
    fflush(stdout);
    std::cout << "--->:REMOVE NON-MAX TIME: " << (long long)s->filter_ms + ms_between(t_rm, clk::now())
              << " ms" << std::endl;
    std::cout << "--->:TOTAL TIME: " << ms_between(t_total, clk::now()) << " ms" << std::endl;
    std::cout << ">:PROGRAM END" << std::endl;
    qc_result_free(r);
    qc_context_free(ctx);
    qc_graph_free(g);
    return 0;
}
