/*
 * qc.h -- C ABI of the B200 maximal gamma-quasi-clique miner (libqc.so).
 *
 * Plain C: pointers, sizes and status codes; no exits inside the library.
 * Ownership: every object the library creates is released with the
 * matching qc_*_free.  Threading: one host thread per qc_context at a time;
 * distinct contexts may be used concurrently (each owns its CUDA stream and
 * device buffers).
 *
 * The reference cuQC (Mike12041204/cuQC) has no library interface; its only
 * "plugin API" is the process CLI (main.cu:416-519) over a serialized graph
 * file (main.cu:82-131) and a result file (main.cu:4641-4652, 4881-4937).
 * Each entry point below names the reference routine whose job it takes
 * over, so a maintainer can see which part of main.cu a call replaces.
 */
#ifndef QC_H
#define QC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    QC_OK = 0,
    QC_ERR_ARGS = 1,            /* argument out of range (gamma, min_size, NULL) */
    QC_ERR_IO = 2,              /* a file could not be opened, read or written   */
    QC_ERR_FORMAT = 3,          /* malformed serialized graph                    */
    QC_ERR_CUDA = 4,            /* CUDA runtime error (message: qc_last_error)   */
    QC_ERR_NOMEM = 5,           /* host or device allocation failed              */
    QC_ERR_TASK_OVERFLOW = 6,   /* device task stack or record arena exhausted   */
    QC_ERR_RESULT_OVERFLOW = 7, /* device result buffer exhausted                */
    QC_ERR_ITER_LIMIT = 8,      /* a bounded device wait gave up                 */
    QC_ERR_TOO_LARGE = 9,       /* a task exceeds the supported vertex count     */
    QC_ERR_NO_DEVICE = 10       /* no CUDA device / library built without it     */
} qc_status;

/* Human-readable text for a status code. */
const char* qc_status_str(qc_status s);
/* Detail of the last failure on the calling thread (never NULL). */
const char* qc_last_error(void);

/* ------------------------------------------------------------------ */
/* graphs                                                               */
/* ------------------------------------------------------------------ */

typedef struct qc_graph qc_graph; /* host CSR (+ 2-hop CSR) of an undirected graph */

/* Parse the reference's serialized graph file: n, 2|E|, #2-hop entries,
 * 1-hop neighbours, 1-hop offsets, 2-hop neighbours, 2-hop offsets,
 * whitespace separated.  Replaces CPU_Graph(ifstream&) (main.cu:96-121). */
qc_status qc_graph_read_serialized(const char* path, qc_graph** out);

/* Adopt a CSR (offsets int64[n+1], sorted neighbour rows int32[off[n]]) and
 * the matching 2-hop CSR.  The arrays are copied.  Replaces the loader's
 * arrays of CPU_Graph (main.cu:89-94). */
qc_status qc_graph_from_csr2(int32_t n, const int64_t* off, const int32_t* adj,
                             const int64_t* off2, const int32_t* adj2, qc_graph** out);

/* Adopt a 1-hop CSR and build the 2-hop lists
 * sorted(N(v) u N(N(v)) minus {v}) on the GPU.  Replaces the offline
 * adjToSer preprocessing (adjToSer.cpp:115-156). */
qc_status qc_graph_from_csr(int32_t n, const int64_t* off, const int32_t* adj, qc_graph** out);

/* Two-hop lists of a graph already in device memory, computed without any
 * device allocation.  No counterpart in the reference (cuQC builds its
 * two-hop lists offline, adjToSer.cpp:115-156, and allocates freely).
 *
 * For callers that cannot call cudaMalloc: applications whose device memory
 * is owned by their own pool or a fixed memory plan, or that must not
 * allocate while serving requests.  The caller passes device buffers:
 * d_off (int64[n+1]) and d_adj (int32[d_off[n]]) hold a 1-hop CSR (the
 * miner wants sorted symmetric rows; these lists follow the rows as given,
 * repeats and one-way rows included, and a self loop keeps v, as adjToSer
 * does); d_off2 (int64[n+1]) receives the two-hop offsets and d_adj2
 * (int32[adj2_cap]) the rows sorted(N(v) u N(N(v)) minus {v}).  With
 * d_adj2 == NULL only d_off2 and *total_out are filled (a size query); if
 * the rows need more than adj2_cap entries the call returns
 * QC_ERR_RESULT_OVERFLOW with *total_out set to the size needed.
 *
 * The CSR is checked on the device before it is used as an index: offsets
 * starting at 0 and non-decreasing, every neighbour id in [0, n), and d_adj
 * not NULL when d_off[n] > 0; a failed check returns QC_ERR_FORMAT and
 * writes no rows.  Only d_off[0..n] and d_adj[0..d_off[n]) are read.
 *
 * Working memory is one 16 MiB array in device memory that every GPU which
 * loads the library holds until the process exits; graphs above
 * qc_twohop_noalloc_max_vertices() vertices are rejected with
 * QC_ERR_TOO_LARGE.  The first call on a device looks up that array's device
 * address (and keeps it for the life of the device's primary context), so
 * make it before any stream capture.  All calls share the array: calls whose
 * work overlaps on the GPU (other threads, other streams) race and must be
 * serialised by the caller.  The call runs on `stream` (a cudaStream_t;
 * NULL = the default stream) and is synchronous: it waits on that stream
 * and returns when the lists are written. */
qc_status qc_twohop_noalloc(int32_t n, const int64_t* d_off, const int32_t* d_adj,
                            int64_t* d_off2, int32_t* d_adj2, int64_t adj2_cap,
                            int64_t* total_out, void* stream);
/* Largest vertex count qc_twohop_noalloc accepts. */
int32_t qc_twohop_noalloc_max_vertices(void);

/* Binary CSR graph file, for graphs whose text form is slow to parse (the
 * reference reads only the text format, main.cu:96-121):
 *   8 bytes "QCSRBIN1"; little-endian int64 n, nnz (= 2|E|), nnz2 (two-hop
 *   entries, -1 when the file has no two-hop lists); int64 off[n+1];
 *   int32 adj[nnz]; zero padding to a multiple of 8 bytes; and when nnz2 >= 0,
 *   int64 off2[n+1] and int32 adj2[nnz2].
 * The file is checked like a serialized one (sizes against the header, sorted
 * symmetric rows, ids in range).  Without two-hop lists they are built on the
 * GPU as qc_graph_from_csr does. */
qc_status qc_graph_read_binary(const char* path, qc_graph** out);
/* Write the graph (with its two-hop lists) in the binary CSR format. */
qc_status qc_graph_write_binary(const qc_graph* g, const char* path);
/* Read a graph file of either format: binary CSR when the file starts with
 * "QCSRBIN1", else the serialized text format. */
qc_status qc_graph_read(const char* path, qc_graph** out);

/* Write the graph in the serialized format (adjToSer.cpp:159-204). */
qc_status qc_graph_write_serialized(const qc_graph* g, const char* path);

int32_t qc_graph_num_vertices(const qc_graph* g);
int64_t qc_graph_num_entries(const qc_graph* g);   /* 2|E|            */
int64_t qc_graph_num_twohop(const qc_graph* g);    /* 2-hop entries  */
/* Read-only views of the host arrays (valid until qc_graph_free). */
const int64_t* qc_graph_offsets(const qc_graph* g);
const int32_t* qc_graph_neighbors(const qc_graph* g);
const int64_t* qc_graph_twohop_offsets(const qc_graph* g);
const int32_t* qc_graph_twohop_neighbors(const qc_graph* g);
void qc_graph_free(qc_graph* g);

/* ------------------------------------------------------------------ */
/* contexts                                                             */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t device;              /* CUDA device ordinal                               */
    int32_t warps_per_block;     /* 0: 8 (qc_tune picks the fastest for a workload)  */
    int32_t blocks_per_sm;       /* 0: 1 (qc_tune picks the fastest for a workload)  */
    int64_t arena_bytes;         /* task-record arena; 0: default                     */
    int64_t stack_slots;         /* task stack capacity; 0: default                   */
    int64_t result_ints;         /* emitted-set buffer (ints); 0: default             */
    int32_t keep_emitted;        /* 1: keep the raw emitted multiset in the result    */
    int32_t wait_limit_ms;       /* bound on any device wait without progress; 0: 10000 */
    int32_t time_limit_ms;       /* stop a run after this long (QC_ERR_ITER_LIMIT); 0: none */
    int32_t split;               /* branches per work item of a task over 32 vertices;
                                    0: for qc_mine 1 up to 256 vertices and 2 above,
                                    for qc_mine_batch 2 */
    int32_t max_blocks;          /* cap on the persistent grid (share the GPU between
                                    contexts running at once); 0: every resident block */
    int32_t stage_max;           /* largest task (vertices) worked on in shared memory;
                                    0: the largest of 256, 192, 160, 128, 96, 64 whose
                                    buffers fit 195 KB a block (L1 keeps 60 KB), -1: none */
    int32_t shared_order;        /* which donated task an idle warp takes: 1 the newest
                                    (depth first), 2 the oldest (the largest subtrees
                                    first); 0: newest for qc_mine, oldest for
                                    qc_mine_batch, whose many instances keep every
                                    warp busy */
} qc_config;

/* Fill a config with defaults (device 0, everything autotuned). */
void qc_config_default(qc_config* cfg);

typedef struct qc_context qc_context;

/* Create a context: CUDA stream + device buffers sized by cfg.
 * Replaces allocate_memory (main.cu:695-843). */
qc_status qc_context_create(const qc_config* cfg, qc_context** out);
void qc_context_free(qc_context* ctx);

/* Copy a graph to the context's device now; later qc_mine calls on the same
 * graph skip the copy.  The reference copies its CSR inside allocate_memory
 * (main.cu:700-711). */
qc_status qc_context_upload(qc_context* ctx, const qc_graph* g);

/* The context's CUDA stream (a cudaStream_t), for callers that time or
 * order their own work against the library's launches. */
void* qc_context_stream(qc_context* ctx);

/* ------------------------------------------------------------------ */
/* mining                                                               */
/* ------------------------------------------------------------------ */

typedef struct {
    double load_ms;        /* host->device copy of the graph                  */
    double enum_ms;        /* level 0 + expansion on the device (CUDA events)  */
    double filter_ms;      /* non-maximal removal on the device               */
    double total_ms;       /* whole call, host wall clock                      */
    int64_t tasks;         /* tasks expanded                                   */
    int64_t branches;      /* add-one-vertex branches                          */
    int64_t children;      /* child tasks written                              */
    int64_t emitted;       /* quasi-cliques emitted before the maximal filter  */
    int64_t emitted_ints;  /* ints of emitted sets (sizes + ids)               */
    int64_t maximal;       /* sets in the result                               */
    int64_t root_size;     /* vertices in the root task                        */
    int64_t max_task;      /* largest task                                     */
    int64_t arena_peak;    /* high-water mark of the task-record arena (bytes) */
    int64_t kernel_launches;
    double kernel_ms;      /* expansion kernel alone (CUDA events)            */
    /* work counters for the algorithmic-byte model (per expanded branch:
     * the parent's vertex records, the added vertex's 1-hop and 2-hop rows,
     * the child's records, the emitted sets) */
    int64_t parent_vertices; /* sum over branches of the parent task size    */
    int64_t p_rows;          /* sum over branches of deg(p) + |N2(p)|        */
    int64_t child_vertices;  /* sum of child task sizes written              */
    int64_t level0_on_device; /* 1: level 0 ran on the device, 0: on the host  */
} qc_stats;

typedef struct qc_result qc_result;

/* Level 0 alone: the root task of the search for (g, gamma, min_size) --
 * the vertices that pass the degree and two-hop tests and the peeling, in the
 * order the search branches them, and how many of them the cover vertex
 * covers.  Replaces initialize_tasks (main.cu:846-998).  ids_out receives the
 * first min(cap, root size) ids; *t_out the root size, *cov_out the covered
 * count.  Runs on the device up to 2^30 vertices. */
qc_status qc_root(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                  int32_t* ids_out, int64_t cap, int32_t* t_out, int32_t* cov_out);

/* One shard of a search split by the root's branches, so that several GPUs
 * (one context each) can mine one graph.  The root's branches are dealt to
 * `nshards` shards round-robin in branching order (the i-th branch taken, i
 * from 0, belongs to shard i mod nshards); this call expands the branches of
 * shard `shard` and everything below them, and returns the maximal sets among
 * the sets they emitted.  The maximal sets of the whole graph are the maximal
 * sets of the union of every shard's result: qc_maximal_sets merges them.  A
 * root that the lookahead accepts whole is emitted by shard 0 only; every
 * shard counts the root in its task counter.  No counterpart in the reference,
 * which mines on one GPU (search, main.cu:535-692). */
qc_status qc_mine_shard(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                        int32_t shard, int32_t nshards, qc_result** out);

/* Work counters of the context's most recent expansion kernel (tasks,
 * branches, emitted sets, kernel_ms, the byte-model counters), also when
 * that run stopped early: after qc_mine returns QC_ERR_ITER_LIMIT because
 * cfg.time_limit_ms ran out, these are the counts of the work done until
 * then (a budgeted measurement of a search too large to finish).  The
 * reference prints its progress only through its DEBUG_TOGGLE size tracker
 * (main.cu:626-660); this takes the place of that read-out. */
qc_status qc_context_last_stats(const qc_context* ctx, qc_stats* out);

/* Enumerate the maximal gamma-quasi-cliques of size >= min_size.
 * gamma in [0.5, 1], min_size > 1 (main.cu:437-446).  sched is accepted for
 * CLI compatibility (0 dynamic / 1 static, main.cu:447-453); the device work
 * queue is always dynamic.  Replaces search() + RemoveNonMax()
 * (main.cu:535-692, 4939-4960). */
qc_status qc_mine(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                  int32_t sched, qc_result** out);

/* Pick the launch settings for this device and workload: mines (g, gamma,
 * min_size) with every candidate launch shape (warps per block, blocks per
 * SM, branches per work item of a task over 32 vertices), then, from the
 * fastest, tries the largest task staged in shared memory (larger task
 * records are read through L2: the spill threshold) and the order in which
 * idle warps take donated tasks; `repeats` timed runs each after one
 * warm-up, the fastest expansion kernel kept in the context's configuration
 * and, if `best` is not NULL, copied there.  Every run must give the same
 * result.  Replaces the reference's compile-time constants (BLOCK_SIZE,
 * NUM_OF_BLOCKS, TASKS_PER_WARP, EXPAND_THRESHOLD, main.cu:21-55). */
qc_status qc_tune(qc_context* ctx, const qc_graph* g, double gamma, int32_t min_size,
                  int32_t repeats, qc_config* best);

/* qc_tune on a sample of a batched workload: the same search, each candidate
 * timed by one qc_mine_batch of the `count` instances (the batched launch's
 * best shape differs from a single instance's: its many instances keep every
 * warp busy, so throughput settings win over latency ones). */
qc_status qc_tune_batch(qc_context* ctx, const qc_graph* const* graphs, const double* gammas,
                        const int32_t* min_sizes, int32_t count, int32_t repeats,
                        qc_config* best);

/* Mine `count` independent instances in one persistent launch (each with
 * its own graph, gamma and min_size).  outs[i] receives instance i's result. */
qc_status qc_mine_batch(qc_context* ctx, const qc_graph* const* graphs, const double* gammas,
                        const int32_t* min_sizes, int32_t count, qc_result** outs);

/* The maximal sets of a family of vertex sets, on the device: the
 * non-maximal removal step alone (RemoveNonMax, main.cu:4571-4960), e.g. to
 * merge the results of instances mined separately over parts of one graph.
 * `flat` holds n_sets sets as [k, id_1 .. id_k] (k >= 1, ids in
 * [0, n_vertices), any order; a set may repeat, a repeated id within a set
 * is an error).  The result lists each maximal set once, in the order of
 * qc_result_sets. */
qc_status qc_maximal_sets(qc_context* ctx, const int32_t* flat, int64_t n_ints,
                          int32_t n_vertices, qc_result** out);

/* Result access.  Sets are sorted ascending and listed in lexicographic
 * order of their id sequences, as the reference's result file. */
int64_t qc_result_count(const qc_result* r);
/* Flat [k, id_1 .. id_k] per set; *n_ints receives the length. */
const int32_t* qc_result_sets(const qc_result* r, int64_t* n_ints);
/* Raw emitted multiset (only with keep_emitted), flat [k, ids..]. */
const int32_t* qc_result_emitted(const qc_result* r, int64_t* n_sets, int64_t* n_ints);
const qc_stats* qc_result_stats(const qc_result* r);
/* Write "<k> v1 .. vk \n" lines (main.cu:4641-4652).  Large results are
 * formatted by several host threads, in chunks written in order. */
qc_status qc_result_write(const qc_result* r, const char* path);
void qc_result_free(qc_result* r);

/* Result files written on a host thread while the caller goes on (mines
 * the next instance, say).  The reference spills every emitted set to
 * temp.txt during enumeration and rebuilds its result file from that spill
 * (main.cu:1218-1246, 4939-4960); here the device filter hands back the
 * maximal sets already in file order, so only their formatting and the
 * write remain, and they overlap the next device work. */
typedef struct qc_writer qc_writer;
/* Start writing sets flat [k, id_1 .. id_k]* (n_ints ints) in the result
 * format.  The array must stay alive and unchanged until qc_writer_wait. */
qc_status qc_sets_write_async(const int32_t* flat, int64_t n_ints, const char* path,
                              qc_writer** out);
/* The same for a result (r must outlive the write). */
qc_status qc_result_write_async(const qc_result* r, const char* path, qc_writer** out);
/* Wait for the write; returns its status (QC_ERR_IO, QC_ERR_FORMAT) and
 * frees the writer. */
qc_status qc_writer_wait(qc_writer* w);

#ifdef __cplusplus
}
#endif
#endif /* QC_H */
