/*
 * qc_oracle.c -- CPU oracle for maximal gamma-quasi-clique enumeration.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT CODE.  This is a serial C restatement of
 * the reference cuQC algorithm (Mike12041204/cuQC, main.cu) used only as the
 * checker for the CUDA path: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it; the product library never links or calls it.
 *
 * It restates, with file:line anchors into the reference:
 *   - the gamma degree table md[k] = ceil(gamma*(k-1))      main.cu:526-533
 *   - level-0 pruning + cover vertex + root task            main.cu:846-998
 *   - per-task expansion (host rules)                        main.cu:1000-1196
 *       lookahead                                            main.cu:1349-1405
 *       remove one vertex                                    main.cu:1408-1462
 *       add one vertex (+ diameter pruning)                  main.cu:1465-1523, 1709-1732
 *       critical-vertex pruning                              main.cu:1526-1707
 *       iterative degree pruning                             main.cu:1735-1855
 *       lower/upper size bounds                              main.cu:1857-1972
 *       clique check                                         main.cu:1974-1995
 *       Q enumeration order                                  main.cu:2059-2104
 *       candidate validity / member extendability            main.cu:2144-2198
 *   - the device variant of the lower bound (lane-0 partial minimum) and
 *     the device's candidate compaction order                main.cu:4122-4289, 3809-4120
 *   - two-hop neighbour lists                                adjToSer.cpp:115-156
 *   - non-maximal removal + lexicographic result order       main.cu:4571-4960
 *     (restated with an inverted-index superset test instead of the
 *      reference's prefix tree; both compute the maximal sets of the emitted
 *      family, written in lexicographic order of the sorted id sequences).
 *
 * Three rule sets (`mode`):
 *   QO_HOST   the reference's host routines exactly, including its shared
 *             vertex->position map (vertex_order_map): the map is empty during
 *             the degree pruning that follows a critical-vertex pass with no
 *             critical-adjacent vertices (main.cu:1574-1580, 1649-1674), and
 *             stale entries survive a partial reset (main.cu:1677-1679).
 *   QO_BINARY the reference binary's split: the root task and the first child
 *             it writes run the host rules (main.cu:576, CPU_LEVELS=1), all
 *             later tasks run the device rules (main.cu:2913-4536), whose only
 *             difference from plain set semantics is the lower-bound start
 *             taken from lane 0's partial minimum indegree (main.cu:4206).
 *   QO_CLEAN  plain set semantics of the same rules (what the CUDA product
 *             implements): every degree is |N(v) cap set|.
 * The maximal sets agree across modes on every tested input; the emitted
 * (pre-filter) multisets can differ, which is why each mode exists.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define QO_HOST 0
#define QO_BINARY 1
#define QO_CLEAN 2

typedef struct {
    int32_t id, label, indeg, exdeg, l2;
} qo_vtx;

typedef struct {
    int64_t tasks;            /* tasks processed (lookahead evaluated)      */
    int64_t lookahead_hits;   /* tasks emitted whole by lookahead          */
    int64_t branches;         /* add-one-vertex calls                      */
    int64_t children;         /* child tasks written                       */
    int64_t emitted;          /* quasi-cliques emitted (incl. non-maximal) */
    int64_t emitted_vertices; /* sum of their sizes                        */
    int64_t parent_vertices;  /* sum over branches of |T_parent|           */
    int64_t p_rows;           /* sum over branches of deg(p)+|N2(p)|       */
    int64_t child_vertices;   /* sum of written child sizes                */
    int64_t max_task;         /* largest task processed                    */
    int64_t root_size;        /* vertices in the root task                 */
    int64_t stale_uses;       /* host rules: map lookups that hit a stale entry */
    int64_t stale_oob;        /*   ... pointing outside the current vertex array */
    int64_t tasks_le32, tasks_le64, tasks_le128, tasks_gt128; /* task size histogram */
    int64_t branches_le32, branches_le64, branches_le128, branches_gt128; /* by parent size */
} qo_stats;

typedef struct {
    int32_t* v;
    int64_t n, cap;
} ivec;

static int iv_push(ivec* a, int32_t x)
{
    if (a->n == a->cap) {
        int64_t nc = a->cap ? a->cap * 2 : 1024;
        int32_t* p = (int32_t*)realloc(a->v, (size_t)nc * sizeof(int32_t));
        if (!p) return -1;
        a->v = p;
        a->cap = nc;
    }
    a->v[a->n++] = x;
    return 0;
}

typedef struct {
    /* graph */
    int n;
    const int64_t *off, *off2;
    const int32_t *adj, *adj2;
    /* parameters */
    double gamma;
    int min_size;
    int* md; /* md[0 .. mdlen) */
    int mdlen;
    /* scratch (the reference's CPU_Data arrays) */
    int* pos; /* vertex id -> position, -1 when unmapped */
    ivec dirty;
    int *rem, *rmv, *cind;
    int nrem, nrmv;
    int* adjc; /* critical-vertex 2-hop counters */
    /* current rule set for the task being processed */
    int host_rules;  /* 1: host map semantics (QO_HOST / first two host tasks) */
    int lane0_quirk; /* 1: device lower-bound start (QO_BINARY device tasks) */
    /* device compaction order emulation (QO_BINARY device tasks) */
    int* ordtmp; /* 2n+2 ints */
    qo_vtx* tmpv; /* n records */
    /* output */
    ivec out;
    int64_t nsets;
    qo_stats st;
    int err;
} qo_ctx;

/* ------------------------------------------------------------------ */
/* gamma table (main.cu:526-533, 2144-2151)                            */
/* ------------------------------------------------------------------ */

static inline int md_at(const qo_ctx* c, int k)
{
    if (k < 0) k = 0;
    if (k >= c->mdlen) k = c->mdlen - 1;
    return c->md[k];
}

static inline int mindeg(const qo_ctx* c, int k)
{
    return md_at(c, k < c->min_size ? c->min_size : k);
}

/* ------------------------------------------------------------------ */
/* position map helpers (the reference's vertex_order_map)             */
/* ------------------------------------------------------------------ */

static void map_set(qo_ctx* c, const qo_vtx* v, int lo, int hi)
{
    for (int i = lo; i < hi; i++) {
        c->pos[v[i].id] = i;
        if (iv_push(&c->dirty, v[i].id)) c->err = 1;
    }
}

/* reset of the ids currently at positions [lo, hi).  Under host rules
 * this is exactly the reference's partial reset; otherwise every id set
 * since the last full clear is cleared. */
static void map_clear(qo_ctx* c, const qo_vtx* v, int lo, int hi)
{
    if (c->host_rules) {
        for (int i = lo; i < hi; i++) c->pos[v[i].id] = -1;
    } else {
        for (int64_t i = 0; i < c->dirty.n; i++) c->pos[c->dirty.v[i]] = -1;
        c->dirty.n = 0;
    }
}

/* diagnostic for host rules: a lookup of id `x` returned position p that
 * does not hold x in the current array v[0..n) */
static inline void note_lookup(qo_ctx* c, const qo_vtx* v, int n, int x, int p)
{
    if (p < 0) return;
    if (p >= n) {
        c->st.stale_uses++;
        c->st.stale_oob++;
    } else if (v[p].id != x) {
        c->st.stale_uses++;
    }
}

static void map_clear_all(qo_ctx* c)
{
    for (int64_t i = 0; i < c->dirty.n; i++) c->pos[c->dirty.v[i]] = -1;
    c->dirty.n = 0;
}

/* ------------------------------------------------------------------ */
/* orders (main.cu:2059-2142)                                          */
/* ------------------------------------------------------------------ */

static inline int label_rank(int l)
{
    switch (l) {
    case 1: return 0;
    case 2: return 1;
    case 0: return 2;
    case 3: return 3;
    default: return 4;
    }
}

static int cmp_q(const void* a, const void* b)
{
    const qo_vtx* x = (const qo_vtx*)a;
    const qo_vtx* y = (const qo_vtx*)b;
    int rx = label_rank(x->label), ry = label_rank(y->label);
    if (rx != ry) return rx < ry ? -1 : 1;
    if (x->indeg != y->indeg) return x->indeg > y->indeg ? -1 : 1;
    if (x->exdeg != y->exdeg) return x->exdeg > y->exdeg ? -1 : 1;
    if (x->l2 != y->l2) return x->l2 > y->l2 ? -1 : 1;
    if (x->id != y->id) return x->id > y->id ? -1 : 1;
    return 0;
}

/* critical-adjacent first; all others compare equal (main.cu:2106-2122) */
static int cmp_cv(const void* a, const void* b)
{
    const qo_vtx* x = (const qo_vtx*)a;
    const qo_vtx* y = (const qo_vtx*)b;
    if (x->label == 4 && y->label != 4) return -1;
    if (x->label != 4 && y->label == 4) return 1;
    return 0;
}

static int cmp_desc(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return x > y ? -1 : (x < y ? 1 : 0);
}

static int cmp_asc(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* stable "critical-adjacent first" partition, as the device's odd-even
 * transposition sort produces it (main.cu:4366-4387, 4454-4464) */
static void stable_cv(qo_ctx* c, qo_vtx* v, int n)
{
    qo_vtx* tmp = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)(n > 0 ? n : 1));
    if (!tmp) { c->err = 1; return; }
    int k = 0;
    for (int i = 0; i < n; i++) if (v[i].label == 4) tmp[k++] = v[i];
    for (int i = 0; i < n; i++) if (v[i].label != 4) tmp[k++] = v[i];
    memcpy(v, tmp, sizeof(qo_vtx) * (size_t)n);
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* validity tests (main.cu:2153-2198)                                  */
/* ------------------------------------------------------------------ */

typedef struct {
    int U, L, med;
} qo_bounds;

static inline int cand_valid(const qo_ctx* c, const qo_vtx* v, int m, const qo_bounds* b)
{
    int tot = v->indeg + v->exdeg;
    if (tot < md_at(c, c->min_size)) return 0;
    if (tot < mindeg(c, m + v->exdeg + 1)) return 0;
    if (tot < b->med) return 0;
    if (v->indeg + b->U - 1 < md_at(c, m + b->L)) return 0;
    if (tot < mindeg(c, m + b->L)) return 0;
    return 1;
}

static inline int vert_extendable(const qo_ctx* c, const qo_vtx* v, int m, const qo_bounds* b)
{
    int tot = v->indeg + v->exdeg;
    if (tot < md_at(c, c->min_size)) return 0;
    if (tot < mindeg(c, m + v->exdeg)) return 0;
    if (tot < b->med) return 0;
    if (v->exdeg == 0 && v->indeg < mindeg(c, m + v->exdeg)) return 0;
    if (v->indeg + b->U < md_at(c, m + b->U)) return 0;
    if (tot < mindeg(c, m + b->L)) return 0;
    return 1;
}

/* ------------------------------------------------------------------ */
/* lower / upper bounds (main.cu:1857-1972; device start main.cu:4206)  */
/* cind[0..ncand) holds candidate indegrees sorted descending.         */
/* Returns 1 when the bounds are invalid.                              */
/* ------------------------------------------------------------------ */

static int lu_bounds(const qo_ctx* c, const qo_vtx* v, int m, int ncand, qo_bounds* b)
{
    const int* cind = c->cind;
    int invalid = 0;
    int min_in = v[0].indeg, min_in_ex = v[0].exdeg;
    int min_tot = v[0].indeg + v[0].exdeg;
    int64_t sum_in = v[0].indeg;
    int lane0_min = v[0].indeg;
    for (int i = 1; i < m; i++) {
        sum_in += v[i].indeg;
        if (v[i].indeg < min_in) {
            min_in = v[i].indeg;
            min_in_ex = v[i].exdeg;
        } else if (v[i].indeg == min_in && v[i].exdeg < min_in_ex) {
            min_in_ex = v[i].exdeg;
        }
        if (v[i].indeg + v[i].exdeg < min_tot) min_tot = v[i].indeg + v[i].exdeg;
        /* lane 0 of the reference's warp visits positions 1, 33, 65, ... */
        if ((i - 1) % 32 == 0 && v[i].indeg < lane0_min) lane0_min = v[i].indeg;
    }
    b->med = mindeg(c, m + 1);
    if (min_in < md_at(c, m)) {
        int lb = mindeg(c, m) - (c->lane0_quirk ? lane0_min : min_in);
        while (lb <= min_in_ex && min_in + lb < md_at(c, m + lb)) lb++;
        if (min_in + lb < md_at(c, m + lb)) {
            lb = ncand + 1;
            invalid = 1;
        }
        int ub = (int)floor((double)min_tot / c->gamma) + 1 - m;
        if (ub > ncand) ub = ncand;
        if (lb < ub) {
            int idx;
            int64_t s = 0;
            for (idx = 0; idx < lb; idx++) s += cind[idx];
            while (idx < ub && sum_in + s < (int64_t)m * md_at(c, m + idx)) {
                s += cind[idx];
                idx++;
            }
            if (sum_in + s < (int64_t)m * md_at(c, m + idx)) {
                lb = ub + 1;
                invalid = 1;
            } else {
                lb = idx;
                int tub = idx;
                while (idx < ub) {
                    s += cind[idx];
                    idx++;
                    if (sum_in + s >= (int64_t)m * md_at(c, m + idx)) tub = idx;
                }
                if (ub > tub) ub = tub;
                if (lb > 1) b->med = mindeg(c, m + lb);
            }
        }
        b->U = ub;
        b->L = lb;
    } else {
        b->U = ncand;
        b->L = m < c->min_size ? c->min_size - m : 0;
    }
    if (m + b->U < c->min_size) invalid = 1;
    if (b->U < 0 || b->U < b->L) invalid = 1;
    return invalid;
}

/* ------------------------------------------------------------------ */
/* degree pruning fixpoint (main.cu:1735-1855; device 3809-4120)       */
/* c->cind[0..c->nrem) holds the indegrees of the diameter survivors.  */
/* Returns 1 on invalid bounds or a non-extendable member.             */
/* ------------------------------------------------------------------ */

/* Filter the candidates listed (in read order) in idx[0..n) into c->rem
 * (kept, in the order the active rules write them) and c->rmv.  Under the
 * device rules lane l reads entries l, l+32, ... and the kept entries are
 * written lane-major (main.cu:3857-3900, 4033-4078); the host keeps read
 * order (main.cu:1759-1768, 1826-1835). */
static void filter_cands(qo_ctx* c, const qo_vtx* v, const int* idx, int n, int m,
                         const qo_bounds* b, int need_label0)
{
    int nr = 0, nm = 0;
    if (c->lane0_quirk) {
        for (int lane = 0; lane < 32; lane++)
            for (int j = lane; j < n; j += 32) {
                const qo_vtx* x = &v[idx[j]];
                if ((!need_label0 || x->label == 0) && cand_valid(c, x, m, b))
                    c->ordtmp[nr++] = idx[j];
                else
                    c->rmv[nm++] = idx[j];
            }
        memcpy(c->rem, c->ordtmp, sizeof(int) * (size_t)nr);
    } else {
        for (int j = 0; j < n; j++) {
            const qo_vtx* x = &v[idx[j]];
            if ((!need_label0 || x->label == 0) && cand_valid(c, x, m, b))
                c->ordtmp[nr++] = idx[j];
            else
                c->rmv[nm++] = idx[j];
        }
        memcpy(c->rem, c->ordtmp, sizeof(int) * (size_t)nr);
    }
    c->nrem = nr;
    c->nrmv = nm;
}

static int degree_prune(qo_ctx* c, qo_vtx* v, int* tot, int* ncand, int m, qo_bounds* b)
{
    int nval;
    qsort(c->cind, (size_t)c->nrem, sizeof(int), cmp_desc);
    if (lu_bounds(c, v, m, c->nrem, b)) return 1;
    for (int k = 0; k < m; k++)
        if (!vert_extendable(c, &v[k], m, b)) return 1;

    /* first filter over positions [m, tot) */
    {
        int n = *tot - m;
        int* idx = c->ordtmp + c->n + 2; /* read order = positions */
        for (int j = 0; j < n; j++) idx[j] = m + j;
        filter_cands(c, v, idx, n, m, b, 1);
    }

    while (c->nrem > 0 && c->nrmv > 0) {
        if (c->nrem < c->nrmv) {
            for (int i = 0; i < *tot; i++) v[i].exdeg = 0;
            for (int r = 0; r < c->nrem; r++) {
                int u = v[c->rem[r]].id;
                for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
                    int p = c->pos[c->adj[e]];
                    if (p > -1) v[p].exdeg++;
                }
            }
        } else {
            for (int r = 0; r < c->nrmv; r++) {
                int u = v[c->rmv[r]].id;
                for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
                    int p = c->pos[c->adj[e]];
                    if (p > -1) v[p].exdeg--;
                }
            }
        }
        nval = 0;
        for (int k = 0; k < c->nrem; k++)
            if (cand_valid(c, &v[c->rem[k]], m, b)) c->cind[nval++] = v[c->rem[k]].indeg;
        qsort(c->cind, (size_t)nval, sizeof(int), cmp_desc);
        if (lu_bounds(c, v, m, nval, b)) return 1;
        for (int k = 0; k < m; k++)
            if (!vert_extendable(c, &v[k], m, b)) return 1;
        {
            int n = c->nrem;
            int* idx = c->ordtmp + c->n + 2;
            memcpy(idx, c->rem, sizeof(int) * (size_t)n);
            filter_cands(c, v, idx, n, m, b, 0);
        }
    }
    /* compact survivors right after the members, in rem order */
    for (int i = 0; i < c->nrem; i++) c->tmpv[i] = v[c->rem[i]];
    for (int i = 0; i < c->nrem; i++) v[m + i] = c->tmpv[i];
    *tot = *tot - *ncand + c->nrem;
    *ncand = c->nrem;
    return 0;
}

/* ------------------------------------------------------------------ */
/* emission                                                            */
/* ------------------------------------------------------------------ */

static void emit(qo_ctx* c, const qo_vtx* v, int k)
{
    if (iv_push(&c->out, k)) c->err = 1;
    for (int i = 0; i < k; i++)
        if (iv_push(&c->out, v[i].id)) c->err = 1;
    c->nsets++;
    c->st.emitted++;
    c->st.emitted_vertices += k;
}

/* main.cu:1974-1995 */
static void check_clique(qo_ctx* c, const qo_vtx* v, int m)
{
    int req = md_at(c, m);
    for (int k = 0; k < m; k++)
        if (v[k].indeg < req) return;
    emit(c, v, m);
}

/* ------------------------------------------------------------------ */
/* lookahead (main.cu:1349-1405; device 3405-3471)                     */
/* ------------------------------------------------------------------ */

static int lookahead(qo_ctx* c, qo_vtx* v, int t, int m, int nc)
{
    int req = md_at(c, t);
    for (int i = 0; i < m; i++)
        if (v[i].indeg + v[i].exdeg < req) return 0;
    map_set(c, v, m, t);
    for (int i = m; i < t; i++) {
        int u = v[i].id;
        for (int64_t e = c->off2[u]; e < c->off2[u + 1]; e++) {
            int p = c->pos[c->adj2[e]];
            note_lookup(c, v, t, c->adj2[e], p);
            /* a stale host-map position can point past this task; the
             * reference's write then lands outside the task's records */
            if (p >= m && p < t) v[p].l2++;
        }
    }
    map_clear(c, v, m, t);
    for (int j = m; j < t; j++)
        if (v[j].l2 < nc - 1 || v[j].indeg + v[j].exdeg < req) return 0;
    emit(c, v, t);
    return 1;
}

/* ------------------------------------------------------------------ */
/* remove the last candidate (main.cu:1408-1462)                       */
/* ------------------------------------------------------------------ */

static int remove_one(qo_ctx* c, qo_vtx* v, int* tot, int* nc, int m)
{
    int need = mindeg(c, m);
    int failed = 0;
    (*nc)--;
    (*tot)--;
    map_set(c, v, 0, *tot);
    int u = v[*tot].id;
    for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
        int p = c->pos[c->adj[e]];
        note_lookup(c, v, *tot, c->adj[e], p);
        if (p > -1 && p < *tot) {
            v[p].exdeg--;
            if (p < m && v[p].indeg + v[p].exdeg < need) {
                failed = 1;
                break;
            }
        }
    }
    map_clear(c, v, 0, *tot);
    return failed;
}

/* ------------------------------------------------------------------ */
/* diameter pruning after adding p (main.cu:1709-1732)                 */
/* ------------------------------------------------------------------ */

static void diameter(qo_ctx* c, qo_vtx* w, int p, int tot, int m)
{
    c->nrem = 0;
    for (int i = m; i < tot; i++) w[i].label = -1;
    for (int64_t e = c->off2[p]; e < c->off2[p + 1]; e++) {
        int q = c->pos[c->adj2[e]];
        note_lookup(c, w, tot, c->adj2[e], q);
        if (q >= m && q < tot) {
            w[q].label = 0;
            c->cind[c->nrem++] = w[q].indeg;
        }
    }
}

/* ------------------------------------------------------------------ */
/* add one vertex (main.cu:1465-1523)                                  */
/* ------------------------------------------------------------------ */

static int add_one(qo_ctx* c, qo_vtx* w, int* tot, int* nc, int* m, qo_bounds* b)
{
    int p = w[*m].id;
    w[*m].label = 1;
    (*m)++;
    (*nc)--;
    map_set(c, w, 0, *tot);
    for (int64_t e = c->off[p]; e < c->off[p + 1]; e++) {
        int q = c->pos[c->adj[e]];
        note_lookup(c, w, *tot, c->adj[e], q);
        if (q > -1 && q < *tot) {
            w[q].indeg++;
            w[q].exdeg--;
        }
    }
    diameter(c, w, p, *tot, *m);
    int r = degree_prune(c, w, tot, nc, *m, b);
    map_clear_all(c);
    return r;
}

/* ------------------------------------------------------------------ */
/* critical-vertex pruning (main.cu:1526-1707; device 3567-3700, 3757)  */
/* returns 2: critical fail, 1: failed member/bounds, 0: ok            */
/* ------------------------------------------------------------------ */

static int crit(qo_ctx* c, qo_vtx* w, int* tot, int* nc, int* m, qo_bounds* b)
{
    int* adjc = c->adjc;
    int nca = 0;
    memset(adjc, 0, sizeof(int) * (size_t)(*tot > 0 ? *tot : 1));
    map_set(c, w, 0, *tot);
    int crit_md = md_at(c, *m + b->L);
    for (int k = 0; k < *m; k++) {
        if (w[k].indeg + w[k].exdeg == crit_md && w[k].exdeg > 0) {
            int u = w[k].id;
            for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
                int q = c->pos[c->adj[e]];
                if (q >= *m && q < *tot) w[q].label = 4;
            }
        }
    }
    map_clear(c, w, 0, *tot);
    if (c->host_rules)
        qsort(w + *m, (size_t)*nc, sizeof(qo_vtx), cmp_cv);
    else
        stable_cv(c, w + *m, *nc);
    for (int i = *m; i < *tot && w[i].label == 4; i++) nca++;

    if (nca > 0) {
        map_set(c, w, 0, *tot);
        for (int i = *m; i < *m + nca; i++) {
            int u = w[i].id;
            for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
                int q = c->pos[c->adj[e]];
                if (q > -1 && q < *tot) {
                    w[q].indeg++;
                    w[q].exdeg--;
                }
            }
            for (int64_t e = c->off2[u]; e < c->off2[u + 1]; e++) {
                int q = c->pos[c->adj2[e]];
                if (q > -1 && q < *tot) adjc[q]++;
            }
        }
        int fail = 0;
        for (int k = 0; k < *m; k++)
            if (adjc[k] != nca) fail = 1;
        if (!fail)
            for (int k = *m; k < *m + nca; k++)
                if (adjc[k] < nca - 1) fail = 1;
        if (fail) {
            map_clear(c, w, 0, *tot);
            return 2;
        }
        for (int k = *m; k < *m + nca; k++) w[k].label = 1;
        *m += nca;
        *nc -= nca;
    } else if (!c->host_rules) {
        /* set semantics: the following degree pruning sees every vertex */
        map_set(c, w, 0, *tot);
    }
    c->nrem = 0;
    for (int k = *m; k < *tot; k++) {
        if (adjc[k] == nca)
            c->cind[c->nrem++] = w[k].indeg;
        else
            w[k].label = -1;
    }
    int r = degree_prune(c, w, tot, nc, *m, b);
    map_clear(c, w, 0, *tot);
    return r;
}

/* ------------------------------------------------------------------ */
/* task stack                                                          */
/* ------------------------------------------------------------------ */

typedef struct {
    qo_vtx* v;
    int64_t n, cap;
    int64_t* toff; /* task start offsets */
    int64_t nt, capt;
} qo_stack;

static int st_push(qo_stack* s, const qo_vtx* v, int k)
{
    if (s->n + k > s->cap) {
        int64_t nc = s->cap ? s->cap : 4096;
        while (nc < s->n + k) nc *= 2;
        qo_vtx* p = (qo_vtx*)realloc(s->v, (size_t)nc * sizeof(qo_vtx));
        if (!p) return -1;
        s->v = p;
        s->cap = nc;
    }
    if (s->nt + 2 > s->capt) {
        int64_t nc = s->capt ? s->capt * 2 : 1024;
        int64_t* p = (int64_t*)realloc(s->toff, (size_t)nc * sizeof(int64_t));
        if (!p) return -1;
        s->toff = p;
        s->capt = nc;
    }
    s->toff[s->nt++] = s->n;
    for (int i = 0; i < k; i++) {
        s->v[s->n + i] = v[i];
        s->v[s->n + i].l2 = 0;
    }
    s->n += k;
    return 0;
}

/* ------------------------------------------------------------------ */
/* expand one task (main.cu:1056-1181)                                  */
/* ------------------------------------------------------------------ */

static void process_task(qo_ctx* c, qo_vtx* v, int t, qo_stack* s, qo_vtx* w)
{
    int m = 0, cov = 0;
    while (m < t && v[m].label == 1) m++;
    while (m + cov < t && v[m + cov].label == 2) cov++;
    int nc = t - m;
    int expansions = nc;
    c->st.tasks++;
    if (t > c->st.max_task) c->st.max_task = t;
    if (t <= 32) c->st.tasks_le32++;
    else if (t <= 64) c->st.tasks_le64++;
    else if (t <= 128) c->st.tasks_le128++;
    else c->st.tasks_gt128++;

    if (lookahead(c, v, t, m, nc)) {
        c->st.lookahead_hits++;
        return;
    }
    for (int j = cov; j < expansions; j++) {
        if (j != cov && remove_one(c, v, &t, &nc, m)) break;

        int mm = m, cc = nc, tt = t;
        for (int i = 0; i < m; i++) w[i] = v[i];
        w[m] = v[t - 1];
        for (int i = m; i < t - 1; i++) w[i + 1] = v[i];
        for (int i = m + 1; i <= m + cov; i++) w[i].label = 0;

        int pid = w[m].id;
        c->st.branches++;
        c->st.parent_vertices += t;
        if (t <= 32) c->st.branches_le32++;
        else if (t <= 64) c->st.branches_le64++;
        else if (t <= 128) c->st.branches_le128++;
        else c->st.branches_gt128++;
        c->st.p_rows += (c->off[pid + 1] - c->off[pid]) + (c->off2[pid + 1] - c->off2[pid]);

        qo_bounds b = {0, 0, 0};
        int r = add_one(c, w, &tt, &cc, &mm, &b);
        if (r == 1) {
            if (mm >= c->min_size) check_clique(c, w, mm);
            continue;
        }
        r = crit(c, w, &tt, &cc, &mm, &b);
        if (r == 2) continue;
        if (mm >= c->min_size) check_clique(c, w, mm);
        if (r == 1) continue;
        qsort(w, (size_t)tt, sizeof(qo_vtx), cmp_q);
        if (cc > 0) {
            if (st_push(s, w, tt)) c->err = 1;
            c->st.children++;
            c->st.child_vertices += tt;
        }
    }
}

/* ------------------------------------------------------------------ */
/* level 0: pruning, cover vertex, root task (main.cu:846-998)         */
/* returns the root size (0: no task)                                  */
/* ------------------------------------------------------------------ */

static int build_root(qo_ctx* c, qo_vtx* vs)
{
    int n = c->n;
    int need = md_at(c, c->min_size);
    int nrem = 0, nrmv = 0;
    int* rem = c->rem;
    int* rmv = c->rmv;
    for (int i = 0; i < n; i++) {
        vs[i].id = i;
        vs[i].indeg = 0;
        vs[i].exdeg = (int)(c->off[i + 1] - c->off[i]);
        vs[i].l2 = (int)(c->off2[i + 1] - c->off2[i]);
        if (vs[i].exdeg >= need && vs[i].l2 >= c->min_size - 1) {
            vs[i].label = 0;
            rem[nrem++] = i;
        } else {
            vs[i].label = -1;
            rmv[nrmv++] = i;
        }
    }
    int ncand = n;
    while (nrem < ncand / 2) {
        ncand = nrem;
        for (int i = 0; i < ncand; i++) vs[rem[i]].exdeg = 0;
        for (int i = 0; i < ncand; i++) {
            int u = rem[i];
            for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
                int w = c->adj[e];
                if (vs[w].label == 0) vs[w].exdeg++;
            }
        }
        nrem = nrmv = 0;
        for (int i = 0; i < ncand; i++) {
            int u = rem[i];
            if (vs[u].exdeg >= need)
                rem[nrem++] = u;
            else {
                vs[u].label = -1;
                rmv[nrmv++] = u;
            }
        }
    }
    ncand = nrem;
    for (int k = 0; k < nrmv; k++) {
        int u = rmv[k];
        for (int64_t e = c->off[u]; e < c->off[u + 1]; e++) {
            int w = c->adj[e];
            if (vs[w].label == 0) {
                vs[w].exdeg--;
                if (vs[w].exdeg < need) {
                    vs[w].label = -1;
                    ncand--;
                    rmv[nrmv++] = w;
                }
            }
        }
    }
    int best = 0, best_i = 0;
    for (int i = 0; i < n; i++)
        if (vs[i].label == 0 && vs[i].exdeg > best) {
            best = vs[i].exdeg;
            best_i = i;
        }
    if (n > 0) {
        vs[best_i].label = 3;
        for (int64_t e = c->off[best_i]; e < c->off[best_i + 1]; e++) {
            int w = c->adj[e];
            if (vs[w].label == 0) vs[w].label = 2;
        }
    }
    qsort(vs, (size_t)n, sizeof(qo_vtx), cmp_q);
    for (int i = 0; i < ncand; i++) vs[i].l2 = 0;
    return ncand;
}

/* ------------------------------------------------------------------ */
/* public: enumerate                                                   */
/* ------------------------------------------------------------------ */

static void ctx_free(qo_ctx* c)
{
    free(c->md);
    free(c->pos);
    free(c->dirty.v);
    free(c->rem);
    free(c->rmv);
    free(c->cind);
    free(c->adjc);
    free(c->ordtmp);
    free(c->tmpv);
}

/* Optional bound on the tasks one qo_mine call may expand (0: none).  A call
 * that would exceed it stops and returns -2; used to screen generated
 * instances by search-tree size. */
static int64_t g_task_budget = 0;
void qo_set_task_budget(int64_t tasks) { g_task_budget = tasks > 0 ? tasks : 0; }

/* Enumerate every quasi-clique the reference's rules emit (maximal or not).
 * Output: out_buf = [k, id_1..id_k, k, ...] (caller frees with qo_free). */
int qo_mine(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
            const int32_t* adj2, double gamma, int min_size, int mode,
            int64_t* out_nsets, int64_t* out_nints, int32_t** out_buf, qo_stats* st)
{
    qo_ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n;
    c.off = off;
    c.adj = adj;
    c.off2 = off2;
    c.adj2 = adj2;
    c.gamma = gamma;
    c.min_size = min_size;
    c.mdlen = (n > min_size ? n : min_size) + 3;
    c.md = (int*)malloc(sizeof(int) * (size_t)c.mdlen);
    int nn = n > 0 ? n : 1;
    c.pos = (int*)malloc(sizeof(int) * (size_t)nn);
    c.rem = (int*)malloc(sizeof(int) * (size_t)(2 * nn + 2));
    c.rmv = (int*)malloc(sizeof(int) * (size_t)(2 * nn + 2));
    c.cind = (int*)malloc(sizeof(int) * (size_t)(2 * nn + 2));
    c.adjc = (int*)malloc(sizeof(int) * (size_t)(nn + 1));
    c.ordtmp = (int*)malloc(sizeof(int) * (size_t)(3 * nn + 4));
    c.tmpv = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)(nn + 1));
    qo_vtx* vs = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)nn);
    qo_vtx* cur = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)(nn + 1));
    qo_vtx* w = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)(nn + 1));
    qo_stack s;
    memset(&s, 0, sizeof(s));
    if (!c.md || !c.pos || !c.rem || !c.rmv || !c.cind || !c.adjc || !c.ordtmp || !c.tmpv ||
        !vs || !cur || !w) {
        ctx_free(&c);
        free(vs); free(cur); free(w);
        return -1;
    }
    c.md[0] = 0;
    for (int i = 1; i < c.mdlen; i++) c.md[i] = (int)ceil(gamma * (double)(i - 1));
    for (int i = 0; i < n; i++) c.pos[i] = -1;

    int rsize = build_root(&c, vs);
    c.st.root_size = rsize;
    if (rsize > 0) {
        /* root: host rules in every mode but CLEAN */
        c.host_rules = (mode != QO_CLEAN);
        c.lane0_quirk = 0;
        process_task(&c, vs, rsize, &s, w);
        /* the first child written by the root is the next host task in
         * the reference (main.cu:2013-2016, 576) */
        if (s.nt > 0) {
            int64_t a = s.toff[0], z = s.nt > 1 ? s.toff[1] : s.n;
            int k = (int)(z - a);
            memcpy(cur, s.v + a, sizeof(qo_vtx) * (size_t)k);
            memmove(s.v + a, s.v + z, sizeof(qo_vtx) * (size_t)(s.n - z));
            for (int64_t i = 1; i < s.nt; i++) s.toff[i - 1] = s.toff[i] - k;
            s.nt--;
            s.n -= k;
            process_task(&c, cur, k, &s, w);
        }
        c.host_rules = (mode == QO_HOST);
        c.lane0_quirk = (mode == QO_BINARY);
        if (!c.host_rules) map_clear_all(&c);
        while (s.nt > 0 && !c.err) {
            if (g_task_budget && c.st.tasks > g_task_budget) {
                c.err = 2;
                break;
            }
            int64_t a = s.toff[--s.nt];
            int k = (int)(s.n - a);
            memcpy(cur, s.v + a, sizeof(qo_vtx) * (size_t)k);
            s.n = a;
            process_task(&c, cur, k, &s, w);
            if (c.dirty.n > 8 * (int64_t)nn) {
                /* drop entries already reset to keep the list short */
                int64_t k2 = 0;
                for (int64_t i = 0; i < c.dirty.n; i++)
                    if (c.pos[c.dirty.v[i]] != -1) c.dirty.v[k2++] = c.dirty.v[i];
                c.dirty.n = k2;
            }
        }
    }
    int err = c.err;
    if (st) *st = c.st;
    *out_nsets = c.nsets;
    *out_nints = c.out.n;
    *out_buf = c.out.v;
    c.out.v = NULL;
    ctx_free(&c);
    free(vs); free(cur); free(w);
    free(s.v);
    free(s.toff);
    return err == 2 ? -2 : (err ? -1 : 0);
}

void qo_free(void* p) { free(p); }

/* ------------------------------------------------------------------ */
/* maximal filter + lexicographic order (main.cu:4571-4960 semantics)  */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t* ids; /* sorted ascending */
    int len;
} qo_set;

static int cmp_set(const void* a, const void* b)
{
    const qo_set* x = (const qo_set*)a;
    const qo_set* y = (const qo_set*)b;
    int k = x->len < y->len ? x->len : y->len;
    for (int i = 0; i < k; i++)
        if (x->ids[i] != y->ids[i]) return x->ids[i] < y->ids[i] ? -1 : 1;
    return x->len < y->len ? -1 : (x->len > y->len ? 1 : 0);
}

static int is_subset(const qo_set* s, const qo_set* t)
{
    int i = 0, j = 0;
    while (i < s->len && j < t->len) {
        if (s->ids[i] == t->ids[j]) { i++; j++; }
        else if (s->ids[i] > t->ids[j]) j++;
        else return 0;
    }
    return i == s->len;
}

/* in: [k, ids...]*nsets ; out: maximal sets, each sorted, in lexicographic
 * order, as [k, ids...]. */
int qo_maximal(const int32_t* in, int64_t nsets, int64_t* out_nsets, int64_t* out_nints,
               int32_t** out_buf)
{
    qo_set* sets = (qo_set*)malloc(sizeof(qo_set) * (size_t)(nsets > 0 ? nsets : 1));
    int64_t total = 0, p = 0;
    int32_t maxid = -1;
    for (int64_t i = 0; i < nsets; i++) {
        int k = in[p];
        total += k;
        for (int j = 0; j < k; j++)
            if (in[p + 1 + j] > maxid) maxid = in[p + 1 + j];
        p += 1 + k;
    }
    int32_t* pool = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
    if (!sets || !pool) { free(sets); free(pool); return -1; }
    p = 0;
    int64_t q = 0;
    for (int64_t i = 0; i < nsets; i++) {
        int k = in[p];
        sets[i].ids = pool + q;
        sets[i].len = k;
        memcpy(pool + q, in + p + 1, sizeof(int32_t) * (size_t)k);
        qsort(pool + q, (size_t)k, sizeof(int32_t), cmp_asc);
        q += k;
        p += 1 + k;
    }
    qsort(sets, (size_t)nsets, sizeof(qo_set), cmp_set);
    int64_t nu = 0;
    for (int64_t i = 0; i < nsets; i++)
        if (nu == 0 || cmp_set(&sets[nu - 1], &sets[i]) != 0) sets[nu++] = sets[i];
    /* inverted index */
    int64_t nv = (int64_t)maxid + 1;
    int64_t* cnt = (int64_t*)calloc((size_t)(nv + 1), sizeof(int64_t));
    int64_t tot2 = 0;
    for (int64_t i = 0; i < nu; i++) tot2 += sets[i].len;
    int64_t* post = (int64_t*)malloc(sizeof(int64_t) * (size_t)(tot2 > 0 ? tot2 : 1));
    char* keep = (char*)malloc((size_t)(nu > 0 ? nu : 1));
    if (!cnt || !post || !keep) { free(sets); free(pool); free(cnt); free(post); free(keep); return -1; }
    for (int64_t i = 0; i < nu; i++)
        for (int j = 0; j < sets[i].len; j++) cnt[sets[i].ids[j] + 1]++;
    for (int64_t v = 0; v < nv; v++) cnt[v + 1] += cnt[v];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nv > 0 ? nv : 1));
    if (!fill) { free(sets); free(pool); free(cnt); free(post); free(keep); return -1; }
    for (int64_t v = 0; v < nv; v++) fill[v] = cnt[v];
    for (int64_t i = 0; i < nu; i++)
        for (int j = 0; j < sets[i].len; j++) post[fill[sets[i].ids[j]]++] = i;
    int64_t nout = 0, nints = 0;
    for (int64_t i = 0; i < nu; i++) {
        keep[i] = 1;
        if (sets[i].len == 0) continue;
        int32_t best = sets[i].ids[0];
        for (int j = 1; j < sets[i].len; j++)
            if (cnt[sets[i].ids[j] + 1] - cnt[sets[i].ids[j]] < cnt[best + 1] - cnt[best])
                best = sets[i].ids[j];
        for (int64_t e = cnt[best]; e < cnt[best + 1]; e++) {
            const qo_set* t = &sets[post[e]];
            if (t->len > sets[i].len && is_subset(&sets[i], t)) {
                keep[i] = 0;
                break;
            }
        }
        if (keep[i]) { nout++; nints += 1 + sets[i].len; }
    }
    int32_t* ob = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nints > 0 ? nints : 1));
    if (!ob) { free(sets); free(pool); free(cnt); free(post); free(keep); free(fill); return -1; }
    int64_t o = 0;
    for (int64_t i = 0; i < nu; i++) {
        if (!keep[i]) continue;
        ob[o++] = sets[i].len;
        memcpy(ob + o, sets[i].ids, sizeof(int32_t) * (size_t)sets[i].len);
        o += sets[i].len;
    }
    *out_nsets = nout;
    *out_nints = nints;
    *out_buf = ob;
    free(sets); free(pool); free(cnt); free(post); free(keep); free(fill);
    return 0;
}

/* result file lines: "<k> v1 v2 ... vk \n" (main.cu:4641-4652) */
int qo_write_result(const char* path, const int32_t* buf, int64_t nsets)
{
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    int64_t p = 0;
    for (int64_t i = 0; i < nsets; i++) {
        int k = buf[p++];
        fprintf(f, "%d ", k);
        for (int j = 0; j < k; j++) fprintf(f, "%d ", buf[p++]);
        fprintf(f, "\n");
    }
    fclose(f);
    return 0;
}

/* ------------------------------------------------------------------ */
/* two-hop lists (adjToSer.cpp:115-156): N2(v) = sorted(N(v) u N(N(v)) \ {v}),
 * where a self loop in N(v) is kept as the reference keeps it.        */
/* ------------------------------------------------------------------ */

int qo_twohop(int n, const int64_t* off, const int32_t* adj, int64_t* off2_out,
              int64_t cap, int32_t* adj2_out, int64_t* n2_out)
{
    char* flag = (char*)calloc((size_t)(n > 0 ? n : 1), 1);
    if (!flag) return -1;
    int64_t k = 0;
    off2_out[0] = 0;
    for (int v = 0; v < n; v++) {
        int64_t a = k;
        for (int64_t e = off[v]; e < off[v + 1]; e++) {
            int u = adj[e];
            if (!flag[u]) {
                if (k >= cap) { free(flag); return -2; }
                adj2_out[k++] = u;
                flag[u] = 1;
            }
            for (int64_t f = off[u]; f < off[u + 1]; f++) {
                int x = adj[f];
                if (!flag[x] && x != v) {
                    if (k >= cap) { free(flag); return -2; }
                    adj2_out[k++] = x;
                    flag[x] = 1;
                }
            }
        }
        for (int64_t i = a; i < k; i++) flag[adj2_out[i]] = 0;
        qsort(adj2_out + a, (size_t)(k - a), sizeof(int32_t), cmp_asc);
        off2_out[v + 1] = k;
    }
    *n2_out = k;
    free(flag);
    return 0;
}

/* ------------------------------------------------------------------ */
/* definitional brute force for n <= 24: every subset, keep the        */
/* quasi-cliques of size >= min_size with no quasi-clique superset.    */
/* ------------------------------------------------------------------ */

int qo_brute(int n, const int64_t* off, const int32_t* adj, double gamma, int min_size,
             int64_t* out_nsets, int64_t* out_nints, int32_t** out_buf)
{
    if (n > 24 || n < 0) return -1;
    uint32_t nb[24];
    int md[26];
    md[0] = 0;
    for (int i = 1; i < 26; i++) md[i] = (int)ceil(gamma * (double)(i - 1));
    for (int v = 0; v < n; v++) {
        nb[v] = 0;
        for (int64_t e = off[v]; e < off[v + 1]; e++)
            if (adj[e] != v) nb[v] |= 1u << adj[e];
    }
    uint32_t full = n ? (uint32_t)((1ull << n) - 1) : 0;
    uint64_t N = 1ull << n;
    uint8_t* qc = (uint8_t*)calloc((size_t)N, 1);
    uint8_t* up = (uint8_t*)calloc((size_t)N, 1);
    if (!qc || !up) { free(qc); free(up); return -1; }
    for (uint64_t s = 1; s < N; s++) {
        int k = __builtin_popcountll(s);
        if (k < min_size) continue;
        int ok = 1;
        for (uint32_t r = (uint32_t)s; r && ok; r &= r - 1) {
            int v = __builtin_ctz(r);
            if (__builtin_popcount(nb[v] & (uint32_t)s) < md[k]) ok = 0;
        }
        qc[s] = (uint8_t)ok;
        up[s] = (uint8_t)ok;
    }
    /* up[S] = OR of qc[T] over T superset of S */
    for (int b = 0; b < n; b++)
        for (uint64_t s = 0; s < N; s++)
            if (!(s >> b & 1)) up[s] |= up[s | (1ull << b)];
    ivec o = {0, 0, 0};
    int64_t ns = 0;
    for (uint64_t s = 1; s < N; s++) {
        if (!qc[s]) continue;
        int maximal = 1;
        for (uint32_t r = full & ~(uint32_t)s; r && maximal; r &= r - 1)
            if (up[s | (1ull << __builtin_ctz(r))]) maximal = 0;
        if (!maximal) continue;
        iv_push(&o, __builtin_popcountll(s));
        for (uint32_t r = (uint32_t)s; r; r &= r - 1) iv_push(&o, __builtin_ctz(r));
        ns++;
    }
    free(qc);
    free(up);
    *out_nsets = ns;
    *out_nints = o.n;
    *out_buf = o.v;
    return 0;
}

/* Level-0 result only: the root task (ids, labels, exdeg in Q order).
 * Returns the root size; arrays need room for n entries. */
int qo_root(int n, const int64_t* off, const int32_t* adj, const int64_t* off2,
            const int32_t* adj2, double gamma, int min_size, int32_t* ids, int32_t* labels,
            int32_t* exdeg)
{
    qo_ctx c;
    memset(&c, 0, sizeof(c));
    c.n = n; c.off = off; c.adj = adj; c.off2 = off2; c.adj2 = adj2;
    c.gamma = gamma; c.min_size = min_size;
    c.mdlen = (n > min_size ? n : min_size) + 3;
    c.md = (int*)malloc(sizeof(int) * (size_t)c.mdlen);
    int nn = n > 0 ? n : 1;
    c.rem = (int*)malloc(sizeof(int) * (size_t)(2 * nn + 2));
    c.rmv = (int*)malloc(sizeof(int) * (size_t)(2 * nn + 2));
    qo_vtx* vs = (qo_vtx*)malloc(sizeof(qo_vtx) * (size_t)nn);
    if (!c.md || !c.rem || !c.rmv || !vs) { free(c.md); free(c.rem); free(c.rmv); free(vs); return -1; }
    c.md[0] = 0;
    for (int i = 1; i < c.mdlen; i++) c.md[i] = (int)ceil(gamma * (double)(i - 1));
    int r = build_root(&c, vs);
    for (int i = 0; i < r; i++) { ids[i] = vs[i].id; labels[i] = vs[i].label; exdeg[i] = vs[i].exdeg; }
    free(c.md); free(c.rem); free(c.rmv); free(vs);
    return r;
}
