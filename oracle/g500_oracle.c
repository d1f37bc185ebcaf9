/*
 * g500_oracle.c -- CPU restatement of the reference's Graph500 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the
 * smoke check and bench.py's CPU-baseline / reference arm are the only code
 * that may load it, and only as the checker or as the timed CPU baseline.
 * The product (the CUDA library under cuda-graph-traversal_b200/) never
 * links, loads or calls it.
 *
 * Every function restates one piece of RuanPetrus/cuda-graph-traversal and
 * cites the file:line it follows.  The Graph500 MRG jump tables are not
 * copied: they are recomputed here by exponentiating the MRG companion
 * matrix, which is the published construction of that table
 * (src/mrg_transitions.cu:10-14 names the generator; the table holds
 * A^(v * 256^b) for byte b and byte value v, src/graph_generation.cu:209-223).
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fPIC -shared (oracle/Makefile).
 * -ffp-contract=off keeps every float expression a plain IEEE binary32
 * operation, as in the reference's kernels.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>

#define MRG_P 0x7FFFFFFFu            /* modulus 2^31 - 1 */
#define MRG_X 107374182u             /* multiplier of z1 */
#define MRG_Y 104480u                /* multiplier of z5 */

typedef struct { uint32_t z[5]; } orc_mrg;        /* z[0] = z1 (newest) .. z[4] = z5 */
typedef struct { uint32_t m[5][5]; } orc_mat;     /* row-major 5x5 matrix mod p      */

static orc_mat g_jump[24][256];                   /* g_jump[b][v] = A^(v * 256^b)     */
static int g_jump_ready = 0;

static inline uint32_t mulmod(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * b) % MRG_P);
}
static inline uint32_t addmod(uint32_t a, uint32_t b) {
    uint32_t s = a + b;
    return s >= MRG_P ? s - MRG_P : s;
}

/* One MRG step: z1' = X*z1 + Y*z5 (mod p), the other words shift down.
 * Follows cuda_mrg_orig_step, src/graph_generation.cu:73-80 (mul_x/mul_y
 * there are Schrage forms of the same products, :38-50). */
static inline uint32_t mrg_next(orc_mrg *s) {
    uint32_t n = addmod(mulmod(MRG_X, s->z[0]), mulmod(MRG_Y, s->z[4]));
    s->z[4] = s->z[3];
    s->z[3] = s->z[2];
    s->z[2] = s->z[1];
    s->z[1] = s->z[0];
    s->z[0] = n;
    return n;
}

static void mat_mul(const orc_mat *a, const orc_mat *b, orc_mat *out) {
    orc_mat r;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) {
            uint64_t acc = 0;
            for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a->m[i][k] * b->m[k][j]) % MRG_P;
            r.m[i][j] = (uint32_t)acc;
        }
    *out = r;
}

static inline void mat_apply(const orc_mat *a, orc_mrg *s) {
    uint32_t in[5];
    memcpy(in, s->z, sizeof in);
    for (int i = 0; i < 5; ++i) {
        uint64_t acc = 0;
        for (int k = 0; k < 5; ++k) acc += (uint64_t)a->m[i][k] * in[k] % MRG_P;
        s->z[i] = (uint32_t)(acc % MRG_P);
    }
}

/* Jump tables: the companion matrix A of the step above, raised to
 * v * 256^b.  Same content as the reference's cuda_mrg_skip_matrices
 * (src/mrg_transitions.cu:14), computed instead of copied. */
static void build_jump_tables(void) {
    if (g_jump_ready) return;
    orc_mat a;
    memset(&a, 0, sizeof a);
    a.m[0][0] = MRG_X;
    a.m[0][4] = MRG_Y;
    for (int i = 1; i < 5; ++i) a.m[i][i - 1] = 1;
    orc_mat p = a; /* A^(256^b) */
    for (int b = 0; b < 24; ++b) {
        memset(&g_jump[b][0], 0, sizeof(orc_mat));
        for (int i = 0; i < 5; ++i) g_jump[b][0].m[i][i] = 1;
        for (int v = 1; v < 256; ++v) mat_mul(&g_jump[b][v - 1], &p, &g_jump[b][v]);
        orc_mat q = p;
        for (int k = 0; k < 8; ++k) mat_mul(&q, &q, &q);
        p = q;
    }
    g_jump_ready = 1;
}

/* Jump ahead by high*2^128 + mid*2^64 + low steps, one table matrix per
 * non-zero byte.  Follows cuda_mrg_skip, src/graph_generation.cu:209-223. */
static void mrg_skip(orc_mrg *s, uint64_t high, uint64_t mid, uint64_t low) {
    for (int b = 0; low; ++b, low >>= 8)
        if (low & 0xFF) mat_apply(&g_jump[b][low & 0xFF], s);
    for (int b = 8; mid; ++b, mid >>= 8)
        if (mid & 0xFF) mat_apply(&g_jump[b][mid & 0xFF], s);
    for (int b = 16; high; ++b, high >>= 8)
        if (high & 0xFF) mat_apply(&g_jump[b][high & 0xFF], s);
}

/* C-ABI views of the jump and the step, for pinning against the reference. */
void orc_mrg_skip(uint32_t z[5], uint64_t high, uint64_t mid, uint64_t low) {
    build_jump_tables();
    orc_mrg s;
    memcpy(s.z, z, sizeof s.z);
    mrg_skip(&s, high, mid, low);
    memcpy(z, s.z, sizeof s.z);
}

void orc_mrg_draw(uint32_t z[5], int n, uint32_t *out) {
    orc_mrg s;
    memcpy(s.z, z, sizeof s.z);
    for (int i = 0; i < n; ++i) out[i] = mrg_next(&s);
    memcpy(z, s.z, sizeof s.z);
}

/* make_mrg_seed, src/graph_generation.cu:248-254. */
void orc_make_mrg_seed(uint64_t s1, uint64_t s2, uint32_t seed[5]) {
    seed[0] = (uint32_t)(s1 & 0x3FFFFFFFu) + 1;
    seed[1] = (uint32_t)((s1 >> 30) & 0x3FFFFFFFu) + 1;
    seed[2] = (uint32_t)(s2 & 0x3FFFFFFFu) + 1;
    seed[3] = (uint32_t)((s2 >> 30) & 0x3FFFFFFFu) + 1;
    seed[4] = (uint32_t)((s2 >> 60) << 4) + (uint32_t)(s1 >> 60) + 1;
}

/* make_random_numbers, src/graph_generation.cu:256-266: reseed, jump by
 * 2*2^128 + 2*position, then draw doubles u * 4.6566128752457969e-10. */
void orc_make_random_numbers(int64_t n, uint64_t s1, uint64_t s2, int64_t position, double *out) {
    build_jump_tables();
    uint32_t seed[5];
    orc_make_mrg_seed(s1, s2, seed);
    orc_mrg s;
    memcpy(s.z, seed, sizeof s.z);
    mrg_skip(&s, 2, 0, 2 * (uint64_t)position);
    for (int64_t i = 0; i < n; ++i) out[i] = (double)mrg_next(&s) * .0000000004656612875245796924106;
}

/* Scrambling keys, src/graph_generation.cu:290-300. */
void orc_scramble_keys(const uint32_t seed[5], uint64_t *val0, uint64_t *val1) {
    build_jump_tables();
    orc_mrg s;
    memcpy(s.z, seed, sizeof s.z);
    mrg_skip(&s, 50, 7, 0);
    uint64_t a = mrg_next(&s);
    a *= 0xFFFFFFFFull;
    a += mrg_next(&s);
    uint64_t b = mrg_next(&s);
    b *= 0xFFFFFFFFull;
    b += mrg_next(&s);
    *val0 = a;
    *val1 = b;
}

static inline uint64_t bitrev64(uint64_t x) {
    x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
    x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((x & 0x0F0F0F0F0F0F0F0Full) << 4);
    x = ((x >> 8) & 0x00FF00FF00FF00FFull) | ((x & 0x00FF00FF00FF00FFull) << 8);
    x = ((x >> 16) & 0x0000FFFF0000FFFFull) | ((x & 0x0000FFFF0000FFFFull) << 16);
    return (x >> 32) | (x << 32);
}

/* Vertex permutation, cuda_scramble src/graph_generation.cu:171-179. */
static inline uint64_t scramble(uint64_t v, int lgN, uint64_t val0, uint64_t val1) {
    v += val0 + val1;
    v *= (val0 | 0x4519840211493211ull);
    v = bitrev64(v) >> (64 - lgN);
    v *= (val1 | 0x3050852102C843A5ull);
    v = bitrev64(v) >> (64 - lgN);
    return v;
}

/* Quadrant draw, cuda_generate_4way_bernoulli src/graph_generation.cu:114-143
 * (SPK_NOISE_LEVEL 0): reject u < 2^31-1 mod 10^4, then thresholds on
 * u mod 10^4 with B = C = 1900/10^4 and A = 5700/10^4. */
static inline int quadrant(orc_mrg *s) {
    const uint32_t limit = MRG_P % 10000u;
    uint32_t u = mrg_next(s);
    while (u < limit) u = mrg_next(s);
    u %= 10000u;
    if (u < 1900u) return 1;
    u -= 1900u;
    if (u < 1900u) return 2;
    u -= 1900u;
    if (u < 5700u) return 0;
    return 3;
}

/* One edge and its weight, cuda_make_one_edge src/graph_generation.cu:186-207
 * plus the weight draw in generate_kronecker_kernel :225-238. */
static void make_edge(const orc_mrg *base, int64_t ei, int lgN, uint64_t val0, uint64_t val1,
                      uint64_t *src, uint64_t *dst, float *w) {
    orc_mrg s = *base;
    mrg_skip(&s, 0, (uint64_t)ei, 0);
    uint64_t nverts = (uint64_t)1 << lgN, bs = 0, bt = 0;
    while (nverts > 1) {
        int q = quadrant(&s);
        int so = q / 2, to = q % 2;
        if (bs == bt && so > to) { int t = so; so = to; to = t; }
        nverts /= 2;
        bs += nverts * (uint64_t)so;
        bt += nverts * (uint64_t)to;
    }
    *src = scramble(bs, lgN, val0, val1);
    *dst = scramble(bt, lgN, val0, val1);
    *w = (float)mrg_next(&s) * .000000000465661287524579692f;
}

/* generate_kronecker_range, src/graph_generation.cu:269-310: edges
 * [start, end) as (v0, v1) u64 pairs plus one float weight each. */
void orc_generate_kronecker_range(const uint32_t seed[5], int lgN, int64_t start, int64_t end,
                                  uint64_t *edges, float *weights, int nthreads) {
    build_jump_tables();
    if (end <= start) return;
    orc_mrg base;
    memcpy(base.z, seed, sizeof base.z);
    uint64_t val0, val1;
    orc_scramble_keys(seed, &val0, &val1);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static, 4096) num_threads(nthreads)
    for (int64_t i = 0; i < end - start; ++i)
        make_edge(&base, start + i, lgN, val0, val1, &edges[2 * i], &edges[2 * i + 1], &weights[i]);
}

/* ------------------------------------------------------------------ CSR */

/* Number of directed CSR entries: 2 per non-self-loop edge
 * (compute_degrees_kernel, src/traversal.cu:15-34). */
uint64_t orc_csr_count(const uint64_t *edges, uint64_t m, uint64_t nverts, uint64_t *deg_out,
                       int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    memset(deg_out, 0, nverts * sizeof(uint64_t));
    uint64_t total = 0;
#pragma omp parallel for reduction(+ : total) num_threads(nthreads)
    for (uint64_t e = 0; e < m; ++e) {
        uint64_t a = edges[2 * e], b = edges[2 * e + 1];
        if (a == b) continue;
        __atomic_fetch_add(&deg_out[a], 1, __ATOMIC_RELAXED);
        __atomic_fetch_add(&deg_out[b], 1, __ATOMIC_RELAXED);
        total += 2;
    }
    return total;
}

static int cmp_entry(const void *pa, const void *pb) {
    uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    return a < b ? -1 : a > b;
}

/* 1-D CSR of oned_graph_from_tuple_graph (src/traversal.cu:342-389) at one
 * rank: rowstarts = exclusive scan of the degrees (:37-46), both directions
 * of every non-loop edge scattered into its row (:48-73), duplicates kept.
 * The reference's in-row order depends on atomic order; with canonical != 0
 * each row is sorted by (dst, weight bits), which is the form parity is
 * checked in.  rowstarts has nverts+1 entries, col/w have orc_csr_count(). */
void orc_csr_build(const uint64_t *edges, const float *weights, uint64_t m, uint64_t nverts,
                   uint64_t *rowstarts, uint32_t *col, float *w, int canonical, int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    uint64_t *cursor = (uint64_t *)malloc(nverts * sizeof(uint64_t));
    orc_csr_count(edges, m, nverts, cursor, nthreads);
    uint64_t sum = 0;
    for (uint64_t v = 0; v < nverts; ++v) {
        rowstarts[v] = sum;
        sum += cursor[v];
        cursor[v] = rowstarts[v];
    }
    rowstarts[nverts] = sum;
#pragma omp parallel for num_threads(nthreads)
    for (uint64_t e = 0; e < m; ++e) {
        uint64_t a = edges[2 * e], b = edges[2 * e + 1];
        if (a == b) continue;
        uint64_t pa = __atomic_fetch_add(&cursor[a], 1, __ATOMIC_RELAXED);
        uint64_t pb = __atomic_fetch_add(&cursor[b], 1, __ATOMIC_RELAXED);
        col[pa] = (uint32_t)b;
        w[pa] = weights[e];
        col[pb] = (uint32_t)a;
        w[pb] = weights[e];
    }
    free(cursor);
    if (!canonical) return;
#pragma omp parallel num_threads(nthreads)
    {
        uint64_t cap = 0;
        uint64_t *tmp = NULL;
#pragma omp for schedule(dynamic, 1024)
        for (uint64_t v = 0; v < nverts; ++v) {
            uint64_t b = rowstarts[v], n = rowstarts[v + 1] - b;
            if (n < 2) continue;
            if (n > cap) { cap = n; tmp = (uint64_t *)realloc(tmp, cap * sizeof(uint64_t)); }
            for (uint64_t i = 0; i < n; ++i) {
                uint32_t wb;
                memcpy(&wb, &w[b + i], 4);
                tmp[i] = ((uint64_t)col[b + i] << 32) | wb;
            }
            qsort(tmp, n, sizeof(uint64_t), cmp_entry);
            for (uint64_t i = 0; i < n; ++i) {
                uint32_t wb = (uint32_t)tmp[i];
                col[b + i] = (uint32_t)(tmp[i] >> 32);
                memcpy(&w[b + i], &wb, 4);
            }
        }
        free(tmp);
    }
}

/* ------------------------------------------------------------- roots */

/* generate_bfs_roots, examples/graph500_runner.cu:43-74, with the
 * isolation test of oned_graph_is_vertex_isolated (src/traversal.cu:391-410). */
int orc_generate_bfs_roots(const uint64_t *rowstarts, uint64_t nverts, uint64_t s1, uint64_t s2,
                           uint64_t *roots, int max_roots) {
    uint64_t counter = 0;
    int count = 0;
    for (; count < max_roots; ++count) {
        uint64_t root = 0;
        int found = 0;
        for (;;) {
            double d[2];
            orc_make_random_numbers(2, s1, s2, (int64_t)counter, d);
            root = (uint64_t)((d[0] + d[1]) * (double)nverts) % nverts;
            counter += 2;
            if (counter > 2 * nverts) break;
            int dup = 0;
            for (int i = 0; i < count; ++i)
                if (roots[i] == root) { dup = 1; break; }
            if (dup) continue;
            if (rowstarts[root] == rowstarts[root + 1]) continue;
            found = 1;
            break;
        }
        if (!found) break;
        roots[count] = root;
    }
    return count;
}

/* --------------------------------------------------------------- BFS */

/* Level-synchronous top-down BFS with a compare-and-swap on the parent of
 * every discovered edge, as bfs_run_kernel does (src/traversal.cu:139-207):
 * pred = -1 for unreached vertices, pred[root] = root.  depth (not produced
 * by the reference's BFS; it is what bfs_compute_dist_from_pred derives,
 * :505-563) is -1 for unreached vertices and the level otherwise.
 * Returns the number of levels. */
void orc_bfs_clear(uint64_t nverts, int64_t *pred, int64_t *depth, int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads)
    for (uint64_t v = 0; v < nverts; ++v) { pred[v] = -1; depth[v] = -1; }
}

/* The search of orc_bfs on arrays already cleared by orc_bfs_clear (the
 * runner keeps oned_graph_bfs_clear outside its timed region,
 * examples/graph500_runner.cu:309-313). */
int orc_bfs_search(const uint64_t *rowstarts, const uint32_t *col, uint64_t nverts, uint64_t root,
                   int64_t *pred, int64_t *depth, int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    uint32_t *cur = (uint32_t *)malloc(nverts * sizeof(uint32_t));
    uint32_t *nxt = (uint32_t *)malloc(nverts * sizeof(uint32_t));
    uint64_t ncur = 1, nnext = 0;
    cur[0] = (uint32_t)root;
    pred[root] = (int64_t)root;
    depth[root] = 0;
    int level = 0;
    while (ncur) {
        nnext = 0;
#pragma omp parallel num_threads(nthreads)
        {
            uint32_t buf[1024];
            int nb = 0;
#pragma omp for schedule(dynamic, 64)
            for (uint64_t i = 0; i < ncur; ++i) {
                uint32_t u = cur[i];
                for (uint64_t e = rowstarts[u]; e < rowstarts[u + 1]; ++e) {
                    uint32_t v = col[e];
                    int64_t expect = -1;
                    if (__atomic_load_n(&pred[v], __ATOMIC_RELAXED) != -1) continue;
                    if (__atomic_compare_exchange_n(&pred[v], &expect, (int64_t)u, 0,
                                                    __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                        depth[v] = level + 1;
                        buf[nb++] = v;
                        if (nb == 1024) {
                            uint64_t at = __atomic_fetch_add(&nnext, (uint64_t)nb, __ATOMIC_RELAXED);
                            memcpy(nxt + at, buf, nb * sizeof(uint32_t));
                            nb = 0;
                        }
                    }
                }
            }
            if (nb) {
                uint64_t at = __atomic_fetch_add(&nnext, (uint64_t)nb, __ATOMIC_RELAXED);
                memcpy(nxt + at, buf, nb * sizeof(uint32_t));
            }
        }
        uint32_t *t = cur; cur = nxt; nxt = t;
        ncur = nnext;
        ++level;
    }
    free(cur);
    free(nxt);
    return level;
}

int orc_bfs(const uint64_t *rowstarts, const uint32_t *col, uint64_t nverts, uint64_t root,
            int64_t *pred, int64_t *depth, int nthreads) {
    orc_bfs_clear(nverts, pred, depth, nthreads);
    return orc_bfs_search(rowstarts, col, nverts, root, pred, depth, nthreads);
}

/* bfs_compute_dist_from_pred, src/traversal.cu:505-563 with the kernels at
 * :75-112: dist = -1 where pred = -1, INT64_MAX otherwise, 0 at the root;
 * then level by level every vertex at level L labels each CSR neighbour dst
 * with pred[dst] == it and dist[dst] == INT64_MAX as L+1, until a level
 * labels nothing. */
void orc_bfs_dist_from_pred(const uint64_t *rowstarts, const uint32_t *col, uint64_t nverts,
                            const int64_t *pred, uint64_t root, int64_t *dist) {
    for (uint64_t v = 0; v < nverts; ++v) dist[v] = pred[v] == -1 ? -1 : INT64_MAX;
    dist[root] = 0;
    for (int64_t level = 0;; ++level) {
        uint64_t labelled = 0;
        for (uint64_t u = 0; u < nverts; ++u) {
            if (dist[u] != level) continue;
            for (uint64_t e = rowstarts[u]; e < rowstarts[u + 1]; ++e) {
                uint32_t v = col[e];
                if (pred[v] != (int64_t)u) continue;
                if (dist[v] == INT64_MAX) { dist[v] = level + 1; ++labelled; }
            }
        }
        if (!labelled) break;
    }
}

/* The runner's seven BFS validation rules, examples/graph500_runner.cu:84-169
 * (init :84-109, edges :111-153, confirmation :155-169).  Returns the error
 * count that kernel sequence accumulates. */
uint64_t orc_bfs_validate(const uint64_t *rowstarts, const uint32_t *col, uint64_t nverts,
                          uint64_t root, const int64_t *pred, const int64_t *dist) {
    uint64_t err = 0;
    uint8_t *confirmed = (uint8_t *)calloc(nverts, 1);
    for (uint64_t v = 0; v < nverts; ++v) {
        int64_t p = pred[v];
        if (p != -1 && (p < 0 || (uint64_t)p >= nverts)) ++err;
        if (v == root) {
            if (p != (int64_t)root || dist[v] != 0) ++err;
            else confirmed[v] = 1;
        }
    }
    for (uint64_t u = 0; u < nverts; ++u) {
        int64_t up = pred[u], ud = dist[u];
        for (uint64_t e = rowstarts[u]; e < rowstarts[u + 1]; ++e) {
            uint64_t v = col[e];
            if (v == u) { ++err; continue; }
            int64_t vp = pred[v], vd = dist[v];
            if ((ud == -1 && vd != -1) || (ud != -1 && vd == -1)) ++err;
            if (ud >= 0 && vd >= 0 && (ud + 1 < vd || vd + 1 < ud)) ++err;
            if (up == (int64_t)v) confirmed[u] = 1;
            if (vp == (int64_t)u) confirmed[v] = 1;
        }
    }
    for (uint64_t v = 0; v < nverts; ++v) {
        if (pred[v] == -1) continue;
        if (dist[v] == INT64_MAX || (v != root && !confirmed[v])) ++err;
    }
    free(confirmed);
    return err;
}

/* TEPS edge count, bfs_edge_count_kernel examples/graph500_runner.cu:171-182:
 * CSR entries col[e] <= v over rows of reached vertices v. */
uint64_t orc_edge_count(const uint64_t *rowstarts, const uint32_t *col, uint64_t nverts,
                        const int64_t *pred) {
    uint64_t n = 0;
#pragma omp parallel for reduction(+ : n) schedule(dynamic, 4096)
    for (uint64_t v = 0; v < nverts; ++v) {
        if (pred[v] == -1) continue;
        for (uint64_t e = rowstarts[v]; e < rowstarts[v + 1]; ++e) n += col[e] <= v;
    }
    return n;
}

/* -------------------------------------------------------------- SSSP */

typedef struct { float d; uint32_t v; } heap_item;

static void heap_push(heap_item *h, uint64_t *n, heap_item x) {
    uint64_t i = (*n)++;
    while (i) {
        uint64_t p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = x;
}

static heap_item heap_pop(heap_item *h, uint64_t *n) {
    heap_item top = h[0], x = h[--(*n)];
    uint64_t i = 0;
    for (;;) {
        uint64_t c = 2 * i + 1;
        if (c >= *n) break;
        if (c + 1 < *n && h[c + 1].d < h[c].d) ++c;
        if (x.d <= h[c].d) break;
        h[i] = h[c];
        i = c;
    }
    h[i] = x;
    return top;
}

/* Single-source shortest paths in binary32.  The reference computes these
 * distances by delta-stepping (oned_graph_sssp_run, src/traversal.cu:638-711,
 * relaxation :211-240): each relaxation is candidate = dist[u] + w in float,
 * kept when it is below the current value, and the export writes -1.0f for
 * unreached vertices (:333-340).  With non-negative weights and monotone
 * rounding the fixed point of those relaxations is unique -- the minimum
 * over paths of the left-to-right float path sum -- so Dijkstra with the
 * same float addition reaches the same bits.  pred[root] = root, -1 for
 * unreached vertices. */
void orc_sssp(const uint64_t *rowstarts, const uint32_t *col, const float *w, uint64_t nverts,
              uint64_t root, float *dist, int64_t *pred) {
    const float inf = INFINITY;
    for (uint64_t v = 0; v < nverts; ++v) { dist[v] = inf; pred[v] = -1; }
    uint64_t cap = rowstarts[nverts] + 1, n = 0;
    heap_item *h = (heap_item *)malloc(cap * sizeof(heap_item));
    uint8_t *done = (uint8_t *)calloc(nverts, 1);
    dist[root] = 0.0f;
    pred[root] = (int64_t)root;
    heap_push(h, &n, (heap_item){0.0f, (uint32_t)root});
    while (n) {
        heap_item it = heap_pop(h, &n);
        uint32_t u = it.v;
        if (done[u]) continue;
        done[u] = 1;
        float du = dist[u];
        for (uint64_t e = rowstarts[u]; e < rowstarts[u + 1]; ++e) {
            uint32_t v = col[e];
            volatile float cand = du + w[e];
            if (cand < dist[v]) {
                dist[v] = cand;
                pred[v] = u;
                heap_push(h, &n, (heap_item){cand, v});
            }
        }
    }
    for (uint64_t v = 0; v < nverts; ++v)
        if (dist[v] == inf) dist[v] = -1.0f;
    free(h);
    free(done);
}

/* SSSP validation.  The reference has none; these are the Graph500 SSSP
 * rules stated for exact binary32 distances (dist = -1 unreached):
 *  1. dist[root] == 0 and pred[root] == root;
 *  2. pred[v] == -1 exactly when dist[v] == -1, and pred is in range;
 *  3. no CSR edge (u, v, w) from a reached u reaches an unreached v or has
 *     dist[u] + w < dist[v] (the distances are a fixed point);
 *  4. every reached v != root has an edge (pred[v], v, w) with
 *     dist[pred[v]] + w == dist[v].
 * Returns the number of violations. */
uint64_t orc_sssp_validate(const uint64_t *rowstarts, const uint32_t *col, const float *w,
                           uint64_t nverts, uint64_t root, const float *dist, const int64_t *pred) {
    uint64_t err = 0;
    uint8_t *confirmed = (uint8_t *)calloc(nverts, 1);
    if (dist[root] != 0.0f || pred[root] != (int64_t)root) ++err;
    confirmed[root] = 1;
    for (uint64_t v = 0; v < nverts; ++v) {
        int64_t p = pred[v];
        if ((p == -1) != (dist[v] == -1.0f)) ++err;
        if (p != -1 && (p < 0 || (uint64_t)p >= nverts)) ++err;
    }
    for (uint64_t u = 0; u < nverts; ++u) {
        float du = dist[u];
        if (du == -1.0f) continue;
        for (uint64_t e = rowstarts[u]; e < rowstarts[u + 1]; ++e) {
            uint32_t v = col[e];
            float dv = dist[v];
            volatile float cand = du + w[e];
            if (dv == -1.0f || cand < dv) ++err;
            if (pred[v] == (int64_t)u && cand == dv) confirmed[v] = 1;
        }
    }
    for (uint64_t v = 0; v < nverts; ++v)
        if (dist[v] != -1.0f && !confirmed[v]) ++err;
    free(confirmed);
    return err;
}

int orc_num_threads(void) { return omp_get_max_threads(); }
