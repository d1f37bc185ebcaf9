// bfs.cu -- K3: direction-optimizing BFS in one persistent cooperative
// kernel (replaces the reference's top-down bfs_run_kernel,
// src/traversal.cu:139-207, and its host wrapper :479-503), plus
// bfs_compute_dist_from_pred (:505-563).
//
// Every level runs inside one launch; the grid meets at a bounded barrier
// after each level and every block takes the same direction decision from
// the same counters, so nothing returns to the host between levels.
//
// Top-down level: the frontier is a queue.  Vertices of degree <= BIG_DEG
// are taken 32 at a time by a warp, which prefix-sums their degrees and
// walks the combined edge list 32 edges per step (each lane finds its
// source by a 5-step shuffle search), so low-degree vertices do not leave
// lanes idle.  Vertices above BIG_DEG sit at the back of the queue and every
// warp of the grid takes BFS_CHUNK-edge chunks of them from one counter
// (g5_frontier.cuh); a chunk is a chain of BFS_CHUNK / 32 dependent steps of
// one warp, so it bounds the longest warp of a level.  Both sizes are
// defaults of g5_bfs_params.big_deg / .chunk, which a tuner may change.  A neighbour is claimed with an atomicOr on the visited bitmap;
// the winner writes pred/depth and appends it to the next queue with one
// atomic per warp.
//
// Bottom-up level: a warp owns a 32-vertex word of the visited bitmap; each
// lane whose vertex is unvisited scans its row until a neighbour is in the
// frontier bitmap.  Both bitmaps are N/8 bytes (8 MiB at SCALE 26) and stay
// resident in the 126 MB L2; the owner warp writes both words without
// atomics.
//
// Switching (Beamer et al.): top-down -> bottom-up when the frontier's edges
// exceed the unvisited vertices' edges / alpha; back when the frontier has
// fewer than N / beta vertices and is shrinking.
//
// Algorithmic bytes per search (one component of n_c vertices and m_c
// undirected edges): 2 m_c * 4 (col) + n_c * (8 rowstarts + 8 pred + 4 depth).
#include <algorithm>
#include <atomic>
#include <mutex>

#include <chrono>
#include <new>

#include "g5_common.cuh"
#include "g5_frontier.cuh"

namespace g5 {

constexpr int BFS_THREADS = 256;
constexpr unsigned BFS_CHUNK = 256;  // default: edges of a long row taken by one warp
constexpr unsigned BFS_BIG_DEG = BIG_DEG;  // default: longest row expanded by one warp
constexpr unsigned BFS_STAGE = 512;  // per-warp staging of the next queue (16 KiB shared per block)
constexpr unsigned long long SOLO_EDGES = 4096;  // levels at most this wide run in block 0 alone
constexpr int BFS_TRACE = 64;                    // levels recorded in the control block

// State every thread keeps identically between levels (also handed from
// the solo prologue to the grid through the control block).
struct LevelState {
    int level, mode, cur, pending, levels, bu_levels;
    unsigned n_f;
    unsigned ucur;  // bottom-up: the unvisited list is q[ucur] (q[ucur ^ 1] takes the survivors)
    unsigned long long m_f, m_u, reached;
};
static_assert(sizeof(LevelState) % 8 == 0, "LevelState is copied in 8-byte words");

struct BfsCtl {
    g5_bfs_stats res;     // the search's result (same layout as the C ABI's)
    const uint32_t *init_used;  // visited bitmap the last reset started from (nullptr: all clear)
    unsigned bar;         // grid barrier arrivals
    unsigned n_small[3];  // per level slot: queue entries of degree <= BIG_DEG
    unsigned long long big[3];  //           big entries << 40 | their chunks
    unsigned grab[3];     //                 work cursor over the small part
    unsigned cgrab[3];    //                 work cursor over the big part's chunks
    unsigned found[3];    //                 vertices found by a bottom-up level
    unsigned ulen[3];     //                 bottom-up: entries of the unvisited list
    unsigned long long m_next[3];  //        degree sum of the next frontier
    // hand-off from the solo prologue to the grid
    unsigned long long go;  // launch sequence << 2 | 1 (continue on the grid) or 2 (finished)
    unsigned heartbeat;     // solo levels completed so far (waiters restart their clock on change)
    unsigned hand_fb;  // 1 when the frontier bitmap is the second buffer
    LevelState hand;
    // per-level trace: time at the level's end, frontier size and edges, direction
    unsigned long long t0;
    unsigned long long t_level[BFS_TRACE];
    unsigned long long m_level[BFS_TRACE];
    unsigned n_level[BFS_TRACE];
    unsigned char mode_level[BFS_TRACE];
    // g5_bfs_export: records appended, blocks finished, the final count
    unsigned long long xcount, xresult;
    unsigned xdone;
};

// What the last search on a workspace wrote, for g5_bfs_reset_touched.
// Only the search kernels write it (every block of the reset reads it): the
// one-block search lists the vertices it reached (the touched list) and
// records its outputs and the visited bitmap its reset started from; any
// other search clears `small`, which makes the next reset a full one.
struct BfsTouch {
    unsigned small;
    unsigned pad;
    unsigned long long count;  // vertices in the touched list
    int64_t *pred;
    int32_t *depth;
    const uint32_t *init;
};

struct BfsArgs {
    const uint64_t *rowptr;
    const int *col;
    uint64_t n;
    uint64_t nwords;
    unsigned root;
    int64_t *pred;
    int *depth;
    unsigned *visited;
    unsigned *fbits;
    unsigned *nbits;
    unsigned *zbits;    // third frontier bitmap: bottom-up levels rotate fb -> zb -> nb
    unsigned *q[2];
    unsigned *base[2];  // chunk bases of each queue's big part
    BfsCtl *ctl;
    float alpha;
    float beta;
    int mode;
    unsigned nblocks;
    unsigned long long limit_ns;
    g5_bfs_stats *stats_out;  // the caller's mapped pinned host statistics, or nullptr
    unsigned long long seq;  // unique per launch: releases only this launch's waiting blocks
    const uint64_t *roots;   // several roots at once (device array) instead of `root`, or nullptr
    unsigned nroots;
    BfsTouch *touch;
    unsigned *tlist;  // touched list of the one-block search (n entries)
    // The one-block search's own export of its result (g5_bfs_query_plan_export):
    // records into xout (device-addressable, xcap of them), then the count to
    // pinned host memory (xcount_map).  nullptr: no export.
    g5_bfs_reached *xout;
    uint64_t xcap;
    unsigned long long *xcount_map;
    unsigned big_deg;       // queue entries with more edges go to the chunked big part
    unsigned chunk;         // edges of a big entry per warp grab (a multiple of 32)
    unsigned lane_entries;  // bottom-up: row head a lane scans alone (a multiple of BU_STEP)
    const unsigned *top;    // bottom-up: each vertex's first row entry, dense (nullptr: none)
};

enum { TOP_DOWN = 0, BOTTOM_UP = 1 };
constexpr int BFS_SMALL = 3;  // g5_bfs_params.mode: one lean block, for a root in a small component

static_assert(sizeof(g5_bfs_reached) == 16, "one 16-byte store a record");

// One record as one 16-byte store (a single bus write when `out` is host
// memory): {vertex, depth} then the parent, the g5_bfs_reached layout.
__device__ __forceinline__ void put_reached(g5_bfs_reached *out, uint64_t i, unsigned v, int d, int64_t p) {
    reinterpret_cast<ulonglong2 *>(out)[i] =
        make_ulonglong2((unsigned long long)v | (unsigned long long)(unsigned)d << 32, (unsigned long long)p);
}


// Bottom-up: entries of a row a lane scans on its own before the rest of
// the row goes to the whole warp (default of g5_bfs_params.lane_entries).
constexpr unsigned BU_LANE_ENTRIES = 8;
constexpr int BU_STEP = 4;  // entries per lane step (loads issued together)

// Claim v for parent u at the next level; appends it to the next queue.
// All 32 lanes must call it (want = this lane has a candidate).
__device__ __forceinline__ void td_visit(const BfsArgs &a, const WarpStage &bq, bool want, unsigned v, unsigned u,
                                         int next_level, unsigned *qn, unsigned *basen, unsigned *n_small,
                                         unsigned long long *n_big, unsigned long long &my_m) {
    if (want && v >= a.n) {  // not a vertex: report it, touch nothing
        atomicOr(&a.ctl->res.error_flags, DEVERR_RANGE);
        want = false;
    }
    bool disc = want && bit_claim(a.visited, v);
    if (!__any_sync(FULL, disc)) return;  // nothing new in this warp step
    uint64_t deg = 0;
    if (disc) {
        a.pred[v] = (int64_t)u;
        if (a.depth) a.depth[v] = next_level;
        deg = __ldg(&a.rowptr[v + 1]) - __ldg(&a.rowptr[v]);
        my_m += deg;
    }
    if (!frontier_append_staged(bq, qn, basen, a.n, n_small, n_big, disc, v, deg, a.big_deg, a.chunk))
        atomicOr(&a.ctl->res.error_flags, DEVERR_CAPACITY);
}

__device__ void td_expand(const BfsArgs &a, const WarpStage &bq, int level, int cur, int s_cur, int s_nxt,
                          unsigned long long &my_m) {
    BfsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const unsigned *Q = a.q[cur];
    unsigned *QN = a.q[cur ^ 1];
    const unsigned *B = a.base[cur];
    unsigned *BN = a.base[cur ^ 1];
    const unsigned ns = ld_volatile(&c->n_small[s_cur]);
    const unsigned long long bp = ld_volatile(&c->big[s_cur]);

    // Small part: g queue entries per grab, edges gathered across the warp.
    const unsigned g = grab_size(ns, ((unsigned long long)gridDim.x * blockDim.x) >> 5);
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&c->grab[s_cur], g);
        base = __shfl_sync(FULL, base, 0);
        if (base >= ns) break;
        const unsigned i = base + lane;
        const bool valid = lane < g && i < ns;
        const unsigned u = valid ? __ldcg(&Q[i]) : 0u;
        const uint64_t rb = valid ? __ldg(&a.rowptr[u]) : 0;
        const unsigned deg = valid ? (unsigned)(__ldg(&a.rowptr[u + 1]) - rb) : 0u;
        const unsigned incl = warp_incl_scan(deg);
        const unsigned total = __shfl_sync(FULL, incl, 31);
        const unsigned excl = incl - deg;
        for (unsigned e0 = 0; e0 < total; e0 += 32) {
            const unsigned e = e0 + lane;
            const bool has = e < total;
            const int j = warp_owner(excl, has ? e : total - 1);
            const unsigned uj = __shfl_sync(FULL, u, j);
            const uint64_t rbj = __shfl_sync(FULL, rb, j);
            const unsigned exj = __shfl_sync(FULL, excl, j);
            const unsigned v = has ? (unsigned)__ldg(&a.col[rbj + (e - exj)]) : 0u;
            td_visit(a, bq, has, v, uj, level + 1, QN, BN, &c->n_small[s_nxt], &c->big[s_nxt], my_m);
        }
    }
    // Big part: chunks of every big vertex from one grid-wide counter.
    const unsigned nb = big_count(bp);
    const unsigned long long nch = big_chunks(bp);
    for (;;) {
        unsigned ch = 0;
        if (lane == 0) ch = atomicAdd(&c->cgrab[s_cur], 1u);
        ch = __shfl_sync(FULL, ch, 0);
        if (ch >= nch) break;
        const unsigned j = chunk_owner(B, nb, ch);
        const unsigned u = __ldcg(&Q[a.n - 1 - j]);
        const uint64_t rb = __ldg(&a.rowptr[u]);
        const uint64_t deg = __ldg(&a.rowptr[u + 1]) - rb;
        const uint64_t cs = (uint64_t)(ch - __ldcg(&B[j])) * a.chunk;
        const uint64_t ce = min(cs + a.chunk, deg);
        for (uint64_t e = cs + lane; e < cs + a.chunk; e += 32) {
            const bool has = e < ce;
            const unsigned v = has ? (unsigned)__ldg(&a.col[rb + e]) : 0u;
            td_visit(a, bq, has, v, u, level + 1, QN, BN, &c->n_small[s_nxt], &c->big[s_nxt], my_m);
        }
    }
    if (!stage_flush_warp(bq, QN, a.n, &c->n_small[s_nxt])) atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
}

__device__ void bu_expand(const BfsArgs &a, const WarpStage &bq, const LevelState &st, int s_cur, int s_nxt,
                          const unsigned *fb, unsigned *nb, unsigned *zb, unsigned long long &my_m,
                          unsigned &my_found) {
    BfsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    // The unvisited vertices are a list (built when the search turned
    // bottom-up, then the survivors of each level), 32 per warp step, so a
    // level costs its unvisited vertices, not N/32 bitmap words with a few
    // live lanes each.  Found vertices set their visited and next-frontier
    // bits with atomics (a word's vertices are spread over warps).
    const unsigned *U = a.q[st.ucur];
    unsigned *UN = a.q[st.ucur ^ 1];
    const uint64_t len = ld_volatile(&c->ulen[s_cur]);
    // zb, the frontier bitmap of the level before, becomes the clean
    // next-frontier bitmap of the level after; nobody reads it now.
    for (uint64_t k = gtid; k < a.nwords; k += nthreads) zb[k] = 0;
    // Software pipeline over the warp's chunks of 32 entries: while chunk j
    // is scanned, the row bounds of chunk j+1 and the list entries of chunk
    // j+2 are in flight.
    constexpr unsigned NONE = 0xffffffffu;
    auto ent = [&](uint64_t ch) -> unsigned {
        const uint64_t i = ch * 32 + lane;
        return i < len ? __ldcg(&U[i]) : NONE;
    };
    auto bounds = [&](unsigned vv, uint64_t &b, uint64_t &e) {
        b = e = 0;
        if (vv < a.n) {
            b = __ldg(&a.rowptr[vv]);
            e = __ldg(&a.rowptr[vv + 1]);
        }
    };
    // Each vertex's first row entry, from the dense array when there is one
    // (coalesced: the list is in vertex order), loaded with the row bounds.
    // Probed on every bottom-up level: S26 main-component searches 1.62 ms
    // against 1.74 ms without it; gating it on the frontier's size (a miss
    // puts a round trip in front of the row scan) measured no better.
    const bool use_top = a.top != nullptr;
    auto first = [&](unsigned vv) -> unsigned { return use_top && vv < a.n ? __ldg(&a.top[vv]) : a.n; };
    const uint64_t nch = (len + 31) / 32;
    unsigned v_n = ent(warp), v_nn = ent(warp + nwarps);
    uint64_t rb_n, re_n;
    bounds(v_n, rb_n, re_n);
    unsigned t_n = first(v_n);
    for (uint64_t ch = warp; ch < nch; ch += nwarps) {
        const unsigned v = v_n;
        const uint64_t rb = rb_n, re = re_n;
        const unsigned t = t_n;
        v_n = v_nn;
        bounds(v_n, rb_n, re_n);
        t_n = first(v_n);
        v_nn = ent(ch + 2 * nwarps);
        if (v != NONE && v >= a.n) atomicOr(&c->res.error_flags, DEVERR_RANGE);
        const bool live = v < a.n;
        int found = -1;
        uint64_t e = rb;  // next entry of the row to look at
        if (use_top && live && rb < re) {
            // The first neighbour (the best connected one, with rows by
            // decreasing degree) without reading the row: most hits.
            if (t < a.n && ((__ldcg(&fb[t >> 5]) >> (t & 31)) & 1u)) found = (int)t;
            else e = rb + 1;  // the lane scan starts after it
        }
        if (live && found < 0) {
            // Each lane scans the head of its own row, BU_STEP neighbours per
            // step: their loads and bitmap probes are independent, so a step
            // costs one memory round trip, not BU_STEP.
            const uint64_t head = min(re, rb + a.lane_entries);
            for (; e < head && found < 0; e += BU_STEP) {
                unsigned u[BU_STEP], word[BU_STEP];
#pragma unroll
                for (int i = 0; i < BU_STEP; ++i) u[i] = e + i < re ? (unsigned)__ldg(&a.col[e + i]) : a.n;
#pragma unroll
                for (int i = 0; i < BU_STEP; ++i) word[i] = u[i] < a.n ? __ldcg(&fb[u[i] >> 5]) : 0u;
#pragma unroll
                for (int i = 0; i < BU_STEP; ++i) {
                    if (e + i < re && u[i] >= a.n) atomicOr(&c->res.error_flags, DEVERR_RANGE);
                    if (found < 0 && u[i] < a.n && ((word[i] >> (u[i] & 31)) & 1u)) found = (int)u[i];
                }
            }
        }
        // The rest of every longer row is scanned by the whole warp, 32
        // consecutive entries per step (coalesced), stopping at the first
        // step with a hit; the row's first frontier neighbour is taken, as
        // in the lane scan.
        unsigned longrows = __ballot_sync(FULL, live && found < 0 && e < re);
        while (longrows) {
            const int src = __ffs(longrows) - 1;
            longrows &= longrows - 1;
            const uint64_t b0 = __shfl_sync(FULL, e, src), end = __shfl_sync(FULL, re, src);
            int hitv = -1;
            for (uint64_t x0 = b0; x0 < end; x0 += 32) {
                const uint64_t xe = x0 + lane;
                const unsigned u = xe < end ? (unsigned)__ldg(&a.col[xe]) : a.n;
                if (xe < end && u >= a.n) atomicOr(&c->res.error_flags, DEVERR_RANGE);
                const bool hit = u < a.n && ((__ldcg(&fb[u >> 5]) >> (u & 31)) & 1u);
                const unsigned m = __ballot_sync(FULL, hit);
                if (m) {
                    hitv = (int)__shfl_sync(FULL, u, __ffs(m) - 1);
                    break;
                }
            }
            if (lane == (unsigned)src) found = hitv;
        }
        if (found >= 0) {
            a.pred[v] = found;
            if (a.depth) a.depth[v] = st.level + 1;
            const unsigned bit = 1u << (v & 31);
            atomicOr(&a.visited[v >> 5], bit);
            atomicOr(&nb[v >> 5], bit);
            my_m += re - rb;
            ++my_found;
        }
        // Vertices still unvisited go on to the next level's list.
        if (!stage_append(bq, live && found < 0, v, UN, a.n, &c->ulen[s_nxt]))
            atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
    }
    if (!stage_flush_warp(bq, UN, a.n, &c->ulen[s_nxt])) atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
}

// The unvisited vertices (visited bit clear) as a list in L, count in
// *count: each warp counts its words' vertices, reserves its range with one
// atomicAdd, then writes them in a second pass over the same words -- 16
// words at a time gathered in the warp's shared staging buffer (at most 512
// vertices) and copied out with coalesced stores.
__device__ void build_unvisited(const BfsArgs &a, const WarpStage &bq, unsigned *L, unsigned *count) {
    const unsigned lane = lane_id();
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    auto live_bits = [&](uint64_t k) -> unsigned {
        if (k >= a.nwords) return 0u;
        unsigned m = ~__ldcg(&a.visited[k]);
        const uint64_t v0 = k * 32;
        if (v0 + 32 > a.n) m &= (1u << (a.n - v0)) - 1u;
        return m;
    };
    static_assert(BFS_STAGE >= 16 * 32, "16 words of vertices fit the staging buffer");
    unsigned long long mine = 0;
    for (uint64_t base = warp * 32; base < a.nwords; base += nwarps * 32) mine += __popc(live_bits(base + lane));
    const unsigned long long total = warp_sum(mine);
    unsigned long long off = 0;
    if (lane == 0 && total) off = atomicAdd(count, (unsigned)total);
    off = __shfl_sync(FULL, off, 0);
    for (uint64_t base = warp * 32; base < a.nwords; base += nwarps * 32) {
        for (unsigned half = 0; half < 32; half += 16) {
            const uint64_t k = base + half + lane;
            unsigned m = lane < 16 ? live_bits(k) : 0u;
            const unsigned p = __popc(m);
            const unsigned incl = warp_incl_scan(p);
            const unsigned t = __shfl_sync(FULL, incl, 31);
            unsigned at = incl - p;
            while (m) {
                bq.buf[at++] = (unsigned)(k * 32 + __ffs(m) - 1);
                m &= m - 1;
            }
            __syncwarp();
            for (unsigned i = lane; i < t; i += 32) L[off + i] = bq.buf[i];
            __syncwarp();
            off += t;
        }
    }
}

// Frontier queue from a bottom-up bitmap (small/big split by degree).
__device__ void bits_to_queue(const BfsArgs &a, const WarpStage &bq, const unsigned *bits, unsigned *qn,
                              unsigned *basen, unsigned *n_small, unsigned long long *n_big) {
    const unsigned lane = lane_id();
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < a.nwords; base += nwarps * 32) {
        const uint64_t k = base + lane;
        unsigned m = k < a.nwords ? __ldcg(&bits[k]) : 0u;
        unsigned cnt = __popc(m);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) cnt = max(cnt, __shfl_xor_sync(FULL, cnt, d));
        for (unsigned it = 0; it < cnt; ++it) {
            const bool has = m != 0;
            unsigned v = 0;
            uint64_t deg = 0;
            if (has) {
                v = (unsigned)(k * 32 + __ffs(m) - 1);
                m &= m - 1;
                deg = __ldg(&a.rowptr[v + 1]) - __ldg(&a.rowptr[v]);
            }
            if (!frontier_append_staged(bq, qn, basen, a.n, n_small, n_big, has, v, deg, a.big_deg, a.chunk))
                atomicOr(&a.ctl->res.error_flags, DEVERR_CAPACITY);
        }
    }
    if (!stage_flush_warp(bq, qn, a.n, n_small)) atomicOr(&a.ctl->res.error_flags, DEVERR_CAPACITY);
}

// Direction of the next level (Beamer's rule; a.mode forces one side).
__device__ __forceinline__ int bfs_decide(const BfsArgs &a, int mode, unsigned n_next, unsigned long long m_next,
                                          unsigned long long m_u, unsigned n_f, unsigned long long reached) {
    if (a.mode == 1) return TOP_DOWN;
    if (a.mode == 2) return BOTTOM_UP;
    // Beamer's rule, plus: a bottom-up level touches every unvisited vertex,
    // so it never pays when the frontier's edges are few next to them (late
    // levels, where unexplored edges belong to other components).
    if (mode == TOP_DOWN)
        return ((double)m_next > (double)m_u / a.alpha && 32.0 * (double)m_next > (double)(a.n - reached))
                   ? BOTTOM_UP
                   : TOP_DOWN;
    return ((double)n_next < (double)a.n / a.beta && n_next < n_f) ? TOP_DOWN : BOTTOM_UP;
}

enum { PEND_NONE = 0, PEND_TO_BITS = 1, PEND_TO_QUEUE = 2 };

// Expands level st.level; adds the next frontier's degree sum and (bottom-up)
// size into slot s_nxt.  No synchronisation.
__device__ __forceinline__ void bfs_expand_level(const BfsArgs &a, const WarpStage &bq, const LevelState &st,
                                                 const unsigned *fb, unsigned *nb, unsigned *zb) {
    BfsCtl *c = a.ctl;
    const int s_cur = st.level % 3, s_nxt = (st.level + 1) % 3, s_clr = (st.level + 2) % 3;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->n_small[s_clr] = 0;
        c->big[s_clr] = 0;
        c->grab[s_clr] = 0;
        c->cgrab[s_clr] = 0;
        c->found[s_clr] = 0;
        c->ulen[s_clr] = 0;
        c->m_next[s_clr] = 0;
    }
    unsigned long long my_m = 0;
    unsigned my_found = 0;
    if (st.mode == TOP_DOWN)
        td_expand(a, bq, st.level, st.cur, s_cur, s_nxt, my_m);
    else
        bu_expand(a, bq, st, s_cur, s_nxt, fb, nb, zb, my_m, my_found);
    my_m = warp_sum(my_m);
    my_found = warp_sum(my_found);
    if (lane_id() == 0) {
        if (my_m) atomicAdd(&c->m_next[s_nxt], my_m);
        if (my_found) atomicAdd(&c->found[s_nxt], my_found);
    }
}

// After the level's barrier: next frontier size/edges, trace, direction.
// Returns false when the search is over.
__device__ __forceinline__ bool bfs_advance(const BfsArgs &a, LevelState &st, unsigned *&fb, unsigned *&nb,
                                            unsigned *&zb) {
    BfsCtl *c = a.ctl;
    const int s_nxt = (st.level + 1) % 3;
    const unsigned long long m_next = ld_volatile(&c->m_next[s_nxt]);
    const unsigned n_next = st.mode == TOP_DOWN ? ld_volatile(&c->n_small[s_nxt]) + big_count(ld_volatile(&c->big[s_nxt]))
                                                : ld_volatile(&c->found[s_nxt]);
    if (blockIdx.x == 0 && threadIdx.x == 0 && st.level < BFS_TRACE) {
        c->t_level[st.level] = globaltimer_ns();
        c->n_level[st.level] = st.n_f;
        c->m_level[st.level] = st.m_f;
        c->mode_level[st.level] = (unsigned char)st.mode;
    }
    ++st.levels;
    st.bu_levels += st.mode == BOTTOM_UP;
    st.m_u -= m_next;
    st.reached += n_next;
    if (n_next == 0) return false;
    const int next = bfs_decide(a, st.mode, n_next, m_next, st.m_u, st.n_f, st.reached);
    if (st.mode == TOP_DOWN) {
        st.cur ^= 1;  // the next frontier queue is now q[cur]
        if (next == BOTTOM_UP) st.pending = PEND_TO_BITS;
    } else {
        unsigned *t = fb;  // the next frontier bitmap is now fb; zb (cleared) the next one's
        fb = nb;
        nb = zb;
        zb = t;
        st.ucur ^= 1;  // the survivors are the next level's unvisited list
        if (next == TOP_DOWN) st.pending = PEND_TO_QUEUE;
    }
    st.mode = next;
    st.n_f = n_next;
    st.m_f = m_next;
    ++st.level;
    return true;
}

// Copies the finished search's statistics to the caller's mapped host
// memory (g5_bfs_query): `levels` last, after a system-scope fence, so a
// host that set it to -1 before the launch and sees it change knows the
// search -- its outputs and every other statistic -- is complete, without
// waiting for the kernel's exit to reach the stream.
__device__ __forceinline__ void bfs_publish_stats(const BfsArgs &a) {
    if (!a.stats_out) return;
    volatile g5_bfs_stats *r = &a.ctl->res;
    volatile g5_bfs_stats *o = a.stats_out;
    o->bottom_up_levels = r->bottom_up_levels;
    o->reached = r->reached;
    o->error_flags = r->error_flags;
    o->solo_levels = r->solo_levels;
    __threadfence_system();
    o->levels = r->levels;
}

__device__ __forceinline__ void bfs_write_stats(const BfsArgs &a, const LevelState &st) {
    a.ctl->res.levels = st.levels;
    a.ctl->res.bottom_up_levels = st.bu_levels;
    a.ctl->res.reached = st.reached;
    bfs_publish_stats(a);
}

__global__ void __launch_bounds__(BFS_THREADS, 4) bfs_persistent_kernel(BfsArgs a) {
    BfsCtl *c = a.ctl;
    unsigned epoch = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    unsigned *fb = a.fbits, *nb = a.nbits, *zb = a.zbits;
    LevelState st;
    __shared__ unsigned s_stage[BFS_THREADS / 32][BFS_STAGE];
    __shared__ unsigned s_stage_cnt[BFS_THREADS / 32];
    if (lane_id() == 0) s_stage_cnt[threadIdx.x >> 5] = 0;
    __syncwarp();
    const WarpStage bq{s_stage[threadIdx.x >> 5], &s_stage_cnt[threadIdx.x >> 5], BFS_STAGE};

    // ---- Solo prologue: block 0 alone runs the first levels while the
    // frontier is small (every search starts with one vertex), syncing with
    // __syncthreads only; the other blocks wait for the hand-off.  A search
    // that stays small -- a root in a small component -- ends here without a
    // single grid barrier.
    if (blockIdx.x == 0) {
        const uint64_t E = __ldg(&a.rowptr[a.n]);
        if (threadIdx.x == 0) {
            // Fresh control state for this launch.  The other blocks read
            // none of it before block 0 releases them below, and they wait
            // for this launch's sequence number, so no leftover from an
            // earlier search on the workspace can release them.
            c->t0 = globaltimer_ns();
            c->res = g5_bfs_stats{0, 0, 0, 0, 0};
            c->xcount = 0;
            c->xdone = 0;
            c->bar = 0;
            a.touch->small = 0;  // the next reset clears everything
            for (int k = 0; k < 3; ++k) {
                c->n_small[k] = c->grab[k] = c->cgrab[k] = c->found[k] = c->ulen[k] = 0;
                c->big[k] = c->m_next[k] = 0;
            }
        }
        if (!a.roots) {
            const unsigned root = a.root;
            const uint64_t root_deg = __ldg(&a.rowptr[root + 1]) - __ldg(&a.rowptr[root]);
            if (threadIdx.x == 0) {
                a.visited[root >> 5] |= 1u << (root & 31);
                a.pred[root] = root;
                if (a.depth) a.depth[root] = 0;
                if (root_deg > a.big_deg) {
                    a.q[0][a.n - 1] = root;
                    a.base[0][0] = 0;
                    c->big[0] = (1ull << BIG_SHIFT) | ((root_deg + a.chunk - 1) / a.chunk);
                } else {
                    a.q[0][0] = root;
                    c->n_small[0] = 1;
                }
            }
            st = LevelState{0, TOP_DOWN, 0, PEND_NONE, 0, 0, 1u, 0u, root_deg, E - root_deg, 1ull};
        } else {
            // Several roots (disjoint graphs packed into one CSR, one root
            // each): level 0 is all of them.  A root is claimed through its
            // parent entry, so a repeated root is queued once.
            __shared__ unsigned long long s_m;
            __shared__ unsigned s_n;
            if (threadIdx.x == 0) s_m = 0, s_n = 0;
            __syncthreads();
            unsigned long long my_m = 0;
            unsigned my_n = 0;
            for (unsigned b0 = 0; b0 < a.nroots; b0 += blockDim.x) {
                const unsigned i = b0 + threadIdx.x;
                bool mine = false;
                unsigned r = 0;
                uint64_t deg = 0;
                if (i < a.nroots) {
                    const uint64_t rr = __ldg(&a.roots[i]);
                    if (rr >= a.n) {
                        atomicOr(&c->res.error_flags, DEVERR_RANGE);
                    } else if (atomicCAS((unsigned long long *)&a.pred[rr], ~0ull, (unsigned long long)rr) == ~0ull) {
                        mine = true;
                        r = (unsigned)rr;
                        atomicOr(&a.visited[r >> 5], 1u << (r & 31));
                        if (a.depth) a.depth[r] = 0;
                        deg = __ldg(&a.rowptr[r + 1]) - __ldg(&a.rowptr[r]);
                        my_m += deg;
                        ++my_n;
                    }
                }
                if (!frontier_append_staged(bq, a.q[0], a.base[0], a.n, &c->n_small[0], &c->big[0], mine, r, deg,
                                            a.big_deg, a.chunk))
                    atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
            }
            if (!stage_flush_warp(bq, a.q[0], a.n, &c->n_small[0])) atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
            my_m = warp_sum(my_m);
            my_n = warp_sum(my_n);
            if (lane_id() == 0) {
                atomicAdd(&s_m, my_m);
                atomicAdd(&s_n, my_n);
            }
            __syncthreads();
            st = LevelState{0, TOP_DOWN, 0, PEND_NONE, 0, 0, s_n, 0u, s_m, E - s_m, (unsigned long long)s_n};
        }
        __syncthreads();
        bool done = false;
        int solo = 0;
        while (a.nblocks == 1 || (st.mode == TOP_DOWN && st.pending == PEND_NONE && st.m_f <= SOLO_EDGES)) {
            if (a.nblocks == 1 && st.pending != PEND_NONE) break;  // conversions run in the grid loop
            bfs_expand_level(a, bq, st, fb, nb, nullptr);  // top-down only (conversions end the loop)
            __threadfence();
            __syncthreads();
            ++solo;
            if (threadIdx.x == 0) atomicAdd(&c->heartbeat, 1u);
            if (!bfs_advance(a, st, fb, nb, zb)) {
                done = true;
                break;
            }
            __syncthreads();  // everyone has read the counters before they are reused
        }
        if (threadIdx.x == 0) {
            c->hand = st;
            c->hand_fb = fb == a.fbits ? 0 : 1;
            c->res.solo_levels = solo;
            if (done) bfs_write_stats(a, st);
            __threadfence();
            atomicExch(&c->go, (a.seq << 2) | (done ? 2ull : 1ull));
        }
        if (done) return;
    } else {
        __shared__ unsigned s_go;
        if (threadIdx.x == 0) {
            // Bounded wait: the clock restarts whenever block 0 finishes a
            // level, so only a stalled prologue times out.
            unsigned long long t0 = globaltimer_ns();
            unsigned beat = ld_volatile(&c->heartbeat);
            unsigned long long go;
            unsigned g = 0;
            while (((go = ld_acquire64(&c->go)) >> 2) != a.seq) {
                const unsigned b = ld_volatile(&c->heartbeat);
                if (b != beat) {
                    beat = b;
                    t0 = globaltimer_ns();
                }
                if (globaltimer_ns() - t0 > a.limit_ns) {
                    atomicOr(&c->res.error_flags, DEVERR_TIMEOUT);
                    g = 2;
                    break;
                }
                __nanosleep(64);
            }
            s_go = g ? g : (unsigned)(go & 3);
        }
        __syncthreads();
        if (s_go == 2) return;
        const unsigned long long *src = (const unsigned long long *)&c->hand;
        unsigned long long *dst = (unsigned long long *)&st;
        for (unsigned i = 0; i < sizeof(LevelState) / 8; ++i) dst[i] = __ldcg(&src[i]);
        if (ld_volatile(&c->hand_fb)) {
            fb = a.nbits;
            nb = a.fbits;
        }
    }

    // ---- Grid loop.
    for (;;) {
        const int s_cur = st.level % 3;
        if (st.pending == PEND_TO_BITS) {
            // Frontier bitmap from the queue q[cur]; a clean next-frontier
            // bitmap; the unvisited list in q[cur ^ 1] (free: its queue was
            // the level before's).
            fb = a.fbits;
            nb = a.nbits;
            zb = a.zbits;
            for (uint64_t k = gtid; k < a.nwords; k += nthreads) fb[k] = nb[k] = 0;
            st.ucur = st.cur ^ 1;
            build_unvisited(a, bq, a.q[st.ucur], &c->ulen[s_cur]);
            if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
            const unsigned *Q = a.q[st.cur];
            const unsigned ns = ld_volatile(&c->n_small[s_cur]), nbg = big_count(ld_volatile(&c->big[s_cur]));
            for (uint64_t i = gtid; i < ns; i += nthreads) {
                const unsigned v = __ldcg(&Q[i]);
                atomicOr(&fb[v >> 5], 1u << (v & 31));
            }
            for (uint64_t i = gtid; i < nbg; i += nthreads) {
                const unsigned v = __ldcg(&Q[a.n - 1 - i]);
                atomicOr(&fb[v >> 5], 1u << (v & 31));
            }
            if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
        } else if (st.pending == PEND_TO_QUEUE) {
            bits_to_queue(a, bq, fb, a.q[st.cur], a.base[st.cur], &c->n_small[s_cur], &c->big[s_cur]);
            if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
        }
        st.pending = PEND_NONE;
        bfs_expand_level(a, bq, st, fb, nb, zb);
        if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
        if (!bfs_advance(a, st, fb, nb, zb)) break;
    }
    if (gtid == 0) bfs_write_stats(a, st);
}

// A search from a root whose component is small (mode BFS_SMALL): one block,
// levels top-down, claims on the visited bitmap -- none of the grid
// machinery (hand-off, grab counters, staging, grid barriers).  The first
// SMALL_Q entries of each frontier live in shared memory together with their
// row bounds: the lane that claims a vertex loads its two row starts in the
// same breath as the claim (both issued before either returns), so a level
// costs one column load and one atomic round trip on its critical path
// instead of queue, row-start, column and bitmap loads in a chain.  Entries
// past SMALL_Q go to the workspace queue (vertex only).  Correct for a
// component of any size, only slow when it is large.
constexpr unsigned SMALL_Q = 1024;

// Row starts of v and v + 1 and the claim of v's visited bit, issued in this
// order without waiting for one another; returns the bit's old word.
__device__ __forceinline__ unsigned claim_with_row(const uint64_t *rowptr, unsigned *visited, unsigned v,
                                                   uint64_t &rb, uint64_t &re) {
    const uint64_t *p = rowptr + v;
    unsigned *w = visited + (v >> 5);
    unsigned old;
    asm volatile("ld.global.nc.u64 %0, [%3];\n\t"
                 "ld.global.nc.u64 %1, [%3+8];\n\t"
                 "atom.global.or.b32 %2, [%4], %5;"
                 : "=l"(rb), "=l"(re), "=r"(old)
                 : "l"(p), "l"(w), "r"(1u << (v & 31))
                 : "memory");
    return old;
}
__global__ void __launch_bounds__(BFS_THREADS) bfs_small_kernel(BfsArgs a) {
    BfsCtl *c = a.ctl;
    __shared__ unsigned s_v[2][SMALL_Q];
    __shared__ uint64_t s_rb[2][SMALL_Q], s_re[2][SMALL_Q];
    __shared__ unsigned s_len[2];
    __shared__ unsigned s_err;
    __shared__ unsigned long long s_reached;
    const unsigned lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) {
        c->t0 = globaltimer_ns();
        c->xcount = 0;
        c->xdone = 0;
        const unsigned long long root = a.root;
        if (root >= a.n) {
            s_err = DEVERR_RANGE;  // the host checks roots; a bad one is reported, not used
            s_len[0] = 0;
        } else {
            uint64_t rb, re;
            claim_with_row(a.rowptr, a.visited, (unsigned)root, rb, re);
            a.pred[root] = (int64_t)root;
            if (a.depth) a.depth[root] = 0;
            a.tlist[0] = (unsigned)root;
            s_v[0][0] = (unsigned)root;
            s_rb[0][0] = rb;
            s_re[0][0] = re;
            s_len[0] = 1;
            s_err = 0;
        }
        s_len[1] = 0;
        s_reached = s_len[0];
    }
    __syncthreads();
    int level = 0;
    for (;; ++level) {
        const int cur = level & 1, nxt = cur ^ 1;
        const unsigned n = s_len[cur];
        if (n == 0) break;
        // One warp per frontier vertex, its lanes over the vertex's row.
        for (unsigned i = wid; i < n; i += nw) {
            unsigned u;
            uint64_t rb, re;
            if (i < SMALL_Q) {
                u = s_v[cur][i];
                rb = s_rb[cur][i];
                re = s_re[cur][i];
            } else {
                u = __ldcg(&a.q[cur][i]);
                rb = __ldg(&a.rowptr[u]);
                re = __ldg(&a.rowptr[u + 1]);
            }
            for (uint64_t e = rb + lane; e < re; e += 32) {
                const unsigned v = (unsigned)__ldg(&a.col[e]);
                if (v >= a.n) {  // not a vertex: report it, touch nothing
                    atomicOr(&s_err, DEVERR_RANGE);
                    continue;
                }
                uint64_t vb, ve;
                if (claim_with_row(a.rowptr, a.visited, v, vb, ve) & (1u << (v & 31))) continue;
                // The next level reads v's row: start bringing it into L2 now.
                if (vb < ve) asm volatile("prefetch.global.L2 [%0];" ::"l"(a.col + vb));
                a.pred[v] = u;
                if (a.depth) a.depth[v] = level + 1;
                const unsigned pos = atomicAdd(&s_len[nxt], 1u);  // each vertex is claimed once: pos < n
                // Touched list: vertices in claim order (s_reached counts the
                // levels before this one), for g5_bfs_reset_touched.
                if (s_reached + pos < a.n) a.tlist[s_reached + pos] = v;
                if (pos < SMALL_Q) {
                    s_v[nxt][pos] = v;
                    s_rb[nxt][pos] = vb;
                    s_re[nxt][pos] = ve;
                } else if (pos < a.n) {
                    a.q[nxt][pos] = v;
                } else {
                    atomicOr(&s_err, DEVERR_CAPACITY);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_reached += s_len[nxt];
            s_len[cur] = 0;
            if (level < BFS_TRACE) {
                c->t_level[level] = globaltimer_ns();
                c->n_level[level] = n;
                c->m_level[level] = 0;
                c->mode_level[level] = TOP_DOWN;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        c->res.levels = level;
        c->res.bottom_up_levels = 0;
        c->res.reached = s_reached;
        c->res.error_flags |= s_err;
        c->res.solo_levels = level;
        // The touched list holds every vertex this search wrote (a search
        // that reported an error leaves the next reset a full one).
        *a.touch = BfsTouch{s_err == 0 && s_reached <= a.n ? 1u : 0u, 0u, s_reached, a.pred, a.depth, c->init_used};
        bfs_publish_stats(a);
    }
    if (a.xout) {
        // The result for the host: a record per touched vertex, then the
        // count (after the statistics above and a system fence).
        __syncthreads();
        const unsigned long long cnt = s_reached < a.n ? s_reached : a.n;
        for (uint64_t i = threadIdx.x; i < cnt && i < a.xcap; i += blockDim.x) {
            const unsigned v = a.tlist[i];
            put_reached(a.xout, i, v, a.depth ? a.depth[v] : -1, a.pred[v]);
        }
        __threadfence_system();
        __syncthreads();
        if (threadIdx.x == 0) {
            c->xresult = cnt;
            *(volatile unsigned long long *)a.xcount_map = cnt;
        }
    }
}

struct BfsWork {
    BfsCtl *ctl;
    BfsTouch *touch;
    unsigned *visited, *fbits, *nbits, *zbits;
    unsigned *q[2], *base[2];
    uint64_t bytes;
};

static BfsWork carve_bfs(void *base, uint64_t n) {
    Carver c(base);
    BfsWork w;
    const uint64_t words = (n + 31) / 32;
    w.ctl = c.take<BfsCtl>(1);
    w.touch = c.take<BfsTouch>(1);
    w.visited = c.take<unsigned>(words);
    w.fbits = c.take<unsigned>(words);
    w.nbits = c.take<unsigned>(words);
    w.zbits = c.take<unsigned>(words);
    for (int i = 0; i < 2; ++i) {
        w.q[i] = c.take<unsigned>(n);
        w.base[i] = c.take<unsigned>(n);
    }
    w.bytes = c.used;
    return w;
}

// Largest co-resident grid of the persistent kernel on this device.
static int bfs_max_blocks(int *out) {
    static int cached[64] = {};
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if (!cached[di.device]) {
        if ((rc = persistent_kernel_setup((const void *)bfs_persistent_kernel))) return rc;
        int per_sm = 0;
        G5_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bfs_persistent_kernel, BFS_THREADS, 0));
        cached[di.device] = std::max(1, per_sm) * di.sms;
    }
    *out = cached[di.device];
    return G5_OK;
}

// ------------------------------------------------ depth from the parents --

// ok bit of v: pred[v] is a CSR neighbour of v (the edge the reference's
// propagation walks, :97-102), so depth can flow along it.
__global__ void dist_init_kernel(const int64_t *__restrict__ pred, uint64_t n, uint64_t root,
                                 int64_t *__restrict__ dist) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        dist[v] = v == root ? 0 : pred[v] == -1 ? -1 : INT64_MAX;
}

__global__ void parent_edge_kernel(const uint64_t *__restrict__ rowptr, const int *__restrict__ col,
                                   const int64_t *__restrict__ pred, uint64_t n, unsigned *__restrict__ okbits) {
    // One warp per vertex; each lane scans a strided part of the row.
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = warp; v < n; v += nwarps) {
        const int64_t p = pred[v];
        bool hit = false;
        if (p >= 0 && (uint64_t)p < n && (uint64_t)p != v) {
            const uint64_t rb = rowptr[v], re = rowptr[v + 1];
            for (uint64_t e = rb + lane_id(); e < re && !hit; e += 32) hit = col[e] == (int)p;
        }
        if (__any_sync(FULL, hit) && lane_id() == 0) atomicOr(&okbits[v >> 5], 1u << (v & 31));
    }
}

__global__ void dist_step_kernel(const int64_t *__restrict__ pred, const unsigned *__restrict__ okbits, uint64_t n,
                                 int64_t level, int64_t *__restrict__ dist, unsigned *__restrict__ changed) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned any = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        if (dist[v] != INT64_MAX || !((okbits[v >> 5] >> (v & 31)) & 1u)) continue;
        if (dist[pred[v]] == level) {
            dist[v] = level + 1;
            any = 1;
        }
    }
    if (__any_sync(__activemask(), any) && any) atomicOr(changed, 1u);
}

}  // namespace g5

using namespace g5;

extern "C" int g5_bfs_workspace_size(uint64_t nverts, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_bfs_workspace_size: bytes is NULL");
    *bytes = carve_bfs(nullptr, nverts).bytes;
    return G5_OK;
}

static int bfs_check(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                     int64_t *d_pred, void *d_work, uint64_t work_bytes, BfsWork *w, const char *who) {
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "%s: nverts outside [1, 2^31]", who);
    G5_CHECK_ARG(root < nverts, "%s: root %llu outside [0, %llu)", who, (unsigned long long)root,
                 (unsigned long long)nverts);
    G5_CHECK_ARG(d_rowstarts && d_col && d_pred && d_work, "%s: NULL argument", who);
    *w = carve_bfs(d_work, nverts);
    if (work_bytes < w->bytes)
        return set_error(G5_ERR_WORKSPACE, "%s: workspace %llu < %llu bytes", who, (unsigned long long)work_bytes,
                         (unsigned long long)w->bytes);
    return G5_OK;
}

// Bit v set when vertex v has no CSR entry (it can only ever be a root).
__global__ void isolated_bits_kernel(const uint64_t *__restrict__ rowptr, uint64_t n, unsigned *__restrict__ bits) {
    const uint64_t words = (n + 31) / 32;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < words; k += stride) {
        unsigned m = 0;
        const uint64_t v0 = k * 32;
        const uint64_t vend = min(v0 + 32, n);
        uint64_t prev = __ldg(&rowptr[v0]);
        for (uint64_t v = v0; v < vend; ++v) {
            const uint64_t next = __ldg(&rowptr[v + 1]);
            if (next == prev) m |= 1u << (v - v0);
            prev = next;
        }
        bits[k] = m;
    }
}

extern "C" int g5_graph_isolated_bitmap(const uint64_t *d_rowstarts, uint64_t nverts, uint32_t *d_bits,
                                        void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31) && d_rowstarts && d_bits, "g5_graph_isolated_bitmap: bad argument");
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    isolated_bits_kernel<<<di.sms * 4, 256, 0, (cudaStream_t)stream>>>(d_rowstarts, nverts, d_bits);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

struct BfsResetArgs {
    uint64_t n;
    int64_t *pred;
    int32_t *depth;
    const uint32_t *init;
    unsigned *visited;
    BfsCtl *ctl;
    BfsTouch *touch;
    const unsigned *tlist;
    int full;  // 1: clear everything whatever the last search touched
};

// The reset before a search: pred (and depth) = -1, visited = the initial
// bitmap (isolated vertices) or zero, a fresh control block.  Each of the
// three arrays is restored vertex by vertex from the touched list when the
// last search was a one-block search that wrote this very array (and
// started from this very bitmap), else cleared in full.  A touched reset
// reads the touch record in every block and leaves it alone; a full reset
// reads none of it and records "nothing touched" for these arrays.
__global__ void bfs_reset_kernel(BfsResetArgs r) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const BfsTouch h = r.full ? BfsTouch{0u, 0u, 0ull, nullptr, nullptr, nullptr} : *r.touch;
    if (r.full && t == 0) *r.touch = BfsTouch{1u, 0u, 0ull, r.pred, r.depth, r.init};
    const bool small = !r.full && h.small && h.count <= r.n;
    const bool pred_t = small && h.pred == r.pred;
    const bool depth_t = small && h.depth == r.depth;
    const bool vis_t = small && h.init == r.init;
    if (blockIdx.x == 0) {
        constexpr unsigned words = sizeof(BfsCtl) / 4;
        static_assert(sizeof(BfsCtl) % 4 == 0, "control block cleared in words");
        for (unsigned i = threadIdx.x; i < words; i += blockDim.x) ((unsigned *)r.ctl)[i] = 0;
        __syncthreads();
        if (threadIdx.x == 0) r.ctl->init_used = r.init;
    }
    if (pred_t || (r.depth && depth_t) || vis_t) {
        for (uint64_t i = t; i < h.count; i += T) {
            const unsigned v = __ldg(&r.tlist[i]);
            if (v >= r.n) continue;
            if (pred_t) r.pred[v] = -1;
            if (r.depth && depth_t) r.depth[v] = -1;
            if (vis_t) {
                const unsigned bit = 1u << (v & 31);
                if (r.init && (__ldg(&r.init[v >> 5]) & bit)) atomicOr(&r.visited[v >> 5], bit);
                else atomicAnd(&r.visited[v >> 5], ~bit);
            }
        }
    }
    if (!pred_t) grid_fill<int64_t>(r.pred, r.n, -1, t, T);
    if (r.depth && !depth_t) grid_fill<int32_t>(r.depth, r.n, -1, t, T);
    if (!vis_t) {
        const uint64_t words = (r.n + 31) / 32;
        if (r.init)
            for (uint64_t k = t; k < words; k += T) r.visited[k] = __ldg(&r.init[k]);
        else
            grid_fill<unsigned>(r.visited, words, 0u, t, T);
    }
}

static int bfs_reset_launch(uint64_t nverts, int64_t *d_pred, int32_t *d_depth, const uint32_t *d_visited_init,
                            void *d_work, uint64_t work_bytes, void *stream, int full, const char *who) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31) && d_pred && d_work, "%s: bad argument", who);
    BfsWork w = carve_bfs(d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "%s: workspace too small", who);
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    BfsResetArgs r{nverts, d_pred, d_depth, d_visited_init, w.visited, w.ctl, w.touch, w.base[0], full};
    const uint64_t want = (nverts + 2047) / 2048;  // 2048 vertices a block when the whole array is cleared
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)di.sms * 8, want));
    bfs_reset_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(r);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_bfs_reset(uint64_t nverts, int64_t *d_pred, int32_t *d_depth, const uint32_t *d_visited_init,
                            void *d_work, uint64_t work_bytes, void *stream) {
    return bfs_reset_launch(nverts, d_pred, d_depth, d_visited_init, d_work, work_bytes, stream, 1, "g5_bfs_reset");
}

extern "C" int g5_bfs_reset_touched(uint64_t nverts, int64_t *d_pred, int32_t *d_depth,
                                    const uint32_t *d_visited_init, void *d_work, uint64_t work_bytes, void *stream) {
    return bfs_reset_launch(nverts, d_pred, d_depth, d_visited_init, d_work, work_bytes, stream, 0,
                            "g5_bfs_reset_touched");
}

// Checks g5_bfs_params (zero tile fields select the defaults).
static int bfs_params_check(const g5_bfs_params &p, const char *who) {
    G5_CHECK_ARG(p.alpha > 0 && p.beta > 0 && p.mode >= 0 && p.mode <= BFS_SMALL, "%s: bad params", who);
    G5_CHECK_ARG(p.big_deg >= 0 && p.big_deg <= (1 << 20), "%s: big_deg %d outside [0, 2^20]", who, p.big_deg);
    G5_CHECK_ARG(p.chunk >= 0 && p.chunk <= (1 << 16) && p.chunk % 32 == 0,
                 "%s: chunk %d is not a multiple of 32 in [0, 65536]", who, p.chunk);
    G5_CHECK_ARG(p.lane_entries >= 0 && p.lane_entries <= 1024 && p.lane_entries % BU_STEP == 0,
                 "%s: lane_entries %d is not a multiple of %d in [0, 1024]", who, p.lane_entries, BU_STEP);
    return G5_OK;
}

// Builds the kernel arguments and launches the persistent BFS;
// d_stats_map (mapped pinned memory, or nullptr) receives the statistics at
// the end of the search.
static int bfs_launch(const BfsWork &w, const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                      uint64_t root, int64_t *d_pred, int32_t *d_depth, const g5_bfs_params *params,
                      cudaStream_t st, const uint64_t *d_roots = nullptr, unsigned nroots = 0,
                      g5_bfs_stats *d_stats_map = nullptr, g5_bfs_reached *xout = nullptr, uint64_t xcap = 0,
                      unsigned long long *xcount_map = nullptr) {
    g5_bfs_params p = {14.0f, 24.0f, 0, 0};
    if (params) p = *params;
    int rc = bfs_params_check(p, "g5_bfs");
    if (rc) return rc;
    int max_blocks = 0;
    rc = bfs_max_blocks(&max_blocks);
    if (rc) return rc;
    int blocks = p.blocks > 0 ? std::min(p.blocks, max_blocks)
                              : (int)std::min<uint64_t>(max_blocks, std::max<uint64_t>(1, nverts / 2048));
    BfsArgs a;
    a.rowptr = d_rowstarts;
    a.col = d_col;
    a.n = nverts;
    a.nwords = (nverts + 31) / 32;
    a.root = (unsigned)root;
    a.pred = d_pred;
    a.depth = d_depth;
    a.visited = w.visited;
    a.fbits = w.fbits;
    a.nbits = w.nbits;
    a.zbits = w.zbits;
    a.q[0] = w.q[0];
    a.q[1] = w.q[1];
    a.base[0] = w.base[0];
    a.base[1] = w.base[1];
    a.ctl = w.ctl;
    a.alpha = p.alpha;
    a.beta = p.beta;
    a.mode = p.mode;
    a.nblocks = (unsigned)blocks;
    a.limit_ns = wait_limit_ns();
    a.stats_out = d_stats_map;
    a.roots = d_roots;
    a.nroots = nroots;
    a.touch = w.touch;
    a.tlist = w.base[0];  // unused by the one-block search, which is the only writer
    a.xout = xout;  // only the one-block search exports by itself
    a.xcap = xcap;
    a.xcount_map = xcount_map;
    a.big_deg = p.big_deg ? (unsigned)p.big_deg : BFS_BIG_DEG;
    a.chunk = p.chunk ? (unsigned)p.chunk : BFS_CHUNK;
    a.lane_entries = p.lane_entries ? (unsigned)p.lane_entries : BU_LANE_ENTRIES;
    a.top = p.top;
    static std::atomic<unsigned long long> next_seq{1};
    a.seq = next_seq.fetch_add(1);
    if (p.mode == BFS_SMALL && !d_roots) {
        bfs_small_kernel<<<1, BFS_THREADS, 0, st>>>(a);
        G5_CUDA_TRY(cudaGetLastError());
        return G5_OK;
    }
    // Cooperative launch; the three bitmaps (visited, frontier, next: N/8
    // bytes each, adjacent in the workspace) get an L2 persisting window so
    // the streaming column reads do not evict them.
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(BFS_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attrs[2];
    attrs[0].id = cudaLaunchAttributeCooperative;
    attrs[0].val.cooperative = blocks > 1;  // one block has nothing to co-schedule
    cfg.attrs = attrs;
    cfg.numAttrs = 1;
    const uint64_t win = (uint64_t)((char *)(w.zbits + a.nwords) - (char *)w.visited);
    uint64_t win_bytes = 0;
    if (blocks > 1 && (rc = l2_persist_window(win, &win_bytes))) return rc;
    if (win_bytes) {
        attrs[1].id = cudaLaunchAttributeAccessPolicyWindow;
        attrs[1].val.accessPolicyWindow.base_ptr = w.visited;
        attrs[1].val.accessPolicyWindow.num_bytes = win_bytes;
        attrs[1].val.accessPolicyWindow.hitRatio = 1.0f;
        attrs[1].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attrs[1].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        cfg.numAttrs = 2;
    }
    G5_CUDA_TRY(cudaLaunchKernelEx(&cfg, bfs_persistent_kernel, a));
    return G5_OK;
}

extern "C" int g5_bfs_traverse(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                               int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                               const g5_bfs_params *params, void *stream) {
    clear_error();
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, root, d_pred, d_work, work_bytes, &w, "g5_bfs_traverse");
    if (rc) return rc;
    return bfs_launch(w, d_rowstarts, d_col, nverts, root, d_pred, d_depth, params, (cudaStream_t)stream);
}

extern "C" int g5_bfs_traverse_multi(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                     const uint64_t *d_roots, uint32_t nroots, int64_t *d_pred, int32_t *d_depth,
                                     void *d_work, uint64_t work_bytes, const g5_bfs_params *params, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_roots && nroots >= 1, "g5_bfs_traverse_multi: no roots");
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, 0, d_pred, d_work, work_bytes, &w, "g5_bfs_traverse_multi");
    if (rc) return rc;
    return bfs_launch(w, d_rowstarts, d_col, nverts, 0, d_pred, d_depth, params, (cudaStream_t)stream, d_roots,
                      nroots);
}

// Device address of pinned host memory `h`, when the device can address it.
// g5_bfs_export: records of the reached vertices.  After a one-block
// search, from its touched list by block 0; otherwise a scan of the parents
// with warp-aggregated appends, the last block to finish publishing the
// count.  A host-mapped count is written after a system fence that follows
// every record.
__global__ void __launch_bounds__(256) bfs_export_kernel(const int64_t *__restrict__ pred,
                                                          const int *__restrict__ depth, uint64_t n,
                                                          const BfsTouch *__restrict__ touch,
                                                          const unsigned *__restrict__ tlist, BfsCtl *c,
                                                          g5_bfs_reached *out, uint64_t cap,
                                                          unsigned long long *count_map) {
    __shared__ unsigned s_last;
    if (touch->small) {
        // The touched list: block 0 alone (it is short), the others leave.
        if (blockIdx.x != 0) return;
        // (clamped and checked: on a workspace no search has written yet the
        // record is whatever the memory held)
        const uint64_t cnt = min((uint64_t)touch->count, n);
        for (uint64_t i = threadIdx.x; i < cnt && i < cap; i += blockDim.x) {
            const unsigned v = tlist[i];
            if (v < n) put_reached(out, i, v, depth ? depth[v] : -1, pred[v]);
            else put_reached(out, i, v, -1, -1);
        }
        __threadfence_system();
        __syncthreads();
        if (threadIdx.x == 0) {
            c->xresult = cnt;
            if (count_map) *(volatile unsigned long long *)count_map = cnt;
        }
        return;
    }
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const unsigned lane = lane_id();
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x - lane; b < n; b += stride) {  // warp-uniform
        const uint64_t v = b + lane;
        const int64_t p = v < n ? pred[v] : -1;
        const bool reached = p != -1;
        const unsigned m = __ballot_sync(FULL, reached);
        if (!m) continue;
        const unsigned leader = __ffs(m) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(&c->xcount, (unsigned long long)__popc(m));
        base = __shfl_sync(FULL, base, leader);
        const unsigned long long pos = base + __popc(m & lanemask_lt());
        if (reached && pos < cap) put_reached(out, pos, (unsigned)v, depth ? depth[v] : -1, p);
    }
    __threadfence_system();  // this thread's records before the count
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&c->xdone, 1u) == gridDim.x - 1;
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        const unsigned long long cnt = atomicAdd(&c->xcount, 0ull);
        c->xresult = cnt;
        c->xcount = 0;  // ready for another export of the same search
        c->xdone = 0;
        if (count_map) {
            __threadfence_system();
            *(volatile unsigned long long *)count_map = cnt;
        }
    }
}

static bool host_mapped(const void *h, void **d) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, h) != cudaSuccess) {
        cudaGetLastError();  // pageable memory on older drivers: not an error here
        return false;
    }
    if (at.type != cudaMemoryTypeHost || !at.devicePointer) return false;
    *d = at.devicePointer;
    return true;
}

// Waits for a query launched with mapped statistics: the kernel writes
// `levels` (set to -1 by the host before the launch) last, after a system
// fence, so a host spin on it sees the search complete a few microseconds
// before a stream synchronisation would.  A search still running after
// QUERY_SPIN_NS (a long one, or one that failed) is waited for with the
// stream synchronisation, which also reports launch and device faults.
constexpr double QUERY_SPIN_NS = 200e3;

static int query_wait(g5_bfs_stats *h_stats, cudaStream_t st, const char *who) {
    volatile int32_t *lv = &h_stats->levels;
    const auto t0 = std::chrono::steady_clock::now();
    while (*lv == -1) {
        if (std::chrono::duration<double, std::nano>(std::chrono::steady_clock::now() - t0).count() > QUERY_SPIN_NS) {
            G5_CUDA_TRY(cudaStreamSynchronize(st));
            break;
        }
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    if (*lv == -1) return set_error(G5_ERR_DEVICE, "%s: the search ended without statistics", who);
    return deverr_to_status(h_stats->error_flags, who);
}

__global__ void first_neighbours_kernel(const uint64_t *__restrict__ rowptr, const int *__restrict__ col,
                                        uint64_t n, unsigned *__restrict__ top) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint64_t b = __ldg(&rowptr[v]), e = __ldg(&rowptr[v + 1]);
        top[v] = b < e ? (unsigned)__ldg(&col[b]) : (unsigned)n;
    }
}

extern "C" int g5_bfs_first_neighbours(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                       uint32_t *d_top, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_bfs_first_neighbours: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_col && d_top, "g5_bfs_first_neighbours: NULL argument");
    DeviceInfo di;
    const int sms = device_info(&di) ? 148 : di.sms;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((nverts + 255) / 256, (uint64_t)sms * 8));
    first_neighbours_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(d_rowstarts, d_col, nverts, d_top);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_bfs_query(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, const uint64_t *h_root,
                            const uint32_t *h_main_bits, int64_t *d_pred, int32_t *d_depth, void *d_work,
                            uint64_t work_bytes, const g5_bfs_params *params, g5_bfs_stats *h_stats, void *stream) {
    clear_error();
    G5_CHECK_ARG(h_root && h_stats, "g5_bfs_query: NULL host pointer");
    const uint64_t root = *h_root;
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, root, d_pred, d_work, work_bytes, &w, "g5_bfs_query");
    if (rc) return rc;
    g5_bfs_params p = {14.0f, 24.0f, 0, 0};
    if (params) p = *params;
    // A root outside the main component reaches a small set: one block
    // runs the whole search, with no grid to launch or wait for.
    if (h_main_bits && p.blocks == 0 && !((h_main_bits[root >> 5] >> (root & 31)) & 1u)) {
        p.blocks = 1;
        p.mode = BFS_SMALL;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // Pinned host statistics that the device can address are written by the
    // kernel itself (no copy call), and the host waits on them.
    void *d_stats_map = nullptr;
    if (host_mapped(h_stats, &d_stats_map)) {
        *(volatile int32_t *)&h_stats->levels = -1;
        if ((rc = bfs_launch(w, d_rowstarts, d_col, nverts, root, d_pred, d_depth, &p, st, nullptr, 0,
                             (g5_bfs_stats *)d_stats_map)))
            return rc;
        return query_wait(h_stats, st, "g5_bfs_query");
    }
    if ((rc = bfs_launch(w, d_rowstarts, d_col, nverts, root, d_pred, d_depth, &p, st))) return rc;
    G5_CUDA_TRY(cudaMemcpyAsync(h_stats, &w.ctl->res, sizeof(g5_bfs_stats), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(h_stats->error_flags, "g5_bfs_query");
}

extern "C" int g5_bfs_export(const int64_t *d_pred, const int32_t *d_depth, uint64_t nverts, void *d_work,
                             uint64_t work_bytes, g5_bfs_reached *out, uint64_t capacity, uint64_t *h_count,
                             void *stream) {
    clear_error();
    G5_CHECK_ARG(h_count && out && d_pred, "g5_bfs_export: NULL argument");
    G5_CHECK_ARG(((uintptr_t)out & 15) == 0, "g5_bfs_export: out is not 16-byte aligned");
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_bfs_export: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_work, "g5_bfs_export: workspace is NULL");
    const BfsWork w = carve_bfs(d_work, nverts);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_bfs_export: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    void *out_dev = out, *cnt_dev = nullptr;
    host_mapped(out, &out_dev);  // pinned host records: the kernel writes them itself
    const bool mapped_count = host_mapped(h_count, &cnt_dev);
    cudaStream_t st = (cudaStream_t)stream;
    DeviceInfo di;
    const int sms = device_info(&di) ? 148 : di.sms;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((nverts + 255) / 256, (uint64_t)sms * 2));
    if (mapped_count) *(volatile uint64_t *)h_count = ~0ull;
    bfs_export_kernel<<<grid, 256, 0, st>>>(d_pred, d_depth, nverts, w.touch, w.base[0], w.ctl,
                                            (g5_bfs_reached *)out_dev, capacity,
                                            mapped_count ? (unsigned long long *)cnt_dev : nullptr);
    G5_CUDA_TRY(cudaGetLastError());
    if (mapped_count) {
        volatile uint64_t *hc = h_count;
        const auto t0 = std::chrono::steady_clock::now();
        while (*hc == ~0ull) {
            if (std::chrono::duration<double, std::nano>(std::chrono::steady_clock::now() - t0).count() >
                QUERY_SPIN_NS) {
                G5_CUDA_TRY(cudaStreamSynchronize(st));
                break;
            }
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        if (*hc == ~0ull) return set_error(G5_ERR_DEVICE, "g5_bfs_export: the export ended without a count");
    } else {
        G5_CUDA_TRY(cudaMemcpyAsync(h_count, &w.ctl->xresult, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        G5_CUDA_TRY(cudaStreamSynchronize(st));
    }
    if (*h_count > capacity)
        return set_error(G5_ERR_INVALID, "g5_bfs_export: %llu reached vertices, capacity %llu",
                         (unsigned long long)*h_count, (unsigned long long)capacity);
    return G5_OK;
}

// A prepared g5_bfs_query: everything but the root checked and resolved
// once, so a query costs one launch and the wait.
struct g5_bfs_query_plan {
    const uint64_t *rowstarts;
    const int32_t *col;
    uint64_t nverts;
    const uint32_t *main_bits;
    int64_t *pred;
    int32_t *depth;
    BfsWork w;
    g5_bfs_params params;
    g5_bfs_stats *h_stats, *d_stats;
    cudaStream_t stream;
    // g5_bfs_query_plan_export: the export buffers last resolved
    g5_bfs_reached *x_out = nullptr;
    void *x_out_dev = nullptr;
    uint64_t *x_count = nullptr;
    void *x_count_dev = nullptr;
    int sms = 148;
};

extern "C" int g5_bfs_query_plan_create(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                        const uint32_t *h_main_bits, int64_t *d_pred, int32_t *d_depth,
                                        void *d_work, uint64_t work_bytes, const g5_bfs_params *params,
                                        g5_bfs_stats *h_stats, void *stream, g5_bfs_query_plan **out) {
    clear_error();
    G5_CHECK_ARG(out && h_stats, "g5_bfs_query_plan_create: NULL argument");
    *out = nullptr;
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, 0, d_pred, d_work, work_bytes, &w, "g5_bfs_query_plan_create");
    if (rc) return rc;
    void *d_stats = nullptr;
    G5_CHECK_ARG(host_mapped(h_stats, &d_stats),
                 "g5_bfs_query_plan_create: h_stats must be pinned host memory the device can address");
    g5_bfs_params p = {14.0f, 24.0f, 0, 0};
    if (params) p = *params;
    if ((rc = bfs_params_check(p, "g5_bfs_query_plan_create"))) return rc;
    int max_blocks = 0;
    if ((rc = bfs_max_blocks(&max_blocks))) return rc;  // resolved (and cached) now, not on the first query
    auto *q = new (std::nothrow) g5_bfs_query_plan{d_rowstarts, d_col, nverts, h_main_bits, d_pred, d_depth, w, p,
                                                   h_stats, (g5_bfs_stats *)d_stats, (cudaStream_t)stream};
    if (!q) return set_error(G5_ERR_INVALID, "g5_bfs_query_plan_create: out of host memory");
    DeviceInfo di;
    if (!device_info(&di)) q->sms = di.sms;
    *out = q;
    return G5_OK;
}

extern "C" int g5_bfs_query_plan_run(g5_bfs_query_plan *q, uint64_t root) {
    clear_error();
    G5_CHECK_ARG(q, "g5_bfs_query_plan_run: NULL plan");
    G5_CHECK_ARG(root < q->nverts, "g5_bfs_query_plan_run: root %llu outside [0, %llu)", (unsigned long long)root,
                 (unsigned long long)q->nverts);
    g5_bfs_params p = q->params;
    if (q->main_bits && p.blocks == 0 && !((q->main_bits[root >> 5] >> (root & 31)) & 1u)) {
        p.blocks = 1;
        p.mode = BFS_SMALL;
    }
    *(volatile int32_t *)&q->h_stats->levels = -1;
    int rc = bfs_launch(q->w, q->rowstarts, q->col, q->nverts, root, q->pred, q->depth, &p, q->stream, nullptr, 0,
                        q->d_stats);
    if (rc) return rc;
    return query_wait(q->h_stats, q->stream, "g5_bfs_query_plan_run");
}

extern "C" int g5_bfs_query_plan_export(g5_bfs_query_plan *q, uint64_t root, g5_bfs_reached *out,
                                        uint64_t capacity, uint64_t *h_count) {
    clear_error();
    G5_CHECK_ARG(q && out && h_count, "g5_bfs_query_plan_export: NULL argument");
    G5_CHECK_ARG(((uintptr_t)out & 15) == 0, "g5_bfs_query_plan_export: out is not 16-byte aligned");
    G5_CHECK_ARG(root < q->nverts, "g5_bfs_query_plan_export: root %llu outside [0, %llu)",
                 (unsigned long long)root, (unsigned long long)q->nverts);
    if (out != q->x_out) {
        q->x_out_dev = out;
        host_mapped(out, &q->x_out_dev);
        q->x_out = out;
    }
    if (h_count != q->x_count) {
        q->x_count_dev = nullptr;
        host_mapped(h_count, &q->x_count_dev);
        q->x_count = h_count;
    }
    g5_bfs_params p = q->params;
    const bool small = q->main_bits && p.blocks == 0 && !((q->main_bits[root >> 5] >> (root & 31)) & 1u);
    if (small) {
        p.blocks = 1;
        p.mode = BFS_SMALL;
    }
    *(volatile int32_t *)&q->h_stats->levels = -1;
    if (q->x_count_dev) *(volatile uint64_t *)h_count = ~0ull;
    // A small search with a host-mapped count writes its records itself at
    // its end; otherwise the export kernel runs right behind the search in
    // the stream (a grid scan of the parents).  The host waits once, on the
    // count.
    const bool fused = small && q->x_count_dev;
    int rc = bfs_launch(q->w, q->rowstarts, q->col, q->nverts, root, q->pred, q->depth, &p, q->stream, nullptr, 0,
                        q->d_stats, fused ? (g5_bfs_reached *)q->x_out_dev : nullptr, capacity,
                        fused ? (unsigned long long *)q->x_count_dev : nullptr);
    if (rc) return rc;
    if (!fused) {
        const int grid = small ? 1 : (int)std::max<uint64_t>(1, std::min<uint64_t>((q->nverts + 255) / 256,
                                                                                  (uint64_t)q->sms * 2));
        bfs_export_kernel<<<grid, 256, 0, q->stream>>>(q->pred, q->depth, q->nverts, q->w.touch, q->w.base[0],
                                                       q->w.ctl, (g5_bfs_reached *)q->x_out_dev, capacity,
                                                       (unsigned long long *)q->x_count_dev);
        G5_CUDA_TRY(cudaGetLastError());
    }
    if (q->x_count_dev) {
        volatile uint64_t *hc = h_count;
        const auto t0 = std::chrono::steady_clock::now();
        while (*hc == ~0ull) {
            if (std::chrono::duration<double, std::nano>(std::chrono::steady_clock::now() - t0).count() >
                QUERY_SPIN_NS) {
                G5_CUDA_TRY(cudaStreamSynchronize(q->stream));
                break;
            }
        }
        std::atomic_thread_fence(std::memory_order_acquire);
        if (*hc == ~0ull) return set_error(G5_ERR_DEVICE, "g5_bfs_query_plan_export: the export ended without a count");
    } else {
        G5_CUDA_TRY(cudaMemcpyAsync(h_count, &q->w.ctl->xresult, sizeof(uint64_t), cudaMemcpyDeviceToHost, q->stream));
        G5_CUDA_TRY(cudaStreamSynchronize(q->stream));
    }
    // The search's statistics landed before the export began (stream order).
    if (*(volatile int32_t *)&q->h_stats->levels == -1)
        return set_error(G5_ERR_DEVICE, "g5_bfs_query_plan_export: the search ended without statistics");
    if ((rc = deverr_to_status(q->h_stats->error_flags, "g5_bfs_query_plan_export"))) return rc;
    if (*h_count > capacity)
        return set_error(G5_ERR_INVALID, "g5_bfs_query_plan_export: %llu reached vertices, capacity %llu",
                         (unsigned long long)*h_count, (unsigned long long)capacity);
    return G5_OK;
}

extern "C" void g5_bfs_query_plan_destroy(g5_bfs_query_plan *q) { delete q; }

extern "C" int g5_bfs_visited_bitmap(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint32_t *d_bits,
                                     void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && d_bits && nverts >= 1 && nverts <= (1ull << 31), "g5_bfs_visited_bitmap: bad argument");
    BfsWork w = carve_bfs((void *)d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_bfs_visited_bitmap: workspace too small");
    G5_CUDA_TRY(cudaMemcpyAsync(d_bits, w.visited, (nverts + 31) / 32 * sizeof(unsigned), cudaMemcpyDeviceToDevice,
                                (cudaStream_t)stream));
    return G5_OK;
}

extern "C" int g5_bfs_run(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                          int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                          const g5_bfs_params *params, void *stream) {
    clear_error();
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, root, d_pred, d_work, work_bytes, &w, "g5_bfs_run");
    if (rc) return rc;
    if ((rc = g5_bfs_reset(nverts, d_pred, d_depth, nullptr, d_work, work_bytes, stream))) return rc;
    return g5_bfs_traverse(d_rowstarts, d_col, nverts, root, d_pred, d_depth, d_work, work_bytes, params, stream);
}

// ---------------------------------------------- allocation-free variant --
//
// Some callers cannot allocate device memory when they search: a process
// whose device memory is handed out entirely by another allocator (an arena
// like the reference's symmetric heap, or a framework's caching pool) would
// fail or fragment it, and cudaMalloc/cudaFree synchronise the device,
// which a latency-bound query loop cannot afford.  For them the BFS scratch
// can live in a fixed array in this library's device image instead of a
// caller-provided workspace: STATIC_BFS_BYTES (5 MiB) on every GPU that
// loads the library, held until the process exits, enough for graphs of up
// to STATIC_BFS_MAX_VERTS (2^18) vertices.

constexpr uint64_t STATIC_BFS_MAX_VERTS = 1ull << 18;
constexpr uint64_t STATIC_BFS_BYTES = 5ull << 20;
static __device__ __align__(256) unsigned char g5_bfs_static_scratch[STATIC_BFS_BYTES];

// Device address of the array in the current context, looked up on every
// call (in host code the array's name is only a stand-in; the lookup is
// cheap once the module is loaded).  Nothing is cached: after a
// cudaDeviceReset the next context holds a new copy of the array at
// another address, and the next call finds that one.
static int static_bfs_scratch(void **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g5_bfs_static_scratch);
    if (e != cudaSuccess || !p)
        return set_error(G5_ERR_CUDA, "g5_bfs_run_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
    *out = p;
    return G5_OK;
}

extern "C" int g5_bfs_run_static(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                                 int64_t *d_pred, int32_t *d_depth, const g5_bfs_params *params, void *stream) {
    clear_error();
    if (nverts > STATIC_BFS_MAX_VERTS)
        return set_error(G5_ERR_INVALID,
                         "g5_bfs_run_static: %llu vertices exceed its fixed scratch limit of %llu; use g5_bfs_run "
                         "with a workspace",
                         (unsigned long long)nverts, (unsigned long long)STATIC_BFS_MAX_VERTS);
    if (carve_bfs(nullptr, nverts).bytes > STATIC_BFS_BYTES)
        return set_error(G5_ERR_WORKSPACE, "g5_bfs_run_static: scratch too small for %llu vertices",
                         (unsigned long long)nverts);
    void *scratch = nullptr;
    int rc = static_bfs_scratch(&scratch);
    if (rc) return rc;
    // g5_bfs_run clears what must start at zero (pred, depth, the visited
    // bitmap, the control block) before the search, so the previous call's
    // contents do not matter.
    return g5_bfs_run(d_rowstarts, d_col, nverts, root, d_pred, d_depth, scratch, STATIC_BFS_BYTES, params, stream);
}

extern "C" int g5_bfs_last_stats(const void *d_work, uint64_t work_bytes, g5_bfs_stats *stats, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && stats, "g5_bfs_last_stats: NULL argument");
    G5_CHECK_ARG(work_bytes >= sizeof(BfsCtl), "g5_bfs_last_stats: workspace too small");
    BfsCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    *stats = c.res;
    return deverr_to_status(c.res.error_flags, "g5_bfs_run");
}

extern "C" int g5_bfs_last_trace(const void *d_work, uint64_t work_bytes, int max_levels, int32_t *mode,
                                  uint64_t *frontier_vertices, uint64_t *frontier_edges, double *level_ms,
                                  int32_t *nlevels, int32_t *solo_levels, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && work_bytes >= sizeof(BfsCtl) && nlevels, "g5_bfs_last_trace: bad argument");
    BfsCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    const int n = std::min(std::min(c.res.levels, BFS_TRACE), std::max(max_levels, 0));
    unsigned long long prev = c.t0;
    for (int i = 0; i < n; ++i) {
        if (mode) mode[i] = c.mode_level[i];
        if (frontier_vertices) frontier_vertices[i] = c.n_level[i];
        if (frontier_edges) frontier_edges[i] = c.m_level[i];
        if (level_ms) level_ms[i] = (double)(c.t_level[i] - prev) * 1e-6;
        prev = c.t_level[i];
    }
    *nlevels = c.res.levels;
    if (solo_levels) *solo_levels = c.res.solo_levels;
    return deverr_to_status(c.res.error_flags, "g5_bfs_run");
}

extern "C" int g5_bfs_dist_from_pred(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                     const int64_t *d_pred, uint64_t root, int64_t *d_dist, void *d_work,
                                     uint64_t work_bytes, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_bfs_dist_from_pred: nverts outside [1, 2^31]");
    G5_CHECK_ARG(root < nverts, "g5_bfs_dist_from_pred: root out of range");
    G5_CHECK_ARG(d_rowstarts && d_col && d_pred && d_dist && d_work, "g5_bfs_dist_from_pred: NULL argument");
    const uint64_t words = (nverts + 31) / 32;
    Carver c(d_work);
    unsigned *okbits = c.take<unsigned>(words);
    unsigned *changed = c.take<unsigned>(64);
    if (work_bytes < c.used) return set_error(G5_ERR_WORKSPACE, "g5_bfs_dist_from_pred: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    const int grid = di.sms * 8;
    G5_CUDA_TRY(cudaMemsetAsync(okbits, 0, words * sizeof(unsigned), st));
    dist_init_kernel<<<grid, 256, 0, st>>>(d_pred, nverts, root, d_dist);
    parent_edge_kernel<<<grid, 256, 0, st>>>(d_rowstarts, d_col, d_pred, nverts, okbits);
    G5_CUDA_TRY(cudaGetLastError());
    // Level by level, as the reference does; a level that labels nothing ends it.
    for (int64_t level = 0; level < (int64_t)nverts; ++level) {
        unsigned h_changed = 0;
        G5_CUDA_TRY(cudaMemsetAsync(changed, 0, sizeof(unsigned), st));
        dist_step_kernel<<<grid, 256, 0, st>>>(d_pred, okbits, nverts, level, d_dist, changed);
        G5_CUDA_TRY(cudaGetLastError());
        G5_CUDA_TRY(cudaMemcpyAsync(&h_changed, changed, sizeof h_changed, cudaMemcpyDeviceToHost, st));
        G5_CUDA_TRY(cudaStreamSynchronize(st));
        if (!h_changed) break;
    }
    return G5_OK;
}

extern "C" int g5_bfs_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks) {
    clear_error();
    G5_CHECK_ARG(blocks && max_blocks, "g5_bfs_grid: NULL argument");
    int mb = 0;
    int rc = bfs_max_blocks(&mb);
    if (rc) return rc;
    *max_blocks = mb;
    *blocks = (int)std::min<uint64_t>(mb, std::max<uint64_t>(1, nverts / 2048));
    return G5_OK;
}
