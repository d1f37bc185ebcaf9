// sssp.cu -- K4: delta-stepping SSSP in one persistent cooperative kernel
// (replaces the reference's host-driven oned_graph_sssp_run,
// src/traversal.cu:638-711, and its kernels :211-340).
//
// Semantics kept from the reference: float32 relaxations cand = d[u] + w,
// a distance is replaced only by a strictly smaller one, buckets
// [b_k, b_{k+1}) with b_0 = 0 and b_{k+1} = b_k + delta accumulated in
// float32 exactly as the reference's `bucket_max += delta`, light edges
// (w < delta) relaxed to a fixed point inside a bucket before its heavy
// edges.  With non-negative weights the float fixed point is unique, so the
// distances equal the reference's bit for bit, whatever the bucket width and
// the order of relaxations -- which lets the kernel use a light threshold
// above the bucket width (the CSR's light/heavy split at 0.1 serves every
// width up to 0.1) and pull instead of push in large heavy phases.
//
// Device-side structure:
//   * dist and parent packed in one u64 (float bits << 32 | parent); a
//     relaxation is one 64-bit atomicMin, which keeps the smallest distance
//     and, among equal distances, the smallest parent -- no locks (the
//     reference spins on a per-vertex lock, :224).
//   * a ring of K bucket queues for the next K-1 buckets; a vertex enters a
//     bucket's queue at most once (its ring stamp only decreases), stale
//     entries are dropped when the bucket opens.  No O(N) bucket scans (the
//     reference scans all vertices per bucket, :297-331).
//   * generation stamps for "already in this frontier" / "already in this
//     bucket's heavy set", so nothing is cleared per iteration (the
//     reference clears N visited flags per light iteration, :270-275).
//   * a settled bitmap (N/8 bytes, L2 resident): edges into vertices of
//     finished buckets are skipped without touching their distance.
//   * frontiers are processed with the warp-gather / big-vertex sharing of
//     the BFS kernel, over the light or the heavy part of each row.
//
// Algorithmic bytes per search: 2 m_c * (4 col + 4 w) + n_c * (8 rowstarts
// + 8 packed dist/parent + 4 dist + 8 parent written out).
#include <algorithm>
#include <cstring>

#include "g5_common.cuh"
#include "g5_frontier.cuh"

namespace g5 {

constexpr int SSSP_THREADS = 256;
constexpr int RING = 32;  // bucket queues; a relaxation may land at most RING-1 buckets ahead
constexpr unsigned STAGE_F = 64;     // per-warp staging: frontier
constexpr unsigned STAGE_S = 64;     //                   heavy set
constexpr unsigned STAGE_R = 16;     //                   each ring queue
constexpr unsigned STAGE_Q = 16;     //                   each sub-bucket queue
constexpr unsigned STAGE_D = 32;     //                   the sub-bucket's expanded set
// stage_append takes up to 32 entries at once; the ring and sub-bucket
// slices are smaller and use stage_push, which writes through when full.
static_assert(STAGE_F >= 32 && STAGE_S >= 32, "staging slices hold one warp step");
static_assert(STAGE_R <= 32 && STAGE_Q <= 32, "stage_push writes a full slice with one lane per entry");
constexpr int SSSP_TRACE = 256;      // phases recorded in the control block
// List entries with more edges to expand than this go to the big part (cut
// into SSSP_CHUNK chunks across the grid), and a warp grabs at most SSSP_GRAB
// small entries at once: a grab holds at most SSSP_GRAB x SSSP_BIG_DEG edges,
// so no warp is left with a long tail of relaxations at the end of a phase.
// Both are defaults of g5_sssp_params.big_deg / .chunk.
constexpr unsigned SSSP_BIG_DEG = 256;
// Chunk of a long row taken by one warp in the frontier, heavy-set and
// expanded-set lists.  A warp's relaxation steps form a chain of dependent
// round trips, so the chunk bounds the longest warp of a phase.  A multiple
// of 32 x SSSP_EDGES (the entries a warp step covers).
constexpr unsigned SSSP_CHUNK = 256;
constexpr unsigned SSSP_GRAB = 32;
// Sub-buckets: once a bucket's light frontier holds SPLIT_MIN light entries,
// the rest of the bucket is processed in SUB equal sub-buckets in order
// (delta-stepping with width delta/SUB for the light edges, nested in the
// bucket), so a vertex is expanded again only when its distance drops
// within its sub-bucket.  On Kronecker graphs the bucket that holds the
// hubs' neighbourhood has most vertices at nearly equal distances; without
// this every one of them is re-expanded several times.
//
// Inside a sub-bucket only the relaxations that can land in the same
// sub-bucket (fl(d_u + w) < its upper bound) are made when a vertex is
// expanded; the others are deferred.  Every vertex expanded in the
// sub-bucket enters its expanded set once; when the sub-bucket's frontier
// is empty their distances are final, and a settle pass relaxes each one's
// deferred light edges once, into later sub-buckets or buckets.  A hub whose
// distance drops several times inside the sub-bucket then re-reads its light
// row (weights only decide) but repeats none of its random relaxations.
constexpr int SUB = 32;
constexpr unsigned long long SPLIT_MIN = 1ull << 25;  // default; g5_sssp_params.sub_min overrides
constexpr float SSSP_PULL_RATIO = 1.0f;  // default heavy-phase pull threshold
constexpr double PULL_WALK = 0.25;       // cost of a pull's bitmap walk, in CSR entries per vertex
constexpr unsigned long long UNREACHED = ~0ull;

// Which capacity check fired: one bit per site above the DEVERR_* flags
// (bit 16 + site), so a status message names where a list overflowed.
enum {
    SITE_PUSH = 0,        // frontier / heavy-set / expanded-set append
    SITE_FINE = 1,        // sub-bucket queue append
    SITE_RING = 2,        // bucket ring queue append
    SITE_HEAVY_SAME = 3,  // a heavy relaxation landed in the open bucket
    SITE_FLUSH = 4,       // end-of-phase flush of the staging slices
    SITE_LIST_F = 5,      // frontier parts overlap
    SITE_LIST_D = 6,      // expanded-set parts overlap
    SITE_LIST_S = 7,      // heavy-set parts overlap
    SITE_PULL = 8,        // pull long-row list append
    SITE_SMALL = 9,       // one-block search list
};
__host__ __device__ constexpr unsigned site_bit(int site) { return 1u << (16 + site); }

// List sizes that every block reads after a grid barrier.  They lead the
// control block, and each block copies them into shared memory once per
// barrier (a few warps, one load per word) instead of every warp reading
// the same words from L2.
struct SsspSnap {
    unsigned long long f_big[3];      // per phase slot: frontier produced for the next phase (big part)
    // Heavy set (vertices settled by the bucket) per bucket slot: the
    // bucket opened i-th uses slot i % 3, cleared when bucket i-1 opens.
    unsigned long long s_big[3];
    unsigned long long s_entries[3];  // CSR entries of the heavy set's rows
    unsigned long long f_entries[3];  // light CSR entries of the frontier's rows
    unsigned long long pl_big;        // heavy-phase pull: rows too long for one warp
    unsigned long long d_big[2];      // expanded set of a sub-bucket (two slots, alternating)
    unsigned f_small[3];
    unsigned s_small[3];
    unsigned ring_len[RING];
    unsigned fq_len[SUB];  // sub-bucket queues of the current bucket
    unsigned d_small[2];
};
constexpr int SNAP_WORDS = (int)(sizeof(SsspSnap) / 4);

// What the last search on a workspace wrote, for g5_sssp_reset_touched.
// Only the search kernels write it (every block of the reset reads it): the
// one-block search lists every vertex it reached in the first heavy-set
// array and records its outputs; a grid search clears `small`, which makes
// the next reset a full one.
struct SsspTouch {
    unsigned small;
    unsigned sparse;           // the outputs were pre-filled and only reached vertices written
    unsigned long long count;  // vertices in the list
    float *dist;
    int64_t *pred;
    const unsigned *inv;  // the search's vertex numbering: output index of listed vertex v (nullptr: v)
};

struct SsspCtl {
    SsspSnap sn;  // first: copied as words 0 .. SNAP_WORDS-1
    unsigned bar;
    unsigned error;
    unsigned grab[3];    // per phase slot: cursor over the input list's small part
    unsigned cgrab[3];   //                 cursor over the input list's big-part chunks
    unsigned pl_small, pl_cgrab;  // heavy-phase pull: long-row list
    unsigned long long pulls;
    unsigned long long splits;
    unsigned long long buckets;
    unsigned long long phases;
    // counters: edges looked at, skipped as settled, atomicMin issued,
    // distances lowered, ring and frontier pushes
    unsigned long long n_edges, n_settled, n_atomic, n_improved, n_ring, n_front;
    // First relaxation that broke a bucket invariant (site SITE_HEAVY_SAME):
    // claimed by dbg_claim, then v, the packed candidate (distance, u), u's
    // packed value when seen, b_B and b_{B+1} bits, the bucket and phase.
    unsigned dbg_claim;
    unsigned long long dbg[7];
    // per-phase trace: end time, kind (0 open, 1 light, 2 heavy push, 3
    // heavy pull), input size, edges looked at so far
    unsigned long long t0;
    unsigned long long t_phase[SSSP_TRACE];
    unsigned long long e_phase[SSSP_TRACE];
    unsigned n_phase[SSSP_TRACE];
    unsigned char kind_phase[SSSP_TRACE];
};

// Output arrays that g5_sssp_reset pre-filled with -1.0f / -1.  When the
// search writes to the same arrays, it stores each vertex's distance and
// parent when the vertex is settled and leaves unreached ones untouched, so
// a search costs O(reached) instead of O(N) (a search in a two-vertex
// component must not sweep a 67M-vertex array).
struct SsspOut {
    float *dist;
    int64_t *pred;
};

struct SsspArgs {
    const uint64_t *rowptr;
    const int *col;
    const float *w;
    const unsigned *ld;  // light degree per vertex (partitioned rows) or nullptr
    const unsigned *td;  // tiny-first light parts: tiny entries per vertex (w < tiny), or nullptr
    float tiny;          // light / G5_TINY_DIV
    uint64_t n;
    unsigned root;
    const uint64_t *roots;  // several sources at once (device array) instead of `root`, or nullptr
    unsigned nroots;
    float delta;       // bucket width
    float light;       // light edges: w < light (light >= delta)
    float pull_ratio;  // heavy phase pulls when its rows' entries >= pull_ratio x unsettled rows' entries; <= 0 never
    unsigned long long split_min;  // frontier light entries that start sub-buckets (~0: never)
    unsigned long long *pack;
    unsigned *fstamp, *sstamp;
    // Queue stamps: the lowest bucket (rstamp) and sub-bucket (jstamp,
    // fine_key) whose queue holds the vertex.  Both only decrease, by
    // atomicMin, so a queue receives a vertex at most once -- however the
    // deferred pushes of several warps interleave -- and every open may
    // take its queue's entries as distinct.
    unsigned *rstamp, *jstamp;
    unsigned *dstamp;        // expanded-set stamp: fine_id of the sub-bucket that expanded the vertex
    unsigned *settled;
    unsigned *cur;           // bitmap of the bucket being pulled from (heavy pull only)
    unsigned *F[2], *FB[2];  // frontiers and the chunk bases of their big parts
    unsigned *S[2], *SB[2];  // heavy sets and chunk bases
    unsigned *ring;
    unsigned *fq;  // SUB sub-bucket queues of n entries
    SsspCtl *ctl;
    SsspTouch *touch;
    const SsspOut *prefilled;
    float *dist;
    int64_t *pred;
    unsigned nblocks;
    unsigned long long limit_ns;
    bool check_opens;  // opens exchange their stamps and flag a vertex met twice (DEVERR_DUPLICATE)
    unsigned big_deg;  // list entries with more edges to expand go to the chunked big part
    unsigned chunk;    // edges of a big entry per warp grab
    // Renumbered search (both set) or not (both nullptr): the CSR is in the
    // search's numbering, roots and outputs in the caller's; perm maps a
    // caller's vertex to the search's, inv back.  Parents in pack are the
    // search's numbers (mapped through inv when written out).
    const unsigned *perm, *inv;
};

__device__ __forceinline__ float pack_dist(unsigned long long p) { return __uint_as_float((unsigned)(p >> 32)); }

// The caller's number of the search's vertex v, and back.
__device__ __forceinline__ unsigned out_id(const SsspArgs &a, unsigned v) { return a.inv ? __ldg(&a.inv[v]) : v; }
__device__ __forceinline__ unsigned in_id(const SsspArgs &a, uint64_t v) {
    return a.perm ? __ldg(&a.perm[v]) : (unsigned)v;
}

// Writes vertex v's final packed value p to the caller's outputs.
__device__ __forceinline__ void write_out(const SsspArgs &a, unsigned v, unsigned long long p) {
    const unsigned o = out_id(a, v);
    a.dist[o] = p == UNREACHED ? -1.0f : pack_dist(p);
    a.pred[o] = p == UNREACHED ? -1 : (int64_t)out_id(a, (unsigned)p);
}

// Row range [b, e) of u's light (heavy = false) or heavy part.  Without
// partition data the whole row is returned and the caller filters by weight.
__device__ __forceinline__ void part_range(const SsspArgs &a, unsigned u, bool heavy, uint64_t &b, uint64_t &e) {
    b = __ldg(&a.rowptr[u]);
    e = __ldg(&a.rowptr[u + 1]);
    if (a.ld) {
        const uint64_t mid = b + __ldg(&a.ld[u]);
        if (heavy) b = mid;
        else e = mid;
    }
}

// Marks u settled; with pre-filled outputs also stores its final distance
// and parent (p = its packed value, final once its bucket's light phases are
// done).
__device__ __forceinline__ void settle(const SsspArgs &a, bool sparse_out, unsigned u, unsigned long long p) {
    atomicOr(&a.settled[u >> 5], 1u << (u & 31));
    if (sparse_out) {
        a.dist[u] = pack_dist(p);
        a.pred[u] = (int64_t)(unsigned)p;
    }
}

// Per-warp shared-memory staging of every list a phase appends to.
struct Stage {
    WarpStage f, s, d;
    unsigned *rbuf;  // RING * STAGE_R, this warp's
    unsigned *rcnt;  // RING, this warp's
    unsigned *qbuf;  // SUB * STAGE_Q, this warp's
    unsigned *qcnt;  // SUB, this warp's
    unsigned long long *bcnt;  // 8 event counts of the block (shared); [7] = frontier light entries
    unsigned *pv, *pw;         // PEND pushes waiting, this warp's: vertex and what (P_*)
    unsigned *pcnt;            // their count, always < 32 between calls
};

// Pushes decided by relaxations wait in a per-warp list and run 32 at a
// time, one per lane, instead of once per warp step with the few lanes that
// lowered a distance: the dependent atomics and loads of a push then serve
// a full warp.
constexpr unsigned PEND = 64;
constexpr unsigned P_SAME = 0x100u;  // this bucket's frontier (and heavy set)
constexpr unsigned P_FINE = 0x200u;  // | j: sub-bucket j's queue (and heavy set)
constexpr unsigned P_RING = 0x300u;  // | j: the ring queue of bucket B + j

// Per-thread event counts, summed into the control block once per phase.
struct Counts {
    unsigned edges, settled, atomics, improved, ring, front;  // per thread and phase: far below 2^32
    unsigned long long s_entries;
};

struct PushCtx {
    Stage st;
    unsigned pid;        // id of the producing phase (frontier stamp)
    unsigned bucket;     // current bucket index (heavy-set stamp)
    int f_slot;          // counter slot of the produced frontier
    unsigned *Fout, *FBout;
    unsigned *Sl, *SBl;  // heavy set of the current bucket
    int s_slot;
    const float *bnd;    // shared: b_B .. b_{B+RING}
    const float *sub;    // shared: sub-bucket bounds t_0 = b_B .. t_SUB = b_{B+1}
    float sub_hi;        // upper bound of the light frontier's range (t_{j+1}, or b_{B+1})
    bool sub_mode;       // the bucket is processed by sub-buckets
    bool tiny_rows;      // sub-bucket expansions read only the rows' tiny prefixes
    unsigned *Dl, *DBl;  // expanded set of the open sub-bucket (borrows the idle heavy-set arrays)
    int d_slot;          // its counter slot
    unsigned d_tag;      // its stamp: fine_id(bucket, sub-bucket)
};

// Expanded-set stamp of sub-bucket j of `bucket` (compared for equality).
__device__ __forceinline__ unsigned fine_id(unsigned bucket, int j) {
    return 0x80000000u | ((bucket * (unsigned)SUB + (unsigned)j) % 0x7fffffffu);
}

// Sub-bucket queue stamp of (bucket, j), compared by order: a vertex is
// queued into sub-buckets of one bucket only (the bucket of its distance,
// which settles it), where the key grows with j and stays below 2^31 - 1, so
// it never meets the reset value ~0u.
__device__ __forceinline__ unsigned fine_key(unsigned bucket, int j) {
    return ((bucket * (unsigned)SUB) & 0x7fffffffu) + (unsigned)j;
}

// Largest j in [0, SUB) with t_j <= d, for d in [t_0, t_SUB).
__device__ __forceinline__ int sub_index(const float *t, float d) {
    int j = 0;
#pragma unroll
    for (int step = SUB / 2; step > 0; step >>= 1)
        if (t[j + step] <= d) j += step;
    return j;
}

// Appends v to the produced frontier and to the bucket's heavy set (each at
// most once).  All 32 lanes call it.  `unique`: the caller's vertices are
// distinct and none of them was pushed in this bucket (or sub-bucket) yet --
// the entries of a bucket's ring queue or a sub-bucket's queue, which hold a
// vertex at most once (rstamp / jstamp) and are read by the first phase of
// their window -- so the stamps are set with plain stores instead of being
// exchanged.  With a.check_opens they are exchanged all the same, and a
// vertex whose stamp is already in place is reported (DEVERR_DUPLICATE) and
// not appended again.
__device__ __forceinline__ void push_same_bucket(const SsspArgs &a, const PushCtx &x, Counts &k, bool want_f,
                                                 bool want_s, unsigned v, bool unique = false) {
    SsspCtl *c = a.ctl;
    bool f, s, d;
    if (unique && !a.check_opens) {
        f = want_f;
        s = want_s;
        d = f && x.sub_mode;
        if (f) a.fstamp[v] = x.pid;
        if (s) a.sstamp[v] = x.bucket;
        if (d) a.dstamp[v] = x.d_tag;
    } else if (unique) {
        const bool df = want_f && atomicExch(&a.fstamp[v], x.pid) == x.pid;
        const bool ds = want_s && atomicExch(&a.sstamp[v], x.bucket) == x.bucket;
        const bool dd = want_f && x.sub_mode && atomicExch(&a.dstamp[v], x.d_tag) == x.d_tag;
        if (df || ds || dd) atomicOr(&c->error, DEVERR_DUPLICATE);
        f = want_f && !df;
        s = want_s && !ds;
        d = f && x.sub_mode && !dd;
    } else {
        f = want_f && atomicExch(&a.fstamp[v], x.pid) != x.pid;
        s = want_s && atomicExch(&a.sstamp[v], x.bucket) != x.bucket;
        // In sub mode a vertex entering the frontier joins the sub-bucket's
        // expanded set (once per sub-bucket).
        d = f && x.sub_mode && atomicExch(&a.dstamp[v], x.d_tag) != x.d_tag;
    }
    uint64_t lb = 0, le = 0, hb = 0, he = 0, dl = 0;
    if (f || s) {
        const uint64_t b = __ldg(&a.rowptr[v]), e = __ldg(&a.rowptr[v + 1]);
        const uint64_t mid = a.ld ? b + __ldg(&a.ld[v]) : e;
        if (f) {
            // A sub-bucket's frontier rows are their tiny prefixes (the
            // expansion's row range, which sets the big part's chunks).
            lb = b;
            le = x.sub_mode && x.tiny_rows ? b + __ldg(&a.td[v]) : mid;
            dl = mid - b;
        }
        if (s) {
            hb = a.ld ? mid : b;
            he = e;
            k.s_entries += e - b;
        }
    }
    // Light entries of the produced frontier, summed per block (they decide
    // whether the bucket goes on by sub-buckets).
    const unsigned long long fe = warp_sum((unsigned long long)(le - lb));
    if (lane_id() == 0 && fe) atomicAdd(&x.st.bcnt[7], fe);
    // Each vertex enters a frontier once per phase and a heavy set once per
    // bucket, so no list exceeds n entries.
    bool ok = frontier_append_staged(x.st.f, x.Fout, x.FBout, a.n, &c->sn.f_small[x.f_slot], &c->sn.f_big[x.f_slot], f, v,
                                     le - lb, a.big_deg, a.chunk);
    ok &= frontier_append_staged(x.st.s, x.Sl, x.SBl, a.n, &c->sn.s_small[x.s_slot], &c->sn.s_big[x.s_slot], s, v, he - hb,
                                 a.big_deg, a.chunk);
    // Once per vertex and sub-bucket, so the set stays within n entries.
    if (x.sub_mode)
        ok &= frontier_append_staged(x.st.d, x.Dl, x.DBl, a.n, &c->sn.d_small[x.d_slot], &c->sn.d_big[x.d_slot], d, v,
                                     dl, a.big_deg, a.chunk);
    if (!ok) atomicOr(&c->error, DEVERR_CAPACITY | site_bit(SITE_PUSH));
}

// Appends v for every lane with `want` to a warp's staging slice of any
// capacity: entries wait in the slice while they fit; otherwise the slice
// and this step's entries go to the global list together under one
// atomicAdd.  A hot queue (all warps pushing to the same few bucket or
// sub-bucket queues) then costs one global atomic per slice-full, not per
// warp step.  All 32 lanes call it.
__device__ __forceinline__ bool stage_push(const WarpStage &q, bool want, unsigned v, unsigned *L, uint64_t n,
                                           unsigned *gcount) {
    const unsigned mask = __ballot_sync(FULL, want);
    if (!mask) return true;
    const unsigned c = *q.cnt;
    const unsigned k = __popc(mask);
    const unsigned rank = __popc(mask & lanemask_lt());
    bool ok = true;
    if (c + k <= q.cap) {
        if (want) q.buf[c + rank] = v;
    } else {
        unsigned base = 0;
        if (lane_id() == 0) base = atomicAdd(gcount, c + k);
        base = __shfl_sync(FULL, base, 0);
        ok = (uint64_t)base + c + k <= n;
        if (ok) {
            if (lane_id() < c) L[base + lane_id()] = q.buf[lane_id()];
            if (want) L[base + c + rank] = v;
        }
    }
    __syncwarp();
    if (lane_id() == 0) *q.cnt = c + k <= q.cap ? c + k : 0u;
    __syncwarp();
    return ok;
}

// Appends v to sub-bucket queue j of the current bucket (lanes with j >= 0)
// unless v already sits in queue j or an earlier one (jstamp <= key): its
// distance, hence its sub-bucket, only decreases, so every queue receives v
// at most once.  Lanes with the same j append together with one atomicAdd.
// All 32 lanes call it.
__device__ __forceinline__ void push_fine(const SsspArgs &a, const PushCtx &x, int j, unsigned v) {
    const unsigned key = j >= 0 ? fine_key(x.bucket, j) : 0u;
    const bool r = j >= 0 && atomicMin(&a.jstamp[v], key) > key;
    unsigned todo = __ballot_sync(FULL, r);
    while (todo) {
        const int q = __shfl_sync(FULL, j, __ffs(todo) - 1);
        const bool mine = r && j == q;
        const unsigned m = __ballot_sync(FULL, mine);
        // A vertex enters each sub-bucket queue at most once per bucket, so
        // no queue exceeds n entries.
        WarpStage st{x.st.qbuf + q * STAGE_Q, x.st.qcnt + q, STAGE_Q};
        if (!stage_push(st, mine, v, a.fq + (uint64_t)q * a.n, a.n, &a.ctl->sn.fq_len[q]))
            atomicOr(&a.ctl->error, DEVERR_CAPACITY | site_bit(SITE_FINE));
        todo &= ~m;
    }
}

// Edges of one warp step, E per lane: their target vertices' settled bits
// and packed distances are loaded together before any is used, so the
// step costs one chain of memory round trips, not E.
#ifndef SSSP_EDGES_PER_LANE
#define SSSP_EDGES_PER_LANE 2
#endif
constexpr int SSSP_EDGES = SSSP_EDGES_PER_LANE;

struct EdgeProbe {
    unsigned v[SSSP_EDGES];
    float wt[SSSP_EDGES];
    unsigned u[SSSP_EDGES];
    float du[SSSP_EDGES];
    bool has[SSSP_EDGES];
    unsigned long long cur[SSSP_EDGES];  // v's packed distance/parent, ~0 if not needed
};

// Fills p.cur for the edges in p (settled targets and non-vertices get
// UNREACHED-free zero so relax() skips them).  In light phases most targets
// are not settled, so the settled bits and the distances are loaded
// together (one memory round trip); in heavy phases most targets are
// settled, so a distance is loaded only after its bit says it is needed.
__device__ __forceinline__ void probe_edges(const SsspArgs &a, Counts &k, EdgeProbe &p, bool heavy) {
    unsigned sw[SSSP_EDGES];
#pragma unroll
    for (int t = 0; t < SSSP_EDGES; ++t) {
        k.edges += p.has[t];
        if (p.has[t] && p.v[t] >= a.n) {  // not a vertex: report it, touch nothing
            atomicOr(&a.ctl->error, DEVERR_RANGE);
            p.has[t] = false;
        }
        sw[t] = p.has[t] ? __ldcg(&a.settled[p.v[t] >> 5]) : 0u;
        p.cur[t] = p.has[t] && !heavy ? __ldcg(&a.pack[p.v[t]]) : 0ull;
    }
#pragma unroll
    for (int t = 0; t < SSSP_EDGES; ++t) {
        const bool settled = (sw[t] >> (p.v[t] & 31)) & 1u;
        k.settled += p.has[t] && settled;
        p.has[t] = p.has[t] && !settled;
        if (heavy) p.cur[t] = p.has[t] ? __ldcg(&a.pack[p.v[t]]) : 0ull;
    }
}

// Offers v the packed distance/parent np (cur = v's packed value as last
// read); queues v when its distance dropped.  All 32 lanes call it (want =
// lane has a candidate for a vertex not settled).
// Runs the pushes of up to 32 waiting entries, one per lane (have = the lane
// holds one: vertex v, what = P_* | argument).  All 32 lanes call it.
__device__ __forceinline__ void run_pushes(const SsspArgs &a, const PushCtx &x, Counts &k, bool have, unsigned v,
                                        unsigned what) {
    const unsigned cls = what & 0xf00u, arg = what & 0xffu;
    const bool same = have && cls == P_SAME;
    const int fine = have && cls == P_FINE ? (int)arg : -1;
    const int target = have && cls == P_RING ? (int)(x.bucket + arg) : -1;
    push_same_bucket(a, x, k, same, same || fine >= 0, v);
    if (x.sub_mode) {
        push_fine(a, x, fine, v);
        k.front += fine >= 0;
    }
    // Ring queue of the target bucket unless v already sits in that queue or
    // an earlier one (rstamp <= target): targets only decrease, so a stale
    // push that runs late (after a lower one) is dropped here and no queue
    // receives v twice.  Staged in the block's shared memory.
    const bool r = target >= 0 && atomicMin(&a.rstamp[v], (unsigned)target) > (unsigned)target;
    k.ring += r;
    k.front += same;
    // Per-slot warp staging: lanes with the same target slot append
    // together; a full slot is flushed to its global queue first.
    const int slot = r ? target % RING : RING;
    unsigned todo = __ballot_sync(FULL, r);
    while (todo) {
        const int sl = __shfl_sync(FULL, slot, __ffs(todo) - 1);
        const bool mine = r && slot == sl;
        const unsigned m = __ballot_sync(FULL, mine);
        WarpStage q{x.st.rbuf + sl * STAGE_R, x.st.rcnt + sl, STAGE_R};
        if (!stage_push(q, mine, v, a.ring + (uint64_t)sl * a.n, a.n, &a.ctl->sn.ring_len[sl]))
            atomicOr(&a.ctl->error, DEVERR_CAPACITY | site_bit(SITE_RING));
        todo &= ~m;
    }
}

// Runs the waiting pushes of this warp (at the end of a phase).  All 32
// lanes call it.
__device__ __forceinline__ void drain_pushes(const SsspArgs &a, const PushCtx &x, Counts &k) {
    __syncwarp();
    const unsigned c = *x.st.pcnt;
    if (!c) return;
    const bool have = lane_id() < c;
    run_pushes(a, x, k, have, have ? x.st.pv[lane_id()] : 0u, have ? x.st.pw[lane_id()] : 0u);
    __syncwarp();
    if (lane_id() == 0) *x.st.pcnt = 0;
    __syncwarp();
}

// Offers v the packed distance/parent np (cur = v's packed value as last
// read); when its distance drops, queues the push it needs (this bucket's
// frontier, a later sub-bucket or a later bucket).  All 32 lanes call it
// (want = lane has a candidate for a vertex not settled).
__device__ __forceinline__ void lower(const SsspArgs &a, const PushCtx &x, Counts &k, bool want, unsigned v,
                                      unsigned long long np, unsigned long long cur, bool heavy_phase) {
    unsigned what = 0;
    if (want) {
        const float cand = pack_dist(np);
        if (np < cur) {
            ++k.atomics;
            const unsigned long long old = atomicMin(&a.pack[v], np);
            if (np < old && (old >> 32) != (np >> 32)) {
                ++k.improved;
                if (cand < x.bnd[1]) {
                    if (heavy_phase) {  // cannot happen: heavy weights are >= delta
                        atomicOr(&a.ctl->error, DEVERR_CAPACITY | site_bit(SITE_HEAVY_SAME));
                        if (atomicCAS(&a.ctl->dbg_claim, 0u, 1u) == 0u) {
                            unsigned long long *d = a.ctl->dbg;
                            d[0] = v;
                            d[1] = np;
                            d[2] = __ldcg(&a.pack[(unsigned)np]);
                            d[3] = __float_as_uint(x.bnd[0]);
                            d[4] = __float_as_uint(x.bnd[1]);
                            d[5] = x.bucket;
                            d[6] = x.pid;
                        }
                    }
                    else if (cand < x.sub_hi) what = P_SAME;
                    else what = P_FINE | (unsigned)sub_index(x.sub, cand);  // a later sub-bucket of this bucket
                } else {
                    // Largest j with b_{B+j} <= cand; the ring holds B+1 .. B+RING-1.
                    int j = 1;
                    while (j < RING && x.bnd[j + 1] <= cand) ++j;
                    if (j >= RING) atomicOr(&a.ctl->error, DEVERR_RING);
                    else what = P_RING | (unsigned)j;
                }
            }
        }
    }
    const unsigned m = __ballot_sync(FULL, what != 0);
    if (!m) return;  // nothing lowered in this warp step
    unsigned c = *x.st.pcnt;  // < 32, so c + 32 <= PEND
    if (what) {
        const unsigned i = c + __popc(m & lanemask_lt());
        x.st.pv[i] = v;
        x.st.pw[i] = what;
    }
    c += __popc(m);
    __syncwarp();
    if (c >= 32) {  // run the last 32 (one per lane); the rest stays below 32
        c -= 32;
        const unsigned pv = x.st.pv[c + lane_id()], pw = x.st.pw[c + lane_id()];
        __syncwarp();
        run_pushes(a, x, k, true, pv, pw);
    }
    if (lane_id() == 0) *x.st.pcnt = c;
    __syncwarp();
}

// Relaxes u -> v with float weight wt from distance du (cur = v's packed
// value read by probe_edges).  All 32 lanes call it.
__device__ __forceinline__ void relax(const SsspArgs &a, const PushCtx &x, Counts &k, bool want, unsigned u, float du,
                                      unsigned v, float wt, unsigned long long cur, bool heavy_phase) {
    const float cand = __fadd_rn(du, wt);
    const unsigned long long np = ((unsigned long long)__float_as_uint(cand) << 32) | u;
    lower(a, x, k, want, v, np, cur, heavy_phase);
}

// Writes every staged entry of this warp to its global list and the warp's
// counts to the control block.  Every thread of the block calls it at the
// end of a phase (it synchronises the block once).
__device__ void stage_flush(const SsspArgs &a, const PushCtx &x, Counts &k) {
    SsspCtl *c = a.ctl;
    drain_pushes(a, x, k);
    {
        unsigned long long v[7] = {k.edges, k.settled, k.atomics, k.improved, k.ring, k.front, k.s_entries};
        unsigned long long *dst[8] = {&c->n_edges, &c->n_settled, &c->n_atomic, &c->n_improved, &c->n_ring,
                                      &c->n_front, &c->sn.s_entries[x.s_slot], &c->sn.f_entries[x.f_slot]};
        // Warp sums meet in the block's shared counters; one thread per
        // block adds them to the control block (a few hundred global atomics
        // per phase instead of several per warp on the same words).
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            const unsigned long long t = warp_sum(v[i]);
            if (lane_id() == 0 && t) atomicAdd(&x.st.bcnt[i], t);
        }
        k = Counts{0, 0, 0, 0, 0, 0, 0ull};
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (x.st.bcnt[i]) atomicAdd(dst[i], x.st.bcnt[i]);
                x.st.bcnt[i] = 0;  // the next phase adds after the grid barrier's __syncthreads
            }
        }
    }
    bool ok = stage_flush_warp(x.st.f, x.Fout, a.n, &c->sn.f_small[x.f_slot]);
    ok &= stage_flush_warp(x.st.s, x.Sl, a.n, &c->sn.s_small[x.s_slot]);
    if (x.sub_mode) ok &= stage_flush_warp(x.st.d, x.Dl, a.n, &c->sn.d_small[x.d_slot]);
    // Only the slices holding entries (one ballot over their counts).
    static_assert(RING <= 32, "one lane per ring slice");
    __syncwarp();
    unsigned todo = __ballot_sync(FULL, lane_id() < RING && x.st.rcnt[lane_id()] != 0);
    while (todo) {
        const int sl = __ffs(todo) - 1;
        todo &= todo - 1;
        WarpStage q{x.st.rbuf + sl * STAGE_R, x.st.rcnt + sl, STAGE_R};
        ok &= stage_flush_warp(q, a.ring + (uint64_t)sl * a.n, a.n, &c->sn.ring_len[sl]);
    }
    for (int j0 = 0; x.sub_mode && j0 < SUB; j0 += 32) {
        todo = __ballot_sync(FULL, j0 + lane_id() < SUB && x.st.qcnt[j0 + lane_id()] != 0);
        while (todo) {
            const int j = j0 + __ffs(todo) - 1;
            todo &= todo - 1;
            WarpStage q{x.st.qbuf + j * STAGE_Q, x.st.qcnt + j, STAGE_Q};
            ok &= stage_flush_warp(q, a.fq + (uint64_t)j * a.n, a.n, &c->sn.fq_len[j]);
        }
    }
    if (!ok && lane_id() == 0) atomicOr(&c->error, DEVERR_CAPACITY | site_bit(SITE_FLUSH));
}

// Which light edges an expansion relaxes: all, only those whose candidate
// distance falls below x.sub_hi (a sub-bucket's frontier), or only the others
// (its settle pass).
enum { SEL_ALL = 0, SEL_SAME = 1, SEL_LATER = 2 };

// Relaxes the light (heavy = false) or heavy edges of every vertex of list L
// (small part [0, ns), big part at the back, `bp` its packed counter).  The
// heavy pass also marks each list vertex settled.
__device__ void expand_list(const SsspArgs &a, const PushCtx &x, Counts &k, const unsigned *L, unsigned ns,
                            unsigned long long bp, const unsigned *B, unsigned *grab, unsigned *cgrab, bool heavy,
                            bool sparse_out, int sel = SEL_ALL) {
    const unsigned lane = lane_id();
    const bool filtered = a.ld == nullptr;
    const unsigned nw = (gridDim.x * blockDim.x) >> 5;
    const unsigned wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned g = grab_size(ns, nw, SSSP_GRAB);
    // Each warp's first grab is static (warp wg takes [wg*g, wg*g + g)); the
    // rest come from the counter, offset past the static range.  A short
    // list then costs no atomics on the shared counter.
    bool first = true;
    for (;;) {
        unsigned long long base;
        if (first) {
            base = (unsigned long long)wg * g;
            first = false;
        } else {
            unsigned b = 0;
            if (lane == 0) b = atomicAdd(grab, g);
            base = (unsigned long long)nw * g + __shfl_sync(FULL, b, 0);
        }
        if (base >= ns) break;
        const unsigned long long i = base + lane;
        const bool valid = lane < g && i < ns;
        const unsigned u = valid ? __ldcg(&L[i]) : 0u;
        uint64_t rb = 0, re = 0;
        float du = 0.0f;
        if (valid) {
            part_range(a, u, heavy, rb, re);
            if (sel == SEL_SAME && x.tiny_rows) re = rb + __ldg(&a.td[u]);
            const unsigned long long pu = __ldcg(&a.pack[u]);
            du = pack_dist(pu);
            if (heavy) settle(a, sparse_out, u, pu);
        }
        const unsigned deg = (unsigned)(re - rb);
        const unsigned incl = warp_incl_scan(deg);
        const unsigned total = __shfl_sync(FULL, incl, 31);
        const unsigned excl = incl - deg;
        for (unsigned e0 = 0; e0 < total; e0 += 32 * SSSP_EDGES) {
            EdgeProbe p;
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) {
                const unsigned e = e0 + 32 * t + lane;
                bool has = e < total;
                const int j = warp_owner(excl, has ? e : total - 1);
                p.u[t] = __shfl_sync(FULL, u, j);
                const uint64_t rbj = __shfl_sync(FULL, rb, j);
                const unsigned exj = __shfl_sync(FULL, excl, j);
                p.du[t] = __shfl_sync(FULL, du, j);
                p.v[t] = 0;
                p.wt[t] = 0.0f;
                if (has) {
                    const uint64_t at = rbj + (e - exj);
                    p.v[t] = (unsigned)__ldg(&a.col[at]);
                    p.wt[t] = __ldg(&a.w[at]);
                    if (filtered) has = heavy ? !(p.wt[t] < a.light) : p.wt[t] < a.light;
                    if (sel != SEL_ALL) has = has && ((__fadd_rn(p.du[t], p.wt[t]) < x.sub_hi) == (sel == SEL_SAME));
                }
                p.has[t] = has;
            }
            probe_edges(a, k, p, heavy);
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) relax(a, x, k, p.has[t], p.u[t], p.du[t], p.v[t], p.wt[t], p.cur[t], heavy);
        }
    }
    const unsigned nb = big_count(bp);
    const unsigned long long nch = big_chunks(bp);
    first = true;
    for (;;) {
        unsigned ch;
        if (first) {
            ch = wg;
            first = false;
        } else {
            unsigned b = 0;
            if (lane == 0) b = atomicAdd(cgrab, 1u);
            ch = nw + __shfl_sync(FULL, b, 0);
        }
        if (ch >= nch) break;
        const unsigned j = chunk_owner(B, nb, ch);
        const unsigned u = __ldcg(&L[a.n - 1 - j]);
        const unsigned cfirst = __ldcg(&B[j]);
        uint64_t rb, re;
        part_range(a, u, heavy, rb, re);
        if (sel == SEL_SAME && x.tiny_rows) re = rb + __ldg(&a.td[u]);
        const unsigned long long pu = __ldcg(&a.pack[u]);
        const float du = pack_dist(pu);
        if (heavy && ch == cfirst && lane == 0) settle(a, sparse_out, u, pu);
        const uint64_t deg = re - rb;
        const uint64_t cs = (uint64_t)(ch - cfirst) * a.chunk;
        const uint64_t ce = min(cs + a.chunk, deg);
        for (uint64_t e0 = cs + lane; e0 < cs + a.chunk; e0 += 32 * SSSP_EDGES) {
            EdgeProbe p;
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) {
                const uint64_t e = e0 + 32 * t;
                bool has = e < ce;
                p.u[t] = u;
                p.du[t] = du;
                p.v[t] = 0;
                p.wt[t] = 0.0f;
                if (has) {
                    p.v[t] = (unsigned)__ldg(&a.col[rb + e]);
                    p.wt[t] = __ldg(&a.w[rb + e]);
                    if (filtered) has = heavy ? !(p.wt[t] < a.light) : p.wt[t] < a.light;
                    if (sel != SEL_ALL) has = has && ((__fadd_rn(du, p.wt[t]) < x.sub_hi) == (sel == SEL_SAME));
                }
                p.has[t] = has;
            }
            probe_edges(a, k, p, heavy);
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) relax(a, x, k, p.has[t], p.u[t], p.du[t], p.v[t], p.wt[t], p.cur[t], heavy);
        }
    }
}

// Grid barrier, then a copy of the control block's list sizes into the
// block's shared snapshot (SNAP_WORDS threads, one word each).  Every read
// of those sizes after a barrier uses the snapshot.
__device__ __forceinline__ bool sssp_sync(const SsspArgs &a, unsigned &epoch, SsspSnap *sp) {
    if (a.nblocks == 1) {
        // One block (a search in a small component): the block barrier
        // orders every global write of the phase before the next phase.
        __syncthreads();
        if (ld_volatile(&a.ctl->error)) return false;
    } else if (!grid_sync(&a.ctl->bar, &a.ctl->error, epoch, a.nblocks, a.limit_ns)) {
        return false;
    }
    static_assert(SNAP_WORDS <= SSSP_THREADS, "one word per thread");
    if (threadIdx.x < SNAP_WORDS)
        ((unsigned *)sp)[threadIdx.x] = ld_volatile(&((const unsigned *)&a.ctl->sn)[threadIdx.x]);
    __syncthreads();
    return true;
}

// A list of capacity n keeps its small part at the front and its big part
// at the back, each append checked against n on its own side only.  The
// parts hold distinct vertices, so together they stay within n; a consumer
// checks the sum all the same (every block reads the same snapshot, so all
// leave together) and reports an overlap instead of reading a list whose
// parts may have overwritten each other.
__device__ __forceinline__ bool list_fits(const SsspArgs &a, unsigned ns, unsigned long long bp, int site) {
    if ((uint64_t)ns + big_count(bp) <= a.n) return true;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctl->error, DEVERR_CAPACITY | site_bit(site));
    return false;
}

// ---- heavy-phase pull -------------------------------------------------------
// When a bucket's rows hold at least pull_ratio times the CSR entries of the
// rows of all vertices not settled yet, its heavy phase runs the other way
// round: every unsettled vertex v scans its own heavy entries (u, w) -- the
// same undirected edges, stored in both rows -- and keeps the smallest
// (fl(d_u + w), u) over the u settled in this bucket.  That is the value the
// pushes from the bucket would leave in pack[v] (their atomicMin sees the
// same candidates), so the distances and parents are the same, but the work
// is proportional to the unsettled vertices' rows, which after the first
// large buckets are a small part of the graph.  Rows with more than BIG_DEG
// heavy entries are cut into BIG_CHUNK chunks taken by warps from one
// grid-wide counter, as in the frontier lists.

constexpr int PULL_EDGES = 2;

// Marks every vertex of the heavy set settled (outputs written when
// pre-filled) and sets its bit in `cur`.
__device__ void pull_settle(const SsspArgs &a, bool sparse_out, const unsigned *L, unsigned ns,
                            unsigned long long bp) {
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t total = (uint64_t)ns + big_count(bp);
    for (uint64_t i = gtid; i < total; i += nthreads) {
        const unsigned u = __ldcg(&L[i < ns ? i : a.n - 1 - (i - ns)]);
        settle(a, sparse_out, u, __ldcg(&a.pack[u]));
        atomicOr(&a.cur[u >> 5], 1u << (u & 31));
    }
}

// Candidates of PULL_EDGES heavy entries (u[t], w[t]) for their row's
// vertex: (fl(d_u + w), u) when u is in `cur`, UNREACHED otherwise.  The
// bitmap probes, then the distance loads, are issued together.
__device__ __forceinline__ void pull_probe(const SsspArgs &a, Counts &k, const unsigned *u, const float *w,
                                           const bool *has, unsigned long long *cand) {
    unsigned cw[PULL_EDGES];
#pragma unroll
    for (int t = 0; t < PULL_EDGES; ++t) {
        bool ok = has[t];
        k.edges += ok;
        if (ok && u[t] >= a.n) {  // not a vertex: report it, touch nothing
            atomicOr(&a.ctl->error, DEVERR_RANGE);
            ok = false;
        }
        cw[t] = ok ? (__ldcg(&a.cur[u[t] >> 5]) >> (u[t] & 31)) & 1u : 0u;
    }
    unsigned long long pu[PULL_EDGES];
#pragma unroll
    for (int t = 0; t < PULL_EDGES; ++t) pu[t] = cw[t] ? __ldcg(&a.pack[u[t]]) : UNREACHED;
#pragma unroll
    for (int t = 0; t < PULL_EDGES; ++t) {
        const float c = __fadd_rn(pack_dist(pu[t]), w[t]);
        cand[t] = cw[t] ? ((unsigned long long)__float_as_uint(c) << 32) | u[t] : UNREACHED;
    }
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x = min(x, __shfl_xor_sync(FULL, x, d));
    return x;
}

// Pull over every 32-vertex word of the settled bitmap: rows of at most
// BIG_DEG heavy entries are gathered by the word's warp (their entries
// walked 32 x PULL_EDGES at a time, each lane's candidates folded into its
// row's slot of s_best with a shared-memory atomicMin); longer rows go to
// the list (LL, LB) for pull_long.
__device__ void pull_words(const SsspArgs &a, const PushCtx &x, Counts &k, unsigned long long *s_best,
                           unsigned *LL, unsigned *LB) {
    SsspCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const bool filtered = a.ld == nullptr;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t nwords = (a.n + 31) >> 5;
    for (uint64_t kw = warp; kw < nwords; kw += nwarps) {
        const unsigned sw = __ldcg(&a.settled[kw]);
        if (sw == FULL) continue;  // warp-uniform
        const uint64_t v = kw * 32 + lane;
        const bool live = v < a.n && !((sw >> lane) & 1u);
        uint64_t hb = 0, he = 0;
        if (live) part_range(a, (unsigned)v, true, hb, he);
        const uint64_t hdeg = he - hb;
        const bool longrow = hdeg > BIG_DEG;
        if (!frontier_append(LL, LB, a.n, &c->pl_small, &c->sn.pl_big, longrow, (unsigned)v, hdeg))
            atomicOr(&c->error, DEVERR_CAPACITY | site_bit(SITE_PULL));
        const unsigned deg = longrow ? 0u : (unsigned)hdeg;
        const unsigned incl = warp_incl_scan(deg);
        const unsigned total = __shfl_sync(FULL, incl, 31);
        if (total == 0) continue;  // warp-uniform
        const unsigned excl = incl - deg;
        s_best[lane] = UNREACHED;
        __syncwarp();
        for (unsigned e0 = 0; e0 < total; e0 += 32 * PULL_EDGES) {
            unsigned u[PULL_EDGES];
            float w[PULL_EDGES];
            bool has[PULL_EDGES];
            int own[PULL_EDGES];
#pragma unroll
            for (int t = 0; t < PULL_EDGES; ++t) {
                const unsigned e = e0 + 32 * t + lane;
                has[t] = e < total;
                own[t] = warp_owner(excl, has[t] ? e : total - 1);
                const uint64_t hbj = __shfl_sync(FULL, hb, own[t]);
                const unsigned exj = __shfl_sync(FULL, excl, own[t]);
                u[t] = 0;
                w[t] = 0.0f;
                if (has[t]) {
                    const uint64_t at = hbj + (e - exj);
                    u[t] = (unsigned)__ldg(&a.col[at]);
                    w[t] = __ldg(&a.w[at]);
                    if (filtered) has[t] = !(w[t] < a.light);
                }
            }
            unsigned long long cand[PULL_EDGES];
            pull_probe(a, k, u, w, has, cand);
#pragma unroll
            for (int t = 0; t < PULL_EDGES; ++t)
                if (cand[t] != UNREACHED) atomicMin(&s_best[own[t]], cand[t]);
        }
        __syncwarp();
        const unsigned long long best = s_best[lane];
        __syncwarp();  // every lane has read its slot before the next word resets it
        const bool want = best != UNREACHED;
        const unsigned long long curv = want ? __ldcg(&a.pack[v]) : 0ull;
        lower(a, x, k, want, (unsigned)v, best, curv, true);
    }
}

// Pull of the long rows listed by pull_words (big part of LL, chunk bases
// LB): one BIG_CHUNK chunk per warp grab, the chunk's best candidate offered
// with one atomicMin.
__device__ void pull_long(const SsspArgs &a, const PushCtx &x, Counts &k, const unsigned *LL, const unsigned *LB,
                          const SsspSnap *sp) {
    SsspCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const bool filtered = a.ld == nullptr;
    const unsigned long long bp = sp->pl_big;
    const unsigned nb = big_count(bp);
    const unsigned long long nch = big_chunks(bp);
    const unsigned nw = (gridDim.x * blockDim.x) >> 5;
    bool first = true;  // first chunk static (the warp's id), then from the counter
    for (;;) {
        unsigned ch;
        if (first) {
            ch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            first = false;
        } else {
            unsigned b = 0;
            if (lane == 0) b = atomicAdd(&c->pl_cgrab, 1u);
            ch = nw + __shfl_sync(FULL, b, 0);
        }
        if (ch >= nch) break;
        const unsigned j = chunk_owner(LB, nb, ch);
        const unsigned v = __ldcg(&LL[a.n - 1 - j]);
        uint64_t hb, he;
        part_range(a, v, true, hb, he);
        const uint64_t cs = (uint64_t)(ch - __ldcg(&LB[j])) * BIG_CHUNK;
        const uint64_t ce = min(cs + BIG_CHUNK, he - hb);
        unsigned long long m = UNREACHED;
        for (uint64_t e0 = cs + lane; e0 < cs + BIG_CHUNK; e0 += 32 * PULL_EDGES) {
            unsigned u[PULL_EDGES];
            float w[PULL_EDGES];
            bool has[PULL_EDGES];
#pragma unroll
            for (int t = 0; t < PULL_EDGES; ++t) {
                const uint64_t e = e0 + 32 * t;
                has[t] = e < ce;
                u[t] = 0;
                w[t] = 0.0f;
                if (has[t]) {
                    u[t] = (unsigned)__ldg(&a.col[hb + e]);
                    w[t] = __ldg(&a.w[hb + e]);
                    if (filtered) has[t] = !(w[t] < a.light);
                }
            }
            unsigned long long cand[PULL_EDGES];
            pull_probe(a, k, u, w, has, cand);
#pragma unroll
            for (int t = 0; t < PULL_EDGES; ++t) m = min(m, cand[t]);
        }
        m = warp_min_u64(m);
        const bool want = lane == 0 && m != UNREACHED;
        const unsigned long long curv = want ? __ldcg(&a.pack[v]) : 0ull;
        lower(a, x, k, want, v, m, curv, true);
    }
}

__device__ __forceinline__ void trace_phase(SsspCtl *c, unsigned phase, int kind, unsigned size) {
    if (phase < SSSP_TRACE) {
        c->t_phase[phase] = globaltimer_ns();
        c->kind_phase[phase] = (unsigned char)kind;
        c->n_phase[phase] = size;
        c->e_phase[phase] = c->n_edges;
    }
}

// Blocks per SM the register allocation is sized for: 3 (80 registers a
// thread) spills 48 bytes a thread where 4 (64 registers) spilled 250, at
// the same S26 search time; 2 (128 registers, no spills) leaves too few
// warps to hide the relaxations' latency (5 % slower).
#ifndef SSSP_MIN_BLOCKS
#define SSSP_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(SSSP_THREADS, SSSP_MIN_BLOCKS) sssp_persistent_kernel(SsspArgs a) {
    SsspCtl *c = a.ctl;
    __shared__ float s_bnd[RING + 1];
    __shared__ float s_sub[SUB + 1];
    __shared__ bool s_tiny_ok;
    constexpr int WARPS = SSSP_THREADS / 32;
    __shared__ unsigned s_fbuf[WARPS][STAGE_F], s_sbuf[WARPS][STAGE_S], s_rbuf[WARPS][RING * STAGE_R];
    __shared__ unsigned s_fcnt[WARPS], s_scnt[WARPS], s_rcnt[WARPS][RING];
    __shared__ unsigned s_qbuf[WARPS][SUB * STAGE_Q], s_qcnt[WARPS][SUB];
    __shared__ unsigned s_pv[WARPS][PEND], s_pw[WARPS][PEND], s_pcnt[WARPS];
    __shared__ unsigned s_dbuf[WARPS][STAGE_D], s_dcnt[WARPS];
    __shared__ unsigned long long s_best[WARPS][32];
    __shared__ unsigned long long s_bcnt[8];
    __shared__ SsspSnap s_snap;
    SsspSnap *const sp = &s_snap;
    if (threadIdx.x < 8) s_bcnt[threadIdx.x] = 0;
    __syncthreads();
    const unsigned wid = threadIdx.x >> 5;
    if (lane_id() == 0) s_fcnt[wid] = s_scnt[wid] = 0;
    if (lane_id() < RING) s_rcnt[wid][lane_id()] = 0;
    for (int j = lane_id(); j < SUB; j += 32) s_qcnt[wid][j] = 0;
    if (lane_id() == 0) s_pcnt[wid] = s_dcnt[wid] = 0;
    __syncwarp();
    const Stage stage{WarpStage{s_fbuf[wid], &s_fcnt[wid], STAGE_F}, WarpStage{s_sbuf[wid], &s_scnt[wid], STAGE_S},
                      WarpStage{s_dbuf[wid], &s_dcnt[wid], STAGE_D}, s_rbuf[wid], s_rcnt[wid], s_qbuf[wid], s_qcnt[wid], s_bcnt, s_pv[wid], s_pw[wid],
                      &s_pcnt[wid]};
    unsigned epoch = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const bool prefilled = __ldcg((const unsigned long long *)&a.prefilled->dist) == (unsigned long long)a.dist &&
                           __ldcg((const unsigned long long *)&a.prefilled->pred) == (unsigned long long)a.pred;
    // Pre-filled outputs are written as vertices settle, unless the search
    // is renumbered: then one pass at the end writes them (in the caller's
    // numbering), which costs less than mapping every settle's writes.
    const bool sparse_out = prefilled && !a.inv;
    const unsigned long long e_total = __ldg(&a.rowptr[a.n]);
    unsigned long long settled_entries = 0;  // CSR entries of the rows of settled vertices

    if (gtid == 0) a.touch->small = 0;  // the next reset clears everything
    if (!a.roots) {
        if (gtid == 0) {
            const unsigned root = in_id(a, a.root);
            a.pack[root] = (unsigned long long)root;  // distance 0.0f, parent = root
            a.ring[0] = root;
            a.rstamp[root] = 0;
            c->sn.ring_len[0] = 1;
        }
    } else {
        // Several sources (disjoint graphs packed into one CSR, one source
        // each) all start in bucket 0; a repeated source is queued once.
        for (uint64_t i = gtid; i < a.nroots; i += nthreads) {
            const uint64_t r0 = __ldg(&a.roots[i]);
            const uint64_t r = r0 < a.n ? in_id(a, r0) : r0;
            if (r >= a.n) {
                atomicOr(&c->error, DEVERR_RANGE);
            } else if (atomicCAS(&a.rstamp[r], 0xffffffffu, 0u) == 0xffffffffu) {
                a.pack[r] = r;
                a.ring[atomicAdd(&c->sn.ring_len[0], 1u)] = (unsigned)r;
            }
        }
    }
    if (!sssp_sync(a, epoch, sp)) return;

    unsigned bucket = 0, phase = 0;
    float blo = 0.0f;
    Counts cnt{0, 0, 0, 0, 0, 0, 0ull};
    if (gtid == 0) c->t0 = globaltimer_ns();
    unsigned long long nbuckets = 0;
    unsigned dgen = 0;  // settle passes so far: the expanded set's counter slot alternates with it
    for (;;) {
        // ---- open the bucket: its ring queue becomes the first frontier.
        if (threadIdx.x == 0) {
            float b = blo;
            for (int j = 0; j <= RING; ++j) {
                s_bnd[j] = b;
                b = __fadd_rn(b, a.delta);
            }
            // t_j = b_B + j * (delta / SUB): monotone, t_0 = b_B, t_SUB = b_{B+1}.
            const float wf = a.delta / (float)SUB;
            for (int j = 0; j < SUB; ++j) s_sub[j] = __fadd_rn(blo, (float)j * wf);
            s_sub[SUB] = s_bnd[1];
            // Tiny prefixes hold every same-sub-bucket relaxation when an
            // entry of weight >= tiny from anywhere in sub-bucket j reaches
            // t_{j+1} or beyond (fl(d + w) is monotone in d and w).
            bool ok = a.td != nullptr;
            for (int j = 0; j < SUB && ok; ++j) ok = __fadd_rn(s_sub[j], a.tiny) >= s_sub[j + 1];
            s_tiny_ok = ok;
        }
        __syncthreads();
        PushCtx x;
        x.st = stage;
        x.bucket = bucket;
        x.bnd = s_bnd;
        x.sub = s_sub;
        x.sub_hi = s_bnd[1];
        x.sub_mode = false;
        x.tiny_rows = s_tiny_ok;
        int sj = -1;  // current sub-bucket in sub mode
        const int sb = (int)(nbuckets % 3);
        x.s_slot = sb;
        x.Sl = a.S[nbuckets & 1];
        x.SBl = a.SB[nbuckets & 1];
        // The other heavy-set arrays are idle until this bucket's heavy phase
        // (a pull borrows them there; the next bucket fills them).
        x.Dl = a.S[(nbuckets + 1) & 1];
        x.DBl = a.SB[(nbuckets + 1) & 1];
        x.d_slot = (int)(dgen & 1);
        x.d_tag = 0;
        bool just_settled = false;  // the snapshot still shows the settled set's size
        {
            const int s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->sn.f_small[s_clr] = 0;
                c->sn.f_big[s_clr] = c->sn.f_entries[s_clr] = 0;
                const int sn = (sb + 1) % 3;  // the next bucket's heavy-set slot
                c->sn.s_small[sn] = 0;
                c->sn.s_big[sn] = 0;
                c->sn.s_entries[sn] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            const unsigned slot = bucket % RING;
            const unsigned len = sp->ring_len[slot];
            const unsigned *R = a.ring + (uint64_t)slot * a.n;
            for (uint64_t base = gtid - lane_id(); base < len; base += nthreads) {
                const uint64_t i = base + lane_id();
                bool ok = false;
                unsigned v = 0;
                if (i < len) {
                    v = __ldcg(&R[i]);
                    const float d = pack_dist(__ldcg(&a.pack[v]));
                    ok = d >= s_bnd[0] && d < s_bnd[1] && !((__ldcg(&a.settled[v >> 5]) >> (v & 31)) & 1u);
                }
                push_same_bucket(a, x, cnt, ok, ok, v, true);
            }
            stage_flush(a, x, cnt);
            if (!sssp_sync(a, epoch, sp)) return;
            // The queue is consumed; nothing can target this slot again before
            // bucket + RING, which lies beyond every push of this bucket.
            if (gtid == 0) {
                c->sn.ring_len[slot] = 0;
                trace_phase(c, phase, 0, len);
            }
            ++phase;
        }
        // ---- light iterations until the bucket's frontier is empty (in sub
        // mode: until every sub-bucket's frontier is).  Every block reads the
        // same counters after a barrier, so all take the same branches.
        for (;;) {
            const int s_cur = phase % 3, s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            const unsigned ns = sp->f_small[s_cur];
            const unsigned long long bp = sp->f_big[s_cur];
            if (!list_fits(a, ns, bp, SITE_LIST_F)) return;
            const unsigned fsize = ns + big_count(bp);
            int nj = -1;
            if (fsize == 0) {
                if (!x.sub_mode) break;
                // Every block must take the same branch here, so it may
                // depend only on counters that no block can change during
                // this phase.  The expanded set's count is not one of them:
                // blocks that pass the barrier first and open the next
                // sub-bucket append to the set while slower blocks are still
                // copying the snapshot.  So an open sub-bucket whose frontier
                // has drained always gets its settle pass, even with an
                // empty expanded set (a sub-bucket whose queue entries were
                // all stale).
                if (!just_settled && sj >= 0) {
                    // Settle pass of sub-bucket sj: every distance in it is
                    // final; its expanded set relaxes the deferred edges.
                    // Nothing appends to the set in this phase, so its
                    // snapshot count is exact.  The other counter slot is
                    // cleared for the next set (appends to it start after
                    // this phase's barrier).
                    const unsigned dn = sp->d_small[x.d_slot];
                    const unsigned long long dbp = sp->d_big[x.d_slot];
                    if (!list_fits(a, dn, dbp, SITE_LIST_D)) return;
                    if (gtid == 0) {
                        c->grab[s_clr] = c->cgrab[s_clr] = c->sn.f_small[s_clr] = 0;
                        c->sn.f_big[s_clr] = c->sn.f_entries[s_clr] = 0;
                        c->sn.d_small[x.d_slot ^ 1] = 0;
                        c->sn.d_big[x.d_slot ^ 1] = 0;
                    }
                    x.pid = phase;
                    x.f_slot = s_nxt;
                    x.Fout = a.F[(phase + 1) & 1];
                    x.FBout = a.FB[(phase + 1) & 1];
                    expand_list(a, x, cnt, x.Dl, dn, dbp, x.DBl, &c->grab[s_cur], &c->cgrab[s_cur], false, sparse_out,
                                SEL_LATER);
                    stage_flush(a, x, cnt);
                    if (!sssp_sync(a, epoch, sp)) return;
                    if (gtid == 0) trace_phase(c, phase, 6, dn + big_count(dbp));
                    ++phase;
                    ++dgen;
                    x.d_slot = (int)(dgen & 1);
                    just_settled = true;
                    continue;
                }
                just_settled = false;
                for (int j = sj + 1; j < SUB; ++j)
                    if (sp->fq_len[j]) {
                        nj = j;
                        break;
                    }
                if (nj < 0) break;
            }
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->sn.f_small[s_clr] = 0;
                c->sn.f_big[s_clr] = c->sn.f_entries[s_clr] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            if (nj >= 0) {
                // Open sub-bucket nj: its queue's entries still in its range
                // become the frontier (they are in the heavy set already).
                sj = nj;
                x.sub_hi = s_sub[sj + 1];
                x.d_tag = fine_id(bucket, sj);
                const unsigned len = sp->fq_len[sj];
                const unsigned *Q = a.fq + (uint64_t)sj * a.n;
                for (uint64_t base = gtid - lane_id(); base < len; base += nthreads) {
                    const uint64_t i = base + lane_id();
                    bool ok = false;
                    unsigned v = 0;
                    if (i < len) {
                        v = __ldcg(&Q[i]);
                        const float d = pack_dist(__ldcg(&a.pack[v]));
                        ok = d >= s_sub[sj] && d < s_sub[sj + 1];
                    }
                    push_same_bucket(a, x, cnt, ok, false, v, true);
                }
                stage_flush(a, x, cnt);
                if (!sssp_sync(a, epoch, sp)) return;
                // Nothing is queued into sub-bucket sj once it is open.
                if (gtid == 0) {
                    c->sn.fq_len[sj] = 0;
                    trace_phase(c, phase, 4, len);
                }
                ++phase;
                continue;
            }
            if (!x.sub_mode && sp->f_entries[s_cur] >= a.split_min) {
                // Split: the frontier goes to the sub-bucket queues of its
                // distances; the bucket continues by sub-buckets in order.
                x.sub_mode = true;
                const uint64_t total = (uint64_t)fsize;
                const unsigned *L = a.F[phase & 1];
                for (uint64_t base = gtid - lane_id(); base < total; base += nthreads) {
                    const uint64_t i = base + lane_id();
                    int j = -1;
                    unsigned v = 0;
                    if (i < total) {
                        v = __ldcg(&L[i < ns ? i : a.n - 1 - (i - ns)]);
                        j = sub_index(s_sub, pack_dist(__ldcg(&a.pack[v])));
                    }
                    push_fine(a, x, j, v);
                }
                stage_flush(a, x, cnt);
                if (!sssp_sync(a, epoch, sp)) return;
                if (gtid == 0) {
                    ++c->splits;
                    trace_phase(c, phase, 5, fsize);
                }
                ++phase;
                continue;
            }
            expand_list(a, x, cnt, a.F[phase & 1], ns, bp, a.FB[phase & 1], &c->grab[s_cur], &c->cgrab[s_cur], false,
                        sparse_out, x.sub_mode ? SEL_SAME : SEL_ALL);
            stage_flush(a, x, cnt);
            if (!sssp_sync(a, epoch, sp)) return;
            if (gtid == 0) trace_phase(c, phase, 1, ns + big_count(bp));
            ++phase;
        }
        // ---- heavy edges of every vertex settled in this bucket.
        {
            const int s_cur = phase % 3, s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->sn.f_small[s_clr] = 0;
                c->sn.f_big[s_clr] = c->sn.f_entries[s_clr] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            const unsigned ns = sp->s_small[sb];
            const unsigned long long bp = sp->s_big[sb];
            if (!list_fits(a, ns, bp, SITE_LIST_S)) return;
            const unsigned long long s_ent = sp->s_entries[sb];
            // Every block reads the same counters after the barrier, so all
            // take the same branch.
            // A pull walks every word of the settled bitmap besides the
            // unsettled rows: that walk counts as PULL_WALK entries a vertex.
            const bool pull = a.pull_ratio > 0.0f &&
                              (double)s_ent >= (double)a.pull_ratio * ((double)(e_total - settled_entries - s_ent) +
                                                                       PULL_WALK * (double)a.n);
            settled_entries += s_ent;
            if (!pull) {
                expand_list(a, x, cnt, x.Sl, ns, bp, x.SBl, &c->grab[s_cur], &c->cgrab[s_cur], true, sparse_out);
                stage_flush(a, x, cnt);
                if (!sssp_sync(a, epoch, sp)) return;
                if (gtid == 0) trace_phase(c, phase, 2, ns + big_count(bp));
            } else {
                // The long-row list borrows the other heavy-set array: the
                // previous bucket is done with it and the next one starts
                // writing it only after this phase's last barrier.
                unsigned *LL = a.S[(nbuckets + 1) & 1], *LB = a.SB[(nbuckets + 1) & 1];
                pull_settle(a, sparse_out, x.Sl, ns, bp);
                if (!sssp_sync(a, epoch, sp)) return;
                pull_words(a, x, cnt, s_best[wid], LL, LB);
                stage_flush(a, x, cnt);
                if (!sssp_sync(a, epoch, sp)) return;
                pull_long(a, x, cnt, LL, LB, sp);
                stage_flush(a, x, cnt);
                if (!sssp_sync(a, epoch, sp)) return;
                // `cur` and the long-row counters are next used by a later
                // bucket's pull, several barriers from here.
                for (uint64_t i = gtid; i < ((a.n + 31) >> 5); i += nthreads) a.cur[i] = 0;
                if (gtid == 0) {
                    c->pl_small = 0;
                    c->sn.pl_big = 0;
                    c->pl_cgrab = 0;
                    ++c->pulls;
                    trace_phase(c, phase, 3, ns + big_count(bp));
                }
            }
            ++phase;
        }
        ++nbuckets;
        // ---- next non-empty bucket within the ring window.
        int step = 0;
        for (int j = 1; j < RING; ++j)
            if (sp->ring_len[(bucket + j) % RING]) {
                step = j;
                break;
            }
        if (!step) break;
        // Ring targets are absolute bucket numbers held in an int.
        if (bucket + (unsigned)step > 0x7fffffffu - RING) {
            if (gtid == 0) atomicOr(&c->error, DEVERR_RING);
            return;
        }
        for (int j = 0; j < step; ++j) blo = __fadd_rn(blo, a.delta);
        bucket += step;
        __syncthreads();  // s_bnd is rewritten at the top of the loop
    }
    if (gtid == 0) {
        c->buckets = nbuckets;
        c->phases = phase;
    }
    // Every distance is final (the last heavy phase ended at a grid barrier).
    // Outputs not written as vertices settled are written here: every
    // vertex, or with pre-filled outputs the reached ones.
    if (!sparse_out) {
        for (uint64_t v = gtid; v < a.n; v += nthreads) {
            const unsigned long long p = __ldcg(&a.pack[v]);
            if (p != UNREACHED || !prefilled) write_out(a, (unsigned)v, p);
        }
    }
}

// A search from a source whose component is small (g5_sssp_params.small):
// one block, label-correcting rounds (every vertex whose distance dropped in
// a round relaxes all its edges in the next) -- no buckets, phases or grid
// machinery.  It reaches the same float fixed point, hence the same
// distances, and the same parents (the smallest u on a tight edge: every
// vertex relaxes its edges again after its last decrease).  The first
// SMALL_L entries of each round's list and of the reached list live in
// shared memory, list entries with their row bounds, which the relaxing
// lane loads together with its atomicMin (issued before either returns);
// the rest go to the workspace lists.  Correct for a component of any size,
// only slow when it is large.
constexpr unsigned SMALL_L = 512;

// Row starts of v and v + 1 and atomicMin(pack[v], np), issued in this
// order without waiting for one another; returns pack[v]'s old value.
__device__ __forceinline__ unsigned long long relax_with_row(const uint64_t *rowptr, unsigned long long *pack,
                                                             unsigned v, unsigned long long np, uint64_t &rb,
                                                             uint64_t &re) {
    unsigned long long old;
    asm volatile("ld.global.nc.u64 %0, [%3];\n\t"
                 "ld.global.nc.u64 %1, [%3+8];\n\t"
                 "atom.global.min.u64 %2, [%4], %5;"
                 : "=l"(rb), "=l"(re), "=l"(old)
                 : "l"(rowptr + v), "l"(pack + v), "l"(np)
                 : "memory");
    return old;
}
__global__ void __launch_bounds__(SSSP_THREADS) sssp_small_kernel(SsspArgs a) {
    SsspCtl *c = a.ctl;
    __shared__ unsigned s_v[2][SMALL_L];
    __shared__ uint64_t s_rb[2][SMALL_L], s_re[2][SMALL_L];
    __shared__ unsigned s_r[SMALL_L];
    __shared__ unsigned s_len[2];
    __shared__ unsigned s_nreach;
    __shared__ unsigned s_err;
    __shared__ bool s_sparse;
    const unsigned lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned *R = a.S[0];  // every vertex reached, once (sstamp): the touched list
    if (threadIdx.x == 32) {
        // Whether the outputs were pre-filled: loaded by another warp while
        // the search runs, read after it.
        s_sparse = __ldcg((const unsigned long long *)&a.prefilled->dist) == (unsigned long long)a.dist &&
                   __ldcg((const unsigned long long *)&a.prefilled->pred) == (unsigned long long)a.pred;
    }
    if (threadIdx.x == 0) {
        c->t0 = globaltimer_ns();
        const unsigned root = in_id(a, a.root);
        a.pack[root] = (unsigned long long)root;  // distance 0.0f, parent = root
        a.sstamp[root] = 0;
        s_v[0][0] = root;
        s_rb[0][0] = __ldg(&a.rowptr[root]);
        s_re[0][0] = __ldg(&a.rowptr[root + 1]);
        s_r[0] = root;
        R[0] = root;
        s_len[0] = 1;
        s_len[1] = 0;
        s_nreach = 1;
        s_err = 0;
    }
    __syncthreads();
    unsigned round = 0;
    for (;; ++round) {
        const int cur = round & 1, nxt = cur ^ 1;
        const unsigned n = s_len[cur];
        if (n == 0) break;
        // One warp per listed vertex, its lanes over the vertex's row.
        for (unsigned i = wid; i < n; i += nw) {
            unsigned u;
            uint64_t rb, re;
            if (i < SMALL_L) {
                u = s_v[cur][i];
                rb = s_rb[cur][i];
                re = s_re[cur][i];
            } else {
                u = __ldcg(&a.F[cur][i]);
                rb = __ldg(&a.rowptr[u]);
                re = __ldg(&a.rowptr[u + 1]);
            }
            const float du = pack_dist(__ldcg(&a.pack[u]));
            for (uint64_t e = rb + lane; e < re; e += 32) {
                const unsigned v = (unsigned)__ldg(&a.col[e]);
                if (v >= a.n) {  // not a vertex: report it, touch nothing
                    atomicOr(&s_err, DEVERR_RANGE);
                    continue;
                }
                const float cand = __fadd_rn(du, __ldg(&a.w[e]));
                const unsigned long long np = ((unsigned long long)__float_as_uint(cand) << 32) | u;
                uint64_t vb, ve;
                const unsigned long long old = relax_with_row(a.rowptr, a.pack, v, np, vb, ve);
                if (!(np < old && (old >> 32) != (np >> 32))) continue;  // distance unchanged
                // The next round reads v's row: start bringing it into L2 now.
                if (vb < ve) {
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.col + vb));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.w + vb));
                }
                const unsigned fold = atomicExch(&a.fstamp[v], round);
                const unsigned sold = atomicExch(&a.sstamp[v], 0u);
                if (fold != round) {
                    const unsigned pos = atomicAdd(&s_len[nxt], 1u);  // once per vertex and round
                    if (pos < SMALL_L) {
                        s_v[nxt][pos] = v;
                        s_rb[nxt][pos] = vb;
                        s_re[nxt][pos] = ve;
                    } else if (pos < a.n) {
                        a.F[nxt][pos] = v;
                    } else {
                        atomicOr(&s_err, DEVERR_CAPACITY | site_bit(SITE_SMALL));
                    }
                }
                if (sold != 0u) {
                    const unsigned pos = atomicAdd(&s_nreach, 1u);
                    if (pos < SMALL_L) s_r[pos] = v;
                    if (pos < a.n) R[pos] = v;
                    else atomicOr(&s_err, DEVERR_CAPACITY | site_bit(SITE_SMALL));
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_len[cur] = 0;
            if (round < SSSP_TRACE) {
                c->t_phase[round] = globaltimer_ns();
                c->kind_phase[round] = 1;
                c->n_phase[round] = n;
                c->e_phase[round] = 0;
            }
        }
        __syncthreads();
    }
    // Outputs: the reached vertices (pre-filled outputs) or every vertex.
    if (s_sparse) {
        const unsigned nr = min(s_nreach, (unsigned)a.n);
        for (unsigned i = threadIdx.x; i < nr; i += blockDim.x) {
            const unsigned v = i < SMALL_L ? s_r[i] : __ldcg(&R[i]);
            write_out(a, v, __ldcg(&a.pack[v]));
        }
    } else {
        for (uint64_t v = threadIdx.x; v < a.n; v += blockDim.x) write_out(a, (unsigned)v, __ldcg(&a.pack[v]));
    }
    if (threadIdx.x == 0) {
        c->buckets = 1;
        c->phases = round;
        c->error |= s_err;
        // R lists every vertex this search wrote (a search that reported an
        // error leaves the next reset a full one).
        *a.touch = SsspTouch{s_err == 0 && s_nreach <= a.n ? 1u : 0u, s_sparse ? 1u : 0u, s_nreach, a.dist, a.pred,
                             a.inv};
    }
}

struct SsspWork {
    SsspCtl *ctl;
    SsspTouch *touch;
    SsspOut *out;
    unsigned long long *pack;
    unsigned *fstamp, *sstamp, *rstamp, *jstamp, *dstamp, *settled, *cur;
    unsigned *F[2], *FB[2], *S[2], *SB[2];
    unsigned *ring;
    unsigned *fq;
    uint64_t bytes;
};

static SsspWork carve_sssp(void *base, uint64_t n) {
    Carver c(base);
    SsspWork w;
    w.ctl = c.take<SsspCtl>(1);
    w.touch = c.take<SsspTouch>(1);
    w.out = c.take<SsspOut>(1);
    w.pack = c.take<unsigned long long>(n);
    w.fstamp = c.take<unsigned>(n);
    w.sstamp = c.take<unsigned>(n);
    w.rstamp = c.take<unsigned>(n);
    w.jstamp = c.take<unsigned>(n);
    w.dstamp = c.take<unsigned>(n);
    w.settled = c.take<unsigned>((n + 31) / 32);
    w.cur = c.take<unsigned>((n + 31) / 32);
    for (int i = 0; i < 2; ++i) {
        w.F[i] = c.take<unsigned>(n);
        w.FB[i] = c.take<unsigned>(n);
        w.S[i] = c.take<unsigned>(n);
        w.SB[i] = c.take<unsigned>(n);
    }
    w.ring = c.take<unsigned>((uint64_t)RING * n);
    w.fq = c.take<unsigned>((uint64_t)SUB * n);
    w.bytes = c.used;
    return w;
}

static int sssp_max_blocks(int *out) {
    static int cached[64] = {};
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if (!cached[di.device]) {
        if ((rc = persistent_kernel_setup((const void *)sssp_persistent_kernel))) return rc;
        int per_sm = 0;
        G5_CUDA_TRY(
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_persistent_kernel, SSSP_THREADS, 0));
        cached[di.device] = std::max(1, per_sm) * di.sms;
    }
    *out = cached[di.device];
    return G5_OK;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_sssp_workspace_size(uint64_t nverts, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_sssp_workspace_size: bytes is NULL");
    *bytes = carve_sssp(nullptr, nverts).bytes;
    return G5_OK;
}

static int sssp_check(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                      uint64_t root, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes, SsspWork *w,
                      const char *who) {
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "%s: nverts outside [1, 2^31]", who);
    G5_CHECK_ARG(root < nverts, "%s: root %llu outside [0, %llu)", who, (unsigned long long)root,
                 (unsigned long long)nverts);
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_dist && d_pred && d_work, "%s: NULL argument", who);
    *w = carve_sssp(d_work, nverts);
    if (work_bytes < w->bytes)
        return set_error(G5_ERR_WORKSPACE, "%s: workspace %llu < %llu bytes", who, (unsigned long long)work_bytes,
                         (unsigned long long)w->bytes);
    return G5_OK;
}

struct SsspResetArgs {
    uint64_t n;
    float *dist;
    int64_t *pred;
    SsspWork w;
    int full;  // 1: clear everything whatever the last search touched
};

// The reset before a search: packed distances ~0, the five stamp arrays ~0,
// settled and pull bitmaps 0, a fresh control block and, with outputs,
// dist = -1.0f / pred = -1 recorded as pre-filled.  After a one-block search
// (which touches only the packed distances, two stamp arrays and the
// outputs of the vertices it reached, all listed) those entries are
// restored one by one; anything else is cleared in full.  A touched reset
// reads the touch record in every block and leaves it alone; a full reset
// reads none of it and records "nothing touched" for these outputs.
__global__ void sssp_reset_kernel(SsspResetArgs r) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const SsspWork &w = r.w;
    const SsspTouch h = r.full ? SsspTouch{0u, 0u, 0ull, nullptr, nullptr, nullptr} : *w.touch;
    if (r.full && t == 0) *w.touch = SsspTouch{1u, r.dist ? 1u : 0u, 0ull, r.dist, r.pred, nullptr};
    const bool small = !r.full && h.small && h.count <= r.n;
    const bool out_t = small && h.sparse && h.dist == r.dist && h.pred == r.pred;
    if (blockIdx.x == 0) {
        constexpr unsigned words = sizeof(SsspCtl) / 4;
        static_assert(sizeof(SsspCtl) % 4 == 0, "control block cleared in words");
        for (unsigned i = threadIdx.x; i < words; i += blockDim.x) ((unsigned *)w.ctl)[i] = 0;
        if (threadIdx.x == 0) *w.out = SsspOut{r.dist, r.pred};
    }
    if (small) {
        const unsigned *L = w.S[0];
        for (uint64_t i = t; i < h.count; i += T) {
            const unsigned v = __ldg(&L[i]);
            if (v >= r.n) continue;
            w.pack[v] = UNREACHED;
            w.fstamp[v] = ~0u;
            w.sstamp[v] = ~0u;
            if (r.dist && out_t) {  // the outputs of a renumbered search are in the caller's numbering
                const unsigned o = h.inv ? __ldg(&h.inv[v]) : v;
                r.dist[o] = -1.0f;
                r.pred[o] = -1;
            }
        }
    } else {
        grid_fill<unsigned long long>(w.pack, r.n, UNREACHED, t, T);
        // fstamp .. dstamp are consecutive carve-outs.
        grid_fill<unsigned>(w.fstamp, (uint64_t)((w.dstamp + r.n) - w.fstamp), ~0u, t, T);
        grid_fill<unsigned>(w.settled, (r.n + 31) / 32, 0u, t, T);
        grid_fill<unsigned>(w.cur, (r.n + 31) / 32, 0u, t, T);
    }
    if (r.dist && !out_t) {
        grid_fill<float>(r.dist, r.n, -1.0f, t, T);
        grid_fill<int64_t>(r.pred, r.n, -1, t, T);
    }
}

static int sssp_reset_launch(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                             void *stream, int full, const char *who) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31) && d_work, "%s: bad argument", who);
    G5_CHECK_ARG((d_dist == nullptr) == (d_pred == nullptr), "%s: give both outputs or neither", who);
    SsspWork w = carve_sssp(d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "%s: workspace too small", who);
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    SsspResetArgs r{nverts, d_dist, d_pred, w, full};
    const uint64_t want = (nverts + 2047) / 2048;  // 2048 vertices a block when everything is cleared
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)di.sms * 8, want));
    sssp_reset_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(r);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_sssp_reset(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                             void *stream) {
    return sssp_reset_launch(nverts, d_dist, d_pred, d_work, work_bytes, stream, 1, "g5_sssp_reset");
}

extern "C" int g5_sssp_reset_touched(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work,
                                     uint64_t work_bytes, void *stream) {
    return sssp_reset_launch(nverts, d_dist, d_pred, d_work, work_bytes, stream, 0, "g5_sssp_reset_touched");
}

static int sssp_launch(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                       const uint32_t *d_light_deg, float light_delta, uint64_t nverts, uint64_t root,
                       const uint64_t *d_roots, unsigned nroots, float *d_dist, int64_t *d_pred, void *d_work,
                       uint64_t work_bytes, const g5_sssp_params *params, void *stream, const char *who) {
    SsspWork w;
    int rc = sssp_check(d_rowstarts, d_col, d_w, nverts, root, d_dist, d_pred, d_work, work_bytes, &w, who);
    if (rc) return rc;
    g5_sssp_params p = {0.1f, 0, 0.0f, 0, 0, nullptr, 0};
    if (params) p = *params;
    G5_CHECK_ARG(p.delta > 0.0f, "g5_sssp_traverse: delta must be positive");
    G5_CHECK_ARG(p.big_deg >= 0 && p.big_deg <= (1 << 20), "%s: big_deg %d outside [0, 2^20]", who, p.big_deg);
    G5_CHECK_ARG(p.chunk >= 0 && p.chunk <= (1 << 16) && p.chunk % (32 * SSSP_EDGES) == 0,
                 "%s: chunk %d is not a multiple of %d in [0, 65536]", who, p.chunk, 32 * SSSP_EDGES);
    G5_CHECK_ARG((p.perm == nullptr) == (p.inv == nullptr), "%s: give both perm and inv or neither", who);
    int max_blocks = 0;
    if ((rc = sssp_max_blocks(&max_blocks))) return rc;
    int blocks = p.blocks > 0 ? std::min(p.blocks, max_blocks)
                              : (int)std::min<uint64_t>(max_blocks, std::max<uint64_t>(1, nverts / 2048));
    cudaStream_t st = (cudaStream_t)stream;
    SsspArgs a;
    a.rowptr = d_rowstarts;
    a.col = d_col;
    a.w = d_w;
    // Rows split at light_delta serve any bucket width up to light_delta:
    // heavy edges (w >= light_delta >= delta) still land beyond the current
    // bucket.  A wider bucket filters every row by weight instead.
    const bool split = d_light_deg && p.delta <= light_delta;
    a.ld = split ? d_light_deg : nullptr;
    a.light = split ? light_delta : p.delta;
    a.td = split ? p.tiny_deg : nullptr;
    a.tiny = light_delta / (float)G5_TINY_DIV;
    a.n = nverts;
    a.root = (unsigned)root;
    a.roots = d_roots;
    a.nroots = nroots;
    a.delta = p.delta;
    a.pull_ratio = p.pull == 0.0f ? SSSP_PULL_RATIO : p.pull;
    a.split_min = p.sub_min == 0 ? SPLIT_MIN : p.sub_min < 0 ? ~0ull : (unsigned long long)p.sub_min;
    a.pack = w.pack;
    a.fstamp = w.fstamp;
    a.sstamp = w.sstamp;
    a.rstamp = w.rstamp;
    a.jstamp = w.jstamp;
    a.dstamp = w.dstamp;
    a.settled = w.settled;
    a.cur = w.cur;
    for (int i = 0; i < 2; ++i) {
        a.F[i] = w.F[i];
        a.FB[i] = w.FB[i];
        a.S[i] = w.S[i];
        a.SB[i] = w.SB[i];
    }
    a.ring = w.ring;
    a.fq = w.fq;
    a.ctl = w.ctl;
    a.touch = w.touch;
    a.prefilled = w.out;
    a.dist = d_dist;
    a.pred = d_pred;
    a.nblocks = (unsigned)blocks;
    a.limit_ns = wait_limit_ns();
    a.check_opens = p.check_opens != 0;
    a.big_deg = p.big_deg ? (unsigned)p.big_deg : SSSP_BIG_DEG;
    a.chunk = p.chunk ? (unsigned)p.chunk : SSSP_CHUNK;
    a.perm = p.perm;
    a.inv = p.inv;
    if (p.small && !d_roots) {
        sssp_small_kernel<<<1, SSSP_THREADS, 0, st>>>(a);
    } else if (blocks == 1) {  // nothing to co-schedule: a plain launch
        sssp_persistent_kernel<<<1, SSSP_THREADS, 0, st>>>(a);
    } else {
        // Cooperative launch.  (An L2 persisting window over the settled
        // bitmap and the packed distances, as the BFS has for its bitmaps,
        // made a SCALE 26 search slower: 41.2 ms against 33.8 ms.)
        void *args[] = {&a};
        G5_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)sssp_persistent_kernel, dim3(blocks),
                                                dim3(SSSP_THREADS), args, 0, st));
    }
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_sssp_traverse(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                const uint32_t *d_light_deg, float light_delta, uint64_t nverts, uint64_t root,
                                float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                                const g5_sssp_params *params, void *stream) {
    clear_error();
    return sssp_launch(d_rowstarts, d_col, d_w, d_light_deg, light_delta, nverts, root, nullptr, 0, d_dist, d_pred,
                       d_work, work_bytes, params, stream, "g5_sssp_traverse");
}

extern "C" int g5_sssp_traverse_multi(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                      const uint32_t *d_light_deg, float light_delta, uint64_t nverts,
                                      const uint64_t *d_roots, uint32_t nroots, float *d_dist, int64_t *d_pred,
                                      void *d_work, uint64_t work_bytes, const g5_sssp_params *params,
                                      void *stream) {
    clear_error();
    G5_CHECK_ARG(d_roots && nroots >= 1, "g5_sssp_traverse_multi: no sources");
    return sssp_launch(d_rowstarts, d_col, d_w, d_light_deg, light_delta, nverts, 0, d_roots, nroots, d_dist, d_pred,
                       d_work, work_bytes, params, stream, "g5_sssp_traverse_multi");
}

extern "C" int g5_sssp_run(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                           const uint32_t *d_light_deg, float light_delta, uint64_t nverts, uint64_t root,
                           float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                           const g5_sssp_params *params, void *stream) {
    clear_error();
    SsspWork w;
    int rc = sssp_check(d_rowstarts, d_col, d_w, nverts, root, d_dist, d_pred, d_work, work_bytes, &w, "g5_sssp_run");
    if (rc) return rc;
    if ((rc = g5_sssp_reset(nverts, d_dist, d_pred, d_work, work_bytes, stream))) return rc;
    return g5_sssp_traverse(d_rowstarts, d_col, d_w, d_light_deg, light_delta, nverts, root, d_dist, d_pred, d_work,
                            work_bytes, params, stream);
}

extern "C" int g5_sssp_last_trace(const void *d_work, uint64_t work_bytes, uint64_t counts[7], int max_phases,
                                   int32_t *kind, uint64_t *size, double *phase_ms, uint64_t *phase_edges,
                                   int32_t *nphases, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && work_bytes >= sizeof(SsspCtl) && nphases, "g5_sssp_last_trace: bad argument");
    SsspCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (counts) {
        counts[0] = c.n_edges;
        counts[1] = c.n_settled;
        counts[2] = c.n_atomic;
        counts[3] = c.n_improved;
        counts[4] = c.n_ring;
        counts[5] = c.n_front;
        counts[6] = c.pulls;
    }
    const int n = (int)std::min<unsigned long long>(std::min<unsigned long long>(c.phases, SSSP_TRACE),
                                                     (unsigned long long)std::max(max_phases, 0));
    unsigned long long prev = c.t0, prev_e = 0;
    for (int i = 0; i < n; ++i) {
        if (kind) kind[i] = c.kind_phase[i];
        if (size) size[i] = c.n_phase[i];
        if (phase_ms) phase_ms[i] = (double)(c.t_phase[i] - prev) * 1e-6;
        if (phase_edges) phase_edges[i] = c.e_phase[i] - prev_e;
        prev = c.t_phase[i];
        prev_e = c.e_phase[i];
    }
    *nphases = (int32_t)c.phases;
    return deverr_to_status(c.error, "g5_sssp_run");
}

extern "C" int g5_sssp_last_status(const void *d_work, uint64_t work_bytes, uint64_t *buckets, uint64_t *phases,
                                   void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && work_bytes >= sizeof(SsspCtl), "g5_sssp_last_status: bad workspace");
    SsspCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (buckets) *buckets = c.buckets;
    if (phases) *phases = c.phases;
    int rc = deverr_to_status(c.error, "g5_sssp_run");
    if (rc && c.dbg_claim) {
        auto f = [](unsigned long long b) {
            float x;
            unsigned u = (unsigned)b;
            memcpy(&x, &u, 4);
            return (double)x;
        };
        char extra[320];
        snprintf(extra, sizeof extra,
                 "%s; first bad relaxation: v %llu, candidate %.9g from u %llu (u now at %.9g), bucket %llu "
                 "[%.9g, %.9g), phase %llu",
                 g5_last_error(), c.dbg[0], f(c.dbg[1] >> 32), c.dbg[1] & 0xffffffffull, f(c.dbg[2] >> 32), c.dbg[5],
                 f(c.dbg[3]), f(c.dbg[4]), c.dbg[6]);
        set_error(rc, "%s", extra);
    }
    return rc;
}

extern "C" int g5_sssp_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks) {
    clear_error();
    G5_CHECK_ARG(blocks && max_blocks, "g5_sssp_grid: NULL argument");
    int mb = 0;
    int rc = sssp_max_blocks(&mb);
    if (rc) return rc;
    *max_blocks = mb;
    *blocks = (int)std::min<uint64_t>(mb, std::max<uint64_t>(1, nverts / 2048));
    return G5_OK;
}
