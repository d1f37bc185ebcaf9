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
// distances equal the reference's bit for bit.
//
// Device-side structure:
//   * dist and parent packed in one u64 (float bits << 32 | parent); a
//     relaxation is one 64-bit atomicMin, which keeps the smallest distance
//     and, among equal distances, the smallest parent -- no locks (the
//     reference spins on a per-vertex lock, :224).
//   * a ring of K bucket queues for the next K-1 buckets; a vertex enters a
//     queue once per bucket (stamp per vertex), stale entries are dropped
//     when the bucket opens.  No O(N) bucket scans (the reference scans all
//     vertices per bucket, :297-331).
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

#include "g5_common.cuh"
#include "g5_frontier.cuh"

namespace g5 {

constexpr int SSSP_THREADS = 256;
constexpr int RING = 16;  // bucket queues; a relaxation may land at most RING-1 buckets ahead
constexpr unsigned STAGE_F = 256;    // per-warp staging: frontier
constexpr unsigned STAGE_S = 256;    //                   heavy set
constexpr unsigned STAGE_R = 32;     //                   each ring queue
constexpr int SSSP_TRACE = 256;      // phases recorded in the control block
constexpr unsigned long long UNREACHED = ~0ull;

struct SsspCtl {
    unsigned bar;
    unsigned error;
    unsigned grab[3];    // per phase slot: cursor over the input list's small part
    unsigned cgrab[3];   //                 cursor over the input list's big-part chunks
    unsigned f_small[3]; // per phase slot: frontier produced for the next phase
    unsigned long long f_big[3];
    unsigned s_small[2]; // per bucket parity: heavy set
    unsigned long long s_big[2];
    unsigned ring_len[RING];
    unsigned long long buckets;
    unsigned long long phases;
    // counters: edges looked at, skipped as settled, atomicMin issued,
    // distances lowered, ring and frontier pushes
    unsigned long long n_edges, n_settled, n_atomic, n_improved, n_ring, n_front;
    // per-phase trace: end time, kind (0 open, 1 light, 2 heavy), input size
    unsigned long long t0;
    unsigned long long t_phase[SSSP_TRACE];
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
    uint64_t n;
    unsigned root;
    const uint64_t *roots;  // several sources at once (device array) instead of `root`, or nullptr
    unsigned nroots;
    float delta;
    unsigned long long *pack;
    unsigned *fstamp, *sstamp, *qstamp;
    unsigned *settled;
    unsigned *F[2], *FB[2];  // frontiers and the chunk bases of their big parts
    unsigned *S[2], *SB[2];  // heavy sets and chunk bases
    unsigned *ring;
    SsspCtl *ctl;
    const SsspOut *prefilled;
    float *dist;
    int64_t *pred;
    unsigned nblocks;
    unsigned long long limit_ns;
};

__device__ __forceinline__ float pack_dist(unsigned long long p) { return __uint_as_float((unsigned)(p >> 32)); }

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
    WarpStage f, s;
    unsigned *rbuf;  // RING * STAGE_R, this warp's
    unsigned *rcnt;  // RING, this warp's
};

// Per-thread event counts, summed into the control block once per phase.
struct Counts {
    unsigned long long edges, settled, atomics, improved, ring, front;
};

struct PushCtx {
    Stage st;
    unsigned pid;        // id of the producing phase (frontier stamp)
    unsigned bucket;     // current bucket index (heavy-set stamp)
    int f_slot;          // counter slot of the produced frontier
    unsigned *Fout, *FBout;
    unsigned *Sl, *SBl;  // heavy set of the current bucket
    int s_par;
    const float *bnd;    // shared: b_B .. b_{B+RING}
};

// Appends v to the produced frontier and to the bucket's heavy set (each at
// most once).  All 32 lanes call it.
__device__ __forceinline__ void push_same_bucket(const SsspArgs &a, const PushCtx &x, bool want, unsigned v) {
    SsspCtl *c = a.ctl;
    bool f = want && atomicExch(&a.fstamp[v], x.pid) != x.pid;
    bool s = want && atomicExch(&a.sstamp[v], x.bucket) != x.bucket;
    uint64_t lb = 0, le = 0, hb = 0, he = 0;
    if (f) part_range(a, v, false, lb, le);
    if (s) part_range(a, v, true, hb, he);
    // Each vertex enters a frontier once per phase and a heavy set once per
    // bucket, so no list exceeds n entries.
    bool ok = frontier_append_staged(x.st.f, x.Fout, x.FBout, a.n, &c->f_small[x.f_slot], &c->f_big[x.f_slot], f, v,
                                     le - lb);
    ok &= frontier_append_staged(x.st.s, x.Sl, x.SBl, a.n, &c->s_small[x.s_par], &c->s_big[x.s_par], s, v, he - hb);
    if (!ok) atomicOr(&c->error, DEVERR_CAPACITY);
}

// Edges of one warp step, E per lane: their target vertices' settled bits
// and packed distances are loaded together before any is used, so the
// step costs one chain of memory round trips, not E.
constexpr int SSSP_EDGES = 2;

struct EdgeProbe {
    unsigned v[SSSP_EDGES];
    float wt[SSSP_EDGES];
    unsigned u[SSSP_EDGES];
    float du[SSSP_EDGES];
    bool has[SSSP_EDGES];
    unsigned long long cur[SSSP_EDGES];  // v's packed distance/parent, ~0 if not needed
};

// Fills p.cur for the edges in p (settled targets and non-vertices get
// UNREACHED-free zero so relax() skips them).
__device__ __forceinline__ void probe_edges(const SsspArgs &a, Counts &k, EdgeProbe &p) {
    unsigned sw[SSSP_EDGES];
#pragma unroll
    for (int t = 0; t < SSSP_EDGES; ++t) {
        k.edges += p.has[t];
        if (p.has[t] && p.v[t] >= a.n) {  // not a vertex: report it, touch nothing
            atomicOr(&a.ctl->error, DEVERR_RANGE);
            p.has[t] = false;
        }
        sw[t] = p.has[t] ? __ldcg(&a.settled[p.v[t] >> 5]) : 0u;
    }
#pragma unroll
    for (int t = 0; t < SSSP_EDGES; ++t) {
        const bool settled = (sw[t] >> (p.v[t] & 31)) & 1u;
        k.settled += p.has[t] && settled;
        p.has[t] = p.has[t] && !settled;
        p.cur[t] = p.has[t] ? __ldcg(&a.pack[p.v[t]]) : 0ull;
    }
}

// Relaxes u -> v with float weight wt from distance du (cur = v's packed
// value read by probe_edges); queues v when its distance dropped.  All 32
// lanes call it (want = lane has an edge to a vertex not settled).
__device__ __forceinline__ void relax(const SsspArgs &a, const PushCtx &x, Counts &k, bool want, unsigned u, float du,
                                      unsigned v, float wt, unsigned long long cur, bool heavy_phase) {
    bool same = false;
    int target = -1;
    if (want) {
        const float cand = __fadd_rn(du, wt);
        const unsigned long long np = ((unsigned long long)__float_as_uint(cand) << 32) | u;
        if (np < cur) {
            ++k.atomics;
            const unsigned long long old = atomicMin(&a.pack[v], np);
            if (np < old && (old >> 32) != (np >> 32)) {
                ++k.improved;
                if (cand < x.bnd[1]) {
                    same = true;
                    if (heavy_phase) atomicOr(&a.ctl->error, DEVERR_CAPACITY);  // cannot happen: w >= delta
                } else {
                    // Largest j with b_{B+j} <= cand; the ring holds B+1 .. B+RING-1.
                    int j = 1;
                    while (j < RING && x.bnd[j + 1] <= cand) ++j;
                    if (j >= RING) atomicOr(&a.ctl->error, DEVERR_RING);
                    else target = (int)x.bucket + j;
                }
            }
        }
    }
    if (!__any_sync(FULL, same || target >= 0)) return;  // nothing lowered in this warp step
    push_same_bucket(a, x, same && !heavy_phase, v);
    // Ring queue of the target bucket, once per (vertex, bucket), staged in
    // the block's shared memory.
    const bool r = target >= 0 && atomicExch(&a.qstamp[v], (unsigned)target) != (unsigned)target;
    k.ring += r;
    k.front += same && !heavy_phase;
    // Per-slot warp staging: lanes with the same target slot append
    // together; a full slot is flushed to its global queue first.
    const int slot = r ? target % RING : RING;
    unsigned todo = __ballot_sync(FULL, r);
    while (todo) {
        const int sl = __shfl_sync(FULL, slot, __ffs(todo) - 1);
        const bool mine = r && slot == sl;
        const unsigned m = __ballot_sync(FULL, mine);
        WarpStage q{x.st.rbuf + sl * STAGE_R, x.st.rcnt + sl, STAGE_R};
        if (!stage_append(q, mine, v, a.ring + (uint64_t)sl * a.n, a.n, &a.ctl->ring_len[sl]))
            atomicOr(&a.ctl->error, DEVERR_CAPACITY);
        todo &= ~m;
    }
}

// Writes every staged entry of this warp to its global list and the warp's
// counts to the control block.  Every warp calls it at the end of a phase.
__device__ void stage_flush(const SsspArgs &a, const PushCtx &x, Counts &k) {
    SsspCtl *c = a.ctl;
    {
        unsigned long long v[6] = {k.edges, k.settled, k.atomics, k.improved, k.ring, k.front};
        unsigned long long *dst[6] = {&c->n_edges, &c->n_settled, &c->n_atomic, &c->n_improved, &c->n_ring,
                                      &c->n_front};
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            const unsigned long long t = warp_sum(v[i]);
            if (lane_id() == 0 && t) atomicAdd(dst[i], t);
        }
        k = Counts{0, 0, 0, 0, 0, 0};
    }
    bool ok = stage_flush_warp(x.st.f, x.Fout, a.n, &c->f_small[x.f_slot]);
    ok &= stage_flush_warp(x.st.s, x.Sl, a.n, &c->s_small[x.s_par]);
    for (int sl = 0; sl < RING; ++sl) {
        WarpStage q{x.st.rbuf + sl * STAGE_R, x.st.rcnt + sl, STAGE_R};
        ok &= stage_flush_warp(q, a.ring + (uint64_t)sl * a.n, a.n, &c->ring_len[sl]);
    }
    if (!ok && lane_id() == 0) atomicOr(&c->error, DEVERR_CAPACITY);
}

// Relaxes the light (heavy = false) or heavy edges of every vertex of list L
// (small part [0, ns), big part at the back, `bp` its packed counter).  The
// heavy pass also marks each list vertex settled.
__device__ void expand_list(const SsspArgs &a, const PushCtx &x, Counts &k, const unsigned *L, unsigned ns,
                            unsigned long long bp, const unsigned *B, unsigned *grab, unsigned *cgrab, bool heavy,
                            bool sparse_out) {
    const unsigned lane = lane_id();
    const bool filtered = a.ld == nullptr;
    const unsigned g = grab_size(ns, ((unsigned long long)gridDim.x * blockDim.x) >> 5);
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(grab, g);
        base = __shfl_sync(FULL, base, 0);
        if (base >= ns) break;
        const unsigned i = base + lane;
        const bool valid = lane < g && i < ns;
        const unsigned u = valid ? __ldcg(&L[i]) : 0u;
        uint64_t rb = 0, re = 0;
        float du = 0.0f;
        if (valid) {
            part_range(a, u, heavy, rb, re);
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
                    if (filtered) has = heavy ? !(p.wt[t] < a.delta) : p.wt[t] < a.delta;
                }
                p.has[t] = has;
            }
            probe_edges(a, k, p);
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) relax(a, x, k, p.has[t], p.u[t], p.du[t], p.v[t], p.wt[t], p.cur[t], heavy);
        }
    }
    const unsigned nb = big_count(bp);
    const unsigned long long nch = big_chunks(bp);
    for (;;) {
        unsigned ch = 0;
        if (lane == 0) ch = atomicAdd(cgrab, 1u);
        ch = __shfl_sync(FULL, ch, 0);
        if (ch >= nch) break;
        const unsigned j = chunk_owner(B, nb, ch);
        const unsigned u = __ldcg(&L[a.n - 1 - j]);
        const unsigned first = __ldcg(&B[j]);
        uint64_t rb, re;
        part_range(a, u, heavy, rb, re);
        const unsigned long long pu = __ldcg(&a.pack[u]);
        const float du = pack_dist(pu);
        if (heavy && ch == first && lane == 0) settle(a, sparse_out, u, pu);
        const uint64_t deg = re - rb;
        const uint64_t cs = (uint64_t)(ch - first) * BIG_CHUNK;
        const uint64_t ce = min(cs + BIG_CHUNK, deg);
        for (uint64_t e0 = cs + lane; e0 < cs + BIG_CHUNK; e0 += 32 * SSSP_EDGES) {
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
                    if (filtered) has = heavy ? !(p.wt[t] < a.delta) : p.wt[t] < a.delta;
                }
                p.has[t] = has;
            }
            probe_edges(a, k, p);
#pragma unroll
            for (int t = 0; t < SSSP_EDGES; ++t) relax(a, x, k, p.has[t], p.u[t], p.du[t], p.v[t], p.wt[t], p.cur[t], heavy);
        }
    }
}

__device__ __forceinline__ void trace_phase(SsspCtl *c, unsigned phase, int kind, unsigned size) {
    if (phase < SSSP_TRACE) {
        c->t_phase[phase] = globaltimer_ns();
        c->kind_phase[phase] = (unsigned char)kind;
        c->n_phase[phase] = size;
    }
}

__global__ void __launch_bounds__(SSSP_THREADS, 4) sssp_persistent_kernel(SsspArgs a) {
    SsspCtl *c = a.ctl;
    __shared__ float s_bnd[RING + 1];
    constexpr int WARPS = SSSP_THREADS / 32;
    __shared__ unsigned s_fbuf[WARPS][STAGE_F], s_sbuf[WARPS][STAGE_S], s_rbuf[WARPS][RING * STAGE_R];
    __shared__ unsigned s_fcnt[WARPS], s_scnt[WARPS], s_rcnt[WARPS][RING];
    const unsigned wid = threadIdx.x >> 5;
    if (lane_id() == 0) s_fcnt[wid] = s_scnt[wid] = 0;
    if (lane_id() < RING) s_rcnt[wid][lane_id()] = 0;
    __syncwarp();
    const Stage stage{WarpStage{s_fbuf[wid], &s_fcnt[wid], STAGE_F}, WarpStage{s_sbuf[wid], &s_scnt[wid], STAGE_S},
                      s_rbuf[wid], s_rcnt[wid]};
    unsigned epoch = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const bool sparse_out = __ldcg((const unsigned long long *)&a.prefilled->dist) == (unsigned long long)a.dist &&
                            __ldcg((const unsigned long long *)&a.prefilled->pred) == (unsigned long long)a.pred;

    if (!a.roots) {
        if (gtid == 0) {
            a.pack[a.root] = (unsigned long long)a.root;  // distance 0.0f, parent = root
            a.ring[0] = a.root;
            a.qstamp[a.root] = 0;
            c->ring_len[0] = 1;
        }
    } else {
        // Several sources (disjoint graphs packed into one CSR, one source
        // each) all start in bucket 0; a repeated source is queued once.
        for (uint64_t i = gtid; i < a.nroots; i += nthreads) {
            const uint64_t r = __ldg(&a.roots[i]);
            if (r >= a.n) {
                atomicOr(&c->error, DEVERR_RANGE);
            } else if (atomicCAS(&a.qstamp[r], 0xffffffffu, 0u) == 0xffffffffu) {
                a.pack[r] = r;
                a.ring[atomicAdd(&c->ring_len[0], 1u)] = (unsigned)r;
            }
        }
    }
    if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;

    unsigned bucket = 0, phase = 0;
    float blo = 0.0f;
    Counts cnt{0, 0, 0, 0, 0, 0};
    if (gtid == 0) c->t0 = globaltimer_ns();
    unsigned long long nbuckets = 0;
    for (;;) {
        // ---- open the bucket: its ring queue becomes the first frontier.
        if (threadIdx.x == 0) {
            float b = blo;
            for (int j = 0; j <= RING; ++j) {
                s_bnd[j] = b;
                b = __fadd_rn(b, a.delta);
            }
        }
        __syncthreads();
        PushCtx x;
        x.st = stage;
        x.bucket = bucket;
        x.bnd = s_bnd;
        x.s_par = bucket & 1;
        x.Sl = a.S[bucket & 1];
        x.SBl = a.SB[bucket & 1];
        {
            const int s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->f_small[s_clr] = 0;
                c->f_big[s_clr] = 0;
                c->s_small[(bucket + 1) & 1] = 0;
                c->s_big[(bucket + 1) & 1] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            const unsigned slot = bucket % RING;
            const unsigned len = ld_volatile(&c->ring_len[slot]);
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
                push_same_bucket(a, x, ok, v);
            }
            stage_flush(a, x, cnt);
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
            // The queue is consumed; nothing can target this slot again before
            // bucket + RING, which lies beyond every push of this bucket.
            if (gtid == 0) {
                c->ring_len[slot] = 0;
                trace_phase(c, phase, 0, len);
            }
            ++phase;
        }
        // ---- light iterations until the bucket's frontier is empty.
        for (;;) {
            const int s_cur = phase % 3, s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            const unsigned ns = ld_volatile(&c->f_small[s_cur]);
            const unsigned long long bp = ld_volatile(&c->f_big[s_cur]);
            if (ns + big_count(bp) == 0) break;
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->f_small[s_clr] = 0;
                c->f_big[s_clr] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            expand_list(a, x, cnt, a.F[phase & 1], ns, bp, a.FB[phase & 1], &c->grab[s_cur], &c->cgrab[s_cur], false,
                        sparse_out);
            stage_flush(a, x, cnt);
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
            if (gtid == 0) trace_phase(c, phase, 1, ns + big_count(bp));
            ++phase;
        }
        // ---- heavy edges of every vertex settled in this bucket.
        {
            const int s_cur = phase % 3, s_nxt = (phase + 1) % 3, s_clr = (phase + 2) % 3;
            if (gtid == 0) {
                c->grab[s_clr] = c->cgrab[s_clr] = c->f_small[s_clr] = 0;
                c->f_big[s_clr] = 0;
            }
            x.pid = phase;
            x.f_slot = s_nxt;
            x.Fout = a.F[(phase + 1) & 1];
            x.FBout = a.FB[(phase + 1) & 1];
            const unsigned ns = ld_volatile(&c->s_small[bucket & 1]);
            const unsigned long long bp = ld_volatile(&c->s_big[bucket & 1]);
            expand_list(a, x, cnt, a.S[bucket & 1], ns, bp, a.SB[bucket & 1], &c->grab[s_cur], &c->cgrab[s_cur], true,
                        sparse_out);
            stage_flush(a, x, cnt);
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
            if (gtid == 0) trace_phase(c, phase, 2, ns + big_count(bp));
            ++phase;
        }
        ++nbuckets;
        // ---- next non-empty bucket within the ring window.
        int step = 0;
        for (int j = 1; j < RING; ++j)
            if (ld_volatile(&c->ring_len[(bucket + j) % RING])) {
                step = j;
                break;
            }
        if (!step) break;
        for (int j = 0; j < step; ++j) blo = __fadd_rn(blo, a.delta);
        bucket += step;
        __syncthreads();  // s_bnd is rewritten at the top of the loop
    }
    if (gtid == 0) {
        c->buckets = nbuckets;
        c->phases = phase;
    }
    // Every distance is final (the last heavy phase ended at a grid barrier).
    // Outputs not pre-filled by the reset are written here in full.
    if (!sparse_out) {
        for (uint64_t v = gtid; v < a.n; v += nthreads) {
            const unsigned long long p = __ldcg(&a.pack[v]);
            a.dist[v] = p == UNREACHED ? -1.0f : pack_dist(p);
            a.pred[v] = p == UNREACHED ? -1 : (int64_t)(unsigned)p;
        }
    }
}

// Fills the outputs with "unreached" and records them as pre-filled.
__global__ void sssp_prefill_kernel(float *__restrict__ dist, int64_t *__restrict__ pred, uint64_t n, SsspOut *hdr) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (uint64_t v = t; v < n; v += stride) {
        dist[v] = -1.0f;
        pred[v] = -1;
    }
    if (t == 0) *hdr = SsspOut{dist, pred};
}

struct SsspWork {
    SsspCtl *ctl;
    SsspOut *out;
    unsigned long long *pack;
    unsigned *fstamp, *sstamp, *qstamp, *settled;
    unsigned *F[2], *FB[2], *S[2], *SB[2];
    unsigned *ring;
    uint64_t bytes;
};

static SsspWork carve_sssp(void *base, uint64_t n) {
    Carver c(base);
    SsspWork w;
    w.ctl = c.take<SsspCtl>(1);
    w.out = c.take<SsspOut>(1);
    w.pack = c.take<unsigned long long>(n);
    w.fstamp = c.take<unsigned>(n);
    w.sstamp = c.take<unsigned>(n);
    w.qstamp = c.take<unsigned>(n);
    w.settled = c.take<unsigned>((n + 31) / 32);
    for (int i = 0; i < 2; ++i) {
        w.F[i] = c.take<unsigned>(n);
        w.FB[i] = c.take<unsigned>(n);
        w.S[i] = c.take<unsigned>(n);
        w.SB[i] = c.take<unsigned>(n);
    }
    w.ring = c.take<unsigned>((uint64_t)RING * n);
    w.bytes = c.used;
    return w;
}

static int sssp_max_blocks(int *out) {
    static int cached[64] = {};
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if (!cached[di.device]) {
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

extern "C" int g5_sssp_reset(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                             void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31) && d_work, "g5_sssp_reset: bad argument");
    G5_CHECK_ARG((d_dist == nullptr) == (d_pred == nullptr), "g5_sssp_reset: give both outputs or neither");
    SsspWork w = carve_sssp(d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_sssp_reset: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    if (d_dist) {
        DeviceInfo di;
        int rc = device_info(&di);
        if (rc) return rc;
        sssp_prefill_kernel<<<di.sms * 8, 256, 0, st>>>(d_dist, d_pred, nverts, w.out);
        G5_CUDA_TRY(cudaGetLastError());
    } else {
        G5_CUDA_TRY(cudaMemsetAsync(w.out, 0, sizeof(SsspOut), st));
    }
    G5_CUDA_TRY(cudaMemsetAsync(w.pack, 0xff, nverts * sizeof(unsigned long long), st));
    // fstamp, sstamp, qstamp are consecutive carve-outs: one memset.
    G5_CUDA_TRY(cudaMemsetAsync(w.fstamp, 0xff, (char *)(w.qstamp + nverts) - (char *)w.fstamp, st));
    G5_CUDA_TRY(cudaMemsetAsync(w.settled, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    return G5_OK;
}

static int sssp_launch(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                       const uint32_t *d_light_deg, float light_delta, uint64_t nverts, uint64_t root,
                       const uint64_t *d_roots, unsigned nroots, float *d_dist, int64_t *d_pred, void *d_work,
                       uint64_t work_bytes, const g5_sssp_params *params, void *stream, const char *who) {
    SsspWork w;
    int rc = sssp_check(d_rowstarts, d_col, d_w, nverts, root, d_dist, d_pred, d_work, work_bytes, &w, who);
    if (rc) return rc;
    g5_sssp_params p = {0.1f, 0};
    if (params) p = *params;
    G5_CHECK_ARG(p.delta > 0.0f, "g5_sssp_traverse: delta must be positive");
    int max_blocks = 0;
    if ((rc = sssp_max_blocks(&max_blocks))) return rc;
    int blocks = p.blocks > 0 ? std::min(p.blocks, max_blocks)
                              : (int)std::min<uint64_t>(max_blocks, std::max<uint64_t>(1, nverts / 2048));
    cudaStream_t st = (cudaStream_t)stream;
    SsspArgs a;
    a.rowptr = d_rowstarts;
    a.col = d_col;
    a.w = d_w;
    a.ld = (d_light_deg && p.delta == light_delta) ? d_light_deg : nullptr;
    a.n = nverts;
    a.root = (unsigned)root;
    a.roots = d_roots;
    a.nroots = nroots;
    a.delta = p.delta;
    a.pack = w.pack;
    a.fstamp = w.fstamp;
    a.sstamp = w.sstamp;
    a.qstamp = w.qstamp;
    a.settled = w.settled;
    for (int i = 0; i < 2; ++i) {
        a.F[i] = w.F[i];
        a.FB[i] = w.FB[i];
        a.S[i] = w.S[i];
        a.SB[i] = w.SB[i];
    }
    a.ring = w.ring;
    a.ctl = w.ctl;
    a.prefilled = w.out;
    a.dist = d_dist;
    a.pred = d_pred;
    a.nblocks = (unsigned)blocks;
    a.limit_ns = wait_limit_ns();
    void *args[] = {&a};
    G5_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(SsspCtl), st));
    G5_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)sssp_persistent_kernel, dim3(blocks), dim3(SSSP_THREADS),
                                            args, 0, st));
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

extern "C" int g5_sssp_last_trace(const void *d_work, uint64_t work_bytes, uint64_t counts[6], int max_phases,
                                   int32_t *kind, uint64_t *size, double *phase_ms, int32_t *nphases, void *stream) {
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
    }
    const int n = (int)std::min<unsigned long long>(std::min<unsigned long long>(c.phases, SSSP_TRACE),
                                                     (unsigned long long)std::max(max_phases, 0));
    unsigned long long prev = c.t0;
    for (int i = 0; i < n; ++i) {
        if (kind) kind[i] = c.kind_phase[i];
        if (size) size[i] = c.n_phase[i];
        if (phase_ms) phase_ms[i] = (double)(c.t_phase[i] - prev) * 1e-6;
        prev = c.t_phase[i];
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
    return deverr_to_status(c.error, "g5_sssp_run");
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
