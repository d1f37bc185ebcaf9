// mssp.cu -- K8: SSSP from up to 32 sources of one graph in one persistent
// cooperative launch (the reference runs one source at a time,
// src/traversal.cu:638-711, and each of its searches is a host-driven loop).
//
// One warp lane per source.  Every vertex holds 32 packed 64-bit words
// (fl(dist) bits << 32 | parent), vertex-major, so a warp relaxing one edge
// for all its sources reads and lowers one 256-byte row with atomicMin: the
// edge's column entry and weight are loaded once for 32 searches.  Work goes
// in distance order, as in delta-stepping, on one bucket index for all
// sources: a vertex whose word for some source dropped has that source's bit
// set in its change mask and its smallest pending bucket (floor(dist /
// delta)) in vbkt; the first bit set since the vertex was last taken queues
// it.  A round of bucket b takes each queued vertex whose vbkt <= b (its mask
// by atomic exchange: later drops queue it again) and relaxes its row for the
// sources whose distance lies in buckets <= b; the other sources go back to
// the mask and vbkt, and vertices whose vbkt > b stay queued untouched.
// Rows longer than MSS_CHUNK entries are cut into chunks spread over the
// grid.  When a round queues nothing in bucket b, b jumps to the smallest
// pending bucket; the search ends when nothing is queued.  Packed minima
// make each source's result the unique limit of every label-correcting
// order, so distances and parents are bit-identical to the single-source
// delta-stepping kernel's (same float sums along the same paths, ties to the
// smaller parent).
//
// HBM bytes per relaxed entry: 8 (column and weight, shared by the sources
// in the bucket) + 8 per active source (its word of the target, read, then
// lowered when improved); per round 12 per queued vertex.
#include "g5_common.cuh"

namespace g5 {

constexpr int MSS_THREADS = 256;
constexpr int MSS_SOURCES = 32;    // one warp lane per source
constexpr unsigned MSS_CHUNK = 256;  // longer rows are cut into chunks of this many entries
constexpr unsigned long long MSS_NONE = ~0ull;
constexpr int MSS_MAX_ROUNDS = 1 << 20;

struct MssCtl {
    unsigned bar;                    // grid barrier arrivals
    unsigned err;                    // DEVERR_* flags
    unsigned qlen[3];                // per round slot: vertices queued for the next round
    unsigned long long big[3];       // per round slot: long-row items << 40 | their chunks
    unsigned minb[3];                // per round slot: smallest pending bucket seen (a lower bound)
    unsigned long long sources[MSS_SOURCES];  // in the CSR's numbering
    g5_sssp_multi_stats res;
};

struct MssWork {
    MssCtl *ctl;
    unsigned long long *pack;  // n * 32: (fl(dist) << 32 | parent) per vertex and source
    unsigned *cmask;           // n: sources whose word dropped since the vertex was last taken
    unsigned *vbkt;            // n: smallest bucket among those sources' distances (a lower bound)
    unsigned *smask;           // n: the mask taken for each entry of the current round
    unsigned *q[2];            // n each: this round's and the next round's vertices
    unsigned *items;           // n: entries of this round whose rows are cut into chunks
    unsigned long long *ibase; // n: their first chunk
    uint64_t bytes;
};

static MssWork carve_mss(void *base, uint64_t n) {
    Carver c(base);
    MssWork w;
    w.ctl = c.take<MssCtl>(1);
    w.pack = c.take<unsigned long long>(n * MSS_SOURCES);
    w.cmask = c.take<unsigned>(n);
    w.vbkt = c.take<unsigned>(n);
    w.smask = c.take<unsigned>(n);
    w.q[0] = c.take<unsigned>(n);
    w.q[1] = c.take<unsigned>(n);
    w.items = c.take<unsigned>(n);
    w.ibase = c.take<unsigned long long>(n);
    w.bytes = c.used;
    return w;
}

struct MssArgs {
    const uint64_t *rowptr;
    const int *col;
    const float *w;
    uint64_t n;
    MssWork ws;
    float inv_delta;
    unsigned nblocks;
    unsigned long long limit_ns;
};

constexpr unsigned MSS_NOBKT = 0xffffffffu;

__device__ __forceinline__ unsigned mss_bucket(float d, float inv_delta) {
    const float b = d * inv_delta;
    return b < 4.0e9f ? (unsigned)b : MSS_NOBKT - 1;
}

__global__ void mss_reset_kernel(MssWork w, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x, t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    grid_fill(w.pack, n * MSS_SOURCES, MSS_NONE, t, stride);
    grid_fill(w.cmask, n, 0u, t, stride);
    grid_fill(w.vbkt, n, MSS_NOBKT, t, stride);
}

// Source s's word at its own vertex, its mask bit, and the vertex queued
// for round 0 (once, however many sources share it).
__global__ void mss_seed_kernel(MssWork w, uint64_t n, unsigned nsrc, const unsigned *perm) {
    const unsigned s = threadIdx.x;
    if (s >= nsrc) return;
    const unsigned long long r = w.ctl->sources[s];
    if (r >= n) {
        atomicOr(&w.ctl->err, DEVERR_RANGE);
        return;
    }
    const unsigned v = perm ? perm[r] : (unsigned)r;
    w.ctl->sources[s] = v;
    w.pack[(uint64_t)v * MSS_SOURCES + s] = (unsigned long long)v;  // distance 0.0f, parent itself
    w.vbkt[v] = 0;
    if (atomicOr(&w.cmask[v], 1u << s) == 0) w.q[0][atomicAdd(&w.ctl->qlen[0], 1u)] = v;
}

// Queues v (append to the next list) on the first bit of its mask, and
// lowers its smallest pending bucket; `bk` = that bucket, MSS_NOBKT for no
// change.  Warp-wide: every lane calls it.
__device__ __forceinline__ void mss_note(const MssArgs &a, unsigned v, unsigned bits, unsigned bk, unsigned *nxt,
                                         unsigned *qlen, unsigned &wmin) {
    bool need = false;
    if (bits) {
        atomicMin(&a.ws.vbkt[v], bk);
        need = atomicOr(&a.ws.cmask[v], bits) == 0;
        wmin = min(wmin, bk);
    }
    const unsigned pos = warp_append(qlen, need);
    if (need) {
        if (pos < a.n) nxt[pos] = v;
        else atomicOr(&a.ws.ctl->err, DEVERR_CAPACITY);
    }
}

// Relaxes entries [b, e) of u's row for the sources in mask m (lane s =
// source s) whose distance lies in buckets <= bk; with `owner` (the row's
// first chunk) the other sources of m go back to u's mask and vbkt.  32
// entries are loaded at a time, one lane each, then each entry's target and
// weight broadcast; lane j records which sources improved entry j's target
// and their smallest new bucket.
__device__ __forceinline__ void mss_relax(const MssArgs &a, unsigned u, unsigned m, uint64_t b, uint64_t e,
                                          unsigned bk, bool owner, unsigned *nxt, unsigned *qlen, unsigned &wmin,
                                          unsigned long long &scanned) {
    const unsigned lane = lane_id();
    const bool inm = (m >> lane) & 1u;
    const unsigned long long pu = inm ? __ldcg(&a.ws.pack[(uint64_t)u * MSS_SOURCES + lane]) : MSS_NONE;
    const float du = __uint_as_float((unsigned)(pu >> 32));
    const unsigned ub = pu != MSS_NONE ? mss_bucket(du, a.inv_delta) : MSS_NOBKT;
    const bool live = pu != MSS_NONE && ub <= bk;
    if (owner) {
        const unsigned later = __ballot_sync(FULL, inm && !live);
        unsigned lb = inm && !live ? ub : MSS_NOBKT;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) lb = min(lb, __shfl_xor_sync(FULL, lb, d));
        mss_note(a, u, lane == 0 ? later : 0u, lb, nxt, qlen, wmin);
    }
    if (!__any_sync(FULL, live)) return;
    if (lane == 0) scanned += e - b;
    for (uint64_t e0 = b; e0 < e; e0 += 32) {
        const uint64_t ej = e0 + lane;
        const bool has = ej < e;
        const unsigned vj = has ? (unsigned)__ldg(&a.col[ej]) : 0u;
        const float wj = has ? __ldg(&a.w[ej]) : 0.0f;
        const unsigned cnt = e - e0 < 32 ? (unsigned)(e - e0) : 32u;
        unsigned mybits = 0, mybk = MSS_NOBKT;
        for (unsigned j = 0; j < cnt; ++j) {
            const unsigned v = __shfl_sync(FULL, vj, j);
            const float wt = __shfl_sync(FULL, wj, j);
            bool imp = false;
            unsigned nb = MSS_NOBKT;
            if (live && v < a.n) {
                const float nd = du + wt;
                const unsigned long long cand = ((unsigned long long)__float_as_uint(nd) << 32) | u;
                unsigned long long *pv = &a.ws.pack[(uint64_t)v * MSS_SOURCES + lane];
                if (cand < __ldcg(pv)) imp = cand < atomicMin(pv, cand);
                if (imp) nb = mss_bucket(nd, a.inv_delta);
            }
            const unsigned bits = __ballot_sync(FULL, imp);
            if (bits) {
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) nb = min(nb, __shfl_xor_sync(FULL, nb, d));
            }
            if (lane == j) {
                mybits = bits;
                mybk = nb;
            }
        }
        if (has && vj >= a.n) atomicOr(&a.ws.ctl->err, DEVERR_RANGE);
        mss_note(a, vj, mybits, mybk, nxt, qlen, wmin);
    }
}

// Largest k < nitems with ibase[k] <= c (ibase increases with k).
__device__ __forceinline__ unsigned mss_item_of(const unsigned long long *ibase, unsigned nitems,
                                                unsigned long long c) {
    unsigned lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const unsigned mid = (lo + hi + 1) >> 1;
        if (__ldcg(&ibase[mid]) <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(MSS_THREADS) mss_persistent_kernel(MssArgs a) {
    MssCtl *c = a.ws.ctl;
    unsigned epoch = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t gwarp = gtid >> 5, nwarps = nthreads >> 5;
    const unsigned long long cmask40 = (1ull << 40) - 1;
    unsigned long long entries = 0, scanned = 0;
    const unsigned lane = lane_id();
    unsigned nf = ld_volatile(&c->qlen[0]);
    unsigned bk = 0;  // the bucket being settled
    int r = 0;
    for (; nf > 0 && r < MSS_MAX_ROUNDS; ++r) {
        const unsigned *cur = (r & 1) ? a.ws.q[1] : a.ws.q[0];  // selects, not a dynamic index (no local copy)
        unsigned *nxt = (r & 1) ? a.ws.q[0] : a.ws.q[1];
        const int sl = r % 3, sn = (r + 1) % 3;
        // Counters: this round appends to qlen[sn] already in this phase, so
        // the queue counter of round r + 1 is cleared here, a round ahead
        // (slot (r + 2) % 3 was last read when round r - 1 began); the long-
        // row and bucket counters of the next round start over here (last
        // used two rounds ago).  Queued vertices whose smallest pending
        // bucket is beyond bk stay queued untouched; the others are taken
        // (mask exchanged, vbkt cleared) and long rows listed with their
        // chunk ranges.
        if (gtid == 0) {
            c->qlen[(r + 2) % 3] = 0;
            c->big[sn] = 0;
            c->minb[sn] = MSS_NOBKT;
            entries += nf;
        }
        unsigned wmin = MSS_NOBKT;
        for (uint64_t i0 = gtid - lane; i0 < nf; i0 += nthreads) {  // warp-uniform
            const uint64_t i = i0 + lane;
            bool keep = false;
            unsigned u = 0;
            if (i < nf) {
                u = __ldcg(&cur[i]);
                const unsigned vb = __ldcg(&a.ws.vbkt[u]);
                unsigned m = 0;
                if (vb > bk) {
                    keep = true;
                    wmin = min(wmin, vb);
                } else {
                    m = atomicExch(&a.ws.cmask[u], 0u);
                    a.ws.vbkt[u] = MSS_NOBKT;
                }
                a.ws.smask[i] = m;
                const uint64_t deg = __ldg(&a.rowptr[u + 1]) - __ldg(&a.rowptr[u]);
                if (deg > MSS_CHUNK && m) {
                    const unsigned long long nch = (deg + MSS_CHUNK - 1) / MSS_CHUNK;
                    const unsigned long long old = atomicAdd(&c->big[sl], (1ull << 40) | nch);
                    const unsigned long long k = old >> 40;
                    if (k < a.n) {
                        a.ws.items[k] = (unsigned)i;
                        a.ws.ibase[k] = old & cmask40;
                    } else {
                        atomicOr(&c->err, DEVERR_CAPACITY);
                    }
                }
            }
            const unsigned pos = warp_append(&c->qlen[sn], keep);
            if (keep) {
                if (pos < a.n) nxt[pos] = u;
                else atomicOr(&c->err, DEVERR_CAPACITY);
            }
        }
        if (!grid_sync(&c->bar, &c->err, epoch, a.nblocks, a.limit_ns)) break;
        // Relax: short rows a warp each, long rows chunk by chunk (the first
        // chunk's warp puts back the sources beyond bk).
        for (uint64_t i = gwarp; i < nf; i += nwarps) {
            const unsigned u = __ldcg(&cur[i]);
            const uint64_t b = __ldg(&a.rowptr[u]), e = __ldg(&a.rowptr[u + 1]);
            if (e - b > MSS_CHUNK) continue;  // warp-uniform
            const unsigned m = __ldcg(&a.ws.smask[i]);
            if (m) mss_relax(a, u, m, b, e, bk, true, nxt, &c->qlen[sn], wmin, scanned);
        }
        const unsigned long long bg = ld_volatile(&c->big[sl]);
        const unsigned nitems = (unsigned)min(bg >> 40, (unsigned long long)a.n);
        const unsigned long long nchunks = nitems ? (bg & cmask40) : 0;
        for (unsigned long long ch = gwarp; ch < nchunks; ch += nwarps) {
            const unsigned k = mss_item_of(a.ws.ibase, nitems, ch);
            const unsigned i = __ldcg(&a.ws.items[k]);
            const unsigned u = __ldcg(&cur[i]);
            const uint64_t rb = __ldg(&a.rowptr[u]), re = __ldg(&a.rowptr[u + 1]);
            const unsigned long long c0 = __ldcg(&a.ws.ibase[k]);
            const uint64_t b = rb + (ch - c0) * MSS_CHUNK;
            mss_relax(a, u, __ldcg(&a.ws.smask[i]), b, min(b + MSS_CHUNK, re), bk, ch == c0, nxt, &c->qlen[sn],
                      wmin, scanned);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) wmin = min(wmin, __shfl_xor_sync(FULL, wmin, d));
        if (lane == 0 && wmin != MSS_NOBKT) atomicMin(&c->minb[sn], wmin);
        if (!grid_sync(&c->bar, &c->err, epoch, a.nblocks, a.limit_ns)) break;
        nf = ld_volatile(&c->qlen[sn]);
        const unsigned mb = ld_volatile(&c->minb[sn]);
        if (nf > a.n) {
            atomicOr(&c->err, DEVERR_CAPACITY);
            break;
        }
        if (mb > bk) bk = mb;  // nothing pending at or below bk: on to the smallest pending bucket
    }
    if (r >= MSS_MAX_ROUNDS && gtid == 0) atomicOr(&c->err, DEVERR_CAPACITY);
    scanned = warp_sum(scanned);
    if (lane_id() == 0 && scanned) atomicAdd((unsigned long long *)&c->res.entries_scanned, scanned);
    if (gtid == 0) {
        c->res.rounds = r;
        c->res.frontier_entries = entries;
    }
}

// Packed words -> per-source outputs dist[s * n + o], pred[s * n + o] in
// the caller's numbering (o = inv[v]; parents renamed through inv).  A warp
// takes 32 vertices: their 32 x 32 words read row by row (coalesced) into
// shared memory, then written source by source.
constexpr int MSS_OUT_WARPS = 4;

__global__ void __launch_bounds__(MSS_OUT_WARPS * 32) mss_output_kernel(const unsigned long long *__restrict__ pack,
                                                                        uint64_t n, unsigned nsrc,
                                                                        const unsigned *__restrict__ inv,
                                                                        float *__restrict__ dist,
                                                                        int64_t *__restrict__ pred) {
    __shared__ unsigned long long s_t[MSS_OUT_WARPS][32][33];
    unsigned long long (*t)[33] = s_t[threadIdx.x >> 5];
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; v0 < n; v0 += nw * 32) {
        for (unsigned j = 0; j < 32; ++j) t[j][lane] = v0 + j < n ? __ldcs(&pack[(v0 + j) * MSS_SOURCES + lane]) : 0;
        __syncwarp();
        const uint64_t v = v0 + lane;
        if (v < n) {
            const uint64_t o = inv ? __ldg(&inv[v]) : v;
            for (unsigned s = 0; s < nsrc; ++s) {
                const unsigned long long p = t[lane][s];
                if (dist) dist[(uint64_t)s * n + o] = p == MSS_NONE ? -1.0f : __uint_as_float((unsigned)(p >> 32));
                if (pred) {
                    const unsigned par = (unsigned)p;
                    pred[(uint64_t)s * n + o] = p == MSS_NONE ? -1 : (int64_t)(inv ? __ldg(&inv[par]) : par);
                }
            }
        }
        __syncwarp();
    }
}

static int mss_max_blocks(int *out) {
    static int cached[64] = {};
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if (!cached[di.device]) {
        if ((rc = persistent_kernel_setup((const void *)mss_persistent_kernel))) return rc;
        int per_sm = 0;
        G5_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mss_persistent_kernel, MSS_THREADS, 0));
        cached[di.device] = std::max(1, per_sm) * di.sms;
    }
    *out = cached[di.device];
    return G5_OK;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_sssp_multi_workspace_size(uint64_t nverts, uint64_t *bytes) {
    clear_error();
    G5_CHECK_ARG(bytes, "g5_sssp_multi_workspace_size: bytes is NULL");
    *bytes = carve_mss(nullptr, nverts).bytes;
    return G5_OK;
}

extern "C" int g5_sssp_multi_run(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                                 const uint32_t *d_perm, const uint32_t *d_inv, const uint64_t *h_sources,
                                 uint32_t nsources, float *d_dist, int64_t *d_pred, void *d_work,
                                 uint64_t work_bytes, float delta, int32_t blocks, g5_sssp_multi_stats *h_stats,
                                 void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts < (1ull << 32) - 1, "g5_sssp_multi_run: nverts outside [1, 2^32 - 1)");
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_work && h_sources, "g5_sssp_multi_run: NULL argument");
    G5_CHECK_ARG(nsources >= 1 && nsources <= MSS_SOURCES, "g5_sssp_multi_run: nsources %u outside [1, 32]",
                 nsources);
    G5_CHECK_ARG(!d_perm == !d_inv, "g5_sssp_multi_run: perm and inv go together");
    G5_CHECK_ARG(delta >= 0.0f && delta < 1e30f, "g5_sssp_multi_run: delta %g is not a width", (double)delta);
    for (uint32_t s = 0; s < nsources; ++s)
        G5_CHECK_ARG(h_sources[s] < nverts, "g5_sssp_multi_run: source %u = %llu outside [0, %llu)", s,
                     (unsigned long long)h_sources[s], (unsigned long long)nverts);
    const MssWork w = carve_mss(d_work, nverts);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_sssp_multi_run: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    int max_blocks = 0, rc;
    if ((rc = mss_max_blocks(&max_blocks))) return rc;
    const int grid = blocks > 0 ? std::min(blocks, max_blocks) : max_blocks;
    DeviceInfo di;
    if ((rc = device_info(&di))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(MssCtl), st));
    G5_CUDA_TRY(cudaMemcpyAsync(w.ctl->sources, h_sources, nsources * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    mss_reset_kernel<<<di.sms * 8, 256, 0, st>>>(w, nverts);
    mss_seed_kernel<<<1, MSS_SOURCES, 0, st>>>(w, nverts, nsources, d_perm);
    G5_CUDA_TRY(cudaGetLastError());
    MssArgs a{d_rowstarts, d_col, d_w, nverts, w, delta > 0.0f ? 1.0f / delta : 0.0f, (unsigned)grid,
              wait_limit_ns()};  // delta 0: one bucket, every pending source relaxed each round
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(MSS_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    G5_CUDA_TRY(cudaLaunchKernelEx(&cfg, mss_persistent_kernel, a));
    if (d_dist || d_pred) {
        const uint64_t warps = (nverts + 31) / 32;
        const int og = (int)std::max<uint64_t>(1, std::min<uint64_t>((warps + MSS_OUT_WARPS - 1) / MSS_OUT_WARPS,
                                                                    (uint64_t)di.sms * 16));
        mss_output_kernel<<<og, MSS_OUT_WARPS * 32, 0, st>>>(w.pack, nverts, nsources, d_inv, d_dist, d_pred);
        G5_CUDA_TRY(cudaGetLastError());
    }
    if (!h_stats) return G5_OK;
    G5_CUDA_TRY(cudaMemcpyAsync(h_stats, &w.ctl->res, sizeof(g5_sssp_multi_stats), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaMemcpyAsync(&h_stats->error_flags, &w.ctl->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(h_stats->error_flags, "g5_sssp_multi_run");
}

extern "C" int g5_sssp_multi_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks) {
    clear_error();
    G5_CHECK_ARG(blocks && max_blocks, "g5_sssp_multi_grid: NULL argument");
    int mb = 0;
    int rc = mss_max_blocks(&mb);
    if (rc) return rc;
    *max_blocks = mb;
    *blocks = (int)std::min<uint64_t>(mb, std::max<uint64_t>(1, nverts / 2048));
    return G5_OK;
}

extern "C" int g5_sssp_multi_last_stats(const void *d_work, uint64_t work_bytes, g5_sssp_multi_stats *stats,
                                        void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && stats, "g5_sssp_multi_last_stats: NULL argument");
    G5_CHECK_ARG(work_bytes >= sizeof(MssCtl), "g5_sssp_multi_last_stats: workspace too small");
    const MssCtl *ctl = (const MssCtl *)d_work;  // the workspace starts with the control block
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(stats, &ctl->res, sizeof(g5_sssp_multi_stats), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaMemcpyAsync(&stats->error_flags, &ctl->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(stats->error_flags, "g5_sssp_multi_run");
}
