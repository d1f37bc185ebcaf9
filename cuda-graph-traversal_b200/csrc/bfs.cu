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
// warp of the grid takes BIG_CHUNK-edge chunks of them from a per-vertex
// cursor.  A neighbour is claimed with an atomicOr on the visited bitmap;
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

#include "g5_common.cuh"

namespace g5 {

constexpr int BFS_THREADS = 256;
constexpr unsigned BIG_DEG = 4096;
constexpr unsigned BIG_CHUNK = 1024;

struct BfsCtl {
    unsigned bar;  // grid barrier arrivals
    unsigned error;
    unsigned n_small[3];  // per level slot: queue entries of degree <= BIG_DEG
    unsigned n_big[3];    //                 queue entries above BIG_DEG
    unsigned grab[3];     //                 work cursor over the small part
    unsigned found[3];    //                 vertices found by a bottom-up level
    unsigned long long m_next[3];  //        degree sum of the next frontier
    int levels;
    int bu_levels;
    unsigned long long reached;
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
    unsigned *q[2];
    unsigned *bigcur[2];
    BfsCtl *ctl;
    float alpha;
    float beta;
    int mode;
    unsigned nblocks;
    unsigned long long limit_ns;
};

enum { TOP_DOWN = 0, BOTTOM_UP = 1 };

// Claim v for parent u at the next level; appends it to the next queue.
// All 32 lanes must call it (want = this lane has a candidate).
__device__ __forceinline__ void td_visit(const BfsArgs &a, bool want, unsigned v, unsigned u, int next_level,
                                         unsigned *qn, unsigned *bcn, unsigned *n_small, unsigned *n_big,
                                         unsigned long long &my_m) {
    if (want && v >= a.n) {  // not a vertex: report it, touch nothing
        atomicOr(&a.ctl->error, DEVERR_RANGE);
        want = false;
    }
    bool disc = want && bit_claim(a.visited, v);
    uint64_t deg = 0;
    if (disc) {
        a.pred[v] = (int64_t)u;
        if (a.depth) a.depth[v] = next_level;
        deg = __ldg(&a.rowptr[v + 1]) - __ldg(&a.rowptr[v]);
        my_m += deg;
    }
    const bool small = disc && deg <= BIG_DEG;
    const bool big = disc && deg > BIG_DEG;
    unsigned ps = warp_append(n_small, small);
    if (small) qn[ps] = v;
    unsigned pb = warp_append(n_big, big);
    if (big) {
        qn[a.n - 1 - pb] = v;
        bcn[pb] = 0;
    }
}

__device__ void td_expand(const BfsArgs &a, int level, int cur, int s_cur, int s_nxt, unsigned long long &my_m) {
    BfsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const unsigned *Q = a.q[cur];
    unsigned *QN = a.q[cur ^ 1];
    unsigned *BC = a.bigcur[cur];
    unsigned *BCN = a.bigcur[cur ^ 1];
    const unsigned ns = ld_volatile(&c->n_small[s_cur]);
    const unsigned nb = ld_volatile(&c->n_big[s_cur]);

    // Small part: 32 queue entries per grab, edges gathered across the warp.
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&c->grab[s_cur], 32u);
        base = __shfl_sync(FULL, base, 0);
        if (base >= ns) break;
        const unsigned i = base + lane;
        const bool valid = i < ns;
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
            td_visit(a, has, v, uj, level + 1, QN, BCN, &c->n_small[s_nxt], &c->n_big[s_nxt], my_m);
        }
    }
    // Big part: every warp takes chunks of every big vertex.
    for (unsigned j = 0; j < nb; ++j) {
        const unsigned u = __ldcg(&Q[a.n - 1 - j]);
        const uint64_t rb = __ldg(&a.rowptr[u]);
        const uint64_t deg = __ldg(&a.rowptr[u + 1]) - rb;
        for (;;) {
            unsigned cstart = 0;
            if (lane == 0) cstart = atomicAdd(&BC[j], BIG_CHUNK);
            cstart = __shfl_sync(FULL, cstart, 0);
            if (cstart >= deg) break;
            const uint64_t cend = min((uint64_t)cstart + BIG_CHUNK, deg);
            for (uint64_t e = cstart + lane; e < (uint64_t)cstart + BIG_CHUNK; e += 32) {
                const bool has = e < cend;
                const unsigned v = has ? (unsigned)__ldg(&a.col[rb + e]) : 0u;
                td_visit(a, has, v, u, level + 1, QN, BCN, &c->n_small[s_nxt], &c->n_big[s_nxt], my_m);
            }
        }
    }
}

__device__ void bu_expand(const BfsArgs &a, int level, const unsigned *fb, unsigned *nb, unsigned long long &my_m,
                          unsigned &my_found) {
    const unsigned lane = lane_id();
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = warp; k < a.nwords; k += nwarps) {
        const unsigned vis = __ldcg(&a.visited[k]);
        const uint64_t v = k * 32 + lane;
        int found = -1;
        uint64_t rb = 0, re = 0;
        if (v < a.n && !((vis >> lane) & 1u)) {
            rb = __ldg(&a.rowptr[v]);
            re = __ldg(&a.rowptr[v + 1]);
            for (uint64_t e = rb; e < re; ++e) {
                const unsigned u = (unsigned)__ldg(&a.col[e]);
                if (u >= a.n) {
                    atomicOr(&a.ctl->error, DEVERR_RANGE);
                    continue;
                }
                if ((__ldcg(&fb[u >> 5]) >> (u & 31)) & 1u) {
                    found = (int)u;
                    break;
                }
            }
        }
        const unsigned mask = __ballot_sync(FULL, found >= 0);
        if (found >= 0) {
            a.pred[v] = found;
            if (a.depth) a.depth[v] = level + 1;
            my_m += re - rb;
        }
        if (lane == 0) {
            if (mask) a.visited[k] = vis | mask;
            nb[k] = mask;
            my_found += __popc(mask);
        }
    }
}

// Next-frontier queue from the bottom-up bitmap (small/big split by degree).
__device__ void bits_to_queue(const BfsArgs &a, const unsigned *bits, unsigned *qn, unsigned *bcn, unsigned *n_small,
                              unsigned *n_big) {
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
            const bool small = has && deg <= BIG_DEG, big = has && deg > BIG_DEG;
            unsigned ps = warp_append(n_small, small);
            if (small) qn[ps] = v;
            unsigned pb = warp_append(n_big, big);
            if (big) {
                qn[a.n - 1 - pb] = v;
                bcn[pb] = 0;
            }
        }
    }
}

__global__ void __launch_bounds__(BFS_THREADS, 4) bfs_persistent_kernel(BfsArgs a) {
    BfsCtl *c = a.ctl;
    unsigned epoch = 0;
    const uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t E = __ldg(&a.rowptr[a.n]);
    const uint64_t root_deg = __ldg(&a.rowptr[a.root + 1]) - __ldg(&a.rowptr[a.root]);

    if (gtid == 0) {
        a.visited[a.root >> 5] |= 1u << (a.root & 31);
        a.pred[a.root] = a.root;
        if (a.depth) a.depth[a.root] = 0;
        if (root_deg > BIG_DEG) {
            a.q[0][a.n - 1] = a.root;
            a.bigcur[0][0] = 0;
            c->n_big[0] = 1;
        } else {
            a.q[0][0] = a.root;
            c->n_small[0] = 1;
        }
    }
    if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;

    int mode = TOP_DOWN;
    int cur = 0;
    unsigned *fb = a.fbits, *nb = a.nbits;
    uint64_t m_u = E - root_deg;
    unsigned n_f = 1;
    unsigned long long reached = 1;
    int levels = 0, bu_levels = 0;

    for (int level = 0;; ++level) {
        const int s_cur = level % 3, s_nxt = (level + 1) % 3, s_clr = (level + 2) % 3;
        if (gtid == 0) {
            c->n_small[s_clr] = 0;
            c->n_big[s_clr] = 0;
            c->grab[s_clr] = 0;
            c->found[s_clr] = 0;
            c->m_next[s_clr] = 0;
        }
        unsigned long long my_m = 0;
        unsigned my_found = 0;
        if (mode == TOP_DOWN)
            td_expand(a, level, cur, s_cur, s_nxt, my_m);
        else
            bu_expand(a, level, fb, nb, my_m, my_found);
        my_m = warp_sum(my_m);
        my_found = warp_sum(my_found);
        if (lane_id() == 0) {
            if (my_m) atomicAdd(&c->m_next[s_nxt], my_m);
            if (my_found) atomicAdd(&c->found[s_nxt], my_found);
        }
        ++levels;
        bu_levels += mode == BOTTOM_UP;
        if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;

        const unsigned long long m_next = ld_volatile(&c->m_next[s_nxt]);
        const unsigned n_next = mode == TOP_DOWN
                                    ? ld_volatile(&c->n_small[s_nxt]) + ld_volatile(&c->n_big[s_nxt])
                                    : ld_volatile(&c->found[s_nxt]);
        m_u -= m_next;
        reached += n_next;
        if (n_next == 0) break;

        int next = mode;
        if (a.mode == 1) {
            next = TOP_DOWN;
        } else if (a.mode == 2) {
            next = BOTTOM_UP;
        } else if (mode == TOP_DOWN) {
            if ((double)m_next > (double)m_u / a.alpha) next = BOTTOM_UP;
        } else {
            if ((double)n_next < (double)a.n / a.beta && n_next < n_f) next = TOP_DOWN;
        }

        if (mode == TOP_DOWN && next == BOTTOM_UP) {
            // Frontier bitmap from the queue just built.
            for (uint64_t k = gtid; k < a.nwords; k += nthreads) fb[k] = 0;
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
            const unsigned *QN = a.q[cur ^ 1];
            const unsigned ns = ld_volatile(&c->n_small[s_nxt]), nbg = ld_volatile(&c->n_big[s_nxt]);
            for (uint64_t i = gtid; i < ns; i += nthreads) {
                unsigned v = __ldcg(&QN[i]);
                atomicOr(&fb[v >> 5], 1u << (v & 31));
            }
            for (uint64_t i = gtid; i < nbg; i += nthreads) {
                unsigned v = __ldcg(&QN[a.n - 1 - i]);
                atomicOr(&fb[v >> 5], 1u << (v & 31));
            }
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
        } else if (mode == BOTTOM_UP && next == BOTTOM_UP) {
            unsigned *t = fb;
            fb = nb;
            nb = t;
        } else if (mode == BOTTOM_UP && next == TOP_DOWN) {
            bits_to_queue(a, nb, a.q[cur ^ 1], a.bigcur[cur ^ 1], &c->n_small[s_nxt], &c->n_big[s_nxt]);
            if (!grid_sync(&c->bar, &c->error, epoch, a.nblocks, a.limit_ns)) return;
        }
        if (next == TOP_DOWN) cur ^= 1;
        mode = next;
        n_f = n_next;
    }
    if (gtid == 0) {
        c->levels = levels;
        c->bu_levels = bu_levels;
        c->reached = reached;
    }
}

struct BfsWork {
    BfsCtl *ctl;
    unsigned *visited, *fbits, *nbits;
    unsigned *q[2], *bigcur[2];
    uint64_t bytes;
};

static BfsWork carve_bfs(void *base, uint64_t n) {
    Carver c(base);
    BfsWork w;
    const uint64_t words = (n + 31) / 32;
    w.ctl = c.take<BfsCtl>(1);
    w.visited = c.take<unsigned>(words);
    w.fbits = c.take<unsigned>(words);
    w.nbits = c.take<unsigned>(words);
    for (int i = 0; i < 2; ++i) {
        w.q[i] = c.take<unsigned>(n);
        w.bigcur[i] = c.take<unsigned>(n);
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

extern "C" int g5_bfs_reset(uint64_t nverts, int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                            void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31) && d_pred && d_work, "g5_bfs_reset: bad argument");
    BfsWork w = carve_bfs(d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_bfs_reset: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(d_pred, 0xff, nverts * sizeof(int64_t), st));
    if (d_depth) G5_CUDA_TRY(cudaMemsetAsync(d_depth, 0xff, nverts * sizeof(int32_t), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.visited, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(BfsCtl), st));
    return G5_OK;
}

extern "C" int g5_bfs_traverse(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                               int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                               const g5_bfs_params *params, void *stream) {
    clear_error();
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, root, d_pred, d_work, work_bytes, &w, "g5_bfs_traverse");
    if (rc) return rc;
    g5_bfs_params p = {14.0f, 24.0f, 0, 0};
    if (params) p = *params;
    G5_CHECK_ARG(p.alpha > 0 && p.beta > 0 && p.mode >= 0 && p.mode <= 2, "g5_bfs_traverse: bad params");

    int max_blocks = 0;
    if ((rc = bfs_max_blocks(&max_blocks))) return rc;
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
    a.q[0] = w.q[0];
    a.q[1] = w.q[1];
    a.bigcur[0] = w.bigcur[0];
    a.bigcur[1] = w.bigcur[1];
    a.ctl = w.ctl;
    a.alpha = p.alpha;
    a.beta = p.beta;
    a.mode = p.mode;
    a.nblocks = (unsigned)blocks;
    a.limit_ns = wait_limit_ns();
    void *args[] = {&a};
    G5_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)bfs_persistent_kernel, dim3(blocks), dim3(BFS_THREADS), args,
                                            0, (cudaStream_t)stream));
    return G5_OK;
}

extern "C" int g5_bfs_run(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                          int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                          const g5_bfs_params *params, void *stream) {
    clear_error();
    BfsWork w;
    int rc = bfs_check(d_rowstarts, d_col, nverts, root, d_pred, d_work, work_bytes, &w, "g5_bfs_run");
    if (rc) return rc;
    if ((rc = g5_bfs_reset(nverts, d_pred, d_depth, d_work, work_bytes, stream))) return rc;
    return g5_bfs_traverse(d_rowstarts, d_col, nverts, root, d_pred, d_depth, d_work, work_bytes, params, stream);
}

extern "C" int g5_bfs_last_stats(const void *d_work, uint64_t work_bytes, g5_bfs_stats *stats, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && stats, "g5_bfs_last_stats: NULL argument");
    G5_CHECK_ARG(work_bytes >= sizeof(BfsCtl), "g5_bfs_last_stats: workspace too small");
    BfsCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    stats->levels = c.levels;
    stats->bottom_up_levels = c.bu_levels;
    stats->reached = c.reached;
    return deverr_to_status(c.error, "g5_bfs_run");
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
