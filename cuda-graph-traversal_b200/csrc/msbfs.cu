// msbfs.cu -- batched BFS: up to 256 roots searched together in one
// persistent cooperative launch, one bit per root.
//
// The reference searches one root per call (oned_graph_bfs_run,
// src/traversal.cu:479-503, kernel :139-207); a Graph500 run repeats it for
// 64 roots.  Here every vertex owns a 256-bit row (8 x u32, one 32-byte
// DRAM sector) in each of these arrays:
//
//   seen[p]     bit i: root i has reached the vertex
//   fr[0/1][p]  bit i: the vertex is in root i's frontier (current / next)
//   plane[k][p] bit i: bit k of root i's depth of the vertex
//
// so one sector read of a neighbour's frontier row serves all 256 searches,
// which is what makes a batch cheaper than 256 single searches.
//
// Vertex positions.  g5_msbfs_prepare renumbers the vertices by decreasing
// degree (p = pos[v]) and keeps a copy of the CSR in that order (rows and
// column values both in positions).  Most CSR entries point at the few
// high-degree vertices, so their rows -- now packed at the front of every
// array -- stay in L2 while the pull levels stream the column past them,
// and the vertices a warp takes together have rows of about equal length.
// Positions [0, H) are heavy rows (more than MS_LIGHT entries), [H, H + L)
// light rows, the rest isolated vertices.
//
// Level L (frontier = vertices at depth L of some root) runs in one of two
// directions, the same in every block:
//   * top-down, while the frontier's CSR entries are few: each frontier
//     vertex u pushes its row fr[u] to every neighbour v, OR-ing the bits
//     v has not seen (fr[u] & ~seen[v]) into next[v] with 64-bit atomics;
//   * pull: every vertex that some live root has not reached ORs the
//     frontier rows of its neighbours and stops as soon as every missing
//     live root is found.  Light rows take one lane each; heavy rows are
//     cut into MS_CHUNK-entry chunks, one warp each, merged with atomics.
// A second pass over the frontier bitmaps then folds next[] into seen[] and
// the depth planes and zeroes the consumed frontier rows, so the frontier
// arrays are all-zero outside the frontier at all times (the next search
// needs no clearing after a clean finish).
//
// Bounds: HBM.  A pull level reads 4 B of column per scanned entry plus the
// neighbour's 32 B row (an L2 hit for most entries); a top-down level reads
// 4 B + one 32 B seen row per frontier entry.
#include <algorithm>
#include <mutex>

#include "g5_common.cuh"

namespace g5 {

constexpr int MS_THREADS = 256;
constexpr int MS_W = 8;              // u32 words per row (256 roots)
constexpr unsigned MS_MAX_ROOTS = 256;
constexpr unsigned MS_LIGHT = 256;   // rows up to this length: one lane per vertex
constexpr unsigned MS_CHUNK = 1024;  // longer rows: chunks of this many entries, one warp each
constexpr int MS_TRACE = 64;
constexpr int MS_DEFAULT_BITS = 6;
constexpr float MS_DEFAULT_ALPHA = 32.0f;  // top-down while frontier entries * alpha < all entries
constexpr unsigned MS_NKEYS = 513;   // degree buckets of the renumbering
constexpr unsigned long long MS_CLEAN = 0x9e3779b97f4a7c15ull;   // frontier arrays known to be zero
constexpr unsigned long long MS_PREPARED = 0x51afd7ed558ccd1dull;

struct MsCtl {
    g5_msbfs_stats res;
    unsigned bar;
    unsigned nheavy;   // H: positions [0, H) have more than MS_LIGHT entries
    unsigned nlight;   // L: positions [H, H + L) have 1..MS_LIGHT entries
    unsigned nchunks;  // chunks of the heavy rows
    unsigned long long prepared;  // MS_PREPARED once g5_msbfs_prepare ran
    unsigned long long prep_n;    // vertex count it ran for
    unsigned long long clean;     // MS_CLEAN when fr[0], fr[1] and both bitmaps are zero
    unsigned long long roots[MS_MAX_ROOTS];
    // per level slot (level % 3)
    unsigned wgrab[3];
    unsigned cgrab[3];
    unsigned n_f[3];
    unsigned long long m_f[3];
    unsigned live[3][MS_W];  // roots with a non-empty frontier at that level
    // trace
    unsigned long long t0;
    unsigned long long t_level[MS_TRACE];
    unsigned long long m_level[MS_TRACE];
    unsigned n_level[MS_TRACE];
    unsigned char mode_level[MS_TRACE];
};

struct MsWork {
    MsCtl *ctl;
    unsigned *seen, *fr[2];
    unsigned *nz;             // ring of frontier bitmaps, one per level (nbufs x words)
    uint64_t words;
    int nbufs;
    unsigned *vis;            // bit p: some root has reached position p
    unsigned *pos, *orig;     // vertex -> position, position -> vertex
    uint64_t *rp;             // row starts in position order (n + 1)
    unsigned *cp;             // column in positions (nentries)
    unsigned *chunk_v, *chunk_off;
    unsigned *hist;           // MS_NKEYS + 1 bucket counters
    unsigned *tmp;            // n: degrees in position order
    uint64_t *scan;           // scan scratch
    unsigned *planes;
    uint64_t maxchunks;
    uint64_t bytes;
};

static uint64_t ms_max_chunks(uint64_t nentries) {
    // A heavy row of d > MS_LIGHT entries has ceil(d / MS_CHUNK) chunks, so
    // all of them together have at most E / MS_CHUNK + E / (MS_LIGHT + 1) + 1.
    return nentries / MS_CHUNK + nentries / (MS_LIGHT + 1) + 1;
}

static MsWork carve_ms(void *base, uint64_t n, uint64_t nentries, int bits) {
    Carver c(base);
    MsWork w{};
    const uint64_t words = (n + 31) / 32;
    w.ctl = c.take<MsCtl>(1);
    w.seen = c.take<unsigned>(n * MS_W);
    w.fr[0] = c.take<unsigned>(n * MS_W);
    w.fr[1] = c.take<unsigned>(n * MS_W);
    w.words = words;
    w.nbufs = (1 << bits) + 2;
    w.nz = c.take<unsigned>(words * w.nbufs);
    w.vis = c.take<unsigned>(words);
    w.pos = c.take<unsigned>(n);
    w.orig = c.take<unsigned>(n);
    w.rp = c.take<uint64_t>(n + 1);
    w.cp = c.take<unsigned>(nentries);
    w.maxchunks = ms_max_chunks(nentries);
    w.chunk_v = c.take<unsigned>(w.maxchunks);
    w.chunk_off = c.take<unsigned>(w.maxchunks);
    w.hist = c.take<unsigned>(MS_NKEYS + 1);
    w.tmp = c.take<unsigned>(n);
    w.scan = c.take<uint64_t>(scan_scratch_words(n));
    w.planes = c.take<unsigned>((uint64_t)bits * n * MS_W);
    w.bytes = c.used;
    return w;
}

// ------------------------------------------------------------ row helpers --

struct Row {
    uint4 a, b;
};

// A whole 32-byte row in one access.  Rows are written earlier in the same
// launch, so they are read from L2 (.cg), optionally with an eviction policy.
__device__ __forceinline__ Row row_ld(const unsigned *base, uint64_t v) {
    const unsigned *p = base + v * MS_W;
    Row r;
    asm volatile("ld.global.cg.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r.a.x), "=r"(r.a.y), "=r"(r.a.z), "=r"(r.a.w), "=r"(r.b.x), "=r"(r.b.y), "=r"(r.b.z),
                   "=r"(r.b.w)
                 : "l"(p));
    return r;
}
__device__ __forceinline__ Row row_ld_hint(const unsigned *base, uint64_t v, uint64_t pol) {
    const unsigned *p = base + v * MS_W;
    Row r;
    asm volatile("ld.global.cg.L2::cache_hint.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8], %9;"
                 : "=r"(r.a.x), "=r"(r.a.y), "=r"(r.a.z), "=r"(r.a.w), "=r"(r.b.x), "=r"(r.b.y), "=r"(r.b.z),
                   "=r"(r.b.w)
                 : "l"(p), "l"(pol));
    return r;
}
__device__ __forceinline__ void row_st(unsigned *base, uint64_t v, const Row &r) {
    unsigned *p = base + v * MS_W;
    asm volatile("st.global.cg.v8.u32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(r.a.x), "r"(r.a.y),
                 "r"(r.a.z), "r"(r.a.w), "r"(r.b.x), "r"(r.b.y), "r"(r.b.z), "r"(r.b.w)
                 : "memory");
}

// L2 eviction policies: the column streams through once per level
// (evict first); frontier and seen rows are re-read by every neighbour
// (evict last).
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Word of the current level's frontier bitmap, through L1.  Safe because
// that bitmap is complete before its level starts (grid barrier) and no
// load ever brought its lines into L1 earlier in the launch: the level that
// builds it reads it with L2-only loads (__ldcg) and atomics only.
__device__ __forceinline__ unsigned ld_l1(const unsigned *p) {
    unsigned v;
    asm("ld.global.ca.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
// Column entry (read-only for the whole launch).
__device__ __forceinline__ unsigned ld_col(const unsigned *p, uint64_t pol) {
    unsigned v;
    asm("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ Row row_zero() { return Row{make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)}; }
__device__ __forceinline__ void row_or_into(Row &d, const Row &s) {
    d.a.x |= s.a.x, d.a.y |= s.a.y, d.a.z |= s.a.z, d.a.w |= s.a.w;
    d.b.x |= s.b.x, d.b.y |= s.b.y, d.b.z |= s.b.z, d.b.w |= s.b.w;
}
__device__ __forceinline__ Row row_and(const Row &x, const Row &y) {
    return Row{make_uint4(x.a.x & y.a.x, x.a.y & y.a.y, x.a.z & y.a.z, x.a.w & y.a.w),
               make_uint4(x.b.x & y.b.x, x.b.y & y.b.y, x.b.z & y.b.z, x.b.w & y.b.w)};
}
__device__ __forceinline__ Row row_andnot(const Row &x, const Row &y) {  // x & ~y
    return Row{make_uint4(x.a.x & ~y.a.x, x.a.y & ~y.a.y, x.a.z & ~y.a.z, x.a.w & ~y.a.w),
               make_uint4(x.b.x & ~y.b.x, x.b.y & ~y.b.y, x.b.z & ~y.b.z, x.b.w & ~y.b.w)};
}
__device__ __forceinline__ bool row_any(const Row &x) {
    return (x.a.x | x.a.y | x.a.z | x.a.w | x.b.x | x.b.y | x.b.z | x.b.w) != 0;
}
__device__ __forceinline__ unsigned row_word(const Row &x, int w) {
    switch (w) {
        case 0: return x.a.x;
        case 1: return x.a.y;
        case 2: return x.a.z;
        case 3: return x.a.w;
        case 4: return x.b.x;
        case 5: return x.b.y;
        case 6: return x.b.z;
        default: return x.b.w;
    }
}
__device__ __forceinline__ unsigned row_popc(const Row &x) {
    return __popc(x.a.x) + __popc(x.a.y) + __popc(x.a.z) + __popc(x.a.w) + __popc(x.b.x) + __popc(x.b.y) +
           __popc(x.b.z) + __popc(x.b.w);
}
__device__ __forceinline__ Row row_bcast(const Row &x, int src) {
    return Row{make_uint4(__shfl_sync(FULL, x.a.x, src), __shfl_sync(FULL, x.a.y, src), __shfl_sync(FULL, x.a.z, src),
                          __shfl_sync(FULL, x.a.w, src)),
               make_uint4(__shfl_sync(FULL, x.b.x, src), __shfl_sync(FULL, x.b.y, src), __shfl_sync(FULL, x.b.z, src),
                          __shfl_sync(FULL, x.b.w, src))};
}
__device__ __forceinline__ Row row_warp_or(Row x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        x.a.x |= __shfl_xor_sync(FULL, x.a.x, d);
        x.a.y |= __shfl_xor_sync(FULL, x.a.y, d);
        x.a.z |= __shfl_xor_sync(FULL, x.a.z, d);
        x.a.w |= __shfl_xor_sync(FULL, x.a.w, d);
        x.b.x |= __shfl_xor_sync(FULL, x.b.x, d);
        x.b.y |= __shfl_xor_sync(FULL, x.b.y, d);
        x.b.z |= __shfl_xor_sync(FULL, x.b.z, d);
        x.b.w |= __shfl_xor_sync(FULL, x.b.w, d);
    }
    return x;
}
// OR of the row into base[v] with 64-bit atomics (only the non-zero halves).
__device__ __forceinline__ void row_atomic_or(unsigned *base, uint64_t v, const Row &x) {
    unsigned long long *p = (unsigned long long *)(base + v * MS_W);
    const unsigned long long w0 = ((unsigned long long)x.a.y << 32) | x.a.x;
    const unsigned long long w1 = ((unsigned long long)x.a.w << 32) | x.a.z;
    const unsigned long long w2 = ((unsigned long long)x.b.y << 32) | x.b.x;
    const unsigned long long w3 = ((unsigned long long)x.b.w << 32) | x.b.z;
    if (w0) atomicOr(p + 0, w0);
    if (w1) atomicOr(p + 1, w1);
    if (w2) atomicOr(p + 2, w2);
    if (w3) atomicOr(p + 3, w3);
}

// ---------------------------------------------------------- preparation --

// Bucket of a degree in decreasing order: heavy rows by their top four
// bits (eight buckets per octave), light rows by exact degree, isolated
// vertices last.
__device__ __forceinline__ unsigned ms_key(uint64_t deg) {
    if (deg == 0) return MS_NKEYS - 1;
    if (deg <= MS_LIGHT) return 256 + (MS_LIGHT - (unsigned)deg);
    const int lg = 63 - __clzll((long long)deg);  // >= 8
    const unsigned hkey = min(255u, (unsigned)(lg - 8) * 8 + (unsigned)((deg >> (lg - 3)) & 7));
    return 255 - hkey;
}

__global__ void ms_prep_hist_kernel(const uint64_t *__restrict__ rowptr, uint64_t n, uint64_t nentries,
                                    unsigned *__restrict__ hist, MsCtl *c) {
    __shared__ unsigned sh[MS_NKEYS];
    for (unsigned i = threadIdx.x; i < MS_NKEYS; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0 && __ldg(&rowptr[n]) != nentries) atomicOr(&c->res.error_flags, DEVERR_RANGE);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        atomicAdd(&sh[ms_key(__ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]))], 1u);
    __syncthreads();
    for (unsigned i = threadIdx.x; i < MS_NKEYS; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// hist[k] := first position of bucket k; heavy and light counts.
__global__ void ms_prep_scan_kernel(unsigned *hist, MsCtl *c) {
    if (threadIdx.x != 0) return;
    unsigned acc = 0, heavy = 0;
    for (unsigned k = 0; k < MS_NKEYS; ++k) {
        const unsigned h = hist[k];
        hist[k] = acc;
        acc += h;
        if (k == 255) heavy = acc;
        if (k == MS_NKEYS - 2) c->nlight = acc - heavy;
    }
    c->nheavy = heavy;
}

__global__ void ms_prep_scatter_kernel(const uint64_t *__restrict__ rowptr, uint64_t n, unsigned *__restrict__ hist,
                                       unsigned *__restrict__ pos, unsigned *__restrict__ orig,
                                       unsigned *__restrict__ deg_p) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v0 = warp * 32; v0 < n; v0 += nwarps * 32) {
        const uint64_t v = v0 + lane_id();
        const bool ok = v < n;
        const uint64_t deg = ok ? __ldg(&rowptr[v + 1]) - __ldg(&rowptr[v]) : 0;
        const unsigned key = ok ? ms_key(deg) : 0xffffffffu;
        // Lanes of one bucket share one atomic.
        const unsigned peers = __match_any_sync(FULL, key);
        const unsigned leader = __ffs(peers) - 1;
        unsigned b = 0;
        if (ok && lane_id() == leader) b = atomicAdd(&hist[key], (unsigned)__popc(peers));
        b = __shfl_sync(FULL, b, leader);
        if (ok) {
            const unsigned p = b + __popc(peers & lanemask_lt());
            pos[v] = p;
            orig[p] = (unsigned)v;
            deg_p[p] = (unsigned)deg;
        }
    }
}

// Column in positions, rows in position order: one warp per row.
__global__ void ms_prep_fill_kernel(const uint64_t *__restrict__ rowptr, const int *__restrict__ col, uint64_t n,
                                    const unsigned *__restrict__ pos, const unsigned *__restrict__ orig,
                                    const uint64_t *__restrict__ rp, unsigned *__restrict__ cp, MsCtl *c) {
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t p = warp; p < n; p += nwarps) {
        const unsigned v = __ldg(&orig[p]);
        const uint64_t rb = __ldg(&rowptr[v]), d = __ldg(&rowptr[v + 1]) - rb;
        const uint64_t out = __ldg(&rp[p]);
        bool bad = false;
        for (uint64_t e = lane_id(); e < d; e += 32) {
            const unsigned u = (unsigned)__ldg(&col[rb + e]);
            bad |= u >= n;
            cp[out + e] = u < n ? __ldg(&pos[u]) : 0xffffffffu;
        }
        if (__any_sync(FULL, bad) && lane_id() == 0) atomicOr(&c->res.error_flags, DEVERR_RANGE);
    }
}

// Chunks of the heavy rows (positions [0, H)).
__global__ void ms_prep_chunks_kernel(const uint64_t *__restrict__ rp, MsCtl *c, unsigned *__restrict__ chunk_v,
                                      unsigned *__restrict__ chunk_off, uint64_t maxchunks) {
    const unsigned H = ld_volatile(&c->nheavy);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < H; p += stride) {
        const uint64_t deg = __ldg(&rp[p + 1]) - __ldg(&rp[p]);
        const unsigned nch = (unsigned)((deg + MS_CHUNK - 1) / MS_CHUNK);
        const unsigned b = atomicAdd(&c->nchunks, nch);
        if ((uint64_t)b + nch > maxchunks) {
            atomicOr(&c->res.error_flags, DEVERR_CAPACITY);
            continue;
        }
        for (unsigned i = 0; i < nch; ++i) {
            chunk_v[b + i] = (unsigned)p;
            chunk_off[b + i] = i * MS_CHUNK;
        }
    }
}

// ---------------------------------------------------------------- search --

struct MsArgs {
    const uint64_t *rp;   // rows in position order
    const unsigned *cp;   // column in positions
    const unsigned *pos;
    uint64_t n, nwords, E;
    unsigned *seen;
    unsigned *fr[2];
    unsigned *nz;  // frontier bitmap of level L at nz + L * nwords
    unsigned *vis;
    unsigned *planes;
    const unsigned *chunk_v, *chunk_off;
    MsCtl *ctl;
    int bits;
    int max_depth;
    float alpha;
    int mode;
    int check_frontier;
    unsigned nblocks;
    unsigned long long limit_ns;
};

enum { MS_TOP_DOWN = 0, MS_PULL = 1 };

__global__ void ms_reset_kernel(MsWork w, uint64_t n) {
    // Every block reads the flag before the seed kernel (the next launch)
    // can change it.
    const bool clean = ld_volatile(&w.ctl->clean) == MS_CLEAN;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (uint64_t i = t0; i < n * 2; i += stride) ((uint4 *)w.seen)[i] = z;
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t k = t0; k < nw; k += stride) w.vis[k] = 0;
    if (!clean) {
        for (uint64_t i = t0; i < n * 2; i += stride) {
            ((uint4 *)w.fr[0])[i] = z;
            ((uint4 *)w.fr[1])[i] = z;
        }
    }
    // Frontier bitmaps a clean search wrote (levels + 1 of them), or all.
    const int used = clean ? min(ld_volatile(&w.ctl->res.levels) + 2, w.nbufs) : w.nbufs;
    for (uint64_t k = t0; k < (uint64_t)used * w.words; k += stride) w.nz[k] = 0;
}

// Level 0: the roots.  One block; thread i takes root i.
__global__ void ms_seed_kernel(MsArgs a, unsigned nroots) {
    MsCtl *c = a.ctl;
    if (threadIdx.x == 0) {
        c->res = g5_msbfs_stats{0, 0, 0, nroots, 0, 0};
        c->bar = 0;
        c->clean = 0;  // the search writes the frontier arrays
        for (int s = 0; s < 3; ++s) {
            c->wgrab[s] = c->cgrab[s] = c->n_f[s] = 0;
            c->m_f[s] = 0;
            for (int w = 0; w < MS_W; ++w) c->live[s][w] = 0;
        }
        if (c->prepared != MS_PREPARED || c->prep_n != a.n) c->res.error_flags |= DEVERR_UNPREPARED;
    }
    __syncthreads();
    const unsigned i = threadIdx.x;
    if (i < nroots && !(ld_volatile(&c->res.error_flags) & DEVERR_UNPREPARED)) {
        const uint64_t r = c->roots[i];
        if (r >= a.n) {
            atomicOr(&c->res.error_flags, DEVERR_RANGE);
        } else {
            const unsigned p = __ldg(&a.pos[r]);
            const unsigned bit = 1u << (i & 31);
            atomicOr(&a.seen[(uint64_t)p * MS_W + (i >> 5)], bit);
            atomicOr(&a.fr[0][(uint64_t)p * MS_W + (i >> 5)], bit);
            atomicOr(&c->live[0][i >> 5], bit);
            atomicOr(&a.vis[p >> 5], 1u << (p & 31));
            // Depth 0: the vertex's planes start at zero (later levels only OR into them).
            for (int k = 0; k < a.bits; ++k) row_st(a.planes + (uint64_t)k * a.n * MS_W, p, row_zero());
            const unsigned pb = 1u << (p & 31);
            if (!(atomicOr(&a.nz[p >> 5], pb) & pb)) {
                atomicAdd(&c->n_f[0], 1u);
                atomicAdd(&c->m_f[0], (unsigned long long)(__ldg(&a.rp[p + 1]) - __ldg(&a.rp[p])));
            }
        }
    }
    if (threadIdx.x == 0) c->res.pairs_reached = nroots;
}

// Pushes fu (a frontier row) to the N neighbours v[i] with ok[i].  The
// vertex bitmap `vis` (any root has reached v) and the next-frontier
// bitmap say whether v's seen and next rows can hold bits at all, so most
// pushes of an early level read neither row; bits already in next[v] need
// no atomic.
template <int N>
__device__ __forceinline__ void ms_push(const MsArgs &a, unsigned *X, unsigned *nzn, const unsigned (&v)[N],
                                        const bool (&ok)[N], const Row &fu, uint64_t keep) {
    unsigned vw[N], nb[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        vw[i] = ok[i] ? __ldcg(&a.vis[v[i] >> 5]) : 0u;
        nb[i] = ok[i] ? __ldcg(&nzn[v[i] >> 5]) : 0u;
    }
    Row sv[N], xv[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const unsigned b = 1u << (v[i] & 31);
        sv[i] = (vw[i] & b) ? row_ld_hint(a.seen, v[i], keep) : row_zero();
        xv[i] = (nb[i] & b) ? row_ld_hint(X, v[i], keep) : row_zero();
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (!ok[i]) continue;
        const Row nw = row_andnot(row_andnot(fu, sv[i]), xv[i]);
        if (!row_any(nw)) continue;
        row_atomic_or(X, v[i], nw);
        const unsigned b = 1u << (v[i] & 31);
        if (!(nb[i] & b)) atomicOr(&nzn[v[i] >> 5], b);
    }
}

__device__ void ms_top_down(const MsArgs &a, int s, const unsigned *F, unsigned *X, const unsigned *nzc,
                            unsigned *nzn) {
    MsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const uint64_t stream = policy_evict_first(), keep = policy_evict_last();
    const unsigned H = ld_volatile(&c->nheavy);
    // Light frontier vertices: a warp takes 32 bitmap words, spreads their
    // set bits over its lanes (one vertex each) and walks the vertices'
    // combined rows 32 entries per step, so one long row does not hold up
    // the warp.
    for (;;) {
        unsigned k0 = 0;
        if (lane == 0) k0 = atomicAdd(&c->wgrab[s], 32u);
        k0 = __shfl_sync(FULL, k0, 0);
        if (k0 >= a.nwords) break;
        const uint64_t k = (uint64_t)k0 + lane;
        unsigned bits = k < a.nwords ? ld_l1(&nzc[k]) : 0u;
        // Heavy positions [0, H) go by chunks below.
        if (k * 32 < H) bits &= (k * 32 + 32 <= H) ? 0u : ~0u << (H - k * 32);
        const unsigned cnt = __popc(bits);
        const unsigned incl = warp_incl_scan(cnt);
        const unsigned total = __shfl_sync(FULL, incl, 31);
        const unsigned excl = incl - cnt;
        for (unsigned r0 = 0; r0 < total; r0 += 32) {
            const unsigned idx = r0 + lane;
            const bool has = idx < total;
            const int j = warp_owner(excl, has ? idx : total - 1);
            const unsigned bj = __shfl_sync(FULL, bits, j);
            const unsigned exj = __shfl_sync(FULL, excl, j);
            uint64_t rb = 0;
            unsigned deg = 0;
            Row fu = row_zero();
            if (has) {
                const unsigned u = (k0 + j) * 32u + __fns(bj, 0, (int)(idx - exj + 1));
                rb = __ldg(&a.rp[u]);
                deg = (unsigned)(__ldg(&a.rp[u + 1]) - rb);
                fu = row_ld(F, u);
            }
            const unsigned dincl = warp_incl_scan(deg);
            const unsigned dtot = __shfl_sync(FULL, dincl, 31);
            const unsigned dex = dincl - deg;
            for (unsigned e0 = 0; e0 < dtot; e0 += 32) {
                const unsigned e = e0 + lane;
                const bool he = e < dtot;
                const int o = warp_owner(dex, he ? e : dtot - 1);
                const uint64_t rbo = __shfl_sync(FULL, rb, o);
                const unsigned exo = __shfl_sync(FULL, dex, o);
                const Row fo = row_bcast(fu, o);
                unsigned v[1] = {he ? ld_col(&a.cp[rbo + (e - exo)], stream) : 0u};
                bool ok[1] = {he && v[0] < a.n};
                if (he && !ok[0]) atomicOr(&c->res.error_flags, DEVERR_RANGE);
                ms_push<1>(a, X, nzn, v, ok, fo, keep);
            }
        }
    }
    // Heavy rows in the frontier: a warp tests 32 chunks at once and
    // expands the ones whose vertex is in the frontier, one at a time.
    const unsigned nch = ld_volatile(&c->nchunks);
    for (;;) {
        unsigned c0 = 0;
        if (lane == 0) c0 = atomicAdd(&c->cgrab[s], 32u);
        c0 = __shfl_sync(FULL, c0, 0);
        if (c0 >= nch) break;
        const unsigned mych = c0 + lane;
        unsigned myu = 0;
        bool hit = false;
        if (mych < nch) {
            myu = __ldg(&a.chunk_v[mych]);
            hit = (ld_l1(&nzc[myu >> 5]) >> (myu & 31)) & 1u;
        }
        unsigned hits = __ballot_sync(FULL, hit);
        while (hits) {
            const int src = __ffs(hits) - 1;
            hits &= hits - 1;
            const unsigned ch = c0 + src;
            const unsigned u = __shfl_sync(FULL, myu, src);
            const Row fu = row_ld(F, u);
            const uint64_t rb = __ldg(&a.rp[u]) + __ldg(&a.chunk_off[ch]);
            const uint64_t re = min(rb + MS_CHUNK, __ldg(&a.rp[u + 1]));
            for (uint64_t e = rb + lane; e < re; e += 64) {
                const bool two = e + 32 < re;
                unsigned v[2] = {ld_col(&a.cp[e], stream), two ? ld_col(&a.cp[e + 32], stream) : 0u};
                bool ok[2] = {v[0] < a.n, two && v[1] < a.n};
                if (!ok[0] || (two && !ok[1])) atomicOr(&c->res.error_flags, DEVERR_RANGE);
                ms_push<2>(a, X, nzn, v, ok, fu, keep);
            }
        }
    }
}

// Frontier row of neighbour u (zero when u is not in the frontier; with
// `check`, the bitmap is tested first so such rows are not read at all).
__device__ __forceinline__ Row ms_pull_row(const MsArgs &a, const unsigned *F, const unsigned *nzc, unsigned u,
                                           bool check, uint64_t keep) {
    if (u >= a.n) return row_zero();
    if (check && !((ld_l1(&nzc[u >> 5]) >> (u & 31)) & 1u)) return row_zero();
    return row_ld_hint(F, u, keep);
}

__device__ void ms_pull(const MsArgs &a, int s, const unsigned *F, unsigned *X, const unsigned *nzc, unsigned *nzn,
                        const unsigned *live_sh, bool check) {
    MsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const uint64_t stream = policy_evict_first(), keep = policy_evict_last();
    const Row live{make_uint4(live_sh[0], live_sh[1], live_sh[2], live_sh[3]),
                   make_uint4(live_sh[4], live_sh[5], live_sh[6], live_sh[7])};
    // Heavy rows first (the long jobs): a warp tests 32 chunks at once and
    // works through those whose vertex still misses a live root.
    const unsigned nch = ld_volatile(&c->nchunks);
    for (;;) {
        unsigned c0 = 0;
        if (lane == 0) c0 = atomicAdd(&c->cgrab[s], 32u);
        c0 = __shfl_sync(FULL, c0, 0);
        if (c0 >= nch) break;
        const unsigned mych = c0 + lane;
        unsigned myv = 0;
        bool want = false;
        if (mych < nch) {
            myv = __ldg(&a.chunk_v[mych]);
            want = row_any(row_andnot(live, row_ld_hint(a.seen, myv, keep)));
        }
        unsigned todo = __ballot_sync(FULL, want);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const unsigned ch = c0 + src;
            const unsigned v = __shfl_sync(FULL, myv, src);
            const Row miss = row_andnot(live, row_ld(a.seen, v));
            // Bits other chunks of v found already (X changes under our
            // feet: take lane 0's copy so the whole warp decides alike).
            const Row have = row_bcast(row_ld(X, v), 0);
            const Row need = row_andnot(miss, have);
            if (!row_any(need)) continue;
            const uint64_t rb = __ldg(&a.rp[v]) + __ldg(&a.chunk_off[ch]);
            const uint64_t re = min(rb + MS_CHUNK, __ldg(&a.rp[v + 1]));
            Row acc = row_zero();
            for (uint64_t e = rb + lane; e < re; e += 128) {
                unsigned u[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) u[t] = e + 32 * t < re ? ld_col(&a.cp[e + 32 * t], stream) : 0xffffffffu;
                const Row f0 = ms_pull_row(a, F, nzc, u[0], check, keep);
                const Row f1 = ms_pull_row(a, F, nzc, u[1], check, keep);
                const Row f2 = ms_pull_row(a, F, nzc, u[2], check, keep);
                const Row f3 = ms_pull_row(a, F, nzc, u[3], check, keep);
                row_or_into(acc, f0);
                row_or_into(acc, f1);
                row_or_into(acc, f2);
                row_or_into(acc, f3);
            }
            acc = row_warp_or(acc);
            const Row x = row_and(acc, need);
            if (row_any(x)) {
                if (lane < MS_W) {
                    const unsigned xw = row_word(x, (int)lane);
                    if (xw) atomicOr(&X[(uint64_t)v * MS_W + lane], xw);
                }
                if (lane == 0) atomicOr(&nzn[v >> 5], 1u << (v & 31));
            }
        }
    }
    // Light rows [H, H + L), one lane per vertex: 32 consecutive positions
    // have rows of about equal length.
    const unsigned H = ld_volatile(&c->nheavy), nl = ld_volatile(&c->nlight);
    for (;;) {
        unsigned i0 = 0;
        if (lane == 0) i0 = atomicAdd(&c->wgrab[s], 32u);
        i0 = __shfl_sync(FULL, i0, 0);
        if (i0 >= nl) break;
        if (i0 + lane >= nl) continue;
        const unsigned v = H + i0 + lane;
        const Row miss = row_andnot(live, row_ld(a.seen, v));
        if (!row_any(miss)) continue;
        const uint64_t rb = __ldg(&a.rp[v]), re = __ldg(&a.rp[v + 1]);
        Row acc = row_zero();
        for (uint64_t e = rb; e < re; e += 4) {
            unsigned u[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) u[t] = e + t < re ? ld_col(&a.cp[e + t], stream) : 0xffffffffu;
            const Row f0 = ms_pull_row(a, F, nzc, u[0], check, keep);
            const Row f1 = ms_pull_row(a, F, nzc, u[1], check, keep);
            const Row f2 = ms_pull_row(a, F, nzc, u[2], check, keep);
            const Row f3 = ms_pull_row(a, F, nzc, u[3], check, keep);
            row_or_into(acc, f0);
            row_or_into(acc, f1);
            row_or_into(acc, f2);
            row_or_into(acc, f3);
            if (!row_any(row_andnot(miss, acc))) break;  // every missing live root found
        }
        const Row x = row_and(acc, miss);
        if (row_any(x)) {
            row_st(X, v, x);
            atomicOr(&nzn[v >> 5], 1u << (v & 31));
        }
    }
}

// Folds the next frontier into seen and the depth planes, zeroes the
// consumed frontier, and counts the next frontier.  A warp reads 32 words
// of both bitmaps at once and visits only the non-empty ones.
__device__ void ms_update(const MsArgs &a, int level, unsigned *F, const unsigned *X, unsigned *nzc,
                          const unsigned *nzn) {
    MsCtl *c = a.ctl;
    const unsigned lane = lane_id();
    const int s1 = (level + 1) % 3;
    const unsigned d = (unsigned)level + 1;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned my_n = 0;
    unsigned long long my_m = 0, my_pairs = 0;
    Row my_live = row_zero();
    bool too_deep = false;
    for (uint64_t k0 = warp * 32; k0 < a.nwords; k0 += nwarps * 32) {
        const uint64_t kl = k0 + lane;
        const unsigned cbl = kl < a.nwords ? ld_l1(&nzc[kl]) : 0u;
        const unsigned nbl = kl < a.nwords ? __ldcg(&nzn[kl]) : 0u;
        unsigned todo = __ballot_sync(FULL, (cbl | nbl) != 0);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const unsigned cb = __shfl_sync(FULL, cbl, src);
            const unsigned nb = __shfl_sync(FULL, nbl, src);
            const uint64_t v = (k0 + src) * 32 + lane;
            if ((cb >> lane) & 1u) row_st(F, v, row_zero());
            if (!((nb >> lane) & 1u)) continue;
            const Row x = row_ld(X, v);
            Row sv = row_ld(a.seen, v);
            const bool first = !row_any(sv);
            if (first) atomicOr(&a.vis[v >> 5], 1u << (v & 31));
            row_or_into(sv, x);
            row_st(a.seen, v, sv);
            if ((int)d > a.max_depth) {
                too_deep = true;
            } else {
                for (int k = 0; k < a.bits; ++k) {
                    unsigned *pl = a.planes + (uint64_t)k * a.n * MS_W;
                    const bool on = (d >> k) & 1u;
                    if (first) {
                        row_st(pl, v, on ? x : row_zero());
                    } else if (on) {
                        Row r = row_ld(pl, v);
                        row_or_into(r, x);
                        row_st(pl, v, r);
                    }
                }
            }
            row_or_into(my_live, x);
            my_pairs += row_popc(x);
            ++my_n;
            my_m += __ldg(&a.rp[v + 1]) - __ldg(&a.rp[v]);
        }
    }
    my_n = warp_sum(my_n);
    my_m = warp_sum(my_m);
    my_pairs = warp_sum(my_pairs);
    my_live = row_warp_or(my_live);
    if (__any_sync(FULL, too_deep) && lane == 0) atomicOr(&c->res.error_flags, DEVERR_DEPTH);
    if (lane == 0 && my_n) {
        atomicAdd(&c->n_f[s1], my_n);
        atomicAdd(&c->m_f[s1], my_m);
        atomicAdd((unsigned long long *)&c->res.pairs_reached, my_pairs);
    }
    if (lane < MS_W && my_n) {
        const unsigned w = row_word(my_live, (int)lane);
        if (w) atomicOr(&c->live[s1][lane], w);
    }
}

__global__ void __launch_bounds__(MS_THREADS, 4) ms_persistent_kernel(MsArgs a) {
    MsCtl *c = a.ctl;
    unsigned epoch = 0;
    __shared__ unsigned s_live[MS_W];
    if (blockIdx.x == 0 && threadIdx.x == 0) c->t0 = globaltimer_ns();
    if (ld_volatile(&c->res.error_flags)) return;  // the seed found a bad root or an unprepared workspace
    int levels = 0, pull_levels = 0;
    unsigned long long fedges = 0;
    for (int level = 0;; ++level) {
        const int s = level % 3;
        const unsigned n_f = ld_volatile(&c->n_f[s]);
        const unsigned long long m_f = ld_volatile(&c->m_f[s]);
        if (n_f == 0) break;
        if (threadIdx.x < MS_W) s_live[threadIdx.x] = ld_volatile(&c->live[s][threadIdx.x]);
        __syncthreads();
        const int mode = a.mode == 1 ? MS_TOP_DOWN
                       : a.mode == 2 ? MS_PULL
                                     : ((double)m_f * a.alpha < (double)a.E ? MS_TOP_DOWN : MS_PULL);
        // The bitmap test pays when few entries lead into the frontier; when
        // most do (the dense middle levels) it only adds work.
        const bool check = a.check_frontier == 1 || (a.check_frontier == 0 && 2.0 * (double)m_f < (double)a.E);
        const unsigned *F = a.fr[level & 1];
        unsigned *X = a.fr[(level + 1) & 1];
        // Each level has a bitmap of its own, never written after its level
        // starts: its words can be read through L1 (ld_l1) safely.
        unsigned *nzc = a.nz + (uint64_t)level * a.nwords;
        unsigned *nzn = nzc + a.nwords;
        if (mode == MS_TOP_DOWN)
            ms_top_down(a, s, F, X, nzc, nzn);
        else
            ms_pull(a, s, F, X, nzc, nzn, s_live, check);
        if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const int s2 = (level + 2) % 3;
            c->wgrab[s2] = c->cgrab[s2] = c->n_f[s2] = 0;
            c->m_f[s2] = 0;
            for (int w = 0; w < MS_W; ++w) c->live[s2][w] = 0;
        }
        ms_update(a, level, (unsigned *)F, X, nzc, nzn);
        if (!grid_sync(&c->bar, &c->res.error_flags, epoch, a.nblocks, a.limit_ns)) return;
        ++levels;
        pull_levels += mode == MS_PULL;
        fedges += m_f;
        if (blockIdx.x == 0 && threadIdx.x == 0 && level < MS_TRACE) {
            c->t_level[level] = globaltimer_ns();
            c->n_level[level] = n_f;
            c->m_level[level] = m_f;
            c->mode_level[level] = (unsigned char)mode;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        c->res.levels = levels;
        c->res.pull_levels = pull_levels;
        c->res.frontier_edges = fedges;
        // Every frontier row and bitmap word was zeroed by the update that
        // consumed it, and the last level found nothing.
        if (!ld_volatile(&c->res.error_flags)) c->clean = MS_CLEAN;
    }
}

// ---------------------------------------------------------------- export --

__global__ void ms_export_one_kernel(const unsigned *__restrict__ seen, const unsigned *__restrict__ planes,
                                     const unsigned *__restrict__ pos, uint64_t n, int bits, unsigned i,
                                     int *__restrict__ depth) {
    const unsigned w = i >> 5, b = i & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint64_t p = __ldg(&pos[v]);
        int d = -1;
        if ((__ldg(&seen[p * MS_W + w]) >> b) & 1u) {
            d = 0;
            for (int k = 0; k < bits; ++k) d |= (int)((__ldg(&planes[((uint64_t)k * n + p) * MS_W + w]) >> b) & 1u) << k;
        }
        depth[v] = d;
    }
}

// All roots: a thread takes 4 consecutive vertices, reads their rows once
// and writes 4 bytes per root (a warp writes 128 contiguous bytes of each
// root's array).
// Word i of b = byte i of a0, a1, a2, a3 (a 4x4 byte transpose).
__device__ __forceinline__ void transpose_bytes4(unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b[4]) {
    const unsigned u0 = __byte_perm(a0, a1, 0x5140), u1 = __byte_perm(a0, a1, 0x7362);
    const unsigned u2 = __byte_perm(a2, a3, 0x5140), u3 = __byte_perm(a2, a3, 0x7362);
    b[0] = __byte_perm(u0, u2, 0x5410), b[1] = __byte_perm(u0, u2, 0x7632);
    b[2] = __byte_perm(u1, u3, 0x5410), b[3] = __byte_perm(u1, u3, 0x7632);
}
// Transpose of an 8x8 bit matrix stored one row per byte (bit j of byte i
// becomes bit i of byte j): the three-stage exchange of Hacker's Delight,
// section 7-3.
__device__ __forceinline__ uint64_t transpose_bits8x8(uint64_t x) {
    uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x ^= t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x ^= t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x ^= t ^ (t << 28);
    return x;
}
// Byte i = 0xFF where bit i of s8 is set, else 0.
__device__ __forceinline__ uint64_t byte_mask_of_bits(unsigned s8) {
    const uint64_t t = ((uint64_t)s8 * 0x0101010101010101ull) & 0x8040201008040201ull;
    return (((t + 0x7F7F7F7F7F7F7F7Full) & 0x8080808080808080ull) >> 7) * 0xFFull;
}

// Depths of every root as bytes, out[r * n + v] (255 = not reached).  A
// block takes EX_V vertices at a time.  First the vertex's seen row and its
// depth-plane rows are loaded whole (32-byte loads) into shared memory, laid
// out [row kind][word][vertex]; the block's two halves take alternate rows,
// so each thread has up to 5 loads in flight.  Then thread (w, q) turns word w
// (32 roots) of vertices 4q..4q+3 into 32 stores of 4 bytes, one per root, a
// warp's stores covering 128 consecutive bytes of one root's output.  The
// bit planes become depth bytes by byte permutes and 8x8 bit transposes
// (about 7 instructions per output byte).  Every row is read once.
constexpr int EX_V = 128;
static_assert(EX_V == 4 * 32, "a warp's 32 threads take the 128 vertices four each");

__global__ void __launch_bounds__(256, 2) ms_export_u8_kernel(const unsigned *__restrict__ seen,
                                                           const unsigned *__restrict__ planes,
                                                           const unsigned *__restrict__ pos, uint64_t n, int bits,
                                                           unsigned nroots, uint8_t *__restrict__ out) {
    __shared__ __align__(16) unsigned s_rows[9][MS_W][EX_V];  // seen, then up to 8 depth planes
    const unsigned t = threadIdx.x;
    const unsigned w = t >> 5, q = t & 31;
    const bool aligned = (n & 3) == 0 && ((uintptr_t)out & 3) == 0;
    for (uint64_t base = (uint64_t)blockIdx.x * EX_V; base < n; base += (uint64_t)gridDim.x * EX_V) {
        {  // the two halves of the block load alternate rows of the same vertex
            const unsigned vi = t & (EX_V - 1), half = t / EX_V;
            const uint64_t v = base + vi;
            const uint64_t p = v < n ? __ldg(&pos[v]) : 0;
            Row r[5];
#pragma unroll
            for (int i = 0; i < 5; ++i) {
                const int k = half + 2 * i;
                r[i] = row_zero();
                if (v < n && k <= bits) r[i] = row_ld(k == 0 ? seen : planes + (uint64_t)(k - 1) * n * MS_W, p);
            }
#pragma unroll
            for (int i = 0; i < 5; ++i) {
                const int k = half + 2 * i;
                if (k <= bits) {
#pragma unroll
                    for (int x = 0; x < MS_W; ++x) s_rows[k][x][vi] = row_word(r[i], x);
                }
            }
        }
        __syncthreads();
        if (w * 32 < nroots) {
            const uint4 S4 = *(const uint4 *)&s_rows[0][w][4 * q];
            const unsigned S[4] = {S4.x, S4.y, S4.z, S4.w};
            // L[j][g] = byte g of planes 0..3 of vertex j, H[j][g] of planes 4..7.
            unsigned L[4][4], H[4][4];
            {
                uint4 P[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    P[k] = k < bits ? *(const uint4 *)&s_rows[1 + k][w][4 * q] : make_uint4(0, 0, 0, 0);
                transpose_bytes4(P[0].x, P[1].x, P[2].x, P[3].x, L[0]);
                transpose_bytes4(P[0].y, P[1].y, P[2].y, P[3].y, L[1]);
                transpose_bytes4(P[0].z, P[1].z, P[2].z, P[3].z, L[2]);
                transpose_bytes4(P[0].w, P[1].w, P[2].w, P[3].w, L[3]);
            }
            if (bits > 4) {
                uint4 P[4];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    P[k] = 4 + k < bits ? *(const uint4 *)&s_rows[5 + k][w][4 * q] : make_uint4(0, 0, 0, 0);
                transpose_bytes4(P[0].x, P[1].x, P[2].x, P[3].x, H[0]);
                transpose_bytes4(P[0].y, P[1].y, P[2].y, P[3].y, H[1]);
                transpose_bytes4(P[0].z, P[1].z, P[2].z, P[3].z, H[2]);
                transpose_bytes4(P[0].w, P[1].w, P[2].w, P[3].w, H[3]);
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
#pragma unroll
                    for (int g = 0; g < 4; ++g) H[j][g] = 0;
            }
            const uint64_t v0 = base + 4 * q;
            const unsigned lim = min(32u, nroots - w * 32);
            const bool whole = aligned && v0 + 4 <= n;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                // D[j] byte i = depth of root 32w + 8g + i at vertex j.
                uint64_t D[4];
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    D[j] = transpose_bits8x8(((uint64_t)H[j][g] << 32) | L[j][g]) |
                           ~byte_mask_of_bits((S[j] >> (8 * g)) & 0xFFu);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    unsigned o[4];
                    transpose_bytes4((unsigned)(D[0] >> (32 * h)), (unsigned)(D[1] >> (32 * h)),
                                     (unsigned)(D[2] >> (32 * h)), (unsigned)(D[3] >> (32 * h)), o);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const unsigned b = 8 * g + 4 * h + i;
                        if (b >= lim) continue;
                        uint8_t *dst = out + (uint64_t)(w * 32 + b) * n + v0;
                        if (whole) {
                            *(unsigned *)dst = o[i];
                        } else {
                            for (unsigned j = 0; j < 4 && v0 + j < n; ++j) dst[j] = (uint8_t)(o[i] >> (8 * j));
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

static int ms_max_blocks(int *out) {
    static int cached[64] = {};
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if (!cached[di.device]) {
        if ((rc = persistent_kernel_setup((const void *)ms_persistent_kernel))) return rc;
        int per_sm = 0;
        G5_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ms_persistent_kernel, MS_THREADS, 0));
        cached[di.device] = std::max(1, per_sm) * di.sms;
    }
    *out = cached[di.device];
    return G5_OK;
}

static int ms_check(uint64_t nverts, uint64_t nentries, int *bits, const void *d_work, uint64_t work_bytes,
                    MsWork *w, const char *who) {
    G5_CHECK_ARG(nverts >= 1 && nverts < (1ull << 31), "%s: nverts outside [1, 2^31)", who);
    G5_CHECK_ARG(nentries < (1ull << 40), "%s: nentries too large", who);
    if (*bits == 0) *bits = MS_DEFAULT_BITS;
    G5_CHECK_ARG(*bits >= 1 && *bits <= 8, "%s: depth_bits %d outside [1, 8]", who, *bits);
    G5_CHECK_ARG(d_work, "%s: NULL workspace", who);
    *w = carve_ms((void *)d_work, nverts, nentries, *bits);
    if (work_bytes < w->bytes)
        return set_error(G5_ERR_WORKSPACE, "%s: workspace %llu < %llu bytes", who, (unsigned long long)work_bytes,
                         (unsigned long long)w->bytes);
    return G5_OK;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_msbfs_workspace_size(uint64_t nverts, uint64_t nentries, int depth_bits, uint64_t *bytes) {
    clear_error();
    G5_CHECK_ARG(bytes, "g5_msbfs_workspace_size: bytes is NULL");
    if (depth_bits == 0) depth_bits = MS_DEFAULT_BITS;
    G5_CHECK_ARG(depth_bits >= 1 && depth_bits <= 8, "g5_msbfs_workspace_size: depth_bits outside [1, 8]");
    *bytes = carve_ms(nullptr, nverts, nentries, depth_bits).bytes;
    return G5_OK;
}

extern "C" int g5_msbfs_prepare(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                uint64_t nentries, int depth_bits, void *d_work, uint64_t work_bytes, void *stream) {
    clear_error();
    MsWork w;
    int rc = ms_check(nverts, nentries, &depth_bits, d_work, work_bytes, &w, "g5_msbfs_prepare");
    if (rc) return rc;
    G5_CHECK_ARG(d_rowstarts && d_col, "g5_msbfs_prepare: NULL graph");
    cudaStream_t st = (cudaStream_t)stream;
    DeviceInfo di;
    if ((rc = device_info(&di))) return rc;
    G5_CUDA_TRY(cudaMemsetAsync(w.ctl, 0, sizeof(MsCtl), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.hist, 0, (MS_NKEYS + 1) * sizeof(unsigned), st));
    const int grid = di.sms * 8;
    ms_prep_hist_kernel<<<grid, 256, 0, st>>>(d_rowstarts, nverts, nentries, w.hist, w.ctl);
    ms_prep_scan_kernel<<<1, 32, 0, st>>>(w.hist, w.ctl);
    ms_prep_scatter_kernel<<<grid, 256, 0, st>>>(d_rowstarts, nverts, w.hist, w.pos, w.orig, w.tmp);
    G5_CUDA_TRY(cudaGetLastError());
    if ((rc = scan_u32_to_u64(w.tmp, nverts, w.rp, w.scan, st))) return rc;
    ms_prep_fill_kernel<<<grid, 256, 0, st>>>(d_rowstarts, d_col, nverts, w.pos, w.orig, w.rp, w.cp, w.ctl);
    ms_prep_chunks_kernel<<<grid, 256, 0, st>>>(w.rp, w.ctl, w.chunk_v, w.chunk_off, w.maxchunks);
    G5_CUDA_TRY(cudaGetLastError());
    MsCtl h;
    G5_CUDA_TRY(cudaMemcpyAsync(&h, w.ctl, sizeof h, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (h.res.error_flags) return deverr_to_status(h.res.error_flags, "g5_msbfs_prepare");
    const unsigned long long tag[2] = {MS_PREPARED, nverts};
    G5_CUDA_TRY(cudaMemcpyAsync(&w.ctl->prepared, tag, sizeof tag, cudaMemcpyHostToDevice, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return G5_OK;
}

extern "C" int g5_msbfs_run(uint64_t nverts, uint64_t nentries, int depth_bits, const uint64_t *h_roots,
                            uint32_t nroots, void *d_work, uint64_t work_bytes, const g5_msbfs_params *params,
                            g5_msbfs_stats *h_stats, void *stream) {
    clear_error();
    MsWork w;
    int rc = ms_check(nverts, nentries, &depth_bits, d_work, work_bytes, &w, "g5_msbfs_run");
    if (rc) return rc;
    G5_CHECK_ARG(h_roots, "g5_msbfs_run: NULL roots");
    G5_CHECK_ARG(nroots >= 1 && nroots <= MS_MAX_ROOTS, "g5_msbfs_run: nroots %u outside [1, 256]", nroots);
    for (uint32_t i = 0; i < nroots; ++i)
        G5_CHECK_ARG(h_roots[i] < nverts, "g5_msbfs_run: root %u = %llu outside [0, %llu)", i,
                     (unsigned long long)h_roots[i], (unsigned long long)nverts);
    g5_msbfs_params p = {MS_DEFAULT_ALPHA, 0, 0, 0};
    if (params) p = *params;
    if (p.alpha <= 0) p.alpha = MS_DEFAULT_ALPHA;
    G5_CHECK_ARG(p.mode >= 0 && p.mode <= 2 && p.check_frontier >= 0 && p.check_frontier <= 2,
                 "g5_msbfs_run: bad params");
    int max_blocks = 0;
    if ((rc = ms_max_blocks(&max_blocks))) return rc;
    const int blocks = p.blocks > 0 ? std::min(p.blocks, max_blocks) : max_blocks;
    cudaStream_t st = (cudaStream_t)stream;
    DeviceInfo di;
    if ((rc = device_info(&di))) return rc;

    MsArgs a;
    a.rp = w.rp;
    a.cp = w.cp;
    a.pos = w.pos;
    a.n = nverts;
    a.nwords = (nverts + 31) / 32;
    a.E = nentries;
    a.seen = w.seen;
    a.fr[0] = w.fr[0];
    a.fr[1] = w.fr[1];
    a.nz = w.nz;
    a.vis = w.vis;
    a.planes = w.planes;
    a.chunk_v = w.chunk_v;
    a.chunk_off = w.chunk_off;
    a.ctl = w.ctl;
    a.bits = depth_bits;
    a.max_depth = (1 << depth_bits) - 1;
    a.alpha = p.alpha;
    a.mode = p.mode;
    a.check_frontier = p.check_frontier;
    a.nblocks = (unsigned)blocks;
    a.limit_ns = wait_limit_ns();

    G5_CUDA_TRY(cudaMemcpyAsync(w.ctl->roots, h_roots, nroots * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    ms_reset_kernel<<<di.sms * 8, 256, 0, st>>>(w, nverts);
    ms_seed_kernel<<<1, MS_MAX_ROOTS, 0, st>>>(a, nroots);
    G5_CUDA_TRY(cudaGetLastError());
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(MS_THREADS);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    G5_CUDA_TRY(cudaLaunchKernelEx(&cfg, ms_persistent_kernel, a));
    if (!h_stats) return G5_OK;
    G5_CUDA_TRY(cudaMemcpyAsync(h_stats, &w.ctl->res, sizeof(g5_msbfs_stats), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(h_stats->error_flags, "g5_msbfs_run");
}

extern "C" int g5_msbfs_depths_u8(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint64_t nentries,
                                  int depth_bits, uint32_t nroots, uint8_t *d_out, void *stream) {
    clear_error();
    MsWork w;
    int rc = ms_check(nverts, nentries, &depth_bits, d_work, work_bytes, &w, "g5_msbfs_depths_u8");
    if (rc) return rc;
    G5_CHECK_ARG(d_out && nroots >= 1 && nroots <= MS_MAX_ROOTS, "g5_msbfs_depths_u8: bad argument");
    DeviceInfo di;
    if ((rc = device_info(&di))) return rc;
    ms_export_u8_kernel<<<di.sms * 2, 256, 0, (cudaStream_t)stream>>>(w.seen, w.planes, w.pos, nverts, depth_bits,
                                                                       nroots, d_out);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_msbfs_depth(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint64_t nentries,
                              int depth_bits, uint32_t root_index, int32_t *d_depth, void *stream) {
    clear_error();
    MsWork w;
    int rc = ms_check(nverts, nentries, &depth_bits, d_work, work_bytes, &w, "g5_msbfs_depth");
    if (rc) return rc;
    G5_CHECK_ARG(d_depth && root_index < MS_MAX_ROOTS, "g5_msbfs_depth: bad argument");
    DeviceInfo di;
    if ((rc = device_info(&di))) return rc;
    ms_export_one_kernel<<<di.sms * 8, 256, 0, (cudaStream_t)stream>>>(w.seen, w.planes, w.pos, nverts, depth_bits,
                                                                        root_index, d_depth);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_msbfs_last_stats(const void *d_work, uint64_t work_bytes, g5_msbfs_stats *stats, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && stats && work_bytes >= sizeof(MsCtl), "g5_msbfs_last_stats: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(stats, &((const MsCtl *)d_work)->res, sizeof *stats, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return deverr_to_status(stats->error_flags, "g5_msbfs_run");
}

extern "C" int g5_msbfs_last_trace(const void *d_work, uint64_t work_bytes, int max_levels, int32_t *mode,
                                   uint64_t *frontier_vertices, uint64_t *frontier_edges, double *level_ms,
                                   int32_t *nlevels, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_work && work_bytes >= sizeof(MsCtl) && nlevels, "g5_msbfs_last_trace: bad argument");
    MsCtl c;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemcpyAsync(&c, d_work, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    const int n = std::min(std::min(c.res.levels, MS_TRACE), std::max(max_levels, 0));
    unsigned long long prev = c.t0;
    for (int i = 0; i < n; ++i) {
        if (mode) mode[i] = c.mode_level[i];
        if (frontier_vertices) frontier_vertices[i] = c.n_level[i];
        if (frontier_edges) frontier_edges[i] = c.m_level[i];
        if (level_ms) level_ms[i] = (double)(c.t_level[i] - prev) * 1e-6;
        prev = c.t_level[i];
    }
    *nlevels = c.res.levels;
    return deverr_to_status(c.res.error_flags, "g5_msbfs_run");
}

extern "C" int g5_msbfs_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks) {
    clear_error();
    G5_CHECK_ARG(blocks && max_blocks, "g5_msbfs_grid: NULL argument");
    int mb = 0;
    int rc = ms_max_blocks(&mb);
    if (rc) return rc;
    *max_blocks = mb;
    // g5_msbfs_run launches every co-resident block by default; this is the
    // grid a caller sharing the device should pass in params.blocks.
    *blocks = (int)std::min<uint64_t>(mb, std::max<uint64_t>(1, nverts / 1024));
    return G5_OK;
}
