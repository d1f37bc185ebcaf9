// csr_sort.cu -- K2 canonical: the CSR with every row sorted by (neighbour,
// weight bits), built by radix partitioning instead of one scattered atomic
// fill (the reference's fill_csr_kernel, src/traversal.cu:48-73, leaves rows
// in atomic order).  Duplicates and their weights are kept unless the
// caller dedupes; self-loops are dropped as in the reference (:20-21).
//
//   partition  each block stages a tile of directed entries (u -> v and
//              v -> u of every edge) in shared memory by source partition
//              (the top 8 bits of the source's index range: 256
//              partitions) and writes each partition's run with one cursor
//              reservation, into a scratch array laid out like the CSR (a
//              partition's entries go exactly where its rows will be).
//   place      one partition at a time across the whole GPU: entries go to
//              their rows with per-row atomic cursors.  A partition's rows
//              span E/256 CSR entries (67 MB of column and weight at SCALE
//              26), so its scattered stores and cursors stay in L2 and reach
//              DRAM as whole lines.
//   sort       rows sorted by the 64-bit key (neighbour << 32 | weight
//              bits): up to 32 entries by a warp in registers (bitonic),
//              up to 4096 by a block in shared memory (bitonic), longer rows
//              cut into 4096-entry tiles spread over the whole grid: every
//              tile sorted in shared memory, then log2(tiles) merge passes,
//              each block producing one 4096-entry tile of output (merge
//              path), ping-ponging with the scratch array.  A hub row of
//              millions of entries thus takes the whole GPU, not one block.
//   dedupe     (optional) keeps the first entry of each run of equal
//              neighbours -- the lightest, rows being sorted -- into new
//              arrays with new row starts.
//   split      the SSSP copy of the CSR: each row stably partitioned into
//              entries below light/G5_TINY_DIV, the other light ones (below
//              light), and the heavy ones, with per-row counts (a warp per
//              row up to 4096 entries; longer rows tiled over the grid: per
//              tile class counts, a scan over tiles, then each tile writes
//              its entries at their final places).
//
// Algorithmic bytes per edge (two entries): partition reads 20 and writes
// 24, place reads 24 and writes 16 (+16 with the u64 column), sort reads and
// writes 16 per pass over the rows (one pass for rows up to 4096 entries).
#include <algorithm>

#include "g5_common.cuh"

namespace g5 {

constexpr int PART_BITS = 8;
constexpr int NPART = 1 << PART_BITS;
constexpr int P1_THREADS = 512;
constexpr int P1_EDGES = 4096;  // edges per tile: 8192 staged entries (96 KB of dynamic shared memory)
constexpr size_t P1_SMEM = (size_t)2 * P1_EDGES * (sizeof(unsigned long long) + sizeof(float));
constexpr int P1_PER_THREAD = P1_EDGES / P1_THREADS;
constexpr int SORT_THREADS = 256;
constexpr unsigned SORT_SMEM_KEYS = 4096;  // rows up to this length sort in shared memory

__host__ __device__ __forceinline__ int part_shift(uint64_t n) {
    int lg = 0;
    while ((1ull << lg) < n) ++lg;
    return lg > PART_BITS ? lg - PART_BITS : 0;
}

// Scratch: keys (u64) and weights of the partitioned entries, row cursors,
// partition cursors, the row lists by size class, error flags.
struct SortWork {
    unsigned long long *tkey;  // E: partitioned entries (src << 32 | dst), then sort ping-pong buffer
    float *tw;                 // E: their weights
    unsigned *rcur;            // N: per-row cursors (place), then dedupe degrees
    unsigned long long *pcur;  // NPART: partition cursors
    unsigned *mid, *big;       // N each: rows of 257..4096 and of more than 4096 entries
    unsigned *cnt;             // [0] mid rows, [1] big rows, [2] errors, [3] big rows (split), [4..5] max length
    // Big rows cut into 4096-entry tiles, spread over the whole grid: per
    // big row its tile count, then (tp) the exclusive prefix of the counts;
    // per tile two class counts and their prefixes (the SSSP split).
    unsigned *tcnt;            // T: per big row tiles, then per tile tiny counts
    unsigned *tcnt2;           // T: per tile light counts
    uint64_t *tp;              // N + 1: tile prefix over the big rows
    uint64_t *tq, *tq2;        // T + 1 each: prefixes of tcnt / tcnt2 over tiles
    uint64_t *scan;            // scan scratch
    uint64_t tmax;             // T: tiles the per-tile arrays hold
    uint64_t bytes;
};

constexpr unsigned BIG_TILE = 4096;  // entries of a big row per block step (chunk sort, merge, split)

// Tiles of all big rows: a row of L > BIG_TILE entries has at most
// L / BIG_TILE + 1, and there are at most e / (BIG_TILE + 1) such rows.
static uint64_t max_tiles(uint64_t n, uint64_t e) { return e / BIG_TILE + std::min(n, e / (BIG_TILE + 1)) + 1; }

static SortWork carve_sort(void *base, uint64_t n, uint64_t e) {
    Carver c(base);
    SortWork w;
    const uint64_t T = max_tiles(n, e);
    w.tmax = T;
    w.tkey = c.take<unsigned long long>(e ? e : 1);
    w.tw = c.take<float>(e ? e : 1);
    w.rcur = c.take<unsigned>(n + 1);
    w.pcur = c.take<unsigned long long>(NPART + 1);
    w.mid = c.take<unsigned>(n);
    w.big = c.take<unsigned>(n);
    w.cnt = c.take<unsigned>(64);
    w.tcnt = c.take<unsigned>(T);
    w.tcnt2 = c.take<unsigned>(T);
    w.tp = c.take<uint64_t>(n + 1);
    w.tq = c.take<uint64_t>(T + 1);
    w.tq2 = c.take<uint64_t>(T + 1);
    w.scan = c.take<uint64_t>(scan_scratch_words(T > n ? T : n));
    w.bytes = c.used;
    return w;
}

enum : unsigned {
    SORTERR_RANGE = 1u,     // an edge endpoint >= nverts
    SORTERR_COUNT = 2u,     // the edges differ from the ones counted
    SORTERR_WAIT = 4u,      // a radix look-back wait gave up
    SORTERR_ORDER = 8u,     // radix output out of order (the edges changed after counting)
    SORTERR_CAPACITY = 16u, // a radix list (gaps, long runs) would have overflowed
};

// ---------------------------------------------------------------- partition

__global__ void csr_part_init_kernel(const uint64_t *__restrict__ rowstarts, uint64_t n, int pshift,
                                     unsigned long long *__restrict__ pcur) {
    const unsigned p = threadIdx.x;
    if (p <= NPART) {
        const uint64_t v = min((uint64_t)p << pshift, n);
        pcur[p] = rowstarts[v];
    }
}

__global__ void __launch_bounds__(P1_THREADS) csr_partition_kernel(const ulonglong2 *__restrict__ edges,
                                                                   const float *__restrict__ weights, uint64_t m,
                                                                   uint64_t n, int pshift,
                                                                   const uint64_t *__restrict__ rowstarts,
                                                                   unsigned long long *__restrict__ pcur,
                                                                   unsigned long long *__restrict__ tkey,
                                                                   float *__restrict__ tw, unsigned *__restrict__ err) {
    extern __shared__ unsigned long long s_key[];  // 2 * P1_EDGES keys, then their weights
    float *s_w = reinterpret_cast<float *>(s_key + 2 * P1_EDGES);
    __shared__ unsigned s_cnt[NPART], s_off[NPART], s_wsum[NPART / 32], s_wbase[NPART / 32];
    __shared__ unsigned long long s_gbase[NPART], s_pend[NPART];
    __shared__ unsigned s_total;
    for (int p = threadIdx.x; p < NPART; p += blockDim.x) s_pend[p] = rowstarts[min((uint64_t)(p + 1) << pshift, n)];
    for (uint64_t tile = blockIdx.x; tile * P1_EDGES < m; tile += gridDim.x) {
        for (int p = threadIdx.x; p < NPART; p += blockDim.x) s_cnt[p] = 0;
        __syncthreads();
        unsigned long long ka[P1_PER_THREAD];
        float wv[P1_PER_THREAD];
        unsigned ra[P1_PER_THREAD], rb[P1_PER_THREAD];
        bool ok[P1_PER_THREAD];
#pragma unroll
        for (int k = 0; k < P1_PER_THREAD; ++k) {
            const uint64_t i = tile * P1_EDGES + (uint64_t)k * P1_THREADS + threadIdx.x;
            ok[k] = false;
            ka[k] = 0;
            wv[k] = 0.0f;
            if (i < m) {
                const ulonglong2 e = edges[i];
                if (e.x >= n || e.y >= n) {
                    atomicOr(err, SORTERR_RANGE);
                } else if (e.x != e.y) {
                    ok[k] = true;
                    ka[k] = (e.x << 32) | e.y;
                    wv[k] = weights[i];
                    ra[k] = atomicAdd(&s_cnt[e.x >> pshift], 1u);
                    rb[k] = atomicAdd(&s_cnt[e.y >> pshift], 1u);
                }
            }
        }
        __syncthreads();
        // Exclusive scan of the partition counts (256 = 8 warps x 32), and
        // one cursor reservation per partition that has entries in the tile.
        unsigned c = 0, incl = 0;
        if (threadIdx.x < NPART) {  // warps 0..7, whole warps
            c = s_cnt[threadIdx.x];
            incl = warp_incl_scan(c);
            if (lane_id() == 31) s_wsum[threadIdx.x >> 5] = incl;
            if (c) s_gbase[threadIdx.x] = atomicAdd(&pcur[threadIdx.x], (unsigned long long)c);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const unsigned ws = threadIdx.x < NPART / 32 ? s_wsum[threadIdx.x] : 0u;
            const unsigned wi = warp_incl_scan(ws);
            if (threadIdx.x < NPART / 32) s_wbase[threadIdx.x] = wi - ws;
            if (threadIdx.x == 31) s_total = wi;
        }
        __syncthreads();
        if (threadIdx.x < NPART) s_off[threadIdx.x] = s_wbase[threadIdx.x >> 5] + incl - c;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < P1_PER_THREAD; ++k) {
            if (!ok[k]) continue;
            const unsigned a = (unsigned)(ka[k] >> 32), b = (unsigned)ka[k];
            const unsigned ja = s_off[a >> pshift] + ra[k], jb = s_off[b >> pshift] + rb[k];
            s_key[ja] = ka[k];
            s_w[ja] = wv[k];
            s_key[jb] = ((unsigned long long)b << 32) | a;
            s_w[jb] = wv[k];
        }
        __syncthreads();
        const unsigned total = s_total;
        for (unsigned j = threadIdx.x; j < total; j += blockDim.x) {
            const unsigned long long key = s_key[j];
            const unsigned p = (unsigned)(key >> 32) >> pshift;
            const unsigned long long pos = s_gbase[p] + (j - s_off[p]);
            if (pos < s_pend[p]) {
                tkey[pos] = key;
                tw[pos] = s_w[j];
            } else {
                atomicOr(err, SORTERR_COUNT);  // the edges differ from the ones the rows were counted on
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------- place

// Entries of partition p (read from the partition cursors' start values,
// i.e. rowstarts of its first and last vertex) into their rows.
__global__ void csr_place_kernel(const unsigned long long *__restrict__ tkey, const float *__restrict__ tw,
                                 uint64_t n, int pshift, unsigned p, const uint64_t *__restrict__ rowstarts,
                                 unsigned *__restrict__ rcur, int *__restrict__ col, float *__restrict__ w,
                                 unsigned *__restrict__ err) {
    const uint64_t b = rowstarts[min((uint64_t)p << pshift, n)];
    const uint64_t e = rowstarts[min((uint64_t)(p + 1) << pshift, n)];
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = b + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e; i += T) {
        const unsigned long long key = __ldcs(&tkey[i]);
        const unsigned src = (unsigned)(key >> 32), dst = (unsigned)key;
        if (src >= n) {  // a slot the partition pass left unwritten (edges that do not match the counts)
            atomicOr(err, SORTERR_COUNT);
            continue;
        }
        const uint64_t pos = rowstarts[src] + atomicAdd(&rcur[src], 1u);
        if (pos >= rowstarts[src + 1]) {
            atomicOr(err, SORTERR_COUNT);
            continue;
        }
        col[pos] = (int)dst;
        w[pos] = __ldcs(&tw[i]);
    }
}

// ---------------------------------------------------------------- row sort

__device__ __forceinline__ unsigned long long row_key(const int *col, const float *w, uint64_t i) {
    return ((unsigned long long)(unsigned)col[i] << 32) | __float_as_uint(w[i]);
}

__device__ __forceinline__ void put_key(int *col, float *w, uint64_t *col64, uint64_t i, unsigned long long k) {
    col[i] = (int)(unsigned)(k >> 32);
    w[i] = __uint_as_float((unsigned)k);
    if (col64) col64[i] = k >> 32;
}

// Rows of 2..256 entries, one warp each: up to 32 entries bitonic in
// registers, 33..256 bitonic in the warp's shared-memory slice.  Longer rows
// are listed for the block kernels (mid: up to 4096 entries, big: more).
constexpr unsigned WARP_SMEM_KEYS = 256;

__global__ void __launch_bounds__(256) csr_sort_warp_kernel(const uint64_t *__restrict__ rowstarts, uint64_t n,
                                                            int *col, float *w, uint64_t *col64,
                                                            unsigned *__restrict__ mid, unsigned *__restrict__ big,
                                                            unsigned *__restrict__ cnt) {
    __shared__ unsigned long long s_rows[8][WARP_SMEM_KEYS];
    unsigned long long *sk = s_rows[threadIdx.x >> 5];
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; v0 < n; v0 += nw * 32) {
        // 32 rows per warp step: each lane reads one row's length and the
        // long rows are listed with one atomic per list and step.
        const uint64_t v = v0 + lane;
        const uint64_t len = v < n ? rowstarts[v + 1] - rowstarts[v] : 0;
        const bool is_mid = len > WARP_SMEM_KEYS && len <= SORT_SMEM_KEYS, is_big = len > SORT_SMEM_KEYS;
        const unsigned pm = warp_append(&cnt[0], is_mid);
        if (is_mid) mid[pm] = (unsigned)v;
        const unsigned pb = warp_append(&cnt[1], is_big);
        if (is_big) big[pb] = (unsigned)v;
        if (col64 && len == 1) col64[rowstarts[v]] = (uint64_t)(unsigned)col[rowstarts[v]];
        unsigned todo = __ballot_sync(FULL, len >= 2 && len <= WARP_SMEM_KEYS);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t r = v0 + l;
            const uint64_t rb = rowstarts[r];
            const unsigned rl = (unsigned)(rowstarts[r + 1] - rb);
            if (rl <= 32) {
                unsigned long long k = lane < rl ? row_key(col, w, rb + lane) : ~0ull;
#pragma unroll
                for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
                    for (int j = size >> 1; j > 0; j >>= 1) {
                        const unsigned long long o = __shfl_xor_sync(FULL, k, j);
                        const bool up = (lane & size) == 0, lower = (lane & j) == 0;
                        k = (lower == up) ? min(k, o) : max(k, o);
                    }
                }
                if (lane < rl) put_key(col, w, col64, rb + lane, k);
                continue;
            }
            unsigned P = 64;
            while (P < rl) P <<= 1;
            for (unsigned i = lane; i < P; i += 32) sk[i] = i < rl ? row_key(col, w, rb + i) : ~0ull;
            __syncwarp();
            for (unsigned size = 2; size <= P; size <<= 1) {
                for (unsigned j = size >> 1; j > 0; j >>= 1) {
                    for (unsigned t = lane; t < P / 2; t += 32) {
                        const unsigned i = 2 * t - (t & (j - 1)), q = i + j;
                        const unsigned long long a = sk[i], b = sk[q];
                        if ((a > b) == ((i & size) == 0)) {
                            sk[i] = b;
                            sk[q] = a;
                        }
                    }
                    __syncwarp();
                }
            }
            for (unsigned i = lane; i < rl; i += 32) put_key(col, w, col64, rb + i, sk[i]);
            __syncwarp();
        }
    }
}

// Bitonic sort of s[0 .. P) (P a power of two) by the whole block.
__device__ void block_bitonic(unsigned long long *s, unsigned P) {
    for (unsigned size = 2; size <= P; size <<= 1) {
        for (unsigned j = size >> 1; j > 0; j >>= 1) {
            for (unsigned t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const unsigned i = 2 * t - (t & (j - 1));
                const unsigned q = i + j;
                const bool up = (i & size) == 0;
                const unsigned long long a = s[i], b = s[q];
                if ((a > b) == up) {
                    s[i] = b;
                    s[q] = a;
                }
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ unsigned next_pow2(unsigned x) {
    unsigned p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Rows of 257..4096 entries: one block per row, in shared memory.
__global__ void __launch_bounds__(SORT_THREADS) csr_sort_mid_kernel(const uint64_t *__restrict__ rowstarts,
                                                                    const unsigned *__restrict__ mid,
                                                                    const unsigned *__restrict__ cnt, int *col,
                                                                    float *w, uint64_t *col64) {
    __shared__ unsigned long long s[SORT_SMEM_KEYS];
    const unsigned nrows = cnt[0];
    for (unsigned k = blockIdx.x; k < nrows; k += gridDim.x) {
        const unsigned v = mid[k];
        const uint64_t rb = rowstarts[v];
        const unsigned L = (unsigned)(rowstarts[v + 1] - rb);
        const unsigned P = next_pow2(L);
        for (unsigned i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < L ? row_key(col, w, rb + i) : ~0ull;
        __syncthreads();
        block_bitonic(s, P);
        for (unsigned i = threadIdx.x; i < L; i += blockDim.x) put_key(col, w, col64, rb + i, s[i]);
        __syncthreads();
    }
}


// Per big row its number of BIG_TILE tiles; the longest row's length.
__global__ void big_tiles_kernel(const uint64_t *__restrict__ rowstarts, const unsigned *__restrict__ big,
                                 unsigned nbig, unsigned *__restrict__ tcnt, unsigned long long *__restrict__ maxlen) {
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < nbig; k += gridDim.x * blockDim.x) {
        const uint64_t L = rowstarts[big[k] + 1] - rowstarts[big[k]];
        tcnt[k] = (unsigned)((L + BIG_TILE - 1) / BIG_TILE);
        atomicMax(maxlen, (unsigned long long)L);
    }
}

// Big row k of tile t: largest k with tp[k] <= t.
__device__ __forceinline__ unsigned tile_row(const uint64_t *tp, unsigned nbig, uint64_t t) {
    unsigned lo = 0, hi = nbig - 1;
    while (lo < hi) {
        const unsigned mid = (lo + hi + 1) >> 1;
        if (tp[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Sorts every BIG_TILE chunk of every big row in shared memory (one block
// per chunk, grid-stride over all chunks) into the scratch array.
__global__ void __launch_bounds__(SORT_THREADS) csr_sort_chunks_kernel(const uint64_t *__restrict__ rowstarts,
                                                                       const unsigned *__restrict__ big, unsigned nbig,
                                                                       const uint64_t *__restrict__ tp, uint64_t ntiles,
                                                                       unsigned long long *tkey, const int *col,
                                                                       const float *w) {
    __shared__ unsigned long long s[BIG_TILE];
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const unsigned k = tile_row(tp, nbig, t);
        const uint64_t rb = rowstarts[big[k]], L = rowstarts[big[k] + 1] - rb;
        const uint64_t c0 = (t - tp[k]) * BIG_TILE;
        const unsigned cl = L - c0 < BIG_TILE ? (unsigned)(L - c0) : BIG_TILE;
        const unsigned P = next_pow2(cl);
        for (unsigned i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < cl ? row_key(col, w, rb + c0 + i) : ~0ull;
        __syncthreads();
        block_bitonic(s, P);
        for (unsigned i = threadIdx.x; i < cl; i += blockDim.x) tkey[rb + c0 + i] = s[i];
        __syncthreads();
    }
}

// A key array in either form: the scratch array (u64) or col/w.
struct KeyBuf {
    unsigned long long *key;  // non-null: the scratch array
    int *col;
    float *w;
    __device__ __forceinline__ unsigned long long get(uint64_t i) const {
        return key ? key[i] : row_key(col, w, i);
    }
    __device__ __forceinline__ void set(uint64_t i, unsigned long long k) const {
        if (key) key[i] = k;
        else {
            col[i] = (int)(unsigned)(k >> 32);
            w[i] = __uint_as_float((unsigned)k);
        }
    }
};

// Elements of A taken among the first d outputs of merging A[0, la) and
// B[0, lb) (merge path; ties to A): the diagonal's crossing point.
template <class GetA, class GetB>
__device__ __forceinline__ uint64_t co_rank(uint64_t d, uint64_t la, uint64_t lb, GetA getA, GetB getB) {
    uint64_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
    while (lo < hi) {
        const uint64_t i = (lo + hi) >> 1;  // A[i] vs B[d - 1 - i]
        if (getA(i) <= getB(d - 1 - i)) lo = i + 1;
        else hi = i;
    }
    return lo;
}

// Merge passes a big row of L entries goes through: one per run length
// R = BIG_TILE * 2^i below L.  Pass 1 writes col/w from the scratch array,
// pass 2 the scratch array, and so on, so after its passes a row sits in
// col/w when their number is odd.
__device__ __forceinline__ int merge_passes(uint64_t L) {
    const uint64_t tiles = (L + BIG_TILE - 1) / BIG_TILE;
    int p = 0;
    while ((1ull << p) < tiles) ++p;
    return p;
}

// One merge pass over the big rows longer than R: sorted runs of R entries
// are merged pairwise (a last run without a partner is copied); shorter
// rows are sorted already and stay where they are.  Each block takes a
// tile of BIG_TILE outputs of some row: it finds where the tile's outputs
// start and end in the two runs (merge path on the row in memory), stages
// those input ranges in shared memory and merges them there, each thread
// placing 16 outputs after a merge-path search of its own in shared memory.
__global__ void __launch_bounds__(SORT_THREADS) csr_merge_pass_kernel(const uint64_t *__restrict__ rowstarts,
                                                                      const unsigned *__restrict__ big, unsigned nbig,
                                                                      const uint64_t *__restrict__ tp, uint64_t ntiles,
                                                                      uint64_t R, KeyBuf src, KeyBuf dst) {
    __shared__ unsigned long long s[BIG_TILE];
    __shared__ uint64_t s_i[2];
    constexpr unsigned PER = BIG_TILE / SORT_THREADS;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const unsigned k = tile_row(tp, nbig, t);
        const uint64_t rb = rowstarts[big[k]], L = rowstarts[big[k] + 1] - rb;
        if (L <= R) continue;  // the same t for the whole block
        const uint64_t o = (t - tp[k]) * BIG_TILE;
        const uint64_t a0 = o / (2 * R) * (2 * R);
        const uint64_t la = min(R, L - a0), b0 = a0 + la, lb = b0 < L ? min(R, L - b0) : 0;
        const uint64_t d0 = o - a0, d1 = min(d0 + BIG_TILE, la + lb);
        if (threadIdx.x < 2) {
            const uint64_t d = threadIdx.x ? d1 : d0;
            s_i[threadIdx.x] = co_rank(
                d, la, lb, [&](uint64_t i) { return src.get(rb + a0 + i); },
                [&](uint64_t j) { return src.get(rb + b0 + j); });
        }
        __syncthreads();
        const uint64_t i0 = s_i[0], i1 = s_i[1], j0 = d0 - i0, j1 = d1 - i1;
        const unsigned na = (unsigned)(i1 - i0), nb = (unsigned)(j1 - j0);
        for (unsigned q = threadIdx.x; q < na + nb; q += blockDim.x)
            s[q] = q < na ? src.get(rb + a0 + i0 + q) : src.get(rb + b0 + j0 + (q - na));
        __syncthreads();
        const unsigned q0 = threadIdx.x * PER;
        if (q0 < na + nb) {
            const unsigned long long *A = s, *B = s + na;
            unsigned i = (unsigned)co_rank(
                q0, na, nb, [&](uint64_t x) { return A[x]; }, [&](uint64_t y) { return B[y]; });
            unsigned j = q0 - i;
            const unsigned qe = min(q0 + PER, na + nb);
            for (unsigned q = q0; q < qe; ++q) {
                const bool takeA = j >= nb || (i < na && A[i] <= B[j]);
                dst.set(rb + a0 + d0 + q, takeA ? A[i++] : B[j++]);
            }
        }
        __syncthreads();
    }
}

// Big rows whose passes left them in the scratch array (an even number)
// back into col/w, and every big row into col64 when it is wanted.
__global__ void csr_big_finish_kernel(const uint64_t *__restrict__ rowstarts, const unsigned *__restrict__ big,
                                      unsigned nbig, const uint64_t *__restrict__ tp, uint64_t ntiles,
                                      const unsigned long long *__restrict__ tkey, int *col, float *w,
                                      uint64_t *col64) {
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const unsigned k = tile_row(tp, nbig, t);
        const uint64_t rb = rowstarts[big[k]], L = rowstarts[big[k] + 1] - rb;
        const bool from_scratch = merge_passes(L) % 2 == 0;
        if (!from_scratch && !col64) continue;
        const uint64_t c0 = (t - tp[k]) * BIG_TILE, c1 = min(c0 + BIG_TILE, L);
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
            const unsigned long long key = from_scratch ? tkey[rb + i] : row_key(col, w, rb + i);
            if (from_scratch) {
                col[rb + i] = (int)(unsigned)(key >> 32);
                w[rb + i] = __uint_as_float((unsigned)key);
            }
            if (col64) col64[rb + i] = key >> 32;
        }
    }
}

// ------------------------------------------------------------------ dedupe

// deg[v] = distinct neighbours of sorted row v (one warp per row).
__global__ void csr_unique_count_kernel(const uint64_t *__restrict__ rowstarts, const int *__restrict__ col,
                                        uint64_t n, unsigned *__restrict__ deg) {
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint64_t rb = rowstarts[v], re = rowstarts[v + 1];
        unsigned c = 0;
        for (uint64_t i = rb + lane; i < re; i += 32) c += i == rb || col[i] != col[i - 1];
        c = warp_sum(c);
        if (lane == 0) deg[v] = c;
    }
}

// The first entry of each run of equal neighbours into the new arrays.
__global__ void csr_unique_copy_kernel(const uint64_t *__restrict__ rowstarts, const int *__restrict__ col,
                                       const float *__restrict__ w, uint64_t n, const uint64_t *__restrict__ rs2,
                                       int *__restrict__ col2, float *__restrict__ w2, uint64_t *__restrict__ col64) {
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint64_t rb = rowstarts[v], re = rowstarts[v + 1];
        uint64_t out = rs2[v];
        for (uint64_t i0 = rb; i0 < re; i0 += 32) {
            const uint64_t i = i0 + lane;
            const bool first = i < re && (i == rb || col[i] != col[i - 1]);
            const unsigned m = __ballot_sync(FULL, first);
            if (first) {
                const uint64_t o = out + __popc(m & lanemask_lt());
                col2[o] = col[i];
                w2[o] = w[i];
                if (col64) col64[o] = (uint64_t)(unsigned)col[i];
            }
            out += __popc(m);
        }
    }
}

// ------------------------------------------------------- BFS degree order

// deg[v] = entries of row v (saturated at 2^32 - 1).
__global__ void row_lengths_kernel(const uint64_t *__restrict__ rowstarts, uint64_t n, unsigned *__restrict__ deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint64_t d = rowstarts[v + 1] - rowstarts[v];
        deg[v] = d > 0xffffffffull ? 0xffffffffu : (unsigned)d;
    }
}

// Sort keys of every entry: (~deg(neighbour), neighbour) in the (col, w)
// slots the row sort orders by, so sorted rows list their neighbours by
// decreasing degree, ties by index.
__global__ void degree_keys_kernel(const int *__restrict__ col, uint64_t e, const unsigned *__restrict__ deg,
                                   uint64_t n, int *__restrict__ ka, float *__restrict__ kb,
                                   unsigned *__restrict__ err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < e; i += stride) {
        const unsigned v = (unsigned)__ldg(&col[i]);
        if (v >= n) atomicOr(err, SORTERR_RANGE);
        ka[i] = (int)(0xffffffffu - (v < n ? __ldg(&deg[v]) : 0u));
        kb[i] = __uint_as_float(v);
    }
}

// --------------------------------------------------- SSSP vertex numbering

// Sort keys of the vertex order: (~degree, index) in the (col, w) slots of
// one row of n entries.
__global__ void vertex_order_keys_kernel(const unsigned *__restrict__ deg, uint64_t n, int *__restrict__ ka,
                                         float *__restrict__ kb) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        ka[v] = (int)(0xffffffffu - __ldg(&deg[v]));
        kb[v] = __uint_as_float((unsigned)v);
    }
}

// perm[inv[i]] = i, and the new rows' lengths.
__global__ void vertex_perm_kernel(const unsigned *__restrict__ inv, const unsigned *__restrict__ deg, uint64_t n,
                                   unsigned *__restrict__ perm, unsigned *__restrict__ len2) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned o = __ldg(&inv[i]);
        perm[o] = (unsigned)i;
        len2[i] = __ldg(&deg[o]);
    }
}

// Row i of the renumbered copy = row inv[i] of the source, in the same
// order, its neighbours renamed by perm.  Rows of at most RENUM_LONG entries
// take a warp each; the longer ones -- a prefix of the new order, which is
// by decreasing length -- a block each (renumber_long_rows_kernel).
constexpr unsigned RENUM_LONG = 2048;

template <int STEP>
__device__ __forceinline__ void renumber_copy(const int *__restrict__ col, const float *__restrict__ w, uint64_t b,
                                              uint64_t len, uint64_t b2, uint64_t n, const unsigned *__restrict__ perm,
                                              int *__restrict__ col2, float *__restrict__ w2, unsigned *err,
                                              unsigned t) {
    for (uint64_t k = t; k < len; k += STEP) {
        const unsigned v = (unsigned)__ldg(&col[b + k]);
        if (v >= n) {
            atomicOr(err, SORTERR_RANGE);
            col2[b2 + k] = (int)v;  // kept out of range: the search reports it
        } else {
            col2[b2 + k] = (int)__ldg(&perm[v]);
        }
        w2[b2 + k] = __ldg(&w[b + k]);
    }
}

__global__ void renumber_rows_kernel(const uint64_t *__restrict__ rs, const int *__restrict__ col,
                                     const float *__restrict__ w, const unsigned *__restrict__ light,
                                     const unsigned *__restrict__ tiny, uint64_t n, const unsigned *__restrict__ perm,
                                     const unsigned *__restrict__ inv, const uint64_t *__restrict__ rs2,
                                     int *__restrict__ col2, float *__restrict__ w2, unsigned *__restrict__ light2,
                                     unsigned *__restrict__ tiny2, unsigned *__restrict__ err) {
    // 32 consecutive new rows per warp step (similar lengths: the new order
    // is by decreasing length).  A row of up to 32 entries is copied by its
    // own lane, longer ones up to RENUM_LONG by the whole warp.
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; i0 < n; i0 += nw * 32) {
        const uint64_t i = i0 + lane;
        uint64_t b = 0, len = 0, b2 = 0;
        if (i < n) {
            const unsigned o = __ldg(&inv[i]);
            b = __ldg(&rs[o]);
            len = __ldg(&rs[o + 1]) - b;
            b2 = __ldg(&rs2[i]);
            light2[i] = __ldg(&light[o]);
            tiny2[i] = __ldg(&tiny[o]);
            if (len <= 32) renumber_copy<1>(col, w, b, len, b2, n, perm, col2, w2, err, 0);
        }
        unsigned todo = __ballot_sync(FULL, len > 32 && len <= RENUM_LONG);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            renumber_copy<32>(col, w, __shfl_sync(FULL, b, l), __shfl_sync(FULL, len, l), __shfl_sync(FULL, b2, l), n,
                              perm, col2, w2, err, lane);
        }
    }
}

__global__ void renumber_long_rows_kernel(const uint64_t *__restrict__ rs, const int *__restrict__ col,
                                          const float *__restrict__ w, uint64_t n, const unsigned *__restrict__ perm,
                                          const unsigned *__restrict__ inv, const uint64_t *__restrict__ rs2,
                                          int *__restrict__ col2, float *__restrict__ w2, unsigned *__restrict__ err) {
    for (uint64_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint64_t b2 = __ldg(&rs2[i]), len = __ldg(&rs2[i + 1]) - b2;
        if (len <= RENUM_LONG) break;  // the rest of the new order is shorter still (block-uniform)
        const uint64_t b = __ldg(&rs[__ldg(&inv[i])]);
        renumber_copy<256>(col, w, b, len, b2, n, perm, col2, w2, err, threadIdx.x);
    }
}

// ------------------------------------------------------------- SSSP split

// Stable three-way partition of a row into tiny (w < tiny), other light
// (w < light) and heavy entries, with the row's light and tiny counts.  The
// warp version takes rows of up to 4096 entries (one warp each); longer
// rows, listed, take a block each.
__device__ __forceinline__ int light_class(float x, float light, float tiny) {
    return x < tiny ? 0 : x < light ? 1 : 2;
}

__global__ void csr_split_light_kernel(const uint64_t *__restrict__ rowstarts, const int *__restrict__ col,
                                       const float *__restrict__ w, uint64_t n, float light, float tiny,
                                       int *__restrict__ scol, float *__restrict__ sw, unsigned *__restrict__ ld,
                                       unsigned *__restrict__ td, unsigned *__restrict__ big,
                                       unsigned *__restrict__ nbig) {
    const unsigned lane = lane_id();
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; v0 < n; v0 += nw * 32) {
        // 32 rows per warp step (coalesced row starts): a row of up to 32
        // entries is split by its own lane (most rows of a Kronecker graph
        // are short: a warp each left most lanes idle), longer ones by the
        // whole warp, rows beyond SORT_SMEM_KEYS listed for the tiled kernels.
        const uint64_t v = v0 + lane;
        const uint64_t rb = v < n ? rowstarts[v] : 0, re = v < n ? rowstarts[v + 1] : 0;
        const uint64_t len = re - rb;
        if (len > SORT_SMEM_KEYS) big[atomicAdd(nbig, 1u)] = (unsigned)v;
        if (v < n && len <= 32) {
            unsigned nt = 0, nl = 0;
            for (uint64_t i = rb; i < re; ++i) {
                const int k = light_class(w[i], light, tiny);
                nt += k == 0;
                nl += k <= 1;
            }
            uint64_t o0 = rb, o1 = rb + nt, o2 = rb + nl;
            for (uint64_t i = rb; i < re; ++i) {
                const float x = w[i];
                const int k = light_class(x, light, tiny);
                const uint64_t o = k == 0 ? o0++ : k == 1 ? o1++ : o2++;
                scol[o] = col[i];
                sw[o] = x;
            }
            ld[v] = nl;
            td[v] = nt;
        }
        unsigned todo = __ballot_sync(FULL, len > 32 && len <= SORT_SMEM_KEYS);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t r = v0 + l;
            const uint64_t b = __shfl_sync(FULL, rb, l), e = __shfl_sync(FULL, re, l);
            unsigned nt = 0, nl = 0;
            for (uint64_t i = b + lane; i < e; i += 32) {
                const int k = light_class(w[i], light, tiny);
                nt += k == 0;
                nl += k <= 1;
            }
            nt = warp_sum(nt);
            nl = warp_sum(nl);
            uint64_t o3[3] = {b, b + nt, b + nl};
            for (uint64_t i0 = b; i0 < e; i0 += 32) {
                const uint64_t i = i0 + lane;
                const bool has = i < e;
                const float x = has ? w[i] : 0.0f;
                const int k = has ? light_class(x, light, tiny) : 3;
                const unsigned lt = lanemask_lt();
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const unsigned m = __ballot_sync(FULL, k == q);
                    if (k == q) {
                        const uint64_t o = o3[q] + __popc(m & lt);
                        scol[o] = col[i];
                        sw[o] = x;
                    }
                    o3[q] += __popc(m);
                }
            }
            if (lane == 0) {
                ld[r] = nl;
                td[r] = nt;
            }
        }
    }
}

// Big rows of the split, tiled as for the sort: per tile its tiny and light
// entry counts (one block per tile) ...
__global__ void __launch_bounds__(SORT_THREADS) csr_split_count_kernel(
    const uint64_t *__restrict__ rowstarts, const float *__restrict__ w, const unsigned *__restrict__ big,
    unsigned nbig, const uint64_t *__restrict__ tp, uint64_t ntiles, float light, float tiny,
    unsigned *__restrict__ ct, unsigned *__restrict__ cl) {
    __shared__ unsigned s_t, s_l;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (threadIdx.x == 0) s_t = s_l = 0;
        __syncthreads();
        const unsigned k = tile_row(tp, nbig, t);
        const uint64_t rb = rowstarts[big[k]], L = rowstarts[big[k] + 1] - rb;
        const uint64_t c0 = (t - tp[k]) * BIG_TILE, c1 = min(c0 + BIG_TILE, L);
        unsigned nt = 0, nl = 0;
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
            const int c = light_class(w[rb + i], light, tiny);
            nt += c == 0;
            nl += c <= 1;
        }
        nt = warp_sum(nt);
        nl = warp_sum(nl);
        if (lane_id() == 0) {
            atomicAdd(&s_t, nt);
            atomicAdd(&s_l, nl);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            ct[t] = s_t;
            cl[t] = s_l;
        }
        __syncthreads();
    }
}

// ... then, with those counts scanned over all tiles (qt, ql), every tile
// writes its entries of each class in order: tiny ones after the row's
// earlier tiny ones, the other light ones after all the row's tiny ones,
// heavy ones after all its light ones.  The block of a row's first tile also
// writes the row's counts.
__global__ void __launch_bounds__(SORT_THREADS) csr_split_write_kernel(
    const uint64_t *__restrict__ rowstarts, const int *__restrict__ col, const float *__restrict__ w,
    const unsigned *__restrict__ big, unsigned nbig, const uint64_t *__restrict__ tp, uint64_t ntiles, float light,
    float tiny, const uint64_t *__restrict__ qt, const uint64_t *__restrict__ ql, int *__restrict__ scol,
    float *__restrict__ sw, unsigned *__restrict__ ld, unsigned *__restrict__ td) {
    constexpr int WARPS = SORT_THREADS / 32;
    __shared__ unsigned s_cnt[3][WARPS];
    __shared__ unsigned long long s_base[3];
    const unsigned lane = lane_id(), wid = threadIdx.x >> 5;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const unsigned k = tile_row(tp, nbig, t);
        const unsigned v = big[k];
        const uint64_t rb = rowstarts[v], L = rowstarts[v + 1] - rb;
        const uint64_t f = tp[k], l = tp[k + 1];  // the row's tiles [f, l)
        const uint64_t c0 = (t - f) * BIG_TILE, c1 = min(c0 + BIG_TILE, L);
        const uint64_t T_row = qt[l] - qt[f], L_row = ql[l] - ql[f];
        const uint64_t t_before = qt[t] - qt[f], l_before = ql[t] - ql[f];
        if (threadIdx.x == 0) {
            s_base[0] = rb + t_before;
            s_base[1] = rb + T_row + (l_before - t_before);
            s_base[2] = rb + L_row + (c0 - l_before);
            if (t == f) {
                ld[v] = (unsigned)L_row;
                td[v] = (unsigned)T_row;
            }
        }
        __syncthreads();
        for (uint64_t i0 = c0; i0 < c1; i0 += blockDim.x) {
            const uint64_t i = i0 + threadIdx.x;
            const bool has = i < c1;
            const float x = has ? w[rb + i] : 0.0f;
            const int c = has ? light_class(x, light, tiny) : 3;
            unsigned m[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                m[q] = __ballot_sync(FULL, c == q);
                if (lane == 0) s_cnt[q][wid] = __popc(m[q]);
            }
            __syncthreads();
            if (has) {
                uint64_t o = s_base[c];
                for (unsigned q = 0; q < wid; ++q) o += s_cnt[c][q];
                o += __popc(m[c] & lanemask_lt());
                scol[o] = col[rb + i];
                sw[o] = x;
            }
            __syncthreads();
            if (threadIdx.x < 3) {
                unsigned long long sum = 0;
                for (int q = 0; q < WARPS; ++q) sum += s_cnt[threadIdx.x][q];
                s_base[threadIdx.x] += sum;
            }
            __syncthreads();
        }
    }
}


// ------------------------------------------------------------ radix build
//
// The canonical CSR as one LSD radix sort of every directed entry by the key
// (src << lg | dst), lg = bits of a vertex index, 8 bits a pass
// (ceil(2 lg / 8) passes: 7 at SCALE 26).  Each pass is one "one-sweep"
// kernel: a block takes the next tile of 4096 entries (tile numbers handed
// out in launch order by an atomic counter, so every earlier tile is held by
// a running block), ranks it by digit in shared memory (warp match plus
// per-warp digit counters: stable), publishes the tile's digit counts, adds
// up the preceding tiles' published counts for its global offsets
// (decoupled look-back with a bounded wait) and writes each digit's run of
// the tile with consecutive stores.  The first pass reads the edge list
// (both directions of each non-loop edge); every pass's digit totals come
// from one counting pass over the edges before it, which also gives the
// entry count before the caller allocates the CSR.  A finish pass writes
// col / w / row starts from the sorted keys and orders each run of equal
// (src, dst) by weight bits: runs of up to 32 by one thread, longer ones
// listed and sorted by the row-sort kernels.
//
// HBM bytes per entry: the counting pass reads 8 (16 per edge), the first
// pass 10 and writes 12, each further pass reads and writes 12, the finish
// reads 12 and writes 8 (16 with the u64 column).

constexpr int RX_BITS = 8;
constexpr int RX_BINS = 1 << RX_BITS;
constexpr int RX_THREADS = 256;  // one thread per digit in the look-back
constexpr int RX_WARPS = RX_THREADS / 32;
#ifndef G5_RX_ITEMS
#define G5_RX_ITEMS 16  // entries a thread takes per tile (even: the first pass takes both directions of ITEMS / 2 edges)
#endif
#ifndef G5_RX_MIN_BLOCKS
#define G5_RX_MIN_BLOCKS 3  // 3 blocks of 256 threads an SM (a few spilled registers; 2 blocks: 18 % slower)
#endif
#ifndef G5_RX_LOOKBACK
#define G5_RX_LOOKBACK 4  // predecessor tiles a look-back step reads at once (8 and 16: slower at SCALE 26)
#endif
constexpr int RX_ITEMS = G5_RX_ITEMS;
constexpr int RX_LOOKBACK = G5_RX_LOOKBACK;
constexpr int RX_TILE = RX_THREADS * RX_ITEMS;  // 4096 entries
constexpr int RX_EDGE_TILE = RX_TILE / 2;       // first pass: 2048 edges, both directions
static_assert(RX_ITEMS % 2 == 0 && RX_ITEMS <= 32, "items: even, at most the valid mask's 32 bits");
constexpr int RX_MAXPASS = 8;                   // 2 lg <= 62 bits
constexpr size_t RX_SMEM = (size_t)RX_TILE * (sizeof(unsigned long long) + sizeof(unsigned));
constexpr unsigned RX_RUN_INLINE = 32;  // duplicate runs up to this long are sorted by one thread
constexpr uint64_t RX_GAP_INLINE = 64;  // empty-row gaps up to this long are filled by one thread

// Look-back status word of (tile, digit): pass epoch (8 bits), flag
// (1 = the tile's own count, 2 = inclusive prefix over tiles 0..t), count.
constexpr int RX_EPOCH_SHIFT = 56, RX_FLAG_SHIFT = 54;
constexpr unsigned long long RX_COUNT_MASK = (1ull << RX_FLAG_SHIFT) - 1;
constexpr unsigned long long RX_AGG = 1, RX_PREFIX = 2;

enum : unsigned { RXC_ERR = 0, RXC_RUNS = 1, RXC_GAPS = 2, RXC_TILES = 8 };  // RadixWork::cnt slots

struct RadixWork {
    unsigned long long *hist;   // RX_MAXPASS x RX_BINS: digit totals per pass
    unsigned long long *base;   // RX_MAXPASS x RX_BINS: their exclusive prefixes
    unsigned long long *total;  // [0] entries counted, [1] edges counted over
    unsigned *cnt;              // 64 counters (RXC_*)
    unsigned *scnt;             // 64: the row sort's list counts ([0] mid runs, [1] big runs, [4..5] longest)
    uint64_t *gaps;             // 3 x gcap: empty-row gaps (first row, end row, start value)
    uint64_t gcap;
    uint64_t *runs;             // 2 x rcap: long duplicate runs as [start, end) "rows" for the row sort
    unsigned *rmid, *rbig;      // rcap each: run numbers 2k by length class
    uint64_t rcap;
    unsigned long long *status; // tmax x RX_BINS
    uint64_t tmax;
    unsigned long long *ka, *kb;  // entry keys, ping-pong (emax each)
    unsigned *va, *vb;            // their weight bits
    uint64_t region;              // bytes from ka to the end (the long-run sort's scratch)
    uint64_t bytes;
};

static int vertex_bits(uint64_t n) {
    int lg = 0;
    while ((1ull << lg) < n) ++lg;
    return lg;
}

static RadixWork carve_radix(void *base, uint64_t n, uint64_t m) {
    Carver c(base);
    RadixWork w;
    const uint64_t emax = 2 * m;
    w.hist = c.take<unsigned long long>(RX_MAXPASS * RX_BINS);
    w.base = c.take<unsigned long long>(RX_MAXPASS * RX_BINS);
    w.total = c.take<unsigned long long>(2);
    w.cnt = c.take<unsigned>(64);
    w.scnt = c.take<unsigned>(64);
    w.gcap = (n + 1) / (RX_GAP_INLINE + 1) + 2;
    w.gaps = c.take<uint64_t>(3 * w.gcap);
    w.rcap = emax / (RX_RUN_INLINE + 1) + 1;
    w.runs = c.take<uint64_t>(2 * w.rcap);
    w.rmid = c.take<unsigned>(w.rcap);
    w.rbig = c.take<unsigned>(w.rcap);
    w.tmax = (m + RX_EDGE_TILE - 1) / RX_EDGE_TILE + 1;
    w.status = c.take<unsigned long long>(w.tmax * RX_BINS);
    const uint64_t before = align_up(c.used, 256);
    w.ka = c.take<unsigned long long>(emax ? emax : 1);
    w.kb = c.take<unsigned long long>(emax ? emax : 1);
    w.va = c.take<unsigned>(emax ? emax : 1);
    w.vb = c.take<unsigned>(emax ? emax : 1);
    w.region = c.used - before;
    w.bytes = c.used;
    return w;
}

// Digit totals of every pass over both directions of every non-loop edge.
__global__ void __launch_bounds__(256) csr_radix_hist_kernel(const ulonglong2 *__restrict__ edges, uint64_t m,
                                                             uint64_t n, int lg, int passes,
                                                             unsigned long long *__restrict__ hist,
                                                             unsigned *__restrict__ err) {
    __shared__ unsigned s_h[RX_MAXPASS * RX_BINS];
    for (int i = threadIdx.x; i < passes * RX_BINS; i += blockDim.x) s_h[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const ulonglong2 e = __ldcs(&edges[i]);
        if (e.x >= n || e.y >= n) {
            atomicOr(err, SORTERR_RANGE);
            continue;
        }
        if (e.x == e.y) continue;
        const unsigned long long k1 = (e.x << lg) | e.y, k2 = (e.y << lg) | e.x;
        for (int p = 0; p < passes; ++p) {
            atomicAdd(&s_h[p * RX_BINS + ((k1 >> (RX_BITS * p)) & (RX_BINS - 1))], 1u);
            atomicAdd(&s_h[p * RX_BINS + ((k2 >> (RX_BITS * p)) & (RX_BINS - 1))], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RX_BINS; i += blockDim.x)
        if (s_h[i]) atomicAdd(&hist[i], (unsigned long long)s_h[i]);
}

// base[p][d] = exclusive prefix of hist[p][*]; total[0] = entries.  One block
// of RX_BINS threads.
__global__ void csr_radix_scan_kernel(const unsigned long long *__restrict__ hist, int passes,
                                      unsigned long long *__restrict__ base, unsigned long long *__restrict__ total) {
    __shared__ unsigned long long s_ws[RX_WARPS];
    const unsigned d = threadIdx.x, lane = lane_id(), wid = d >> 5;
    for (int p = 0; p < passes; ++p) {
        const unsigned long long x = hist[p * RX_BINS + d];
        const unsigned long long incl = warp_incl_scan(x);
        if (lane == 31) s_ws[wid] = incl;
        __syncthreads();
        unsigned long long wb = 0, all = 0;
        for (int q = 0; q < RX_WARPS; ++q) {
            if (q < (int)wid) wb += s_ws[q];
            all += s_ws[q];
        }
        base[p * RX_BINS + d] = wb + incl - x;
        if (p == 0 && d == 0) total[0] = all;
        __syncthreads();
    }
}

struct RxPass {
    const ulonglong2 *edges;  // first pass: the edge list and its weights
    const float *weights;
    uint64_t m;
    const unsigned long long *kin;  // later passes: the previous pass's output
    const unsigned *vin;
    unsigned long long *kout;
    unsigned *vout;
    uint64_t n, E, ntiles;
    int lg, shift;
    unsigned long long epoch;
    const unsigned long long *base, *hist;  // this pass's digit starts and totals
    unsigned long long *status;
    unsigned *tilectr, *err;
    unsigned long long limit_ns;
};

__device__ __forceinline__ void st_status(unsigned long long *p, unsigned long long x) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(x) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

template <bool FIRST>
__global__ void __launch_bounds__(RX_THREADS, G5_RX_MIN_BLOCKS) csr_radix_pass_kernel(RxPass a) {
    extern __shared__ unsigned long long s_key[];  // RX_TILE keys, then their values
    unsigned *s_val = reinterpret_cast<unsigned *>(s_key + RX_TILE);
    __shared__ unsigned s_wcnt[RX_WARPS][RX_BINS];
    __shared__ unsigned s_wsum[RX_WARPS];
    __shared__ unsigned long long s_gdelta[RX_BINS];
    __shared__ unsigned s_tile, s_total;
    const unsigned tid = threadIdx.x, lane = lane_id(), wid = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(a.tilectr, 1u);
    for (int i = tid; i < RX_WARPS * RX_BINS; i += RX_THREADS) (&s_wcnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= a.ntiles) return;  // block-uniform (the grid has ntiles blocks)

    // The tile's items, warp-striped (item k of lane l of warp w is entry
    // w * 512 + k * 32 + l of the tile): coalesced loads, and that order is
    // the ranking's, which keeps the pass stable.
    unsigned long long key[RX_ITEMS];
    unsigned val[RX_ITEMS];
    unsigned valid = 0;
    if (FIRST) {
        const uint64_t e0 = tile * RX_EDGE_TILE + wid * (RX_EDGE_TILE / RX_WARPS) + lane;
#pragma unroll
        for (int k = 0; k < RX_ITEMS / 2; ++k) {
            const uint64_t i = e0 + (uint64_t)k * 32;
            unsigned long long u = 0, v = 0;
            unsigned wb = 0;
            if (i < a.m) {
                const ulonglong2 e = __ldcs(&a.edges[i]);
                u = e.x;
                v = e.y;
                if (u >= a.n || v >= a.n) {
                    atomicOr(a.err, SORTERR_RANGE);
                } else if (u != v) {
                    valid |= 1u << k | 1u << (k + RX_ITEMS / 2);
                    wb = __float_as_uint(__ldcs(&a.weights[i]));
                }
            }
            key[k] = (u << a.lg) | v;
            key[k + RX_ITEMS / 2] = (v << a.lg) | u;
            val[k] = val[k + RX_ITEMS / 2] = wb;
        }
    } else {
        const uint64_t p0 = tile * RX_TILE + wid * (RX_TILE / RX_WARPS) + lane;
#pragma unroll
        for (int k = 0; k < RX_ITEMS; ++k) {
            const uint64_t i = p0 + (uint64_t)k * 32;
            key[k] = 0;
            val[k] = 0;
            if (i < a.E) {
                key[k] = __ldcs(&a.kin[i]);
                val[k] = __ldcs(&a.vin[i]);
                valid |= 1u << k;
            }
        }
    }

    // Rank: per warp, items in order k = 0, 1, ...; lanes of one digit
    // (match) take consecutive slots after the warp's earlier items of it.
    unsigned rank[RX_ITEMS / 2];  // two 16-bit ranks a register (a rank is below 32 * RX_ITEMS)
    unsigned *wc = s_wcnt[wid];
#pragma unroll
    for (int k = 0; k < RX_ITEMS; ++k) {
        const bool ok = (valid >> k) & 1u;
        const unsigned d = ok ? (unsigned)(key[k] >> a.shift) & (RX_BINS - 1) : RX_BINS;
        const unsigned peers = __match_any_sync(FULL, d);
        const unsigned leader = __ffs(peers) - 1;
        unsigned c = 0;
        if (ok && lane == leader) {
            c = wc[d];
            wc[d] = c + __popc(peers);
        }
        c = __shfl_sync(FULL, c, leader);
        const unsigned r = c + __popc(peers & lanemask_lt());
        rank[k / 2] = (k & 1) ? rank[k / 2] | r << 16 : r;
        __syncwarp();
    }
    __syncthreads();

    // Thread d: digit d's warp offsets, tile count, tile offset, look-back.
    const unsigned d = tid;
    unsigned tot = 0;
#pragma unroll
    for (int q = 0; q < RX_WARPS; ++q) {
        const unsigned c = s_wcnt[q][d];
        s_wcnt[q][d] = tot;
        tot += c;
    }
    unsigned long long *my = a.status + tile * RX_BINS + d;
    const unsigned long long ep = a.epoch << RX_EPOCH_SHIFT;
    st_status(my, ep | ((tile == 0 ? RX_PREFIX : RX_AGG) << RX_FLAG_SHIFT) | tot);
    const unsigned incl = warp_incl_scan(tot);
    if (lane == 31) s_wsum[wid] = incl;
    __syncthreads();
    unsigned wb = 0, all = 0;
#pragma unroll
    for (int q = 0; q < RX_WARPS; ++q) {
        const unsigned x = s_wsum[q];
        if (q < (int)wid) wb += x;
        all += x;
    }
    // Tile offsets folded into the warp offsets: s_wcnt[w][d] = where warp
    // w's digit-d items start in the tile.
    const unsigned toff = wb + incl - tot;
#pragma unroll
    for (int q = 0; q < RX_WARPS; ++q) s_wcnt[q][d] += toff;
    if (tid == 0) s_total = all;
    __syncthreads();

    // Into shared memory in tile order by digit (the items' registers are
    // free from here on).
#pragma unroll
    for (int k = 0; k < RX_ITEMS; ++k) {
        if ((valid >> k) & 1u) {
            const unsigned dk = (unsigned)(key[k] >> a.shift) & (RX_BINS - 1);
            const unsigned pos = s_wcnt[wid][dk] + ((rank[k / 2] >> (16 * (k & 1))) & 0xffffu);
            s_key[pos] = key[k];
            s_val[pos] = val[k];
        }
    }

    // Look-back for digit d, after the scatter (read later, the status
    // words are further along): RX_LOOKBACK predecessors' words in flight at
    // once, taken in order from the nearest; a predecessor that has not
    // published yet is waited for (bounded), a prefix ends the walk.
    unsigned long long excl = 0;
    if (tile > 0) {
        int64_t j = (int64_t)tile - 1;
        const unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        bool done = false;
        while (!done) {
            unsigned long long sw[RX_LOOKBACK];
#pragma unroll
            for (int q = 0; q < RX_LOOKBACK; ++q)
                sw[q] = j - q >= 0 ? ld_relaxed64(a.status + (uint64_t)(j - q) * RX_BINS + d) : 0ull;
#pragma unroll
            for (int q = 0; q < RX_LOOKBACK; ++q) {
                if (done) break;
                if (j - q < 0) {  // tile 0 publishes a prefix: a walk past it means a broken status
                    atomicOr(a.err, SORTERR_WAIT);
                    done = true;
                    break;
                }
                unsigned long long x = sw[q];
                while ((x >> RX_EPOCH_SHIFT) != a.epoch || ((x >> RX_FLAG_SHIFT) & 3ull) == 0) {
                    if (++spins > 64) {
                        if (ld_volatile(a.err) & SORTERR_WAIT) break;  // another tile gave up: so do the rest
                        if (globaltimer_ns() - t0 > a.limit_ns) {
                            atomicOr(a.err, SORTERR_WAIT);
                            break;
                        }
                        __nanosleep(32);
                    }
                    x = ld_relaxed64(a.status + (uint64_t)(j - q) * RX_BINS + d);
                }
                if ((x >> RX_EPOCH_SHIFT) != a.epoch || ((x >> RX_FLAG_SHIFT) & 3ull) == 0) {  // gave up
                    done = true;
                    break;
                }
                excl += x & RX_COUNT_MASK;
                if (((x >> RX_FLAG_SHIFT) & 3ull) == RX_PREFIX) done = true;
            }
            j -= RX_LOOKBACK;
        }
        st_status(my, ep | (RX_PREFIX << RX_FLAG_SHIFT) | ((excl + tot) & RX_COUNT_MASK));
    }
    // Entry i of the tile (digit d) goes to s_gdelta[d] + i (mod 2^64).
    s_gdelta[d] = a.base[d] + excl - toff;
    if (tile + 1 == a.ntiles && excl + tot != a.hist[d]) atomicOr(a.err, SORTERR_COUNT);
    __syncthreads();

    // Out, run by run.
    const unsigned total = s_total;
    for (unsigned i = tid; i < total; i += RX_THREADS) {
        const unsigned long long k = s_key[i];
        const unsigned dk = (unsigned)(k >> a.shift) & (RX_BINS - 1);
        const unsigned long long pos = s_gdelta[dk] + i;
        if (pos < a.E) {
            a.kout[pos] = k;
            a.vout[pos] = s_val[i];
        } else {
            atomicOr(a.err, SORTERR_COUNT);
        }
    }
}

// rowstarts[r] = x for rows [r0, r1): short gaps here, long ones listed.
__device__ __forceinline__ void rx_gap(uint64_t *rowstarts, uint64_t r0, uint64_t r1, uint64_t x, uint64_t *gaps,
                                       uint64_t gcap, unsigned *cnt, unsigned *err) {
    if (r1 - r0 <= RX_GAP_INLINE) {
        for (uint64_t r = r0; r < r1; ++r) rowstarts[r] = x;
        return;
    }
    const unsigned g = atomicAdd(&cnt[RXC_GAPS], 1u);
    if (g >= gcap) {
        atomicOr(err, SORTERR_CAPACITY);
        return;
    }
    gaps[3 * g] = r0;
    gaps[3 * g + 1] = r1;
    gaps[3 * g + 2] = x;
}

// Entry i of the sorted keys (kp, k, kn: keys i - 1, i, i + 1, ~0 past
// the ends) -> col / w / row starts; a run of equal (src, dst) is ordered by
// weight bits by its first entry's thread.
__device__ __forceinline__ void rx_finish_entry(uint64_t i, unsigned long long kp, unsigned long long k,
                                                unsigned long long kn, const unsigned long long *__restrict__ K,
                                                const unsigned *__restrict__ V, unsigned v, uint64_t E, uint64_t n,
                                                int lg, uint64_t *__restrict__ rowstarts, int *__restrict__ col,
                                                float *__restrict__ w, uint64_t *__restrict__ col64,
                                                const RadixWork &rw) {
    unsigned *err = &rw.cnt[RXC_ERR];
    const uint64_t src = k >> lg, dst = k & ((1ull << lg) - 1);
    if ((i && kp > k) || src >= n) {
        atomicOr(err, SORTERR_ORDER);
        return;
    }
    col[i] = (int)dst;
    if (col64) col64[i] = dst;
    if (i == 0) rx_gap(rowstarts, 0, src + 1, 0, rw.gaps, rw.gcap, rw.cnt, err);
    else if ((kp >> lg) != src) rx_gap(rowstarts, (kp >> lg) + 1, src + 1, i, rw.gaps, rw.gcap, rw.cnt, err);
    if (i + 1 == E) rx_gap(rowstarts, src + 1, n + 1, E, rw.gaps, rw.gcap, rw.cnt, err);
    if (kp != k && kn != k) {
        w[i] = __uint_as_float(v);
    } else if (kp != k) {  // the first of a run of equal keys: the run's weights, sorted
        uint64_t j = i + 1;
        while (j < E && K[j] == k) ++j;
        const uint64_t L = j - i;
        if (L <= RX_RUN_INLINE) {
            unsigned x[RX_RUN_INLINE];
            for (unsigned q = 0; q < (unsigned)L; ++q) {
                const unsigned y = V[i + q];
                unsigned b = q;
                while (b > 0 && x[b - 1] > y) {
                    x[b] = x[b - 1];
                    --b;
                }
                x[b] = y;
            }
            for (unsigned q = 0; q < (unsigned)L; ++q) w[i + q] = __uint_as_float(x[q]);
        } else {
            for (uint64_t q = i; q < j; ++q) w[q] = __uint_as_float(V[q]);
            const unsigned r = atomicAdd(&rw.cnt[RXC_RUNS], 1u);
            if (r >= rw.rcap) {
                atomicOr(err, SORTERR_CAPACITY);
            } else {
                rw.runs[2 * r] = i;
                rw.runs[2 * r + 1] = j;
                if (L <= SORT_SMEM_KEYS) rw.rmid[atomicAdd(&rw.scnt[0], 1u)] = 2 * r;
                else rw.rbig[atomicAdd(&rw.scnt[1], 1u)] = 2 * r;
            }
        }
    }
}

// Sorted keys -> col / w / row starts, RX_FIN consecutive entries a thread
// (16-byte loads of the keys and weights; the neighbours' keys from L1).
constexpr int RX_FIN = 4;  // the loads below are written for 4

__global__ void csr_radix_finish_kernel(const unsigned long long *__restrict__ K, const unsigned *__restrict__ V,
                                        uint64_t E, uint64_t n, int lg, uint64_t *__restrict__ rowstarts,
                                        int *__restrict__ col, float *__restrict__ w, uint64_t *__restrict__ col64,
                                        RadixWork rw) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g * RX_FIN < E; g += stride) {
        const uint64_t i0 = g * RX_FIN;
        unsigned long long k[RX_FIN + 2];  // keys i0 - 1 .. i0 + RX_FIN
        unsigned v[RX_FIN];
        k[0] = i0 ? K[i0 - 1] : ~0ull;
        if (i0 + RX_FIN <= E) {  // K and V are 256-byte aligned, i0 a multiple of 4: 16-byte aligned
            const ulonglong2 a = *reinterpret_cast<const ulonglong2 *>(K + i0);
            const ulonglong2 b = *reinterpret_cast<const ulonglong2 *>(K + i0 + 2);
            const uint4 c = *reinterpret_cast<const uint4 *>(V + i0);
            k[1] = a.x;
            k[2] = a.y;
            k[3] = b.x;
            k[4] = b.y;
            v[0] = c.x;
            v[1] = c.y;
            v[2] = c.z;
            v[3] = c.w;
            k[RX_FIN + 1] = i0 + RX_FIN < E ? K[i0 + RX_FIN] : ~0ull;
        } else {
#pragma unroll
            for (int q = 0; q < RX_FIN; ++q) {
                k[q + 1] = i0 + q < E ? K[i0 + q] : ~0ull;
                v[q] = i0 + q < E ? V[i0 + q] : 0u;
            }
            k[RX_FIN + 1] = ~0ull;
        }
#pragma unroll
        for (int q = 0; q < RX_FIN; ++q)
            if (i0 + q < E) rx_finish_entry(i0 + q, k[q], k[q + 1], k[q + 2], K, V, v[q], E, n, lg, rowstarts, col, w,
                                            col64, rw);
    }
}

// The listed long gaps of empty rows, a block each.
__global__ void csr_radix_gaps_kernel(const uint64_t *__restrict__ gaps, const unsigned *__restrict__ cnt,
                                      uint64_t gcap, uint64_t *__restrict__ rowstarts) {
    const uint64_t ng = min((uint64_t)cnt[RXC_GAPS], gcap);
    for (uint64_t g = blockIdx.x; g < ng; g += gridDim.x) {
        const uint64_t r0 = gaps[3 * g], r1 = gaps[3 * g + 1], x = gaps[3 * g + 2];
        for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) rowstarts[r] = x;
    }
}

static int sort_grid(int per_sm) {
    DeviceInfo di;
    if (device_info(&di)) return 148 * per_sm;
    return di.sms * per_sm;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_csr_sorted_workspace_size(uint64_t nverts, uint64_t nentries, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_csr_sorted_workspace_size: bytes is NULL");
    *bytes = carve_sort(nullptr, nverts, nentries).bytes;
    return G5_OK;
}

// Tile prefix over the big rows listed in w.big (count in w.cnt[cidx]):
// returns their number, their tiles and the longest row's length (one
// synchronisation).
static int big_rows_prepare(const uint64_t *d_rowstarts, const SortWork &w, int cidx, cudaStream_t st,
                            unsigned *nbig, uint64_t *ntiles, unsigned long long *maxlen) {
    G5_CUDA_TRY(cudaMemsetAsync(&w.cnt[4], 0, 2 * sizeof(unsigned), st));
    unsigned nb = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(&nb, &w.cnt[cidx], sizeof nb, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    *nbig = nb;
    *ntiles = 0;
    *maxlen = 0;
    if (!nb) return G5_OK;
    big_tiles_kernel<<<std::max(1u, std::min(nb / 256 + 1, 1024u)), 256, 0, st>>>(
        d_rowstarts, w.big, nb, w.tcnt, (unsigned long long *)&w.cnt[4]);
    int rc = scan_u32_to_u64(w.tcnt, nb, w.tp, w.scan, st);
    if (rc) return rc;
    G5_CUDA_TRY(cudaMemcpyAsync(ntiles, w.tp + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaMemcpyAsync(maxlen, &w.cnt[4], sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (*ntiles > w.tmax)
        return set_error(G5_ERR_INVALID, "canonical CSR: rows hold more entries than nentries (%llu tiles > %llu)",
                         (unsigned long long)*ntiles, (unsigned long long)w.tmax);
    return G5_OK;
}

// The listed big rows (w.big, count w.cnt[cidx]) sorted in place: every
// BIG_TILE chunk in shared memory, then merge passes over the whole grid.
static int sort_big_rows(const uint64_t *d_rowstarts, int32_t *d_col, float *d_w, uint64_t *d_col64,
                         const SortWork &w, int cidx, cudaStream_t st) {
    unsigned nbig = 0;
    uint64_t ntiles = 0;
    unsigned long long maxlen = 0;
    int rc = big_rows_prepare(d_rowstarts, w, cidx, st, &nbig, &ntiles, &maxlen);
    if (rc || !nbig) return rc;
    const int grid = (int)std::min<uint64_t>(ntiles, (uint64_t)sort_grid(4));
    csr_sort_chunks_kernel<<<grid, SORT_THREADS, 0, st>>>(d_rowstarts, w.big, nbig, w.tp, ntiles, w.tkey, d_col, d_w);
    const KeyBuf K{w.tkey, nullptr, nullptr}, C{nullptr, d_col, d_w};
    bool in_scratch = true;
    for (uint64_t R = BIG_TILE; R < maxlen; R <<= 1) {
        csr_merge_pass_kernel<<<grid, SORT_THREADS, 0, st>>>(d_rowstarts, w.big, nbig, w.tp, ntiles, R,
                                                             in_scratch ? K : C, in_scratch ? C : K);
        in_scratch = !in_scratch;
    }
    csr_big_finish_kernel<<<grid, 256, 0, st>>>(d_rowstarts, w.big, nbig, w.tp, ntiles, w.tkey, d_col, d_w, d_col64);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

// Sorts rows in place (any CSR: the rows of g5_csr_fill or of the fused
// Kronecker fill come out canonical too).
static int sort_rows(const uint64_t *d_rowstarts, uint64_t nverts, int32_t *d_col, float *d_w, uint64_t *d_col64,
                     const SortWork &w, cudaStream_t st) {
    G5_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, 2 * sizeof(unsigned), st));
    const uint64_t warps = (nverts + 31) / 32;
    const int wblocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sort_grid(8), (warps + 7) / 8));
    csr_sort_warp_kernel<<<wblocks, 256, 0, st>>>(d_rowstarts, nverts, d_col, d_w, d_col64, w.mid, w.big, w.cnt);
    csr_sort_mid_kernel<<<sort_grid(4), SORT_THREADS, 0, st>>>(d_rowstarts, w.mid, w.cnt, d_col, d_w, d_col64);
    G5_CUDA_TRY(cudaGetLastError());
    return sort_big_rows(d_rowstarts, d_col, d_w, d_col64, w, 1, st);
}

extern "C" int g5_csr_fill_sorted(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                                  const uint64_t *d_rowstarts, uint64_t nentries, void *d_work, uint64_t work_bytes,
                                  int32_t *d_col, float *d_w, uint64_t *d_col64, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_fill_sorted: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_work && (nentries == 0 || (d_col && d_w)), "g5_csr_fill_sorted: NULL argument");
    G5_CHECK_ARG(nedges == 0 || (d_edges && d_weights), "g5_csr_fill_sorted: edges or weights NULL");
    SortWork w = carve_sort(d_work, nverts, nentries);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_csr_fill_sorted: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    cudaStream_t st = (cudaStream_t)stream;
    const int pshift = part_shift(nverts);
    G5_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, 64 * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.rcur, 0, nverts * sizeof(unsigned), st));
    if (nedges && nentries) {
        csr_part_init_kernel<<<1, NPART + 32, 0, st>>>(d_rowstarts, nverts, pshift, w.pcur);
        const uint64_t tiles = (nedges + P1_EDGES - 1) / P1_EDGES;
        const int pblocks = (int)std::min<uint64_t>(tiles, (uint64_t)sort_grid(2));
        static bool smem_set[64] = {};  // the function attribute, once per device
        int dev = 0;
        G5_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64 || !smem_set[dev]) {
            G5_CUDA_TRY(cudaFuncSetAttribute(csr_partition_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)P1_SMEM));
            if (dev >= 0 && dev < 64) smem_set[dev] = true;
        }
        csr_partition_kernel<<<pblocks, P1_THREADS, P1_SMEM, st>>>((const ulonglong2 *)d_edges, d_weights, nedges, nverts,
                                                             pshift, d_rowstarts, w.pcur, w.tkey, w.tw, &w.cnt[2]);
        const uint64_t nparts = std::min<uint64_t>(NPART, (nverts + (1ull << pshift) - 1) >> pshift);
        const int gblocks = (int)std::max<uint64_t>(
            1, std::min<uint64_t>((uint64_t)sort_grid(8), (nentries / nparts + 255) / 256));
        for (unsigned p = 0; p < nparts; ++p)
            csr_place_kernel<<<gblocks, 256, 0, st>>>(w.tkey, w.tw, nverts, pshift, p, d_rowstarts, w.rcur, d_col,
                                                      d_w, &w.cnt[2]);
        G5_CUDA_TRY(cudaGetLastError());
    }
    int rc = sort_rows(d_rowstarts, nverts, d_col, d_w, d_col64, w, st);
    if (rc) return rc;
    unsigned err = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(&err, &w.cnt[2], sizeof err, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (err & SORTERR_RANGE) return set_error(G5_ERR_INVALID, "g5_csr_fill_sorted: an edge endpoint is >= nverts");
    if (err) return set_error(G5_ERR_INVALID, "g5_csr_fill_sorted: the edges differ from those the rows were counted on");
    return G5_OK;
}

// ------------------------------------------------------------ radix build

static int radix_passes(uint64_t n) { return (2 * vertex_bits(n) + RX_BITS - 1) / RX_BITS; }

extern "C" int g5_csr_radix_workspace_size(uint64_t nverts, uint64_t nedges, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_csr_radix_workspace_size: bytes is NULL");
    *bytes = carve_radix(nullptr, nverts, nedges).bytes;
    return G5_OK;
}

extern "C" int g5_csr_radix_count(const uint64_t *d_edges, uint64_t nedges, uint64_t nverts, void *d_work,
                                  uint64_t work_bytes, uint64_t *nentries, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_radix_count: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_work && nentries && (nedges == 0 || d_edges), "g5_csr_radix_count: NULL argument");
    RadixWork w = carve_radix(d_work, nverts, nedges);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_csr_radix_count: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    cudaStream_t st = (cudaStream_t)stream;
    const int lg = vertex_bits(nverts), passes = radix_passes(nverts);
    G5_CUDA_TRY(cudaMemsetAsync(w.hist, 0, 2 * RX_MAXPASS * RX_BINS * sizeof(unsigned long long), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.total, 0, 2 * sizeof(unsigned long long), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, 64 * sizeof(unsigned), st));
    if (nedges) {  // (with one vertex there are no passes, but the endpoints are still checked)
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((nedges + 255) / 256, (uint64_t)sort_grid(8)));
        csr_radix_hist_kernel<<<grid, 256, 0, st>>>((const ulonglong2 *)d_edges, nedges, nverts, lg, passes, w.hist,
                                                    &w.cnt[RXC_ERR]);
        if (passes) csr_radix_scan_kernel<<<1, RX_BINS, 0, st>>>(w.hist, passes, w.base, w.total);
        G5_CUDA_TRY(cudaGetLastError());
    }
    const unsigned long long m = nedges;
    G5_CUDA_TRY(cudaMemcpyAsync(&w.total[1], &m, sizeof m, cudaMemcpyHostToDevice, st));
    unsigned long long total = 0;
    unsigned err = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(&total, w.total, sizeof total, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaMemcpyAsync(&err, &w.cnt[RXC_ERR], sizeof err, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (err & SORTERR_RANGE) return set_error(G5_ERR_INVALID, "g5_csr_radix_count: an edge endpoint is >= nverts");
    *nentries = total;
    return G5_OK;
}

extern "C" int g5_csr_radix_fill(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                                 uint64_t nentries, void *d_work, uint64_t work_bytes, uint64_t *d_rowstarts,
                                 int32_t *d_col, float *d_w, uint64_t *d_col64, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_radix_fill: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_work && d_rowstarts && (nentries == 0 || (d_col && d_w)), "g5_csr_radix_fill: NULL argument");
    G5_CHECK_ARG(nedges == 0 || (d_edges && d_weights), "g5_csr_radix_fill: edges or weights NULL");
    G5_CHECK_ARG(nentries <= 2 * nedges, "g5_csr_radix_fill: nentries > 2 * nedges");
    RadixWork w = carve_radix(d_work, nverts, nedges);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_csr_radix_fill: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    cudaStream_t st = (cudaStream_t)stream;
    unsigned long long counted[2] = {0, 0};
    G5_CUDA_TRY(cudaMemcpyAsync(counted, w.total, sizeof counted, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (counted[0] != nentries || counted[1] != nedges)
        return set_error(G5_ERR_INVALID, "g5_csr_radix_fill: run g5_csr_radix_count on the same edges first "
                         "(counted %llu entries of %llu edges, given %llu of %llu)", counted[0], counted[1],
                         (unsigned long long)nentries, (unsigned long long)nedges);
    const int lg = vertex_bits(nverts), passes = radix_passes(nverts);
    const uint64_t E = nentries;
    G5_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, 64 * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.scnt, 0, 64 * sizeof(unsigned), st));
    if (E == 0) {
        G5_CUDA_TRY(cudaMemsetAsync(d_rowstarts, 0, (nverts + 1) * sizeof(uint64_t), st));
        G5_CUDA_TRY(cudaStreamSynchronize(st));
        return G5_OK;
    }
    static bool smem_set[64][2] = {};  // the function attributes, once per device
    int dev = 0;
    G5_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || !smem_set[dev][0]) {
        G5_CUDA_TRY(cudaFuncSetAttribute(csr_radix_pass_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)RX_SMEM));
        G5_CUDA_TRY(cudaFuncSetAttribute(csr_radix_pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)RX_SMEM));
        if (dev >= 0 && dev < 64) smem_set[dev][0] = true;
    }
    const uint64_t t_first = (nedges + RX_EDGE_TILE - 1) / RX_EDGE_TILE, t_rest = (E + RX_TILE - 1) / RX_TILE;
    G5_CUDA_TRY(cudaMemsetAsync(w.status, 0, t_first * RX_BINS * sizeof(unsigned long long), st));
    RxPass a{};
    a.edges = (const ulonglong2 *)d_edges;
    a.weights = d_weights;
    a.m = nedges;
    a.n = nverts;
    a.E = E;
    a.lg = lg;
    a.status = w.status;
    a.err = &w.cnt[RXC_ERR];
    a.limit_ns = wait_limit_ns();
    unsigned long long *kin = nullptr, *kout = w.ka;
    unsigned *vin = nullptr, *vout = w.va;
    for (int p = 0; p < passes; ++p) {
        a.kin = kin;
        a.vin = vin;
        a.kout = kout;
        a.vout = vout;
        a.shift = RX_BITS * p;
        a.epoch = (unsigned long long)(p + 1);
        a.base = w.base + p * RX_BINS;
        a.hist = w.hist + p * RX_BINS;
        a.tilectr = &w.cnt[RXC_TILES + p];
        a.ntiles = p == 0 ? t_first : t_rest;
        if (a.ntiles > 0x7fffffffull) return set_error(G5_ERR_INVALID, "g5_csr_radix_fill: too many tiles");
        if (p == 0) csr_radix_pass_kernel<true><<<(unsigned)a.ntiles, RX_THREADS, RX_SMEM, st>>>(a);
        else csr_radix_pass_kernel<false><<<(unsigned)a.ntiles, RX_THREADS, RX_SMEM, st>>>(a);
        G5_CUDA_TRY(cudaGetLastError());
        kin = kout;
        vin = vout;
        kout = kout == w.ka ? w.kb : w.ka;
        vout = vout == w.va ? w.vb : w.va;
    }
    const int fgrid = (int)std::max<uint64_t>(1, std::min<uint64_t>((E / RX_FIN + 256) / 256, (uint64_t)sort_grid(8)));
    csr_radix_finish_kernel<<<fgrid, 256, 0, st>>>(kin, vin, E, nverts, lg, d_rowstarts, d_col, d_w, d_col64, w);
    csr_radix_gaps_kernel<<<sort_grid(2), 256, 0, st>>>(w.gaps, w.cnt, w.gcap, d_rowstarts);
    G5_CUDA_TRY(cudaGetLastError());
    unsigned c[3] = {0, 0, 0};
    G5_CUDA_TRY(cudaMemcpyAsync(c, w.cnt, sizeof c, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    const unsigned err = c[RXC_ERR];
    if (err & SORTERR_RANGE) return set_error(G5_ERR_INVALID, "g5_csr_radix_fill: an edge endpoint is >= nverts");
    if (err & SORTERR_WAIT) return set_error(G5_ERR_TIMEOUT, "g5_csr_radix_fill: a look-back wait gave up");
    if (err & SORTERR_CAPACITY) return set_error(G5_ERR_DEVICE, "g5_csr_radix_fill: internal list overflow");
    if (err) return set_error(G5_ERR_INVALID, "g5_csr_radix_fill: the edges differ from the ones counted");
    if (c[RXC_RUNS]) {
        // Long runs of one (row, neighbour): sorted as "rows" [start, end)
        // by the row-sort kernels, with the key buffers as their scratch.
        const uint64_t nruns = std::min<uint64_t>(c[RXC_RUNS], w.rcap);
        SortWork sw = carve_sort(w.ka, 2 * nruns + 1, E);
        if (sw.bytes > w.region) return set_error(G5_ERR_DEVICE, "g5_csr_radix_fill: run-sort scratch too small");
        sw.mid = w.rmid;
        sw.big = w.rbig;
        sw.cnt = w.scnt;
        csr_sort_mid_kernel<<<sort_grid(4), SORT_THREADS, 0, st>>>(w.runs, w.rmid, w.scnt, d_col, d_w, d_col64);
        G5_CUDA_TRY(cudaGetLastError());
        int rc = sort_big_rows(w.runs, d_col, d_w, d_col64, sw, 1, st);
        if (rc) return rc;
        G5_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return G5_OK;
}

extern "C" int g5_csr_sort_rows(const uint64_t *d_rowstarts, uint64_t nverts, uint64_t nentries, int32_t *d_col,
                                float *d_w, uint64_t *d_col64, void *d_work, uint64_t work_bytes, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_sort_rows: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_work && (nentries == 0 || (d_col && d_w)), "g5_csr_sort_rows: NULL argument");
    SortWork w = carve_sort(d_work, nverts, nentries);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_sort_rows: workspace too small");
    return sort_rows(d_rowstarts, nverts, d_col, d_w, d_col64, w, (cudaStream_t)stream);
}

extern "C" int g5_csr_dedupe_count(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                   uint64_t nentries, uint64_t *d_rowstarts_out, void *d_work, uint64_t work_bytes,
                                   uint64_t *nentries_out, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_dedupe_count: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_rowstarts_out && d_work && nentries_out && (nentries == 0 || d_col),
                 "g5_csr_dedupe_count: NULL argument");
    SortWork w = carve_sort(d_work, nverts, nentries);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_dedupe_count: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sort_grid(8), (nverts + 7) / 8));
    csr_unique_count_kernel<<<blocks, 256, 0, st>>>(d_rowstarts, d_col, nverts, w.rcur);
    G5_CUDA_TRY(cudaGetLastError());
    int rc = scan_u32_to_u64(w.rcur, nverts, d_rowstarts_out, w.scan, st);
    if (rc) return rc;
    G5_CUDA_TRY(cudaMemcpyAsync(nentries_out, d_rowstarts_out + nverts, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return G5_OK;
}

extern "C" int g5_csr_dedupe_copy(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                  uint64_t nverts, const uint64_t *d_rowstarts_out, int32_t *d_col_out,
                                  float *d_w_out, uint64_t *d_col64_out, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_dedupe_copy: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_rowstarts_out && d_col_out && d_w_out,
                 "g5_csr_dedupe_copy: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sort_grid(8), (nverts + 7) / 8));
    csr_unique_copy_kernel<<<blocks, 256, 0, st>>>(d_rowstarts, d_col, d_w, nverts, d_rowstarts_out, d_col_out,
                                                   d_w_out, d_col64_out);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_csr_degree_order_workspace_size(uint64_t nverts, uint64_t nentries, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_csr_degree_order_workspace_size: bytes is NULL");
    *bytes = carve_sort(nullptr, nverts, nentries).bytes + align_up(nentries * 4, 256) + align_up(nverts * 4, 256);
    return G5_OK;
}

extern "C" int g5_csr_degree_order(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                   uint64_t nentries, int32_t *d_out_col, void *d_work, uint64_t work_bytes,
                                   void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_degree_order: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_work && (nentries == 0 || (d_col && d_out_col)),
                 "g5_csr_degree_order: NULL argument");
    G5_CHECK_ARG(nentries == 0 || d_out_col != d_col, "g5_csr_degree_order: d_out_col must not be d_col");
    uint64_t need = 0;
    g5_csr_degree_order_workspace_size(nverts, nentries, &need);
    if (work_bytes < need) return set_error(G5_ERR_WORKSPACE, "g5_csr_degree_order: workspace too small");
    if (nentries == 0) return G5_OK;
    SortWork w = carve_sort(d_work, nverts, nentries);
    int *ka = (int *)((char *)d_work + w.bytes);
    unsigned *deg = (unsigned *)((char *)ka + align_up(nentries * 4, 256));
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(&w.cnt[2], 0, sizeof(unsigned), st));
    row_lengths_kernel<<<sort_grid(8), 256, 0, st>>>(d_rowstarts, nverts, deg);
    degree_keys_kernel<<<sort_grid(8), 256, 0, st>>>(d_col, nentries, deg, nverts, ka, (float *)d_out_col, &w.cnt[2]);
    G5_CUDA_TRY(cudaGetLastError());
    int rc = sort_rows(d_rowstarts, nverts, ka, (float *)d_out_col, nullptr, w, st);
    if (rc) return rc;
    unsigned errs = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(&errs, &w.cnt[2], sizeof errs, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (errs) return set_error(G5_ERR_INVALID, "g5_csr_degree_order: a column entry is not a vertex");
    return G5_OK;
}

// Scratch of g5_csr_sssp_renumber: the row sort's for one row of n
// entries, the degrees and new lengths, the sort keys, a scan's scratch.
static uint64_t renumber_bytes(uint64_t n, uint64_t *off_deg, uint64_t *off_len, uint64_t *off_ka,
                               uint64_t *off_rs, uint64_t *off_scan) {
    uint64_t b = align_up(carve_sort(nullptr, 1, n).bytes, 256);
    *off_deg = b;
    b += align_up(n * 4, 256);
    *off_len = b;
    b += align_up(n * 4, 256);
    *off_ka = b;
    b += align_up(n * 4, 256);
    *off_rs = b;
    b += 256;
    *off_scan = b;
    b += align_up(scan_scratch_words(n) * 8, 256);
    return b;
}

extern "C" int g5_csr_sssp_renumber_workspace_size(uint64_t nverts, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_csr_sssp_renumber_workspace_size: bytes is NULL");
    uint64_t a, b, c, d, e;
    *bytes = renumber_bytes(nverts, &a, &b, &c, &d, &e);
    return G5_OK;
}

extern "C" int g5_csr_sssp_renumber(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                    const uint32_t *d_light_deg, const uint32_t *d_tiny_deg, uint64_t nverts,
                                    uint64_t nentries, uint32_t *d_perm, uint32_t *d_inv, uint64_t *d_rowstarts_out,
                                    int32_t *d_col_out, float *d_w_out, uint32_t *d_light_out, uint32_t *d_tiny_out,
                                    void *d_work, uint64_t work_bytes, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_sssp_renumber: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_light_deg && d_tiny_deg && d_perm && d_inv && d_rowstarts_out && d_light_out &&
                     d_tiny_out && d_work && (nentries == 0 || (d_col && d_w && d_col_out && d_w_out)),
                 "g5_csr_sssp_renumber: NULL argument");
    uint64_t off_deg, off_len, off_ka, off_rs, off_scan;
    if (work_bytes < renumber_bytes(nverts, &off_deg, &off_len, &off_ka, &off_rs, &off_scan))
        return set_error(G5_ERR_WORKSPACE, "g5_csr_sssp_renumber: workspace too small");
    char *base = (char *)d_work;
    SortWork w = carve_sort(d_work, 1, nverts);
    unsigned *deg = (unsigned *)(base + off_deg), *len2 = (unsigned *)(base + off_len);
    int *ka = (int *)(base + off_ka);
    uint64_t *rs1 = (uint64_t *)(base + off_rs), *scan = (uint64_t *)(base + off_scan);
    cudaStream_t st = (cudaStream_t)stream;
    const int grid = sort_grid(8);
    // The vertex order: decreasing degree, ties by index (a row sort of one
    // row of n keys); inv = the order, perm its inverse.
    const uint64_t one_row[2] = {0, nverts};
    G5_CUDA_TRY(cudaMemcpyAsync(rs1, one_row, sizeof one_row, cudaMemcpyHostToDevice, st));
    G5_CUDA_TRY(cudaMemsetAsync(&w.cnt[2], 0, sizeof(unsigned), st));
    row_lengths_kernel<<<grid, 256, 0, st>>>(d_rowstarts, nverts, deg);
    vertex_order_keys_kernel<<<grid, 256, 0, st>>>(deg, nverts, ka, (float *)d_inv);
    G5_CUDA_TRY(cudaGetLastError());
    int rc = sort_rows(rs1, 1, ka, (float *)d_inv, nullptr, w, st);
    if (rc) return rc;
    vertex_perm_kernel<<<grid, 256, 0, st>>>(d_inv, deg, nverts, d_perm, len2);
    G5_CUDA_TRY(cudaGetLastError());
    if ((rc = scan_u32_to_u64(len2, nverts, d_rowstarts_out, scan, st))) return rc;
    renumber_rows_kernel<<<grid, 256, 0, st>>>(d_rowstarts, d_col, d_w, d_light_deg, d_tiny_deg, nverts, d_perm, d_inv,
                                               d_rowstarts_out, d_col_out, d_w_out, d_light_out, d_tiny_out,
                                               &w.cnt[2]);
    renumber_long_rows_kernel<<<grid, 256, 0, st>>>(d_rowstarts, d_col, d_w, nverts, d_perm, d_inv, d_rowstarts_out,
                                                    d_col_out, d_w_out, &w.cnt[2]);
    G5_CUDA_TRY(cudaGetLastError());
    unsigned errs = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(&errs, &w.cnt[2], sizeof errs, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (errs) return set_error(G5_ERR_INVALID, "g5_csr_sssp_renumber: a column entry is not a vertex");
    return G5_OK;
}

extern "C" int g5_csr_split_light(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                  uint64_t nverts, uint64_t nentries, float light_delta, int32_t *d_scol, float *d_sw,
                                  uint32_t *d_light_deg, uint32_t *d_tiny_deg, void *d_work, uint64_t work_bytes,
                                  void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_split_light: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_light_deg && d_tiny_deg && d_work &&
                     (nentries == 0 || (d_col && d_w && d_scol && d_sw)),
                 "g5_csr_split_light: NULL argument");
    G5_CHECK_ARG(light_delta > 0.0f, "g5_csr_split_light: light_delta must be positive");
    SortWork w = carve_sort(d_work, nverts, nentries);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_split_light: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const float tiny = light_delta / (float)G5_TINY_DIV;
    G5_CUDA_TRY(cudaMemsetAsync(&w.cnt[3], 0, sizeof(unsigned), st));
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)sort_grid(8), (nverts + 7) / 8));
    csr_split_light_kernel<<<blocks, 256, 0, st>>>(d_rowstarts, d_col, d_w, nverts, light_delta, tiny, d_scol, d_sw,
                                                   d_light_deg, d_tiny_deg, w.big, &w.cnt[3]);
    G5_CUDA_TRY(cudaGetLastError());
    unsigned nbig = 0;
    uint64_t ntiles = 0;
    unsigned long long maxlen = 0;
    int rc = big_rows_prepare(d_rowstarts, w, 3, st, &nbig, &ntiles, &maxlen);
    if (rc || !nbig) return rc;
    const int grid = (int)std::min<uint64_t>(ntiles, (uint64_t)sort_grid(4));
    csr_split_count_kernel<<<grid, SORT_THREADS, 0, st>>>(d_rowstarts, d_w, w.big, nbig, w.tp, ntiles, light_delta,
                                                          tiny, w.tcnt, w.tcnt2);
    if ((rc = scan_u32_to_u64(w.tcnt, ntiles, w.tq, w.scan, st))) return rc;
    if ((rc = scan_u32_to_u64(w.tcnt2, ntiles, w.tq2, w.scan, st))) return rc;
    csr_split_write_kernel<<<grid, SORT_THREADS, 0, st>>>(d_rowstarts, d_col, d_w, w.big, nbig, w.tp, ntiles,
                                                          light_delta, tiny, w.tq, w.tq2, d_scol, d_sw, d_light_deg,
                                                          d_tiny_deg);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}
