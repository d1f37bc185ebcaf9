// validate.cu -- K5: Graph500 BFS validation, SSSP validation and the TEPS
// edge count.
//
// The BFS rules and the edge count are the runner's
// (examples/graph500_runner.cu:84-201): same rules, same error count.  The
// reference walks each row with one thread (a hub row of millions of entries
// serialises on that thread); here every edge pass is edge-parallel: a block
// takes a tile of 4096 CSR entries, caches the row starts of the rows the
// tile spans in shared memory, and each thread walks 16 consecutive entries,
// finding its first row by a binary search in shared memory and the next
// ones by stepping forward -- no per-entry search through rowptr in memory.
// (A tile spanning more rows than the cache holds -- many empty rows --
// searches rowptr per entry instead.)  The first row of every tile comes
// from a pre-pass (one thread per tile, all searches in parallel), so no
// block waits on a 26-step dependent search through rowptr per tile.  A
// neighbour's two values the rules compare (BFS: dist and pred; SSSP: dist
// and pred) are packed by a pre-pass into one 16-byte record, so each entry
// reads one sector of it; a thread issues the record loads of its 16
// entries before it tests any of them.
//
// HBM bytes per pass: E * 4 (col) [+ E * 4 w] + one random 16-byte record
// per entry (a 32-byte sector).
#include "g5_common.cuh"

namespace g5 {

constexpr int VAL_THREADS = 256;
constexpr int VAL_ITEMS = 16;                       // consecutive entries a thread walks
constexpr int VAL_TILE = VAL_THREADS * VAL_ITEMS;   // entries per tile
constexpr unsigned VAL_SPAN = 4096;                 // row starts cached per tile

// Largest v in [lo, hi] with rowptr[v] <= e.
__device__ __forceinline__ uint64_t row_of(const uint64_t *__restrict__ rowptr, uint64_t lo, uint64_t hi, uint64_t e) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&rowptr[mid]) <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Tile table: trow[t] = row of entry t * VAL_TILE for every tile t, and
// trow[ntiles] = row of the last entry, when the table has room (the
// pre-pass sets ok[0]).
__global__ void val_tile_rows_kernel(const uint64_t *__restrict__ rowptr, uint64_t n, unsigned *__restrict__ trow,
                                     uint64_t cap, unsigned long long *__restrict__ ok) {
    const uint64_t E = rowptr[n];
    const uint64_t ntiles = (E + VAL_TILE - 1) / VAL_TILE;
    if (E == 0 || ntiles + 1 > cap) return;  // ok stays 0: tiles search rowptr themselves
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += stride)
        trow[t] = (unsigned)row_of(rowptr, 0, n - 1, t < ntiles ? t * VAL_TILE : E - 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) *ok = 1;
}

// Row span of the tile [e0, e1) of the CSR, into shared memory: from the
// tile table when it is there (the row of the next tile's first entry
// bounds the span; rows beyond the tile's last entry start after it and are
// never stepped into), else by two searches.
__device__ __forceinline__ void tile_rows(const uint64_t *__restrict__ rowptr, uint64_t n, uint64_t e0, uint64_t e1,
                                          const unsigned *__restrict__ trow, bool table, uint64_t *s_lo,
                                          uint64_t *s_hi) {
    if (threadIdx.x == 0) {
        if (table) {
            const uint64_t t = e0 / VAL_TILE;
            *s_lo = __ldg(&trow[t]);
            *s_hi = __ldg(&trow[t + 1]);
        } else {
            *s_lo = row_of(rowptr, 0, n - 1, e0);
            *s_hi = row_of(rowptr, *s_lo, n - 1, e1 - 1);
        }
    }
    __syncthreads();
}

// Entries of tile [e0, e1): calls visit(u, eb, ne, c) once per thread with
// the thread's ne <= 16 consecutive entries eb.. (u[k] the row of entry
// eb + k, c[k] its column entry).  Thread t takes [e0 + 16 t, e0 + 16 t +
// 16).  The tile's row starts are cached in s_rp (when its rows fit) and
// each thread steps from row to row; the column is read 16 bytes at a time
// where it is aligned.  Every thread of the block calls it.
template <class Visit>
__device__ __forceinline__ void tile_walk(const uint64_t *__restrict__ rowptr, const int *__restrict__ col, uint64_t n,
                                          uint64_t e0, uint64_t e1, const unsigned *__restrict__ trow, bool table,
                                          uint64_t *s_rp, uint64_t *s_lo, uint64_t *s_hi, Visit visit) {
    tile_rows(rowptr, n, e0, e1, trow, table, s_lo, s_hi);
    const uint64_t lo = *s_lo, span64 = *s_hi - lo + 1;
    const unsigned span = span64 <= VAL_SPAN ? (unsigned)span64 : 0u;
    for (unsigned r = threadIdx.x; span && r <= span; r += blockDim.x) s_rp[r] = __ldg(&rowptr[lo + r]);
    __syncthreads();
    const uint64_t eb = e0 + (uint64_t)threadIdx.x * VAL_ITEMS;
    if (eb < e1) {
        const uint64_t ee = min(eb + VAL_ITEMS, e1);
        int c[VAL_ITEMS];
        if (ee - eb == VAL_ITEMS && ((uintptr_t)(col + eb) & 15) == 0) {
            const int4 *p = reinterpret_cast<const int4 *>(col + eb);
#pragma unroll
            for (int k = 0; k < VAL_ITEMS / 4; ++k) {
                const int4 q = __ldg(p + k);
                c[4 * k] = q.x;
                c[4 * k + 1] = q.y;
                c[4 * k + 2] = q.z;
                c[4 * k + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < VAL_ITEMS; ++k) c[k] = eb + k < ee ? __ldg(&col[eb + k]) : 0;
        }
        unsigned r = 0;
        if (span) {
            unsigned a = 0, b = span - 1;  // largest r with s_rp[r] <= eb
            while (a < b) {
                const unsigned mid = (a + b + 1) >> 1;
                if (s_rp[mid] <= eb) a = mid;
                else b = mid - 1;
            }
            r = a;
        }
        const unsigned ne = (unsigned)(ee - eb);
        unsigned u[VAL_ITEMS];
#pragma unroll
        for (int k = 0; k < VAL_ITEMS; ++k) {
            const uint64_t e = eb + k;
            u[k] = 0;
            if (k < ne) {
                if (span) {
                    while (s_rp[r + 1] <= e) ++r;
                    u[k] = (unsigned)(lo + r);
                } else {
                    u[k] = (unsigned)row_of(rowptr, lo, *s_hi, e);
                }
            }
        }
        visit(u, eb, ne, c);
    }
    __syncthreads();
}

__device__ __forceinline__ void block_add(unsigned long long *dst, unsigned long long v) {
    v = warp_sum(v);
    if (lane_id() == 0 && v) atomicAdd(dst, v);
}

__global__ void __launch_bounds__(VAL_THREADS) edge_count_kernel(const uint64_t *__restrict__ rowptr,
                                                                 const int *__restrict__ col, uint64_t n,
                                                                 const int64_t *__restrict__ pred,
                                                                 const unsigned *__restrict__ trow,
                                                                 const unsigned long long *__restrict__ table,
                                                                 unsigned long long *__restrict__ out) {
    __shared__ uint64_t s_lo, s_hi;
    __shared__ uint64_t s_rp[VAL_SPAN + 1];
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    unsigned long long cnt = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        tile_walk(rowptr, col, n, e0, min(e0 + VAL_TILE, E), trow, tab, s_rp, &s_lo, &s_hi,
                  [&](const unsigned *u, uint64_t, unsigned ne, const int *c) {
                      // rows change rarely within 16 entries: one pred load per row
                      unsigned ur = ~0u;
                      bool reached = false;
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          if (k >= ne) break;
                          if (u[k] != ur) {
                              ur = u[k];
                              reached = __ldg(&pred[ur]) != -1;
                          }
                          if (reached && (unsigned)c[k] <= u[k]) ++cnt;
                      }
                  });
    }
    block_add(out, cnt);
}

// A neighbour's values for the edge rules, packed into one 16-byte record:
// BFS {dist, pred}; SSSP {dist bits, pred}.
__global__ void val_pack_bfs_kernel(const int64_t *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                    longlong2 *__restrict__ vx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        vx[v] = make_longlong2(dist[v], pred[v]);
}

__global__ void val_pack_sssp_kernel(const float *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                     longlong2 *__restrict__ vx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        vx[v] = make_longlong2((long long)__float_as_uint(dist[v]), pred[v]);
}

// Rules 1-2 (examples/graph500_runner.cu:84-109).
__global__ void bfs_val_vertex_kernel(const int64_t *__restrict__ pred, const int64_t *__restrict__ dist, uint64_t n,
                                      uint64_t root, unsigned *__restrict__ confirmed,
                                      unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const int64_t p = pred[v];
        if (p != -1 && (p < 0 || (uint64_t)p >= n)) ++err;
        if (v == root) {
            if (p != (int64_t)root || dist[v] != 0) ++err;
            else atomicOr(&confirmed[v >> 5], 1u << (v & 31));
        }
    }
    block_add(errors, err);
}

// Rules 3-6 (examples/graph500_runner.cu:111-153), one thread per CSR entry.
__global__ void __launch_bounds__(VAL_THREADS, 2) bfs_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                   const int *__restrict__ col, uint64_t n,
                                                                   const int64_t *__restrict__ pred,
                                                                   const int64_t *__restrict__ dist,
                                                                   const longlong2 *__restrict__ vx,
                                                                   const unsigned *__restrict__ trow,
                                                                   const unsigned long long *__restrict__ table,
                                                                   unsigned *__restrict__ confirmed,
                                                                   unsigned long long *__restrict__ errors) {
    __shared__ uint64_t s_lo, s_hi;
    __shared__ uint64_t s_rp[VAL_SPAN + 1];
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    unsigned long long err = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        tile_walk(rowptr, col, n, e0, min(e0 + VAL_TILE, E), trow, tab, s_rp, &s_lo, &s_hi,
                  [&](const unsigned *u, uint64_t, unsigned ne, const int *c) {
                      // every neighbour record in flight before the first test
                      longlong2 xv[VAL_ITEMS];
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          const unsigned x = (unsigned)c[k];
                          xv[k] = k < ne && x < n ? __ldg(&vx[x]) : make_longlong2(0, 0);
                      }
                      unsigned ur = ~0u;
                      int64_t ud = 0, up = 0;
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          if (k >= ne) break;
                          const unsigned uu = u[k];
                          const uint64_t x = (unsigned)c[k];
                          if (x == uu || x >= n) {  // a self-loop entry, or not a vertex (counted once, nothing else compared)
                              ++err;
                              continue;
                          }
                          if (uu != ur) {
                              ur = uu;
                              ud = __ldg(&dist[uu]);
                              up = __ldg(&pred[uu]);
                          }
                          const int64_t xd = xv[k].x, xp = xv[k].y;
                          if ((ud == -1) != (xd == -1)) ++err;
                          if (ud >= 0 && xd >= 0 && (ud + 1 < xd || xd + 1 < ud)) ++err;
                          if (up == (int64_t)x) atomicOr(&confirmed[uu >> 5], 1u << (uu & 31));
                          if (xp == (int64_t)uu) atomicOr(&confirmed[x >> 5], 1u << (x & 31));
                      }
                  });
    }
    block_add(errors, err);
}

// Rule 7 (examples/graph500_runner.cu:155-169).
__global__ void bfs_val_confirm_kernel(const int64_t *__restrict__ pred, const int64_t *__restrict__ dist, uint64_t n,
                                       uint64_t root, const unsigned *__restrict__ confirmed,
                                       unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        if (pred[v] == -1) continue;
        const bool conf = (confirmed[v >> 5] >> (v & 31)) & 1u;
        if (dist[v] == INT64_MAX || (v != root && !conf)) ++err;
    }
    block_add(errors, err);
}

__global__ void sssp_val_vertex_kernel(const float *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                       uint64_t root, unsigned *__restrict__ confirmed,
                                       unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const int64_t p = pred[v];
        const float d = dist[v];
        if (v == root) {
            if (d != 0.0f || p != (int64_t)root) ++err;
            atomicOr(&confirmed[v >> 5], 1u << (v & 31));
        }
        if ((p == -1) != (d == -1.0f)) ++err;
        if (p != -1 && (p < 0 || (uint64_t)p >= n)) ++err;
    }
    block_add(errors, err);
}

__global__ void __launch_bounds__(VAL_THREADS, 2) sssp_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                    const int *__restrict__ col,
                                                                    const float *__restrict__ w, uint64_t n,
                                                                    const float *__restrict__ dist,
                                                                    const longlong2 *__restrict__ vx,
                                                                    const unsigned *__restrict__ trow,
                                                                    const unsigned long long *__restrict__ table,
                                                                    unsigned *__restrict__ confirmed,
                                                                    unsigned long long *__restrict__ errors) {
    __shared__ uint64_t s_lo, s_hi;
    __shared__ uint64_t s_rp[VAL_SPAN + 1];
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    unsigned long long err = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        tile_walk(rowptr, col, n, e0, min(e0 + VAL_TILE, E), trow, tab, s_rp, &s_lo, &s_hi,
                  [&](const unsigned *u, uint64_t eb, unsigned ne, const int *c) {
                      // the rows' distances first (one load per row), then every
                      // record of a reached row in flight before the first test
                      float du[VAL_ITEMS];
                      unsigned ur = ~0u;
                      float d = -1.0f;
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          if (k < ne && u[k] != ur) {
                              ur = u[k];
                              d = __ldg(&dist[ur]);
                          }
                          du[k] = k < ne ? d : -1.0f;
                      }
                      longlong2 xv[VAL_ITEMS];
                      float wk[VAL_ITEMS];
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          const unsigned x = (unsigned)c[k];
                          const bool live = du[k] != -1.0f && x < n;
                          xv[k] = live ? __ldg(&vx[x]) : make_longlong2(0, 0);
                          wk[k] = live ? __ldg(&w[eb + k]) : 0.0f;
                      }
#pragma unroll
                      for (int k = 0; k < VAL_ITEMS; ++k) {
                          if (du[k] == -1.0f) continue;
                          const uint64_t x = (unsigned)c[k];
                          if (x >= n) {
                              ++err;
                              continue;
                          }
                          const float dx = __uint_as_float((unsigned)xv[k].x);
                          const float cand = __fadd_rn(du[k], wk[k]);
                          if (dx == -1.0f || cand < dx) ++err;
                          if (xv[k].y == (int64_t)u[k] && cand == dx) atomicOr(&confirmed[x >> 5], 1u << (x & 31));
                      }
                  });
    }
    block_add(errors, err);
}

__global__ void sssp_val_confirm_kernel(const float *__restrict__ dist, uint64_t n,
                                        const unsigned *__restrict__ confirmed,
                                        unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        if (dist[v] != -1.0f && !((confirmed[v >> 5] >> (v & 31)) & 1u)) ++err;
    block_add(errors, err);
}

struct ValWork {
    unsigned *confirmed;
    unsigned long long *counter;  // [0] the result, [1] the tile table is valid
    longlong2 *vx;  // packed neighbour records (16 bytes per vertex)
    unsigned *trow;  // tile table (val_tile_rows_kernel)
    uint64_t tcap;   // its entries: room for graphs of up to 256 entries per vertex on average
    uint64_t bytes;
};

static ValWork carve_val(void *base, uint64_t n) {
    Carver c(base);
    ValWork w;
    w.confirmed = c.take<unsigned>((n + 31) / 32);
    w.counter = c.take<unsigned long long>(32);
    w.vx = c.take<longlong2>(n);
    w.tcap = n / 16 + 2;
    w.trow = c.take<unsigned>(w.tcap);
    w.bytes = c.used;
    return w;
}

// Zeroes the result and the table flag, then builds the tile table.
static int val_tiles(const uint64_t *d_rowstarts, uint64_t n, const ValWork &w, int grid, cudaStream_t st) {
    G5_CUDA_TRY(cudaMemsetAsync(w.counter, 0, 2 * sizeof(unsigned long long), st));
    val_tile_rows_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, n, w.trow, w.tcap, &w.counter[1]);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

static int val_prepare(uint64_t n, void *d_work, uint64_t work_bytes, ValWork *w, int *grid, const char *who) {
    G5_CHECK_ARG(n >= 1 && n <= (1ull << 31), "%s: nverts outside [1, 2^31]", who);
    G5_CHECK_ARG(d_work, "%s: workspace is NULL", who);
    *w = carve_val(d_work, n);
    if (work_bytes < w->bytes) return set_error(G5_ERR_WORKSPACE, "%s: workspace too small", who);
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    *grid = di.sms * 8;
    return G5_OK;
}

static int val_finish(const ValWork &w, uint64_t *out, cudaStream_t st) {
    unsigned long long v = 0;
    G5_CUDA_TRY(cudaGetLastError());
    G5_CUDA_TRY(cudaMemcpyAsync(&v, w.counter, sizeof v, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    *out = v;
    return G5_OK;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_validate_workspace_size(uint64_t nverts, uint64_t *bytes) {
    G5_CHECK_ARG(bytes, "g5_validate_workspace_size: bytes is NULL");
    *bytes = carve_val(nullptr, nverts).bytes;
    return G5_OK;
}

extern "C" int g5_edge_count(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                             const int64_t *d_pred, void *d_work, uint64_t work_bytes, uint64_t *count, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_rowstarts && d_col && d_pred && count, "g5_edge_count: NULL argument");
    ValWork w;
    int grid = 0;
    int rc = val_prepare(nverts, d_work, work_bytes, &w, &grid, "g5_edge_count");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = val_tiles(d_rowstarts, nverts, w, grid, st))) return rc;
    edge_count_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, nverts, d_pred, w.trow, &w.counter[1],
                                                    w.counter);
    return val_finish(w, count, st);
}

extern "C" int g5_bfs_validate(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                               const int64_t *d_pred, const int64_t *d_dist, void *d_work, uint64_t work_bytes,
                               uint64_t *errors, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_rowstarts && d_col && d_pred && d_dist && errors, "g5_bfs_validate: NULL argument");
    G5_CHECK_ARG(root < nverts, "g5_bfs_validate: root out of range");
    ValWork w;
    int grid = 0;
    int rc = val_prepare(nverts, d_work, work_bytes, &w, &grid, "g5_bfs_validate");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.confirmed, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    if ((rc = val_tiles(d_rowstarts, nverts, w, grid, st))) return rc;
    bfs_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_pred, d_dist, nverts, root, w.confirmed, w.counter);
    val_pack_bfs_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, w.vx);
    bfs_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, nverts, d_pred, d_dist, w.vx, w.trow,
                                                      &w.counter[1], w.confirmed, w.counter);
    bfs_val_confirm_kernel<<<grid, VAL_THREADS, 0, st>>>(d_pred, d_dist, nverts, root, w.confirmed, w.counter);
    return val_finish(w, errors, st);
}

extern "C" int g5_sssp_validate(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                                uint64_t root, const float *d_dist, const int64_t *d_pred, void *d_work,
                                uint64_t work_bytes, uint64_t *errors, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_pred && d_dist && errors, "g5_sssp_validate: NULL argument");
    G5_CHECK_ARG(root < nverts, "g5_sssp_validate: root out of range");
    ValWork w;
    int grid = 0;
    int rc = val_prepare(nverts, d_work, work_bytes, &w, &grid, "g5_sssp_validate");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.confirmed, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    if ((rc = val_tiles(d_rowstarts, nverts, w, grid, st))) return rc;
    sssp_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, root, w.confirmed, w.counter);
    val_pack_sssp_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, w.vx);
    sssp_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, d_w, nverts, d_dist, w.vx, w.trow,
                                                       &w.counter[1], w.confirmed, w.counter);
    sssp_val_confirm_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, nverts, w.confirmed, w.counter);
    return val_finish(w, errors, st);
}
