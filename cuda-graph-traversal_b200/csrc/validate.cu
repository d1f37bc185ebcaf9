// validate.cu -- K5: Graph500 BFS validation, SSSP validation and the TEPS
// edge count.
//
// The BFS rules and the edge count are the runner's
// (examples/graph500_runner.cu:84-201): same rules, same error count.  The
// reference walks each row with one thread (a hub row of millions of entries
// serialises on that thread); here every edge pass is edge-parallel: a block
// takes a fixed tile of CSR entries and each entry finds its row by a short
// binary search inside the tile's row span, so the work per thread is the
// same whatever the degree distribution.
//
// HBM bytes per pass: E * 4 (col) [+ E * 4 w] + random 8-byte reads of the
// neighbour's pred/dist per entry.
#include "g5_common.cuh"

namespace g5 {

constexpr int VAL_THREADS = 256;
constexpr int VAL_TILE = VAL_THREADS * 8;

// Largest v in [lo, hi] with rowptr[v] <= e.
__device__ __forceinline__ uint64_t row_of(const uint64_t *__restrict__ rowptr, uint64_t lo, uint64_t hi, uint64_t e) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&rowptr[mid]) <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Row span of the tile [e0, e1) of the CSR, into shared memory.
__device__ __forceinline__ void tile_rows(const uint64_t *__restrict__ rowptr, uint64_t n, uint64_t e0, uint64_t e1,
                                          uint64_t *s_lo, uint64_t *s_hi) {
    if (threadIdx.x == 0) {
        *s_lo = row_of(rowptr, 0, n - 1, e0);
        *s_hi = row_of(rowptr, *s_lo, n - 1, e1 - 1);
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
                                                                 unsigned long long *__restrict__ out) {
    __shared__ uint64_t s_lo, s_hi;
    const uint64_t E = rowptr[n];
    unsigned long long cnt = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        const uint64_t e1 = min(e0 + VAL_TILE, E);
        tile_rows(rowptr, n, e0, e1, &s_lo, &s_hi);
        for (uint64_t e = e0 + threadIdx.x; e < e1; e += VAL_THREADS) {
            const uint64_t v = row_of(rowptr, s_lo, s_hi, e);
            if (pred[v] != -1 && (uint64_t)(unsigned)__ldg(&col[e]) <= v) ++cnt;
        }
        __syncthreads();
    }
    block_add(out, cnt);
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
__global__ void __launch_bounds__(VAL_THREADS) bfs_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                   const int *__restrict__ col, uint64_t n,
                                                                   const int64_t *__restrict__ pred,
                                                                   const int64_t *__restrict__ dist,
                                                                   unsigned *__restrict__ confirmed,
                                                                   unsigned long long *__restrict__ errors) {
    __shared__ uint64_t s_lo, s_hi;
    const uint64_t E = rowptr[n];
    unsigned long long err = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        const uint64_t e1 = min(e0 + VAL_TILE, E);
        tile_rows(rowptr, n, e0, e1, &s_lo, &s_hi);
        for (uint64_t e = e0 + threadIdx.x; e < e1; e += VAL_THREADS) {
            const uint64_t u = row_of(rowptr, s_lo, s_hi, e);
            const uint64_t x = (unsigned)__ldg(&col[e]);
            if (x == u) {
                ++err;
                continue;
            }
            if (x >= n) {  // not a vertex: counted once, nothing else to compare
                ++err;
                continue;
            }
            const int64_t ud = dist[u], xd = dist[x], up = pred[u], xp = pred[x];
            if ((ud == -1) != (xd == -1)) ++err;
            if (ud >= 0 && xd >= 0 && (ud + 1 < xd || xd + 1 < ud)) ++err;
            if (up == (int64_t)x) atomicOr(&confirmed[u >> 5], 1u << (u & 31));
            if (xp == (int64_t)u) atomicOr(&confirmed[x >> 5], 1u << (x & 31));
        }
        __syncthreads();
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

__global__ void __launch_bounds__(VAL_THREADS) sssp_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                    const int *__restrict__ col,
                                                                    const float *__restrict__ w, uint64_t n,
                                                                    const float *__restrict__ dist,
                                                                    const int64_t *__restrict__ pred,
                                                                    unsigned *__restrict__ confirmed,
                                                                    unsigned long long *__restrict__ errors) {
    __shared__ uint64_t s_lo, s_hi;
    const uint64_t E = rowptr[n];
    unsigned long long err = 0;
    for (uint64_t e0 = (uint64_t)blockIdx.x * VAL_TILE; e0 < E; e0 += (uint64_t)gridDim.x * VAL_TILE) {
        const uint64_t e1 = min(e0 + VAL_TILE, E);
        tile_rows(rowptr, n, e0, e1, &s_lo, &s_hi);
        for (uint64_t e = e0 + threadIdx.x; e < e1; e += VAL_THREADS) {
            const uint64_t u = row_of(rowptr, s_lo, s_hi, e);
            const float du = dist[u];
            if (du == -1.0f) continue;
            const uint64_t x = (unsigned)__ldg(&col[e]);
            if (x >= n) {
                ++err;
                continue;
            }
            const float dx = dist[x];
            const float cand = __fadd_rn(du, __ldg(&w[e]));
            if (dx == -1.0f || cand < dx) ++err;
            if (pred[x] == (int64_t)u && cand == dx) atomicOr(&confirmed[x >> 5], 1u << (x & 31));
        }
        __syncthreads();
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
    unsigned long long *counter;
    uint64_t bytes;
};

static ValWork carve_val(void *base, uint64_t n) {
    Carver c(base);
    ValWork w;
    w.confirmed = c.take<unsigned>((n + 31) / 32);
    w.counter = c.take<unsigned long long>(32);
    w.bytes = c.used;
    return w;
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
    G5_CUDA_TRY(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), st));
    edge_count_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, nverts, d_pred, w.counter);
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
    G5_CUDA_TRY(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), st));
    bfs_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_pred, d_dist, nverts, root, w.confirmed, w.counter);
    bfs_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, nverts, d_pred, d_dist, w.confirmed,
                                                      w.counter);
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
    G5_CUDA_TRY(cudaMemsetAsync(w.counter, 0, sizeof(unsigned long long), st));
    sssp_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, root, w.confirmed, w.counter);
    sssp_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, d_w, nverts, d_dist, d_pred, w.confirmed,
                                                       w.counter);
    sssp_val_confirm_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, nverts, w.confirmed, w.counter);
    return val_finish(w, errors, st);
}
