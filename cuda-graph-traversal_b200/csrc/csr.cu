// csr.cu -- K2: CSR build from the Kronecker edge list (the reference's
// oned_graph_from_tuple_graph, src/traversal.cu:342-389, at one rank).
//
//   count:  degree of every vertex over non-self-loop edges (one 32-bit
//           atomic per endpoint, as compute_degrees_kernel :15-34), then a
//           three-pass parallel exclusive scan into rowstarts (the
//           reference uses one GPU thread for it, :37-46).
//   fill:   both directions of every non-loop edge scattered into its row
//           (fill_csr_kernel :48-73): light entries (w < delta) from the row
//           start upward, heavy ones from the row end downward, so every row
//           is split for delta-stepping with no extra pass.  Duplicates are
//           kept, like the reference; in-row order depends on atomic order
//           in both.
//
// HBM bytes per edge: count reads 16; fill reads 20 and writes 2 x (4 col +
// 4 w [+ 8 col64]) scattered.
#include "g5_common.cuh"
#include "g5_mrg.cuh"

namespace g5 {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
static_assert(SCAN_TILE == 4096, "scan_scratch_words assumes 4096-item tiles");

__global__ void csr_degree_kernel(const ulonglong2 *__restrict__ edges, uint64_t m, uint64_t n,
                                  unsigned *__restrict__ deg, unsigned *__restrict__ err) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        ulonglong2 e = edges[i];
        if (e.x >= n || e.y >= n) {
            atomicOr(err, DEVERR_RANGE);
            continue;
        }
        if (e.x == e.y) continue;
        atomicAdd(&deg[e.x], 1u);
        atomicAdd(&deg[e.y], 1u);
    }
}

// Tile sums of a u32 array (first pass of the scan).
__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_sums(const unsigned *__restrict__ in, uint64_t n,
                                                               uint64_t *__restrict__ tile_sums) {
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint64_t s = 0;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        uint64_t i = base + (uint64_t)j * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    s = warp_sum(s);
    __shared__ uint64_t ws[SCAN_THREADS / 32];
    if (lane_id() == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t v = threadIdx.x < SCAN_THREADS / 32 ? ws[threadIdx.x] : 0;
        v = warp_sum(v);
        if (threadIdx.x == 0) tile_sums[blockIdx.x] = v;
    }
}

// Exclusive scan of the tile sums in place by one block; total -> *total.
__global__ void __launch_bounds__(1024) scan_tile_offsets(uint64_t *__restrict__ tile_sums, uint64_t ntiles,
                                                          uint64_t *__restrict__ total) {
    __shared__ uint64_t wsum[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < ntiles; base += 1024) {
        uint64_t i = base + threadIdx.x;
        uint64_t v = i < ntiles ? tile_sums[i] : 0;
        uint64_t incl = warp_incl_scan(v);
        if (lane_id() == 31) wsum[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            uint64_t w = wsum[threadIdx.x];
            uint64_t wi = warp_incl_scan(w);
            wsum[threadIdx.x] = wi - w;
        }
        __syncthreads();
        uint64_t excl = carry + wsum[threadIdx.x >> 5] + incl - v;
        if (i < ntiles) tile_sums[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// out[i] = offset(tile) + exclusive prefix within the tile; out[n] = total.
// The tile is staged in shared memory (padded one slot per 32) so that both
// the loads and the stores stay coalesced while each thread scans 16
// consecutive items.
__device__ __forceinline__ int scan_pad(int i) { return i + (i >> 5); }

__global__ void __launch_bounds__(SCAN_THREADS) scan_tile_apply(const unsigned *__restrict__ in, uint64_t n,
                                                                const uint64_t *__restrict__ tile_offsets,
                                                                const uint64_t *__restrict__ total,
                                                                uint64_t *__restrict__ out) {
    __shared__ uint64_t s[SCAN_TILE + SCAN_TILE / 32];
    __shared__ uint64_t s_warp[SCAN_THREADS / 32];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int k = j * SCAN_THREADS + threadIdx.x;
        s[scan_pad(k)] = base + k < n ? in[base + k] : 0u;
    }
    __syncthreads();
    uint64_t sum = 0;
    for (int j = 0; j < SCAN_ITEMS; ++j) sum += s[scan_pad(threadIdx.x * SCAN_ITEMS + j)];
    uint64_t incl = warp_incl_scan(sum);
    if (lane_id() == 31) s_warp[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t w = threadIdx.x < SCAN_THREADS / 32 ? s_warp[threadIdx.x] : 0;
        uint64_t wi = warp_incl_scan(w);
        if (threadIdx.x < SCAN_THREADS / 32) s_warp[threadIdx.x] = wi - w;
    }
    __syncthreads();
    uint64_t run = tile_offsets[blockIdx.x] + s_warp[threadIdx.x >> 5] + incl - sum;
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int k = scan_pad(threadIdx.x * SCAN_ITEMS + j);
        uint64_t v = s[k];
        s[k] = run;
        run += v;
    }
    __syncthreads();
    for (int j = 0; j < SCAN_ITEMS; ++j) {
        int k = j * SCAN_THREADS + threadIdx.x;
        if (base + k < n) out[base + k] = s[scan_pad(k)];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *total;
}

// out[0..n] = exclusive prefix of in[0..n) (u32 -> u64); `scratch` holds
// ceil(n / 4096) + 1 u64.
int scan_u32_to_u64(const unsigned *in, uint64_t n, uint64_t *out, uint64_t *scratch, cudaStream_t st) {
    const uint64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    uint64_t *total = scratch + ntiles;
    if (ntiles == 0) {
        G5_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(uint64_t), st));
        return G5_OK;
    }
    scan_tile_sums<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(in, n, scratch);
    scan_tile_offsets<<<1, 1024, 0, st>>>(scratch, ntiles, total);
    scan_tile_apply<<<(unsigned)ntiles, SCAN_THREADS, 0, st>>>(in, n, scratch, total, out);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

__global__ void csr_fill_kernel(const ulonglong2 *__restrict__ edges, const float *__restrict__ weights, uint64_t m,
                                uint64_t n, const uint64_t *__restrict__ rowstarts, float delta,
                                unsigned *__restrict__ lo, unsigned *__restrict__ hi, int *__restrict__ col,
                                float *__restrict__ w, uint64_t *__restrict__ col64) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        ulonglong2 e = edges[i];
        if (e.x >= n || e.y >= n || e.x == e.y) continue;
        const float wt = weights[i];
        const bool light = wt < delta;
        uint64_t pa, pb;
        if (light) {
            pa = rowstarts[e.x] + atomicAdd(&lo[e.x], 1u);
            pb = rowstarts[e.y] + atomicAdd(&lo[e.y], 1u);
        } else {
            pa = rowstarts[e.x + 1] - 1 - atomicAdd(&hi[e.x], 1u);
            pb = rowstarts[e.y + 1] - 1 - atomicAdd(&hi[e.y], 1u);
        }
        // Counted by g5_csr_count over the same edges, each row has exactly
        // the room its entries need; other input could not stay in bounds.
        if (pa >= rowstarts[e.x + 1] || pa < rowstarts[e.x] || pb >= rowstarts[e.y + 1] || pb < rowstarts[e.y])
            continue;
        col[pa] = (int)e.y;
        w[pa] = wt;
        col[pb] = (int)e.x;
        w[pb] = wt;
        if (col64) {
            col64[pa] = e.y;
            col64[pb] = e.x;
        }
    }
}

// Generator fused into the CSR passes: each thread walks its edges of the
// Kronecker stream (as kron_generate_kernel) and counts (FILL = false) or
// scatters (FILL = true) them directly, so the 20-byte-per-edge edge list is
// never written or read.  Both passes regenerate the same edges.
template <bool FILL>
__global__ void __launch_bounds__(256) kron_csr_kernel(KronLaunch k, uint64_t n, const uint64_t *__restrict__ rowstarts,
                                                       float delta, unsigned *__restrict__ lo,
                                                       unsigned *__restrict__ hi, int *__restrict__ col,
                                                       float *__restrict__ w, uint64_t *__restrict__ col64) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    if (t >= k.count) return;
    MrgState z = kron_thread_start(k, t);
    for (int64_t i = t; i < k.count; i += T) {
        uint64_t a, b;
        float wt;
        kron_edge(z, k.log_n, k.val0, k.val1, a, b, wt);
        mrg_apply(k.stride_jump, z);
        if (a == b) continue;  // ids are < 2^log_n = n by construction
        if (!FILL) {
            atomicAdd(&lo[a], 1u);
            atomicAdd(&lo[b], 1u);
            continue;
        }
        uint64_t pa, pb;
        if (wt < delta) {
            pa = rowstarts[a] + atomicAdd(&lo[a], 1u);
            pb = rowstarts[b] + atomicAdd(&lo[b], 1u);
        } else {
            pa = rowstarts[a + 1] - 1 - atomicAdd(&hi[a], 1u);
            pb = rowstarts[b + 1] - 1 - atomicAdd(&hi[b], 1u);
        }
        if (pa >= rowstarts[a + 1] || pa < rowstarts[a] || pb >= rowstarts[b + 1] || pb < rowstarts[b]) continue;
        col[pa] = (int)b;
        w[pa] = wt;
        col[pb] = (int)a;
        w[pb] = wt;
        if (col64) {
            col64[pa] = b;
            col64[pb] = a;
        }
    }
}

struct CsrWork {
    unsigned *deg;    // degrees, then heavy cursors
    unsigned *lo;     // light cursors when the caller keeps no light degrees
    uint64_t *scan;   // scan scratch
    unsigned *err;
    uint64_t bytes;
};

static CsrWork carve_csr(void *base, uint64_t n) {
    Carver c(base);
    CsrWork w;
    w.deg = c.take<unsigned>(n);
    w.lo = c.take<unsigned>(n);
    w.scan = c.take<uint64_t>((n + SCAN_TILE - 1) / SCAN_TILE + 1);
    w.err = c.take<unsigned>(64);
    w.bytes = c.used;
    return w;
}

// One graph's CSR copied into a larger one at vertex offset vbase and
// entry offset ebase (disjoint graphs packed into one CSR).
__global__ void csr_pack_rows_kernel(const uint64_t *__restrict__ src_rs, uint64_t n, uint64_t vbase, uint64_t ebase,
                                     const uint32_t *__restrict__ src_ld, uint64_t *__restrict__ dst_rs,
                                     uint32_t *__restrict__ dst_ld) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
        dst_rs[vbase + i] = ebase + src_rs[i];
        if (src_ld && i < n) dst_ld[vbase + i] = src_ld[i];
    }
}

__global__ void csr_pack_entries_kernel(const int *__restrict__ src_col, const float *__restrict__ src_w, uint64_t m,
                                        uint64_t vbase, int *__restrict__ dst_col, float *__restrict__ dst_w) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
        dst_col[e] = (int)((uint64_t)src_col[e] + vbase);
        if (src_w) dst_w[e] = src_w[e];
    }
}

static int grid_for(uint64_t items, int threads) {
    DeviceInfo di;
    if (device_info(&di)) return 1;
    uint64_t b = (items + threads - 1) / threads;
    uint64_t cap = (uint64_t)di.sms * (di.max_threads_per_sm / threads) * 4;
    if (b > cap) b = cap;
    return b ? (int)b : 1;
}

}  // namespace g5

using namespace g5;

extern "C" int g5_csr_workspace_size(uint64_t nverts, uint64_t nedges, uint64_t *bytes) {
    (void)nedges;
    G5_CHECK_ARG(bytes, "g5_csr_workspace_size: bytes is NULL");
    *bytes = carve_csr(nullptr, nverts).bytes;
    return G5_OK;
}

extern "C" int g5_csr_count(const uint64_t *d_edges, uint64_t nedges, uint64_t nverts, uint64_t *d_rowstarts,
                            void *d_work, uint64_t work_bytes, uint64_t *nentries, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_count: nverts %llu outside [1, 2^31]",
                 (unsigned long long)nverts);
    G5_CHECK_ARG(d_rowstarts && d_work && nentries, "g5_csr_count: NULL argument");
    G5_CHECK_ARG(nedges == 0 || d_edges, "g5_csr_count: edges is NULL");
    CsrWork w = carve_csr(d_work, nverts);
    if (work_bytes < w.bytes)
        return set_error(G5_ERR_WORKSPACE, "g5_csr_count: workspace %llu < %llu bytes",
                         (unsigned long long)work_bytes, (unsigned long long)w.bytes);
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.deg, 0, nverts * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.err, 0, sizeof(unsigned), st));
    if (nedges) {
        csr_degree_kernel<<<grid_for(nedges, 256), 256, 0, st>>>((const ulonglong2 *)d_edges, nedges, nverts, w.deg,
                                                                 w.err);
        G5_CUDA_TRY(cudaGetLastError());
    }
    int rc = scan_u32_to_u64(w.deg, nverts, d_rowstarts, w.scan, st);
    if (rc) return rc;
    unsigned err = 0;
    G5_CUDA_TRY(cudaMemcpyAsync(nentries, d_rowstarts + nverts, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaMemcpyAsync(&err, w.err, sizeof err, cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    if (err) return set_error(G5_ERR_INVALID, "g5_csr_count: an edge endpoint is >= nverts");
    return G5_OK;
}

extern "C" int g5_csr_fill(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                           const uint64_t *d_rowstarts, float light_delta, void *d_work, uint64_t work_bytes,
                           int32_t *d_col, float *d_w, uint64_t *d_col64, uint32_t *d_light_deg, void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_fill: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_work && d_col && d_w, "g5_csr_fill: NULL argument");
    G5_CHECK_ARG(nedges == 0 || (d_edges && d_weights), "g5_csr_fill: edges or weights NULL");
    CsrWork w = carve_csr(d_work, nverts);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_fill: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *lo = d_light_deg ? d_light_deg : w.lo;
    G5_CUDA_TRY(cudaMemsetAsync(lo, 0, nverts * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.deg, 0, nverts * sizeof(unsigned), st));
    if (nedges) {
        csr_fill_kernel<<<grid_for(nedges, 256), 256, 0, st>>>((const ulonglong2 *)d_edges, d_weights, nedges, nverts,
                                                               d_rowstarts, light_delta, lo, w.deg, d_col, d_w,
                                                               d_col64);
        G5_CUDA_TRY(cudaGetLastError());
    }
    return G5_OK;
}

extern "C" int g5_csr_count_kronecker(const uint32_t seed[5], uint32_t log_n, uint64_t nedges, uint64_t *d_rowstarts,
                                      void *d_work, uint64_t work_bytes, uint64_t *nentries, void *stream) {
    clear_error();
    G5_CHECK_ARG(log_n >= 1 && log_n <= 31, "g5_csr_count_kronecker: log_n %u outside [1, 31]", log_n);
    G5_CHECK_ARG(d_rowstarts && d_work && nentries, "g5_csr_count_kronecker: NULL argument");
    const uint64_t n = 1ull << log_n;
    KronLaunch k;
    int blocks = 0;
    int rc = kron_prepare(seed, log_n, 0, (int64_t)nedges, 256, &k, &blocks, "g5_csr_count_kronecker");
    if (rc) return rc;
    CsrWork w = carve_csr(d_work, n);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_count_kronecker: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.deg, 0, n * sizeof(unsigned), st));
    if (nedges) {
        kron_csr_kernel<false><<<blocks, 256, 0, st>>>(k, n, nullptr, 0.0f, w.deg, nullptr, nullptr, nullptr, nullptr);
        G5_CUDA_TRY(cudaGetLastError());
    }
    if ((rc = scan_u32_to_u64(w.deg, n, d_rowstarts, w.scan, st))) return rc;
    G5_CUDA_TRY(cudaMemcpyAsync(nentries, d_rowstarts + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    G5_CUDA_TRY(cudaStreamSynchronize(st));
    return G5_OK;
}

extern "C" int g5_csr_fill_kronecker(const uint32_t seed[5], uint32_t log_n, uint64_t nedges,
                                     const uint64_t *d_rowstarts, float light_delta, void *d_work, uint64_t work_bytes,
                                     int32_t *d_col, float *d_w, uint64_t *d_col64, uint32_t *d_light_deg,
                                     void *stream) {
    clear_error();
    G5_CHECK_ARG(log_n >= 1 && log_n <= 31, "g5_csr_fill_kronecker: log_n %u outside [1, 31]", log_n);
    G5_CHECK_ARG(d_rowstarts && d_work && d_col && d_w, "g5_csr_fill_kronecker: NULL argument");
    const uint64_t n = 1ull << log_n;
    KronLaunch k;
    int blocks = 0;
    int rc = kron_prepare(seed, log_n, 0, (int64_t)nedges, 256, &k, &blocks, "g5_csr_fill_kronecker");
    if (rc) return rc;
    CsrWork w = carve_csr(d_work, n);
    if (work_bytes < w.bytes) return set_error(G5_ERR_WORKSPACE, "g5_csr_fill_kronecker: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *lo = d_light_deg ? d_light_deg : w.lo;
    G5_CUDA_TRY(cudaMemsetAsync(lo, 0, n * sizeof(unsigned), st));
    G5_CUDA_TRY(cudaMemsetAsync(w.deg, 0, n * sizeof(unsigned), st));
    if (nedges) {
        kron_csr_kernel<true><<<blocks, 256, 0, st>>>(k, n, d_rowstarts, light_delta, lo, w.deg, d_col, d_w, d_col64);
        G5_CUDA_TRY(cudaGetLastError());
    }
    return G5_OK;
}

// Tiny-first order of each row's light part.  One warp per row.  Short
// parts (at most 32 entries) are reordered in registers; longer ones are
// counted (t tiny entries), then every non-tiny entry among the first t is
// swapped with a tiny entry after them, the k-th with the k-th, both found
// by warp-wide scans that queue up to 63 positions of each kind; each round
// swaps up to 32 pairs (one per lane).  In place, the multiset of the row
// unchanged.
__global__ void __launch_bounds__(256) csr_split_tiny_kernel(const uint64_t *__restrict__ rowptr, int *col, float *w,
                                                             uint64_t *col64, const unsigned *__restrict__ ld,
                                                             uint64_t n, float tiny, unsigned *__restrict__ td) {
    __shared__ unsigned s_q[8][2][64];  // per warp: queued head / tail positions (row offsets)
    const unsigned lane = lane_id(), wib = threadIdx.x >> 5;
    unsigned *hq = s_q[wib][0], *tq = s_q[wib][1];
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint64_t rb = __ldg(&rowptr[v]);
        const unsigned L = __ldg(&ld[v]);
        if (L <= 32) {
            const bool has = lane < L;
            const float wt = has ? w[rb + lane] : 0.0f;
            const int c = has ? col[rb + lane] : 0;
            const uint64_t c64 = has && col64 ? col64[rb + lane] : 0;
            const bool t = has && wt < tiny;
            const unsigned tm = __ballot_sync(FULL, t), om = __ballot_sync(FULL, has && !t);
            const unsigned nt = __popc(tm);
            __syncwarp();
            if (has) {
                const unsigned to = t ? __popc(tm & lanemask_lt()) : nt + __popc(om & lanemask_lt());
                w[rb + to] = wt;
                col[rb + to] = c;
                if (col64) col64[rb + to] = c64;
            }
            if (lane == 0) td[v] = nt;
            continue;
        }
        unsigned t = 0;
        for (unsigned i = lane; i < L; i += 32) t += w[rb + i] < tiny;
        t = warp_sum(t);
        unsigned h = 0, tc = t, nh = 0, nt = 0;
        for (;;) {
            // Refill both queues to at least 32 entries (or to the end of their range).
            while (nh < 32 && h < t) {
                const unsigned i = h + lane;
                const bool m = i < t && !(w[rb + i] < tiny);
                const unsigned bm = __ballot_sync(FULL, m);
                if (m) hq[nh + __popc(bm & lanemask_lt())] = i;
                nh += __popc(bm);
                h += 32;
                __syncwarp();
            }
            while (nt < 32 && tc < L) {
                const unsigned i = tc + lane;
                const bool m = i < L && w[rb + i] < tiny;
                const unsigned bm = __ballot_sync(FULL, m);
                if (m) tq[nt + __popc(bm & lanemask_lt())] = i;
                nt += __popc(bm);
                tc += 32;
                __syncwarp();
            }
            const unsigned k = min(min(nh, nt), 32u);  // one pair per lane
            if (k == 0) break;  // equal counts of misplaced entries: both queues run dry together
            if (lane < k) {
                const uint64_t a = rb + hq[lane], b = rb + tq[lane];
                const float wa = w[a], wb = w[b];
                const int ca = col[a], cb = col[b];
                w[a] = wb;
                w[b] = wa;
                col[a] = cb;
                col[b] = ca;
                if (col64) {
                    const uint64_t xa = col64[a], xb = col64[b];
                    col64[a] = xb;
                    col64[b] = xa;
                }
            }
            __syncwarp();
            // Drop the k swapped positions from the front of each queue (up
            // to 63 entries stay: two per lane).
            const unsigned hr = nh - k, tr = nt - k;
            const unsigned h0 = lane < hr ? hq[k + lane] : 0u, h1 = lane + 32 < hr ? hq[k + lane + 32] : 0u;
            const unsigned t0 = lane < tr ? tq[k + lane] : 0u, t1 = lane + 32 < tr ? tq[k + lane + 32] : 0u;
            __syncwarp();
            if (lane < hr) hq[lane] = h0;
            if (lane + 32 < hr) hq[lane + 32] = h1;
            if (lane < tr) tq[lane] = t0;
            if (lane + 32 < tr) tq[lane + 32] = t1;
            nh = hr;
            nt = tr;
            __syncwarp();
        }
        if (lane == 0) td[v] = t;
    }
}

extern "C" int g5_csr_split_tiny(const uint64_t *d_rowstarts, int32_t *d_col, float *d_w, uint64_t *d_col64,
                                 const uint32_t *d_light_deg, uint64_t nverts, float light_delta, uint32_t *d_tiny_deg,
                                 void *stream) {
    clear_error();
    G5_CHECK_ARG(nverts >= 1 && nverts <= (1ull << 31), "g5_csr_split_tiny: nverts outside [1, 2^31]");
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_light_deg && d_tiny_deg, "g5_csr_split_tiny: NULL argument");
    G5_CHECK_ARG(light_delta > 0.0f, "g5_csr_split_tiny: light_delta must be positive");
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    const float tiny = light_delta / (float)G5_TINY_DIV;
    const uint64_t want = (nverts + 7) / 8;  // blocks of 8 warps, one row each
    const unsigned blocks = (unsigned)std::min<uint64_t>(want, (uint64_t)di.sms * 8);
    csr_split_tiny_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d_rowstarts, d_col, d_w, d_col64, d_light_deg,
                                                                    nverts, tiny, d_tiny_deg);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}

extern "C" int g5_csr_pack_append(const uint64_t *d_src_rowstarts, const int32_t *d_src_col, const float *d_src_w,
                                  const uint32_t *d_src_light_deg, uint64_t src_nverts, uint64_t src_nentries,
                                  uint64_t vbase, uint64_t ebase, uint64_t *d_dst_rowstarts, int32_t *d_dst_col,
                                  float *d_dst_w, uint32_t *d_dst_light_deg, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_src_rowstarts && d_dst_rowstarts && (src_nentries == 0 || (d_src_col && d_dst_col)),
                 "g5_csr_pack_append: NULL argument");
    G5_CHECK_ARG(!d_src_w == !d_dst_w && !d_src_light_deg == !d_dst_light_deg,
                 "g5_csr_pack_append: weights / light counts given on one side only");
    G5_CHECK_ARG(vbase + src_nverts <= (1ull << 31), "g5_csr_pack_append: packed graph above 2^31 vertices");
    cudaStream_t st = (cudaStream_t)stream;
    csr_pack_rows_kernel<<<grid_for(src_nverts + 1, 256), 256, 0, st>>>(d_src_rowstarts, src_nverts, vbase, ebase,
                                                                         d_src_light_deg, d_dst_rowstarts,
                                                                         d_dst_light_deg);
    if (src_nentries)
        csr_pack_entries_kernel<<<grid_for(src_nentries, 256), 256, 0, st>>>(
            d_src_col, d_src_w, src_nentries, vbase, d_dst_col + ebase, d_dst_w ? d_dst_w + ebase : nullptr);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}
