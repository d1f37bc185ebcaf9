// validate.cu -- K5: Graph500 BFS validation, SSSP validation and the TEPS
// edge count.
//
// The BFS rules and the edge count are the runner's
// (examples/graph500_runner.cu:84-201): same rules, same error count.  The
// reference walks each row with one thread (a hub row of millions of entries
// serialises on that thread); here every edge pass is edge-parallel and
// free of block barriers: a warp takes a tile of 512 consecutive CSR
// entries, each lane 16 of them.  The rows the warp tile spans come from a
// pre-pass table (the row of every tile's first entry, all searched in
// parallel); a lane finds the row of its first entry by a binary search
// inside that span (a few row starts, cached) and steps forward from row to
// row.  The column is read 16 bytes at a time.  A neighbour's two values
// the rules compare (BFS: dist and pred; SSSP: dist and pred) are packed by
// a pre-pass into one 16-byte record, so each entry reads one sector of
// it; a lane issues the record loads of its 16 entries before it tests any
// of them.
//
// HBM bytes per pass: E * 4 (col) [+ E * 4 w] + one random 16-byte record
// per entry (a 32-byte sector).
#include "g5_common.cuh"

namespace g5 {

constexpr int VAL_THREADS = 256;
constexpr int VAL_WTILE = 512;  // entries per warp tile (the tile table's unit)
constexpr int COUNT_ITEMS = 16; // consecutive entries a lane takes per step: edge count
constexpr int RULE_ITEMS = 8;   //   the validators (their neighbour records held in registers)
constexpr int VAL_WIN = 128;    // rows a warp tile's shared window holds

// Largest v in [lo, hi] with rowptr[v] <= e.
__device__ __forceinline__ uint64_t row_of(const uint64_t *__restrict__ rowptr, uint64_t lo, uint64_t hi, uint64_t e) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&rowptr[mid]) <= e) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Tile table: trow[t] = row of entry t * VAL_WTILE for every warp tile t,
// and trow[ntiles] = row of the last entry, when the table has room (the
// pre-pass then sets ok[0]).
__global__ void val_tile_rows_kernel(const uint64_t *__restrict__ rowptr, uint64_t n, unsigned *__restrict__ trow,
                                     uint64_t cap, unsigned long long *__restrict__ ok) {
    const uint64_t E = rowptr[n];
    const uint64_t ntiles = (E + VAL_WTILE - 1) / VAL_WTILE;
    if (E == 0 || ntiles + 1 > cap) return;  // ok stays 0: lanes search all of rowptr themselves
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles; t += stride)
        trow[t] = (unsigned)row_of(rowptr, 0, n - 1, t < ntiles ? t * VAL_WTILE : E - 1);
    if (blockIdx.x == 0 && threadIdx.x == 0) *ok = 1;
}

// Every CSR entry, warp tile by warp tile: calls visit(u, eb, ne, c) per
// lane and step with the lane's ne <= ITEMS consecutive entries eb.. (u[k]
// the row of entry eb + k, c[k] its column entry; lanes past the last
// entry have ne = 0).  A warp tile of VAL_WTILE entries takes
// VAL_WTILE / (32 ITEMS) steps.  No block barrier: each warp runs on its
// own.  With the table, the rows a warp tile spans are known (the row of
// the next tile's first entry bounds them; rows after a lane's entries
// start beyond them and are never stepped into).  When they are fewer
// than VAL_WIN - 1, the warp's shared window holds the starts of the
// tile's rows (coalesced loads of just those rows) and each lane finds the
// row of its first entry by a binary search of the window; otherwise it
// searches rowptr.  From there a lane keeps the next row's start in a
// register: an entry costs one compare unless a row ends there.  All 32
// lanes call it.
template <int ITEMS, class Visit>
__device__ __forceinline__ void warp_walk(const uint64_t *__restrict__ rowptr, const int *__restrict__ col, uint64_t n,
                                          uint64_t E, const unsigned *__restrict__ trow, bool table, Visit visit) {
    static_assert(ITEMS % 4 == 0 && VAL_WTILE % (32 * ITEMS) == 0, "whole int4 loads, whole steps");
    __shared__ int s_win[VAL_THREADS / 32][VAL_WIN];
    int *wrp = s_win[threadIdx.x >> 5];
    const unsigned lane = lane_id();
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t * VAL_WTILE < E; t += nwarps) {
        uint64_t lo = 0, hi = n - 1;
        if (table) {
            lo = __ldg(&trow[t]);
            hi = __ldg(&trow[t + 1]);
        }
        // The window: starts of rows lo .. lo + hi - lo + 1 (the last one
        // starts after the tile's last entry), as 32-bit offsets from the
        // tile's first entry (starts before it clamp to -1, far ones and the
        // unused slots to 2^30), so the lookups below compare 32-bit
        // numbers.
        const uint64_t t0 = t * VAL_WTILE;
        const bool win = table && hi - lo < VAL_WIN - 1;
        __syncwarp();  // the last tile's window is read
        if (win) {
            for (unsigned i = lane; i < VAL_WIN; i += 32) {
                int rp = 1 << 30;
                if (i <= hi - lo + 1 && lo + i <= n) {
                    const uint64_t x = __ldg(&rowptr[lo + i]);
                    rp = x < t0 ? -1 : x - t0 > (1u << 30) ? 1 << 30 : (int)(x - t0);
                }
                wrp[i] = rp;
            }
        }
        __syncwarp();
#pragma unroll 1
        for (int step = 0; step < VAL_WTILE / (32 * ITEMS); ++step) {
            const uint64_t eb = t * VAL_WTILE + (uint64_t)step * 32 * ITEMS + (uint64_t)lane * ITEMS;
            const uint64_t ee = eb < E ? min(eb + (uint64_t)ITEMS, E) : eb;
            const unsigned ne = (unsigned)(ee - eb);
            int c[ITEMS];
            if (ne == ITEMS && ((uintptr_t)(col + eb) & 15) == 0) {
                const int4 *p = reinterpret_cast<const int4 *>(col + eb);
#pragma unroll
                for (int k = 0; k < ITEMS / 4; ++k) {
                    const int4 q = __ldg(p + k);
                    c[4 * k] = q.x;
                    c[4 * k + 1] = q.y;
                    c[4 * k + 2] = q.z;
                    c[4 * k + 3] = q.w;
                }
            } else {
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) c[k] = k < ne ? __ldg(&col[eb + k]) : 0;
            }
            unsigned u[ITEMS];
            if (win) {
                const int el = (int)(eb - t0);  // < VAL_WTILE
                unsigned j = 0;  // largest window row starting at or before eb
#pragma unroll
                for (unsigned s = VAL_WIN / 2; s >= 1; s >>= 1)
                    if (wrp[j + s] <= el) j += s;  // j + s <= VAL_WIN - 1
                // d: this lane's entries before row j + 1 starts.  The row of
                // a real entry is at most hi - lo <= VAL_WIN - 2, and window
                // row hi - lo + 1 starts after the tile's last entry, so the
                // stepping stops by itself (the guard only bounds the index).
                int d = (j + 1 < VAL_WIN ? wrp[j + 1] : 1 << 30) - el;
                const unsigned ul = (unsigned)lo;
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) {
                    if (k < (int)ne) {
                        while (k >= d) {  // a later row starts at or before this entry (past empty rows too)
                            ++j;
                            d = (j + 1 < VAL_WIN ? wrp[j + 1] : 1 << 30) - el;
                        }
                    }
                    u[k] = ul + j;
                }
            } else {
                uint64_t r = ne ? row_of(rowptr, lo, hi, eb) : 0;
                uint64_t next = ne ? __ldg(&rowptr[r + 1]) : ~0ull;
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) {
                    const uint64_t e = eb + k;
                    if (k < ne && e >= next) {  // into a later row: the next one, or past empty rows a search
                        ++r;
                        next = __ldg(&rowptr[r + 1]);
                        if (next <= e) {
                            r = row_of(rowptr, r + 1, hi, e);
                            next = __ldg(&rowptr[r + 1]);
                        }
                    }
                    u[k] = (unsigned)r;
                }
            }
            visit(u, eb, ne, c);
        }
    }
}

__device__ __forceinline__ void block_add(unsigned long long *dst, unsigned long long v) {
    v = warp_sum(v);
    if (lane_id() == 0 && v) atomicAdd(dst, v);
}

// The TEPS edge count walks the CSR as warp_walk does, with two changes for
// its one cheap test per entry: the window also holds each row's reached
// flag (pred != -1, loaded with the row starts, coalesced), and a lane keeps
// its current row, its flag and where the next row starts in registers, so
// an entry costs a compare and an add unless a row ends at it.
__global__ void __launch_bounds__(VAL_THREADS) edge_count_kernel(const uint64_t *__restrict__ rowptr,
                                                                 const int *__restrict__ col, uint64_t n,
                                                                 const int64_t *__restrict__ pred,
                                                                 const unsigned *__restrict__ trow,
                                                                 const unsigned long long *__restrict__ table,
                                                                 unsigned long long *__restrict__ out) {
    constexpr int ITEMS = COUNT_ITEMS;
    __shared__ int s_win[VAL_THREADS / 32][VAL_WIN];
    __shared__ unsigned char s_reach[VAL_THREADS / 32][VAL_WIN];
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    int *wrp = s_win[threadIdx.x >> 5];
    unsigned char *wrc = s_reach[threadIdx.x >> 5];
    const unsigned lane = lane_id();
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long cnt = 0;
    for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; t * VAL_WTILE < E; t += nwarps) {
        uint64_t lo = 0, hi = n - 1;
        if (tab) {
            lo = __ldg(&trow[t]);
            hi = __ldg(&trow[t + 1]);
        }
        const uint64_t t0 = t * VAL_WTILE;
        const bool win = tab && hi - lo < VAL_WIN - 1;
        __syncwarp();  // the last tile's window is read
        if (win) {
            for (unsigned i = lane; i < VAL_WIN; i += 32) {
                int rp = 1 << 30;
                unsigned char rc = 0;
                if (i <= hi - lo + 1 && lo + i <= n) {
                    const uint64_t x = __ldg(&rowptr[lo + i]);
                    rp = x < t0 ? -1 : x - t0 > (1u << 30) ? 1 << 30 : (int)(x - t0);
                    rc = lo + i < n && __ldg(&pred[lo + i]) != -1;
                }
                wrp[i] = rp;
                wrc[i] = rc;
            }
        }
        __syncwarp();
#pragma unroll 1
        for (int step = 0; step < VAL_WTILE / (32 * ITEMS); ++step) {
            const uint64_t eb = t0 + (uint64_t)step * 32 * ITEMS + (uint64_t)lane * ITEMS;
            const uint64_t ee = eb < E ? min(eb + (uint64_t)ITEMS, E) : eb;
            const unsigned ne = (unsigned)(ee - eb);
            if (!ne) continue;
            int c[ITEMS];
            if (ne == ITEMS && ((uintptr_t)(col + eb) & 15) == 0) {
                const int4 *p = reinterpret_cast<const int4 *>(col + eb);
#pragma unroll
                for (int k = 0; k < ITEMS / 4; ++k) {
                    const int4 q = __ldg(p + k);
                    c[4 * k] = q.x;
                    c[4 * k + 1] = q.y;
                    c[4 * k + 2] = q.z;
                    c[4 * k + 3] = q.w;
                }
            } else {
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) c[k] = k < ne ? __ldg(&col[eb + k]) : 0;
            }
            unsigned local = 0;
            if (win) {
                const int el = (int)(eb - t0);
                unsigned j = 0;  // largest window row starting at or before eb
#pragma unroll
                for (unsigned s2 = VAL_WIN / 2; s2 >= 1; s2 >>= 1)
                    if (wrp[j + s2] <= el) j += s2;
                int d = (j + 1 < VAL_WIN ? wrp[j + 1] : 1 << 30) - el;
                unsigned u = (unsigned)lo + j;
                bool reached = wrc[j];
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) {
                    if (k < (int)ne) {
                        if (k >= d) {  // a later row starts at or before this entry (past empty rows too)
                            do {
                                ++j;
                                d = (j + 1 < VAL_WIN ? wrp[j + 1] : 1 << 30) - el;
                            } while (k >= d);
                            u = (unsigned)lo + j;
                            reached = wrc[j];
                        }
                        local += reached && (unsigned)c[k] <= u;
                    }
                }
            } else {
                uint64_t r = row_of(rowptr, lo, hi, eb);
                uint64_t next = __ldg(&rowptr[r + 1]);
                bool reached = __ldg(&pred[r]) != -1;
#pragma unroll
                for (int k = 0; k < ITEMS; ++k) {
                    const uint64_t e = eb + k;
                    if (k < (int)ne) {
                        if (e >= next) {  // into a later row: the next one, or past empty rows a search
                            ++r;
                            next = __ldg(&rowptr[r + 1]);
                            if (next <= e) {
                                r = row_of(rowptr, r + 1, hi, e);
                                next = __ldg(&rowptr[r + 1]);
                            }
                            reached = __ldg(&pred[r]) != -1;
                        }
                        local += reached && (unsigned)c[k] <= (unsigned)r;
                    }
                }
            }
            cnt += local;
        }
    }
    block_add(out, cnt);
}

// A vertex's values for the edge rules, packed into one 16-byte record in
// the CSR's numbering: BFS {dist, pred}; SSSP {dist bits, pred}.  With a
// renumbered CSR (perm: caller's vertex -> CSR's, inv back) record v holds
// caller's vertex inv[v], its parent renamed by perm (-1 kept; a parent
// that is not a vertex becomes -2, which equals no vertex, as the raw value
// did).
__device__ __forceinline__ int64_t val_parent(int64_t p, uint64_t n, const unsigned *perm) {
    if (!perm || p == -1) return p;
    return p >= 0 && (uint64_t)p < n ? (int64_t)__ldg(&perm[p]) : -2;
}

__global__ void val_pack_bfs_kernel(const int64_t *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                    const unsigned *__restrict__ perm, const unsigned *__restrict__ inv,
                                    longlong2 *__restrict__ vx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint64_t o = inv ? __ldg(&inv[v]) : v;
        vx[v] = make_longlong2(dist[o], val_parent(pred[o], n, perm));
    }
}

__global__ void val_pack_sssp_kernel(const float *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                     const unsigned *__restrict__ perm, const unsigned *__restrict__ inv,
                                     longlong2 *__restrict__ vx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const uint64_t o = inv ? __ldg(&inv[v]) : v;
        vx[v] = make_longlong2((long long)__float_as_uint(dist[o]), val_parent(pred[o], n, perm));
    }
}

// Rules 1-2 (examples/graph500_runner.cu:84-109).
__global__ void bfs_val_vertex_kernel(const int64_t *__restrict__ pred, const int64_t *__restrict__ dist, uint64_t n,
                                      uint64_t root, const unsigned *__restrict__ perm,
                                      unsigned *__restrict__ confirmed, unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const int64_t p = pred[v];
        if (p != -1 && (p < 0 || (uint64_t)p >= n)) ++err;
        if (v == root) {
            if (p != (int64_t)root || dist[v] != 0) ++err;
            else {
                const uint64_t r = perm ? __ldg(&perm[v]) : v;  // the bitmap is in the CSR's numbering
                atomicOr(&confirmed[r >> 5], 1u << (r & 31));
            }
        }
    }
    block_add(errors, err);
}

// Rules 3-6 (examples/graph500_runner.cu:111-153), one thread per CSR entry.
__global__ void __launch_bounds__(VAL_THREADS, 2) bfs_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                   const int *__restrict__ col, uint64_t n,
                                                                   const longlong2 *__restrict__ vx,
                                                                   const unsigned *__restrict__ trow,
                                                                   const unsigned long long *__restrict__ table,
                                                                   unsigned *__restrict__ confirmed,
                                                                   unsigned long long *__restrict__ errors) {
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    unsigned long long err = 0;
    warp_walk<RULE_ITEMS>(rowptr, col, n, E, trow, tab,
              [&](const unsigned *u, uint64_t, unsigned ne, const int *c) {
                  // every neighbour record in flight before the first test
                  longlong2 xv[RULE_ITEMS];
#pragma unroll
                  for (int k = 0; k < RULE_ITEMS; ++k) {
                      const unsigned x = (unsigned)c[k];
                      xv[k] = k < ne && x < n ? __ldg(&vx[x]) : make_longlong2(0, 0);
                  }
                  unsigned ur = ~0u;
                  int64_t ud = 0, up = 0;
#pragma unroll
                  for (int k = 0; k < RULE_ITEMS; ++k) {
                      if (k >= ne) break;
                      const unsigned uu = u[k];
                      const uint64_t x = (unsigned)c[k];
                      if (x == uu || x >= n) {  // a self-loop entry, or not a vertex (counted once, nothing else compared)
                          ++err;
                          continue;
                      }
                      if (uu != ur) {  // the row's own record
                          ur = uu;
                          const longlong2 uv = __ldg(&vx[uu]);
                          ud = uv.x;
                          up = uv.y;
                      }
                      const int64_t xd = xv[k].x, xp = xv[k].y;
                      if ((ud == -1) != (xd == -1)) ++err;
                      if (ud >= 0 && xd >= 0 && (ud + 1 < xd || xd + 1 < ud)) ++err;
                      if (up == (int64_t)x) atomicOr(&confirmed[uu >> 5], 1u << (uu & 31));
                      if (xp == (int64_t)uu) atomicOr(&confirmed[x >> 5], 1u << (x & 31));
                  }
              });
    block_add(errors, err);
}

// Rule 7 (examples/graph500_runner.cu:155-169), over the records (the
// CSR's numbering; root = the root's number there).
__global__ void bfs_val_confirm_kernel(const longlong2 *__restrict__ vx, uint64_t n, uint64_t root,
                                       const unsigned *__restrict__ confirmed,
                                       unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const longlong2 r = vx[v];
        if (r.y == -1) continue;
        const bool conf = (confirmed[v >> 5] >> (v & 31)) & 1u;
        if (r.x == INT64_MAX || (v != root && !conf)) ++err;
    }
    block_add(errors, err);
}

__global__ void sssp_val_vertex_kernel(const float *__restrict__ dist, const int64_t *__restrict__ pred, uint64_t n,
                                       uint64_t root, const unsigned *__restrict__ perm,
                                       unsigned *__restrict__ confirmed, unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
        const int64_t p = pred[v];
        const float d = dist[v];
        if (v == root) {
            if (d != 0.0f || p != (int64_t)root) ++err;
            const uint64_t r = perm ? __ldg(&perm[v]) : v;  // the bitmap is in the CSR's numbering
            atomicOr(&confirmed[r >> 5], 1u << (r & 31));
        }
        if ((p == -1) != (d == -1.0f)) ++err;
        if (p != -1 && (p < 0 || (uint64_t)p >= n)) ++err;
    }
    block_add(errors, err);
}

__global__ void __launch_bounds__(VAL_THREADS, 3) sssp_val_edge_kernel(const uint64_t *__restrict__ rowptr,
                                                                    const int *__restrict__ col,
                                                                    const float *__restrict__ w, uint64_t n,
                                                                    const longlong2 *__restrict__ vx,
                                                                    const unsigned *__restrict__ trow,
                                                                    const unsigned long long *__restrict__ table,
                                                                    unsigned *__restrict__ confirmed,
                                                                    unsigned long long *__restrict__ errors) {
    const uint64_t E = rowptr[n];
    const bool tab = *table != 0;
    unsigned long long err = 0;
    warp_walk<RULE_ITEMS>(rowptr, col, n, E, trow, tab,
              [&](const unsigned *u, uint64_t eb, unsigned ne, const int *c) {
                  // the rows' distances first (one load per row), then every
                  // record of a reached row in flight before the first test
                  float du[RULE_ITEMS];
                  unsigned ur = ~0u;
                  float d = -1.0f;
#pragma unroll
                  for (int k = 0; k < RULE_ITEMS; ++k) {
                      if (k < ne && u[k] != ur) {  // the row's own record
                          ur = u[k];
                          d = __uint_as_float((unsigned)__ldg(&vx[ur]).x);
                      }
                      du[k] = k < ne ? d : -1.0f;
                  }
                  longlong2 xv[RULE_ITEMS];
                  float wk[RULE_ITEMS];
#pragma unroll
                  for (int k = 0; k < RULE_ITEMS; ++k) {
                      const unsigned x = (unsigned)c[k];
                      const bool live = du[k] != -1.0f && x < n;
                      xv[k] = live ? __ldg(&vx[x]) : make_longlong2(0, 0);
                      wk[k] = live ? __ldg(&w[eb + k]) : 0.0f;
                  }
#pragma unroll
                  for (int k = 0; k < RULE_ITEMS; ++k) {
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
    block_add(errors, err);
}

__global__ void sssp_val_confirm_kernel(const longlong2 *__restrict__ vx, uint64_t n,
                                        const unsigned *__restrict__ confirmed,
                                        unsigned long long *__restrict__ errors) {
    unsigned long long err = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
        if (__uint_as_float((unsigned)vx[v].x) != -1.0f && !((confirmed[v >> 5] >> (v & 31)) & 1u)) ++err;
    block_add(errors, err);
}

struct ValWork {
    unsigned *confirmed;
    unsigned long long *counter;  // [0] the result, [1] the tile table is valid
    longlong2 *vx;  // packed neighbour records (16 bytes per vertex)
    unsigned *trow;  // tile table (val_tile_rows_kernel)
    uint64_t tcap;   // its entries: room for graphs of up to 128 entries per vertex on average
    uint64_t bytes;
};

static ValWork carve_val(void *base, uint64_t n) {
    Carver c(base);
    ValWork w;
    w.confirmed = c.take<unsigned>((n + 31) / 32);
    w.counter = c.take<unsigned long long>(32);
    w.vx = c.take<longlong2>(n);
    w.tcap = n / 4 + 2;
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

extern "C" int g5_bfs_validate_renumbered(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                                          uint64_t root, const int64_t *d_pred, const int64_t *d_dist,
                                          const uint32_t *d_perm, const uint32_t *d_inv, void *d_work,
                                          uint64_t work_bytes, uint64_t *errors, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_rowstarts && d_col && d_pred && d_dist && errors, "g5_bfs_validate: NULL argument");
    G5_CHECK_ARG(root < nverts, "g5_bfs_validate: root out of range");
    G5_CHECK_ARG((d_perm == nullptr) == (d_inv == nullptr), "g5_bfs_validate: give both perm and inv or neither");
    ValWork w;
    int grid = 0;
    int rc = val_prepare(nverts, d_work, work_bytes, &w, &grid, "g5_bfs_validate");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.confirmed, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    if ((rc = val_tiles(d_rowstarts, nverts, w, grid, st))) return rc;
    uint64_t root_csr = root;
    if (d_perm) {
        uint32_t r = 0;
        G5_CUDA_TRY(cudaMemcpyAsync(&r, d_perm + root, sizeof r, cudaMemcpyDeviceToHost, st));
        G5_CUDA_TRY(cudaStreamSynchronize(st));
        root_csr = r;
    }
    bfs_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_pred, d_dist, nverts, root, d_perm, w.confirmed,
                                                        w.counter);
    val_pack_bfs_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, d_perm, d_inv, w.vx);
    bfs_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, nverts, w.vx, w.trow, &w.counter[1],
                                                      w.confirmed, w.counter);
    bfs_val_confirm_kernel<<<grid, VAL_THREADS, 0, st>>>(w.vx, nverts, root_csr, w.confirmed, w.counter);
    return val_finish(w, errors, st);
}

extern "C" int g5_bfs_validate(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                               const int64_t *d_pred, const int64_t *d_dist, void *d_work, uint64_t work_bytes,
                               uint64_t *errors, void *stream) {
    return g5_bfs_validate_renumbered(d_rowstarts, d_col, nverts, root, d_pred, d_dist, nullptr, nullptr, d_work,
                                      work_bytes, errors, stream);
}

extern "C" int g5_sssp_validate_renumbered(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                                           uint64_t nverts, uint64_t root, const float *d_dist,
                                           const int64_t *d_pred, const uint32_t *d_perm, const uint32_t *d_inv,
                                           void *d_work, uint64_t work_bytes, uint64_t *errors, void *stream) {
    clear_error();
    G5_CHECK_ARG(d_rowstarts && d_col && d_w && d_pred && d_dist && errors, "g5_sssp_validate: NULL argument");
    G5_CHECK_ARG(root < nverts, "g5_sssp_validate: root out of range");
    G5_CHECK_ARG((d_perm == nullptr) == (d_inv == nullptr), "g5_sssp_validate: give both perm and inv or neither");
    ValWork w;
    int grid = 0;
    int rc = val_prepare(nverts, d_work, work_bytes, &w, &grid, "g5_sssp_validate");
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    G5_CUDA_TRY(cudaMemsetAsync(w.confirmed, 0, (nverts + 31) / 32 * sizeof(unsigned), st));
    if ((rc = val_tiles(d_rowstarts, nverts, w, grid, st))) return rc;
    sssp_val_vertex_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, root, d_perm, w.confirmed,
                                                         w.counter);
    val_pack_sssp_kernel<<<grid, VAL_THREADS, 0, st>>>(d_dist, d_pred, nverts, d_perm, d_inv, w.vx);
    sssp_val_edge_kernel<<<grid, VAL_THREADS, 0, st>>>(d_rowstarts, d_col, d_w, nverts, w.vx, w.trow, &w.counter[1],
                                                       w.confirmed, w.counter);
    sssp_val_confirm_kernel<<<grid, VAL_THREADS, 0, st>>>(w.vx, nverts, w.confirmed, w.counter);
    return val_finish(w, errors, st);
}

extern "C" int g5_sssp_validate(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                                uint64_t root, const float *d_dist, const int64_t *d_pred, void *d_work,
                                uint64_t work_bytes, uint64_t *errors, void *stream) {
    return g5_sssp_validate_renumbered(d_rowstarts, d_col, d_w, nverts, root, d_dist, d_pred, nullptr, nullptr,
                                       d_work, work_bytes, errors, stream);
}
