// g5_frontier.cuh -- vertex lists ("frontiers") shared by the BFS and SSSP
// persistent kernels.
//
// A list of capacity n holds vertices whose edge range has at most BIG_DEG
// entries at the front ("small" part, counted by a u32) and the others at
// the back ("big" part).  Small vertices are expanded a few at a time (the
// grab size adapts to the list length, up to 32) by a warp that gathers
// their edges across its lanes, so a short list of heavy vertices still
// spreads over the whole grid.  Big vertices are cut into BIG_CHUNK-edge
// chunks and every warp of the grid takes chunks from one counter, so no
// vertex's edges serialise on one warp.  Big entries are
// appended with one 64-bit atomicAdd per warp on a packed counter
// (entry count << 40 | chunk count), which hands out slots and first-chunk
// ids in the same order, so chunk bases are sorted by slot and a chunk id
// maps back to its vertex by binary search.
#pragma once

#include "g5_common.cuh"

namespace g5 {

constexpr unsigned BIG_DEG = 1024;
constexpr unsigned BIG_CHUNK = 1024;

// Entries per grab over a small part of ns entries: about four grabs per
// warp, between 1 and `cap` (at most 32).
__host__ __device__ __forceinline__ unsigned grab_size(unsigned ns, unsigned long long nwarps, unsigned cap = 32) {
    unsigned long long g = ns / (4 * nwarps);
    return g < 1 ? 1u : g > cap ? cap : (unsigned)g;
}
constexpr int BIG_SHIFT = 40;
constexpr unsigned long long BIG_LOW = (1ull << BIG_SHIFT) - 1;

#ifdef __CUDACC__

__device__ __forceinline__ unsigned big_count(unsigned long long packed) { return (unsigned)(packed >> BIG_SHIFT); }
__device__ __forceinline__ unsigned long long big_chunks(unsigned long long packed) { return packed & BIG_LOW; }

// Appends v, whose edge range to expand has `deg` entries, to list L of
// capacity n (base[] = chunk bases of the big part): the small part when
// deg <= big_deg, else the big part.  All 32 lanes call it.  Returns false
// (and writes nothing) when the list would overflow, which the callers'
// once-per-list invariants rule out.
__device__ __forceinline__ bool frontier_append(unsigned *L, unsigned *base, uint64_t n, unsigned *n_small,
                                                unsigned long long *big, bool want, unsigned v, uint64_t deg,
                                                unsigned big_deg = BIG_DEG, unsigned chunk = BIG_CHUNK) {
    const bool sm = want && deg <= big_deg;
    const bool bg = want && deg > big_deg;
    bool ok = true;
    const unsigned p = warp_append(n_small, sm);
    if (sm) {
        if (p < n) L[p] = v;
        else ok = false;
    }
    const unsigned bmask = __ballot_sync(FULL, bg);
    if (bmask) {
        const unsigned nch = bg ? (unsigned)((deg + chunk - 1) / chunk) : 0u;
        const unsigned incl = warp_incl_scan(nch);
        const unsigned total = __shfl_sync(FULL, incl, 31);
        const unsigned leader = __ffs(bmask) - 1;
        unsigned long long old = 0;
        if (lane_id() == leader) old = atomicAdd(big, ((unsigned long long)__popc(bmask) << BIG_SHIFT) | total);
        old = __shfl_sync(FULL, old, leader);
        if (bg) {
            const uint64_t j = (old >> BIG_SHIFT) + __popc(bmask & lanemask_lt());
            if (j < n) {
                L[n - 1 - j] = v;
                base[j] = (unsigned)((old & BIG_LOW) + incl - nch);
            } else {
                ok = false;
            }
        }
    }
    return ok;
}

// Per-warp staging of a list's small part in shared memory.  A warp
// appends into its own slice with ballots only, and when the slice is full
// it reserves a range of the global list with one atomicAdd and copies the
// slice out (coalesced).  A frontier of millions of vertices then costs one
// global atomic per `cap` entries instead of one per warp step on a single
// counter, and no block-wide synchronisation is needed.
struct WarpStage {
    unsigned *buf;  // this warp's slice (shared), cap entries, cap >= 32
    unsigned *cnt;  // this warp's fill count (shared)
    unsigned cap;
};

__device__ __forceinline__ bool stage_flush_warp(const WarpStage &q, unsigned *L, uint64_t n, unsigned *gcount) {
    __syncwarp();
    const unsigned c = *q.cnt;
    if (!c) return true;
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(gcount, c);
    base = __shfl_sync(FULL, base, 0);
    const bool ok = (uint64_t)base + c <= n;
    if (ok)
        for (unsigned i = lane_id(); i < c; i += 32) L[base + i] = q.buf[i];
    __syncwarp();
    if (lane_id() == 0) *q.cnt = 0;
    __syncwarp();
    return ok;
}

// Appends v for every lane with `want`.  All 32 lanes call it.
__device__ __forceinline__ bool stage_append(const WarpStage &q, bool want, unsigned v, unsigned *L, uint64_t n,
                                             unsigned *gcount) {
    const unsigned mask = __ballot_sync(FULL, want);
    if (!mask) return true;
    bool ok = true;
    unsigned c = *q.cnt;
    if (c + __popc(mask) > q.cap) {
        ok = stage_flush_warp(q, L, n, gcount);
        c = 0;
    }
    if (want) q.buf[c + __popc(mask & lanemask_lt())] = v;
    __syncwarp();
    if (lane_id() == 0) *q.cnt = c + __popc(mask);
    __syncwarp();
    return ok;
}

// frontier_append with the small part staged per warp.  All lanes call it.
__device__ __forceinline__ bool frontier_append_staged(const WarpStage &q, unsigned *L, unsigned *basearr, uint64_t n,
                                                       unsigned *n_small, unsigned long long *big, bool want,
                                                       unsigned v, uint64_t deg, unsigned big_deg = BIG_DEG,
                                                       unsigned chunk = BIG_CHUNK) {
    bool ok = stage_append(q, want && deg <= big_deg, v, L, n, n_small);
    ok &= frontier_append(L, basearr, n, n_small, big, want && deg > big_deg, v, deg, big_deg, chunk);
    return ok;
}

// Slot j of the big part whose chunks contain chunk c (largest j with
// base[j] <= c); base[0] == 0.
__device__ __forceinline__ unsigned chunk_owner(const unsigned *base, unsigned nb, unsigned c) {
    unsigned lo = 0, hi = nb - 1;
    while (lo < hi) {
        const unsigned mid = (lo + hi + 1) >> 1;
        if (__ldcg(&base[mid]) <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

#endif  // __CUDACC__

}  // namespace g5
