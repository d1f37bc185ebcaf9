// g5_frontier.cuh -- vertex lists ("frontiers") shared by the BFS and SSSP
// persistent kernels.
//
// A list of capacity n holds vertices whose edge range has at most BIG_DEG
// entries at the front ("small" part, counted by a u32) and the others at
// the back ("big" part).  Small vertices are expanded 32 at a time by a
// warp that gathers their edges across its lanes.  Big vertices are cut
// into BIG_CHUNK-edge chunks and every warp of the grid takes chunks from
// one counter: a big entry is appended with a single 64-bit atomicAdd on a
// packed counter (entry count << 40 | chunk count), which hands it both its
// slot j and the id of its first chunk, so chunk bases are sorted by slot
// and a chunk id maps back to its vertex by binary search.
#pragma once

#include "g5_common.cuh"

namespace g5 {

constexpr unsigned BIG_DEG = 4096;
constexpr unsigned BIG_CHUNK = 1024;
constexpr int BIG_SHIFT = 40;
constexpr unsigned long long BIG_LOW = (1ull << BIG_SHIFT) - 1;

#ifdef __CUDACC__

__device__ __forceinline__ unsigned big_count(unsigned long long packed) { return (unsigned)(packed >> BIG_SHIFT); }
__device__ __forceinline__ unsigned long long big_chunks(unsigned long long packed) { return packed & BIG_LOW; }

// Appends v, whose edge range to expand has `deg` entries, to list L of
// capacity n (base[] = chunk bases of the big part).  All 32 lanes call it.
// Returns false (and writes nothing) when the list would overflow, which
// the callers' once-per-list invariants rule out.
__device__ __forceinline__ bool frontier_append(unsigned *L, unsigned *base, uint64_t n, unsigned *n_small,
                                                unsigned long long *big, bool want, unsigned v, uint64_t deg) {
    const bool sm = want && deg <= BIG_DEG;
    const bool bg = want && deg > BIG_DEG;
    bool ok = true;
    const unsigned p = warp_append(n_small, sm);
    if (sm) {
        if (p < n) L[p] = v;
        else ok = false;
    }
    if (bg) {
        const unsigned long long nch = (deg + BIG_CHUNK - 1) / BIG_CHUNK;
        const unsigned long long old = atomicAdd(big, (1ull << BIG_SHIFT) | nch);
        const uint64_t j = old >> BIG_SHIFT;
        if (j < n) {
            L[n - 1 - j] = v;
            base[j] = (unsigned)(old & BIG_LOW);
        } else {
            ok = false;
        }
    }
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
