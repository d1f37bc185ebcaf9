// g5_common.cuh -- shared host and device helpers of libg500b.
//
// Host side: thread-local error message, CUDA error mapping, workspace
// carving, device properties.  Device side: bounded grid barrier for the
// persistent cooperative kernels, warp scans and warp-aggregated appends,
// bitmap helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>

#include "g500b.h"

namespace g5 {

// ------------------------------------------------------------------ host --

int set_error(int code, const char *fmt, ...);
void clear_error();

#define G5_CUDA_TRY(call)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return ::g5::set_error(G5_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,  \
                                   cudaGetErrorString(e_));                                 \
    } while (0)

#define G5_CHECK_ARG(cond, ...)                                                             \
    do {                                                                                    \
        if (!(cond)) return ::g5::set_error(G5_ERR_INVALID, __VA_ARGS__);                   \
    } while (0)

inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Sequential carve-out of a caller-provided workspace, 256-byte aligned.
struct Carver {
    char *base;
    uint64_t used = 0;
    explicit Carver(void *b) : base((char *)b) {}
    template <class T>
    T *take(uint64_t count) {
        used = align_up(used, 256);
        T *p = base ? (T *)(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
};

struct DeviceInfo {
    int device;
    int sms;
    int max_threads_per_sm;
};
int device_info(DeviceInfo *out);

// Device-side error flags reported through a control word.
enum : unsigned {
    DEVERR_TIMEOUT = 1u,    // a bounded wait gave up
    DEVERR_RANGE = 2u,      // an input value outside its documented range
    DEVERR_CAPACITY = 4u,   // an internal list would have overflowed
    DEVERR_DEPTH = 8u,      // a batched search went deeper than its depth planes hold
    DEVERR_UNPREPARED = 16u, // a batched-search workspace was not prepared for this graph
    DEVERR_RING = 32u,      // an SSSP relaxation landed beyond the bucket ring (delta too small for the weights)
    DEVERR_DUPLICATE = 64u, // an SSSP queue held a vertex twice (reported only by the checked opens)
};
int deverr_to_status(unsigned flags, const char *what);

// Bytes of an L2 persisting access-policy window to use for a region of
// `want` bytes (0 = none): min(want, the device's window limit), after
// reserving that much persisting L2 for this process's context once per
// device.  G5_L2_PERSIST=0 disables it.
int l2_persist_window(uint64_t want, uint64_t *bytes);

// Exclusive scan (csr.cu): out[0..n] = prefix sums of in[0..n) widened to
// u64, out[n] = total; `scratch` holds scan_scratch_words(n) u64.
int scan_u32_to_u64(const unsigned *in, uint64_t n, uint64_t *out, uint64_t *scratch, cudaStream_t st);
inline uint64_t scan_scratch_words(uint64_t n) { return (n + 4095) / 4096 + 1; }

// Function attributes shared by the persistent (cooperative) search kernels,
// set before their occupancy is first queried.
int persistent_kernel_setup(const void *fn);

// Wait limit of the persistent kernels' grid barriers, nanoseconds
// (G5_WAIT_LIMIT_MS overrides; default 2000 ms).
unsigned long long wait_limit_ns();

// -------------------------------------------------------------- device --

#ifdef __CUDACC__

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

template <class T>
__device__ __forceinline__ T ld_volatile(const T *p) {
    return *(const volatile T *)p;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Grid-wide barrier for a cooperative launch.  `count` only grows: the
// barrier with sequence number `epoch` (1, 2, ...) completes when
// count == epoch * nblocks.  The wait is bounded by `limit_ns`; on expiry
// (or when another block already flagged an error) it sets `*error`,
// returns false and the caller must leave its loop.  Returns true when every
// block arrived.
__device__ __forceinline__ bool grid_sync(unsigned *count, unsigned *error, unsigned &epoch, unsigned nblocks,
                                          unsigned long long limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        const unsigned target = epoch * nblocks;
        const unsigned long long t0 = globaltimer_ns();
        int ok = 1;
        while (ld_acquire(count) < target) {
            if (ld_volatile(error)) { ok = 0; break; }
            if (globaltimer_ns() - t0 > limit_ns) {
                atomicOr(error, DEVERR_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        s_ok = ok && !ld_volatile(error);
    }
    __syncthreads();
    return s_ok;
}

template <class T>
__device__ __forceinline__ T warp_incl_scan(T x) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(FULL, x, d);
        if ((int)lane_id() >= d) x += y;
    }
    return x;
}

template <class T>
__device__ __forceinline__ T warp_sum(T x) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(FULL, x, d);
    return x;
}

// Warp-aggregated append: every lane with `want` gets a distinct slot of
// `*counter`; returns the slot (undefined for lanes without `want`).  All 32
// lanes must call it.
__device__ __forceinline__ unsigned warp_append(unsigned *counter, bool want) {
    unsigned mask = __ballot_sync(FULL, want);
    if (!mask) return 0;
    unsigned leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
    base = __shfl_sync(FULL, base, leader);
    return base + __popc(mask & lanemask_lt());
}

// Lane j (largest) with excl_j <= e, over a warp's exclusive prefix values.
__device__ __forceinline__ int warp_owner(unsigned excl, unsigned e) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        unsigned v = __shfl_sync(FULL, excl, lo + step < 32 ? lo + step : 31);
        if (lo + step < 32 && v <= e) lo += step;
    }
    return lo;
}

// p[0 .. n) = x for the calling grid (thread t of T), with 16-byte stores
// once p is 16-byte aligned (sizeof(T) is 4 or 8).
template <class T>
__device__ __forceinline__ void grid_fill(T *p, uint64_t n, T x, uint64_t t, uint64_t T_) {
    constexpr uint64_t per = 16 / sizeof(T);
    const uint64_t mis = ((uintptr_t)p & 15) / sizeof(T);
    const uint64_t head = mis ? (per - mis < n ? per - mis : n) : 0;
    if (t < head) p[t] = x;
    const uint64_t nvec = (n - head) / per;
    T v[per];
#pragma unroll
    for (uint64_t k = 0; k < per; ++k) v[k] = x;
    const uint4 q = *reinterpret_cast<const uint4 *>(v);
    uint4 *pv = reinterpret_cast<uint4 *>(p + head);
    for (uint64_t i = t; i < nvec; i += T_) pv[i] = q;
    for (uint64_t i = head + nvec * per + t; i < n; i += T_) p[i] = x;
}

__device__ __forceinline__ bool bit_test(const unsigned *bm, unsigned v) { return (bm[v >> 5] >> (v & 31)) & 1u; }

// Sets bit v; true when this call changed it from 0 to 1.
__device__ __forceinline__ bool bit_claim(unsigned *bm, unsigned v) {
    const unsigned bit = 1u << (v & 31);
    if (bm[v >> 5] & bit) return false;
    return !(atomicOr(&bm[v >> 5], bit) & bit);
}

#endif  // __CUDACC__

}  // namespace g5
