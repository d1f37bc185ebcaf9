/*
 * nvshmem.h -- single-PE stand-in for the NVSHMEM calls that
 * RuanPetrus/cuda-graph-traversal makes (src/base.cu:41,69,
 * src/traversal.cu:26-233, src/worker.cu:46-61,
 * examples/graph500_runner.cu:96-168,213-244).
 *
 * With one processing element every remote operation targets this GPU's own
 * memory, so:
 *   get / put        -> volatile load / store (bypasses a stale L1 line)
 *   atomics          -> the matching CUDA atomic in L2
 *   nvshmem_quiet    -> __threadfence()
 *   barrier_all      -> __threadfence() on the device, cudaDeviceSynchronize()
 *                       on the host
 *   malloc / free    -> cudaMalloc / cudaFree
 * The `pe` arguments must be 0; they are otherwise ignored.
 */
#ifndef G5_SHIM_NVSHMEM_H
#define G5_SHIM_NVSHMEM_H

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#define G5_SHMEM_HD static inline __host__ __device__
#define G5_SHMEM_D static inline __device__

G5_SHMEM_HD int nvshmem_my_pe(void) { return 0; }
G5_SHMEM_HD int nvshmem_n_pes(void) { return 1; }

G5_SHMEM_HD void nvshmem_quiet(void) {
#ifdef __CUDA_ARCH__
    __threadfence();
#endif
}
G5_SHMEM_HD void nvshmem_fence(void) { nvshmem_quiet(); }

G5_SHMEM_HD void nvshmem_barrier_all(void) {
#ifdef __CUDA_ARCH__
    __threadfence();
#else
    cudaDeviceSynchronize();
#endif
}

static inline void *nvshmem_malloc(size_t bytes) {
    void *p = NULL;
    if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) return NULL;
    return p;
}
static inline void nvshmem_free(void *p) {
    if (p) cudaFree(p);
}
static inline void nvshmem_init(void) {}
static inline void nvshmem_finalize(void) {}

/* Typed get / put / atomics.  NAME is the NVSHMEM type tag, T the C type,
 * A the type CUDA's atomic intrinsics take for the same bits. */
#define G5_SHMEM_RMA(NAME, T)                                                         \
    G5_SHMEM_D T nvshmem_##NAME##_g(const T *src, int pe) {                           \
        (void)pe;                                                                     \
        return *(const volatile T *)src;                                              \
    }                                                                                 \
    G5_SHMEM_D void nvshmem_##NAME##_p(T *dst, T value, int pe) {                     \
        (void)pe;                                                                     \
        *(volatile T *)dst = value;                                                   \
    }

#define G5_SHMEM_AMO(NAME, T, A)                                                      \
    G5_SHMEM_D void nvshmem_##NAME##_atomic_add(T *dst, T value, int pe) {            \
        (void)pe;                                                                     \
        atomicAdd((A *)dst, (A)value);                                                \
    }                                                                                 \
    G5_SHMEM_D T nvshmem_##NAME##_atomic_fetch_add(T *dst, T value, int pe) {         \
        (void)pe;                                                                     \
        return (T)atomicAdd((A *)dst, (A)value);                                      \
    }                                                                                 \
    G5_SHMEM_D void nvshmem_##NAME##_atomic_inc(T *dst, int pe) {                     \
        (void)pe;                                                                     \
        atomicAdd((A *)dst, (A)1);                                                    \
    }                                                                                 \
    G5_SHMEM_D T nvshmem_##NAME##_atomic_compare_swap(T *dst, T cond, T value, int pe) { \
        (void)pe;                                                                     \
        return (T)atomicCAS((A *)dst, (A)cond, (A)value);                             \
    }                                                                                 \
    G5_SHMEM_D T nvshmem_##NAME##_atomic_fetch(const T *src, int pe) {                \
        (void)pe;                                                                     \
        return *(const volatile T *)src;                                              \
    }

G5_SHMEM_RMA(int, int)
G5_SHMEM_RMA(uint, unsigned int)
G5_SHMEM_RMA(int32, int32_t)
G5_SHMEM_RMA(uint32, uint32_t)
G5_SHMEM_RMA(int64, int64_t)
G5_SHMEM_RMA(uint64, uint64_t)
G5_SHMEM_RMA(longlong, long long)
G5_SHMEM_RMA(ulonglong, unsigned long long)
G5_SHMEM_RMA(float, float)
G5_SHMEM_RMA(double, double)

G5_SHMEM_AMO(int, int, int)
G5_SHMEM_AMO(uint, unsigned int, unsigned int)
G5_SHMEM_AMO(int32, int32_t, int)
G5_SHMEM_AMO(uint32, uint32_t, unsigned int)
G5_SHMEM_AMO(int64, int64_t, unsigned long long)
G5_SHMEM_AMO(uint64, uint64_t, unsigned long long)
G5_SHMEM_AMO(longlong, long long, unsigned long long)
G5_SHMEM_AMO(ulonglong, unsigned long long, unsigned long long)

#undef G5_SHMEM_RMA
#undef G5_SHMEM_AMO

#endif /* G5_SHIM_NVSHMEM_H */
