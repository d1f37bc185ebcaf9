/*
 * nvshmemx.h -- single-PE stand-in for the NVSHMEM extension calls of
 * RuanPetrus/cuda-graph-traversal: bootstrap (src/worker.cu:46-50) and the
 * collective kernel launch (src/worker.cu:69-101).
 *
 * A collective launch is a CUDA cooperative launch: the runtime refuses a
 * grid that cannot be co-resident, so kernels that spin on a software grid
 * barrier never wait on a block that has not been scheduled.  Both launch
 * calls return 0 on success and non-zero otherwise, as NVSHMEM does.
 */
#ifndef G5_SHIM_NVSHMEMX_H
#define G5_SHIM_NVSHMEMX_H

#include "nvshmem.h"

typedef struct nvshmemx_init_attr {
    void *mpi_comm;
    size_t heap_size;
    void *args;
} nvshmemx_init_attr_t;

#define NVSHMEMX_INIT_THREAD_PES 0x1
#define NVSHMEMX_INIT_WITH_MPI_COMM 0x2
#define NVSHMEMX_INIT_WITH_SHMEM 0x4
#define NVSHMEMX_INIT_WITH_UNIQUEID 0x8

static inline int nvshmemx_init_attr(unsigned int flags, nvshmemx_init_attr_t *attr) {
    (void)flags; (void)attr;
    return 0;
}

static inline int nvshmemx_collective_launch_query_gridsize(const void *kernel, dim3 block, void **args,
                                                            size_t smem, int *grid) {
    (void)args;
    int per_sm = 0, sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)(block.x * block.y * block.z),
                                                      smem) != cudaSuccess)
        return 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
    *grid = per_sm * sms;
    return *grid > 0 ? 0 : 1;
}

static inline int nvshmemx_collective_launch(const void *kernel, dim3 grid, dim3 block, void **args, size_t smem,
                                             cudaStream_t stream) {
    return cudaLaunchCooperativeKernel(kernel, grid, block, args, smem, stream) == cudaSuccess ? 0 : 1;
}

#endif /* G5_SHIM_NVSHMEMX_H */
