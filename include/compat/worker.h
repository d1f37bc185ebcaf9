/*
 * worker.h -- drop-in for RuanPetrus/cuda-graph-traversal src/worker.h.
 *
 * Worker_State keeps the reference's layout (src/worker.h:6-12).  This
 * implementation is one process on one GPU: rank 0 of 1, no MPI and no
 * NVSHMEM; the GPU arena is plain device memory.  worker_kernel_launch runs
 * any kernel as a CUDA cooperative launch capped at the co-resident grid and
 * synchronises, like the reference's NVSHMEM collective launch
 * (src/worker.cu:69-101).
 */
#ifndef WORKER_H
#define WORKER_H
#include "base.h"

typedef struct Worker_State Worker_State;
struct Worker_State {
    Arena cpu_arena;
    Arena gpu_arena;
    i32 rank;
    i32 rank_size;
    i32 pes_on_device;
};

/* gpu_memory_size 0: the reference's default sizing -- free device memory
 * minus max(half of it, 512 MiB) (src/worker.cu:28-38). */
Worker_State worker_init(i32 argc, char **argv, u64 gpu_memory_size);
void worker_finalize(Worker_State *ws);
void worker_abort(Worker_State *ws, i32 return_code);
i32 worker_kernel_block_count(Worker_State *ws, const void *kernel, void **args, u64 work_count,
                              i32 threads_per_block, const char *label);
i32 worker_kernel_launch(Worker_State *ws, const void *kernel, void **args, u64 work_count, i32 threads_per_block,
                         const char *label);
void *_worker_arena_push_array(Worker_State *ws, u64 local_count, u64 elem_size, u64 alignment, u64 *max_count_out);

#define worker_arena_push_array(ws, count, type, max_count_out) \
    ((type *)_worker_arena_push_array((ws), (count), sizeof(type), alignof(type), (max_count_out)))

#endif /* WORKER_H */
