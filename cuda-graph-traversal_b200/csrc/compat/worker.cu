// worker.cu -- Worker_State of the reference's src/worker.h on one GPU
// (src/worker.cu:6-109 without MPI and NVSHMEM).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "compat_internal.h"
#include "worker.h"

Worker_State worker_init(i32 argc, char **argv, u64 gpu_memory_size) {
    (void)argc;
    (void)argv;
    Worker_State ws;
    memset(&ws, 0, sizeof ws);
    ws.rank = 0;
    ws.rank_size = 1;
    ws.pes_on_device = 1;
    i32 devices = 0;
    CHECK_CUDA(cudaGetDeviceCount(&devices));
    if (devices <= 0) {
        ERROR("Rank %d: no CUDA devices available", ws.rank);
        exit(1);
    }
    CHECK_CUDA(cudaSetDevice(ws.rank % devices));
    if (gpu_memory_size == 0) {
        // The reference's default: free memory minus max(half, 512 MiB).
        size_t free_b = 0, total_b = 0;
        CHECK_CUDA(cudaMemGetInfo(&free_b, &total_b));
        u64 avail = (u64)free_b / (u64)ws.pes_on_device;
        u64 reserve = MAX(avail / 2, (u64)MEGABYTE(512));
        gpu_memory_size = avail > reserve ? avail - reserve : avail / 2;
    }
    ws.cpu_arena = arena_create_cpu(MEGABYTE(256));
    ws.gpu_arena = arena_create_gpu(gpu_memory_size);
    return ws;
}

void worker_finalize(Worker_State *ws) {
    CHECK_CUDA(cudaDeviceSynchronize());
    arena_release_gpu(&ws->gpu_arena);
    arena_release_cpu(&ws->cpu_arena);
}

void worker_abort(Worker_State *ws, i32 return_code) {
    worker_finalize(ws);
    exit(return_code);
}

i32 worker_kernel_block_count(Worker_State *ws, const void *kernel, void **args, u64 work_count,
                              i32 threads_per_block, const char *label) {
    (void)args;
    i32 per_sm = 0, sms = 0, dev = 0;
    CHECK_CUDA(cudaGetDevice(&dev));
    CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads_per_block, 0));
    CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    i32 resident = per_sm * sms / MAX(ws->pes_on_device, 1);
    if (resident <= 0) {
        ERROR("Kernel %s cannot be resident with %d threads per block", label, threads_per_block);
        worker_abort(ws, 1);
    }
    u64 needed = MAX(INT_CEIL(work_count, (u64)threads_per_block), (u64)1);
    return needed > (u64)resident ? resident : (i32)needed;
}

i32 worker_kernel_launch(Worker_State *ws, const void *kernel, void **args, u64 work_count, i32 threads_per_block,
                         const char *label) {
    i32 blocks = worker_kernel_block_count(ws, kernel, args, work_count, threads_per_block, label);
    cudaError_t e = cudaLaunchCooperativeKernel(kernel, dim3(blocks), dim3(threads_per_block), args, 0, 0);
    if (e != cudaSuccess) {
        ERROR("Cooperative launch failed for %s: %s", label, cudaGetErrorString(e));
        worker_abort(ws, 1);
    }
    CHECK_CUDA(cudaDeviceSynchronize());
    return blocks;
}

void *_worker_arena_push_array(Worker_State *ws, u64 local_count, u64 elem_size, u64 alignment, u64 *max_count_out) {
    // One rank: the maximum over ranks is the local count.
    if (max_count_out) *max_count_out = local_count;
    return _arena_push(&ws->gpu_arena, local_count * elem_size, alignment);
}

namespace g5compat {

static std::mutex g_mu;
static std::unordered_map<const void *, GraphExt> g_graphs;
static std::unordered_map<const void *, BfsExt> g_bfs;
static std::unordered_map<const void *, SsspExt> g_sssp;

void put_graph(const u64 *k, const GraphExt &x) {
    std::lock_guard<std::mutex> l(g_mu);
    g_graphs[k] = x;
}
GraphExt *get_graph(const Oned_Graph *g, Worker_State *ws) {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_graphs.find(g->rowstarts);
    if (it == g_graphs.end()) {
        ERROR("Oned_Graph was not built by oned_graph_from_tuple_graph of this library");
        worker_abort(ws, 1);
    }
    return &it->second;
}
void drop_graph(const u64 *k) {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_graphs.find(k);
    if (it != g_graphs.end() && it->second.main_host) free(it->second.main_host);
    g_graphs.erase(k);
}
void put_bfs(const i64 *k, const BfsExt &x) {
    std::lock_guard<std::mutex> l(g_mu);
    g_bfs[k] = x;
}
const BfsExt *get_bfs(const i64 *k) {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_bfs.find(k);
    return it == g_bfs.end() ? nullptr : &it->second;
}
void drop_bfs(const i64 *k) {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_bfs.find(k);
    if (it != g_bfs.end() && it->second.root_host) cudaFreeHost(it->second.root_host);
    g_bfs.erase(k);
}
void put_sssp(const i64 *k, const SsspExt &x) {
    std::lock_guard<std::mutex> l(g_mu);
    g_sssp[k] = x;
}
const SsspExt *get_sssp(const i64 *k) {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_sssp.find(k);
    return it == g_sssp.end() ? nullptr : &it->second;
}
void drop_sssp(const i64 *k) {
    std::lock_guard<std::mutex> l(g_mu);
    g_sssp.erase(k);
}

void die(Worker_State *ws, int rc, const char *what) {
    ERROR("%s failed (%d): %s", what, rc, g5_last_error());
    worker_abort(ws, 1);
}

void *gpu_push(Worker_State *ws, uint64_t bytes, const char *what) {
    void *p = _arena_push(&ws->gpu_arena, std::max<uint64_t>(bytes, 256), 256);
    if (!p) {
        ERROR("GPU arena too small for %s (%llu bytes)", what, (unsigned long long)bytes);
        worker_abort(ws, 1);
    }
    return p;
}

}  // namespace g5compat
