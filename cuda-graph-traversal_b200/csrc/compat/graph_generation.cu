// graph_generation.cu -- the reference's src/graph_generation.h API over
// libg500b (replaces src/graph_generation.cu:248-396).
#include <fcntl.h>
#include <unistd.h>

#include "compat_internal.h"
#include "graph_generation.h"

using namespace g5compat;

void make_mrg_seed(u64 userseed1, u64 userseed2, u32 *seed) { g5_make_mrg_seed(userseed1, userseed2, seed); }

void make_random_numbers(i64 nvalues, u64 userseed1, u64 userseed2, i64 position, f64 *result) {
    g5_make_random_numbers(nvalues, userseed1, userseed2, position, result);
}

void generate_kronecker_range(Worker_State *ws, u32 seed[5], u32 logN, i64 start_edge, i64 end_edge,
                              Tuple_Graph *tg) {
    const i64 count = end_edge - start_edge;
    const u64 local = count > 0 ? (u64)count : 0;
    tg->edges_size = local;
    tg->edges = worker_arena_push_array(ws, local, Packed_Edge, &tg->max_edges_size);
    u64 wcount = 0;
    tg->weights = worker_arena_push_array(ws, local, f32, &wcount);
    if (wcount != tg->max_edges_size) {
        ERROR("Mismatched tuple graph allocation sizes");
        ABORT();
    }
    if (count <= 0) return;
    check(ws, g5_generate_kronecker_range(seed, logN, start_edge, end_edge, (uint64_t *)tg->edges, tg->weights, 0),
          "generate_kronecker_range");
    CHECK_CUDA(cudaDeviceSynchronize());
}

static const char *kDumpEdges = "graph-refactor.bin";
static const char *kDumpWeights = "graph-refactor.bin.weights";

static void file_io(const char *path, bool write_, u64 offset, void *buf, u64 bytes, u64 file_size) {
    int fd = write_ ? open(path, O_WRONLY | O_CREAT, 0644) : open(path, O_RDONLY);
    if (fd < 0) {
        ERROR("Cannot open %s", path);
        ABORT();
    }
    if (write_ && ftruncate(fd, (off_t)file_size) != 0) {
        ERROR("Cannot size %s", path);
        ABORT();
    }
    char *p = (char *)buf;
    while (bytes) {
        ssize_t n = write_ ? pwrite(fd, p, bytes, (off_t)offset) : pread(fd, p, bytes, (off_t)offset);
        if (n <= 0) {
            ERROR("I/O error on %s", path);
            ABORT();
        }
        p += n;
        offset += (u64)n;
        bytes -= (u64)n;
    }
    close(fd);
}

void tuple_graph_dump(const Tuple_Graph *tg, i64 start_edge) {
    const u64 eb = tg->edges_size * sizeof(Packed_Edge), wb = tg->edges_size * sizeof(f32);
    void *he = eb ? malloc(eb) : 0, *hw = wb ? malloc(wb) : 0;
    if ((eb && !he) || (wb && !hw)) {
        ERROR("Failed to allocate host graph dump buffers");
        ABORT();
    }
    if (eb) CHECK_CUDA(cudaMemcpy(he, tg->edges, eb, cudaMemcpyDeviceToHost));
    if (wb) CHECK_CUDA(cudaMemcpy(hw, tg->weights, wb, cudaMemcpyDeviceToHost));
    file_io(kDumpEdges, true, (u64)start_edge * sizeof(Packed_Edge), he, eb, tg->nglobaledges * sizeof(Packed_Edge));
    file_io(kDumpWeights, true, (u64)start_edge * sizeof(f32), hw, wb, tg->nglobaledges * sizeof(f32));
    free(he);
    free(hw);
}

void tuple_graph_load(Worker_State *ws, Tuple_Graph *tg, i64 start_edge, i64 edge_count) {
    const u64 local = edge_count > 0 ? (u64)edge_count : 0;
    tg->edges_size = local;
    tg->edges = worker_arena_push_array(ws, local, Packed_Edge, &tg->max_edges_size);
    u64 wcount = 0;
    tg->weights = worker_arena_push_array(ws, local, f32, &wcount);
    if (wcount != tg->max_edges_size) {
        ERROR("Mismatched tuple graph load allocation sizes");
        ABORT();
    }
    const u64 eb = local * sizeof(Packed_Edge), wb = local * sizeof(f32);
    void *he = eb ? malloc(eb) : 0, *hw = wb ? malloc(wb) : 0;
    if ((eb && !he) || (wb && !hw)) {
        ERROR("Failed to allocate host graph load buffers");
        ABORT();
    }
    if (eb) file_io(kDumpEdges, false, (u64)start_edge * sizeof(Packed_Edge), he, eb, 0);
    if (wb) file_io(kDumpWeights, false, (u64)start_edge * sizeof(f32), hw, wb, 0);
    if (eb) CHECK_CUDA(cudaMemcpy(tg->edges, he, eb, cudaMemcpyHostToDevice));
    if (wb) CHECK_CUDA(cudaMemcpy(tg->weights, hw, wb, cudaMemcpyHostToDevice));
    free(he);
    free(hw);
}
