// Test program for tests/test_gpu_dump_load.py: the reference's edge-list
// dump format (graph-refactor.bin / .weights, raw Packed_Edge and f32)
// through the compat API, src/graph_generation.cu:314-396.  The graph is
// generated in two edge ranges, as two ranks would, and each range dumped
// at its offset; then the whole list and a sub-range starting at an odd
// offset are loaded back and compared byte for byte with a fresh
// generation, and the CSR built from the loaded list is compared with the
// one built from the generated list.  Usage: compat_dump_load SCALE EF;
// prints "ok <edges> <file bytes>" or the first mismatch and exits 1.
#include <mpi.h>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "graph_generation.h"
#include "traversal.h"
#include "worker.h"

template <class T>
static std::vector<T> to_host(const T *d, u64 n) {
    std::vector<T> h(n);
    if (n) CHECK_CUDA(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}

static int fail(const char *what) {
    printf("mismatch: %s\n", what);
    return 1;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s SCALE EF\n", argv[0]);
        return 2;
    }
    const int scale = atoi(argv[1]), ef = atoi(argv[2]);
    const i64 m = (i64)ef << scale;
    const u64 n = 1ull << scale;
    Worker_State ws = worker_init(1, argv, 0);
    u32 seed[5];
    make_mrg_seed(2, 3, seed);

    // Two ranges dumped at their offsets (the file is sized to nglobaledges
    // by each writer, as the reference does).
    const i64 half = m / 2 + 1;  // odd split: the second range starts mid-block
    for (int part = 0; part < 2; ++part) {
        Arena saved = ws.gpu_arena;
        Tuple_Graph tg;
        memset(&tg, 0, sizeof tg);
        tg.nglobaledges = (u64)m;
        const i64 a = part ? half : 0, b = part ? m : half;
        generate_kronecker_range(&ws, seed, (u32)scale, a, b, &tg);
        tuple_graph_dump(&tg, a);
        ws.gpu_arena = saved;
    }

    Tuple_Graph gen;
    memset(&gen, 0, sizeof gen);
    gen.nglobaledges = (u64)m;
    generate_kronecker_range(&ws, seed, (u32)scale, 0, m, &gen);
    const std::vector<Packed_Edge> ge = to_host(gen.edges, (u64)m);
    const std::vector<f32> gw = to_host(gen.weights, (u64)m);

    Tuple_Graph ld;
    memset(&ld, 0, sizeof ld);
    ld.nglobaledges = (u64)m;
    tuple_graph_load(&ws, &ld, 0, m);
    if (ld.edges_size != (u64)m) return fail("loaded edge count");
    {
        const std::vector<Packed_Edge> le = to_host(ld.edges, (u64)m);
        const std::vector<f32> lw = to_host(ld.weights, (u64)m);
        if (memcmp(le.data(), ge.data(), (size_t)m * sizeof(Packed_Edge))) return fail("edges");
        if (memcmp(lw.data(), gw.data(), (size_t)m * sizeof(f32))) return fail("weights");
    }

    // A sub-range at an odd offset.
    {
        Arena saved = ws.gpu_arena;
        const i64 off = m / 3 + 7, cnt = m / 5 + 3;
        Tuple_Graph sub;
        memset(&sub, 0, sizeof sub);
        sub.nglobaledges = (u64)m;
        tuple_graph_load(&ws, &sub, off, cnt);
        const std::vector<Packed_Edge> se = to_host(sub.edges, (u64)cnt);
        const std::vector<f32> sw = to_host(sub.weights, (u64)cnt);
        if (memcmp(se.data(), ge.data() + off, (size_t)cnt * sizeof(Packed_Edge))) return fail("sub-range edges");
        if (memcmp(sw.data(), gw.data() + off, (size_t)cnt * sizeof(f32))) return fail("sub-range weights");
        ws.gpu_arena = saved;
    }

    // CSRs of the generated and of the loaded lists.
    Oned_Graph g1 = oned_graph_from_tuple_graph(&ws, &gen, n);
    Oned_Graph g2 = oned_graph_from_tuple_graph(&ws, &ld, n);
    if (g1.nlocaledges != g2.nlocaledges) return fail("CSR entry counts");
    if (to_host(g1.rowstarts, n + 1) != to_host(g2.rowstarts, n + 1)) return fail("rowstarts");
    printf("ok %lld %llu\n", (long long)m, (unsigned long long)((u64)m * sizeof(Packed_Edge)));
    worker_finalize(&ws);
    return 0;
}
