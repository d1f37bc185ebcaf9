// ref_dump.cu -- runs the reference library (RuanPetrus/cuda-graph-traversal,
// compiled from its own sources by oracle/ref.mk) on one GPU and writes its
// raw outputs for the golden fixtures (tests/golden/make_golden.py).
//
// TEST INFRASTRUCTURE ONLY.  Usage: ref_dump SCALE EDGEFACTOR NROOTS OUTDIR
//
// Files written to OUTDIR (little-endian raw arrays):
//   edges.u64 (2 per edge) weights.f32      generate_kronecker_range output
//   rowstarts.u64 column.u64 csrw.f32       oned_graph_from_tuple_graph output
//   roots.u64                               roots chosen as the runner does
//   bfs_pred.i64 bfs_dist.i64               per root, concatenated (N each)
//   sssp_dist.f32 sssp_pred.i64             per root, concatenated (N each)
#include "graph_generation.h"
#include "traversal.h"
#include "worker.h"

#include <stdio.h>
#include <stdlib.h>
#include <vector>

static void dump(const char *dir, const char *name, const void *host, size_t bytes, bool append) {
    char path[1024];
    snprintf(path, sizeof path, "%s/%s", dir, name);
    FILE *f = fopen(path, append ? "ab" : "wb");
    if (!f || fwrite(host, 1, bytes, f) != bytes) {
        fprintf(stderr, "ref_dump: cannot write %s\n", path);
        exit(1);
    }
    fclose(f);
}

template <class T>
static std::vector<T> fetch(const T *dev, size_t n) {
    std::vector<T> h(n);
    if (n) CHECK_CUDA(cudaMemcpy(h.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s SCALE EDGEFACTOR NROOTS OUTDIR\n", argv[0]);
        return 2;
    }
    int scale = atoi(argv[1]), ef = atoi(argv[2]), nroots_max = atoi(argv[3]);
    const char *out = argv[4];
    Worker_State ws = worker_init(1, argv, 0);

    // Same seeds and edge range as examples/graph500_runner.cu:270-284.
    u64 seed1 = 2, seed2 = 3;
    u32 seed[5];
    make_mrg_seed(seed1, seed2, seed);
    Tuple_Graph tg = {0};
    tg.nglobaledges = (u64)ef << scale;
    generate_kronecker_range(&ws, seed, (u32)scale, 0, (i64)tg.nglobaledges, &tg);
    auto edges = fetch((const u64 *)tg.edges, 2 * tg.edges_size);
    auto weights = fetch(tg.weights, tg.edges_size);
    dump(out, "edges.u64", edges.data(), edges.size() * 8, false);
    dump(out, "weights.f32", weights.data(), weights.size() * 4, false);

    u64 n = (u64)1 << scale;
    Oned_Graph g = oned_graph_from_tuple_graph(&ws, &tg, n);
    auto rowstarts = fetch(g.rowstarts, n + 1);
    auto column = fetch(g.column, g.nlocaledges);
    auto csrw = fetch(g.weights, g.nlocaledges);
    dump(out, "rowstarts.u64", rowstarts.data(), rowstarts.size() * 8, false);
    dump(out, "column.u64", column.data(), column.size() * 8, false);
    dump(out, "csrw.f32", csrw.data(), csrw.size() * 4, false);

    // Root choice of generate_bfs_roots (examples/graph500_runner.cu:43-74),
    // through the reference's own make_random_numbers and isolation test.
    std::vector<u64> roots;
    u64 counter = 0;
    while ((int)roots.size() < nroots_max) {
        bool found = false;
        u64 root = 0;
        for (;;) {
            f64 d[2];
            make_random_numbers(2, seed1, seed2, (i64)counter, d);
            root = (u64)((d[0] + d[1]) * (f64)n) % n;
            counter += 2;
            if (counter > 2 * n) break;
            bool dup = false;
            for (u64 r : roots) dup |= r == root;
            if (dup) continue;
            if (oned_graph_is_vertex_isolated(&ws, &g, root)) continue;
            found = true;
            break;
        }
        if (!found) break;
        roots.push_back(root);
    }
    dump(out, "roots.u64", roots.data(), roots.size() * 8, false);

    Bfs_State bfs = oned_graph_bfs_create(&ws, &g);
    Sssp_State sssp = oned_graph_sssp_create(&ws, &g);
    for (size_t i = 0; i < roots.size(); ++i) {
        oned_graph_bfs_clear(&ws, &bfs);
        oned_graph_bfs_run(&ws, &g, &bfs, roots[i]);
        i64 *dist = bfs_compute_dist_from_pred(&ws, &g, &bfs, roots[i]);
        auto pred = fetch(bfs.pred, n);
        auto depth = fetch(dist, n);
        dump(out, "bfs_pred.i64", pred.data(), n * 8, i > 0);
        dump(out, "bfs_dist.i64", depth.data(), n * 8, i > 0);

        oned_graph_sssp_clear(&ws, &sssp);
        oned_graph_sssp_run(&ws, &g, &sssp, roots[i]);
        auto sd = fetch(sssp.dist, n);
        auto sp = fetch(sssp.pred, n);
        dump(out, "sssp_dist.f32", sd.data(), n * 4, i > 0);
        dump(out, "sssp_pred.i64", sp.data(), n * 8, i > 0);
    }
    printf("ref_dump: scale %d ef %d edges %llu csr %llu roots %zu\n", scale, ef,
           (unsigned long long)tg.edges_size, (unsigned long long)g.nlocaledges, roots.size());
    worker_finalize(&ws);
    return 0;
}
