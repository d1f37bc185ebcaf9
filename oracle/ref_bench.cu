// ref_bench.cu -- times the reference library (RuanPetrus/cuda-graph-traversal,
// compiled from its own sources by oracle/ref.mk with the single-process
// shims) on one GPU, with its runner's protocol: generation + CSR untimed,
// then per root oned_graph_*_clear outside and oned_graph_*_run inside the
// timer (examples/graph500_runner.cu:303-313, 402-408), nedge from the
// runner's rule.  Unlike the runner, the number of BFS and SSSP roots is a
// parameter, so the SCALE 26 SSSP can be sampled.
//
// TEST/MEASUREMENT INFRASTRUCTURE.  Usage: ref_bench SCALE EF NBFS NSSSP
// Prints one JSON line with per-root times and harmonic-mean TEPS.
#include <mpi.h>

#include "graph_generation.h"
#include "traversal.h"
#include "worker.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <vector>

static double now() { return MPI_Wtime(); }

// TEPS edge count on the host: CSR entries col <= v over rows of reached v.
static double nedge_of(const std::vector<u64> &rs, const std::vector<u64> &col, const std::vector<i64> &pred) {
    double n = 0;
    for (size_t v = 0; v + 1 < rs.size(); ++v) {
        if (pred[v] == -1) continue;
        for (u64 e = rs[v]; e < rs[v + 1]; ++e) n += col[e] <= v;
    }
    return n;
}

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s SCALE EF NBFS NSSSP\n", argv[0]);
        return 2;
    }
    int scale = atoi(argv[1]), ef = atoi(argv[2]), nbfs = atoi(argv[3]), nsssp = atoi(argv[4]);
    Worker_State ws = worker_init(1, argv, 0);
    u64 seed1 = 2, seed2 = 3;
    u32 seed[5];
    make_mrg_seed(seed1, seed2, seed);
    Tuple_Graph tg = {0};
    tg.nglobaledges = (u64)ef << scale;
    double t0 = now();
    generate_kronecker_range(&ws, seed, (u32)scale, 0, (i64)tg.nglobaledges, &tg);
    double t1 = now();
    u64 n = (u64)1 << scale;
    Oned_Graph g = oned_graph_from_tuple_graph(&ws, &tg, n);
    double t2 = now();
    std::vector<u64> rs(n + 1), col(g.nlocaledges);
    CHECK_CUDA(cudaMemcpy(rs.data(), g.rowstarts, rs.size() * 8, cudaMemcpyDeviceToHost));
    CHECK_CUDA(cudaMemcpy(col.data(), g.column, col.size() * 8, cudaMemcpyDeviceToHost));

    std::vector<u64> roots;  // generate_bfs_roots, examples/graph500_runner.cu:43-74
    u64 counter = 0;
    int want = nbfs > nsssp ? nbfs : nsssp;
    while ((int)roots.size() < want) {
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
            if (dup || rs[root] == rs[root + 1]) continue;
            found = true;
            break;
        }
        if (!found) break;
        roots.push_back(root);
    }
    std::vector<i64> pred(n);
    printf("{\"scale\": %d, \"edgefactor\": %d, \"generation_s\": %.6g, \"construction_s\": %.6g", scale, ef, t1 - t0,
           t2 - t1);
    Bfs_State bfs = oned_graph_bfs_create(&ws, &g);
    oned_graph_bfs_clear(&ws, &bfs);
    oned_graph_bfs_run(&ws, &g, &bfs, roots[0]);  // warm-up, like the runner
    double inv = 0;
    std::vector<double> bfs_nedge;
    printf(", \"bfs\": [");
    for (int i = 0; i < nbfs && i < (int)roots.size(); ++i) {
        oned_graph_bfs_clear(&ws, &bfs);
        double a = now();
        oned_graph_bfs_run(&ws, &g, &bfs, roots[i]);
        double b = now();
        CHECK_CUDA(cudaMemcpy(pred.data(), bfs.pred, n * 8, cudaMemcpyDeviceToHost));
        double ne = nedge_of(rs, col, pred);
        bfs_nedge.push_back(ne);
        inv += (b - a) / ne;
        printf("%s[%llu, %.9g, %.0f]", i ? ", " : "", (unsigned long long)roots[i], b - a, ne);
    }
    printf("], \"bfs_hmean_teps\": %.6g", nbfs ? 1.0 / (inv / nbfs) : 0.0);
    Sssp_State sssp = oned_graph_sssp_create(&ws, &g);
    if (nsssp > 0) {
        oned_graph_sssp_clear(&ws, &sssp);
        oned_graph_sssp_run(&ws, &g, &sssp, roots[0]);
    }
    inv = 0;
    printf(", \"sssp\": [");
    for (int i = 0; i < nsssp && i < (int)roots.size(); ++i) {
        oned_graph_sssp_clear(&ws, &sssp);
        double a = now();
        oned_graph_sssp_run(&ws, &g, &sssp, roots[i]);
        double b = now();
        // SSSP reaches the root's component, as BFS does: the same TEPS edge
        // count, so a root already searched by BFS reuses it.
        double ne;
        if (i < (int)bfs_nedge.size()) {
            ne = bfs_nedge[i];
        } else {
            CHECK_CUDA(cudaMemcpy(pred.data(), sssp.pred, n * 8, cudaMemcpyDeviceToHost));
            ne = nedge_of(rs, col, pred);
        }
        inv += (b - a) / ne;
        printf("%s[%llu, %.9g, %.0f]", i ? ", " : "", (unsigned long long)roots[i], b - a, ne);
    }
    printf("], \"sssp_hmean_teps\": %.6g}\n", nsssp ? 1.0 / (inv / nsssp) : 0.0);
    worker_finalize(&ws);
    return 0;
}
