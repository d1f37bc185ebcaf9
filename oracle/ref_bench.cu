// ref_bench.cu -- times the reference library (RuanPetrus/cuda-graph-traversal,
// compiled from its own sources by oracle/ref.mk with the single-process
// shims) on one GPU, with its runner's protocol: generation + CSR untimed,
// then per root oned_graph_*_clear outside and oned_graph_*_run inside the
// timer (examples/graph500_runner.cu:303-313, 402-408), nedge from the
// runner's rule.  Unlike the runner, the number of BFS and SSSP roots is a
// parameter, so the SCALE 26 SSSP can be sampled.
//
// TEST/MEASUREMENT INFRASTRUCTURE.
// Usage: ref_bench SCALE EF NBFS NSSSP [FIRST [NEDGE [SSSP_ROOT_INDEX ...]]]
//   BFS from roots FIRST .. FIRST+NBFS-1 of the runner's 64 (wrapping), SSSP
//   from roots FIRST .. FIRST+NSSSP-1 or, when indices are listed, from those
//   roots; NEDGE=0 skips the host-side TEPS edge count (printed as 0: the
//   caller counts edges on its own copy of the same graph).
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
    if (argc < 5) {
        fprintf(stderr, "usage: %s SCALE EF NBFS NSSSP [FIRST [NEDGE [SSSP_ROOT_INDEX ...]]]\n", argv[0]);
        return 2;
    }
    int scale = atoi(argv[1]), ef = atoi(argv[2]), nbfs = atoi(argv[3]), nsssp = atoi(argv[4]);
    const int first = argc > 5 ? atoi(argv[5]) : 0;
    const bool count_edges = argc > 6 ? atoi(argv[6]) != 0 : true;
    std::vector<int> sssp_idx;
    for (int i = 7; i < argc; ++i) sssp_idx.push_back(atoi(argv[i]));
    if (!sssp_idx.empty()) nsssp = (int)sssp_idx.size();
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
    std::vector<u64> rs(n + 1), col(count_edges ? g.nlocaledges : 0);
    CHECK_CUDA(cudaMemcpy(rs.data(), g.rowstarts, rs.size() * 8, cudaMemcpyDeviceToHost));
    if (count_edges) CHECK_CUDA(cudaMemcpy(col.data(), g.column, col.size() * 8, cudaMemcpyDeviceToHost));

    std::vector<u64> roots;  // generate_bfs_roots, examples/graph500_runner.cu:43-74
    u64 counter = 0;
    const int want = 64;  // the runner's root count; roots are taken by index, wrapping
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
    const int nr = (int)roots.size();
    auto root_at = [&](int i) { return roots[(size_t)i % (size_t)nr]; };
    oned_graph_bfs_run(&ws, &g, &bfs, root_at(first));  // warm-up, like the runner
    double inv = 0;
    std::vector<double> bfs_nedge;
    printf(", \"bfs\": [");
    for (int i = 0; i < nbfs && nr > 0; ++i) {
        const u64 r = root_at(first + i);
        oned_graph_bfs_clear(&ws, &bfs);
        double a = now();
        oned_graph_bfs_run(&ws, &g, &bfs, r);
        double b = now();
        double ne = 0;
        if (count_edges) {
            CHECK_CUDA(cudaMemcpy(pred.data(), bfs.pred, n * 8, cudaMemcpyDeviceToHost));
            ne = nedge_of(rs, col, pred);
            inv += (b - a) / ne;
        }
        bfs_nedge.push_back(ne);
        printf("%s[%llu, %.9g, %.0f]", i ? ", " : "", (unsigned long long)r, b - a, ne);
    }
    printf("], \"bfs_hmean_teps\": %.6g", nbfs && count_edges ? 1.0 / (inv / nbfs) : 0.0);
    Sssp_State sssp = oned_graph_sssp_create(&ws, &g);
    auto sssp_index = [&](int i) { return sssp_idx.empty() ? first + i : sssp_idx[(size_t)i]; };
    if (nsssp > 0 && nr > 0) {
        oned_graph_sssp_clear(&ws, &sssp);
        oned_graph_sssp_run(&ws, &g, &sssp, root_at(sssp_index(0)));
    }
    inv = 0;
    printf(", \"sssp\": [");
    for (int i = 0; i < nsssp && nr > 0; ++i) {
        const int k = sssp_index(i);
        const u64 r = root_at(k);
        oned_graph_sssp_clear(&ws, &sssp);
        double a = now();
        oned_graph_sssp_run(&ws, &g, &sssp, r);
        double b = now();
        // SSSP reaches the root's component, as BFS does: the same TEPS edge
        // count, so a root already searched by BFS reuses it.
        double ne = 0;
        if (count_edges) {
            if (k >= first && k - first < (int)bfs_nedge.size()) {
                ne = bfs_nedge[(size_t)(k - first)];
            } else {
                CHECK_CUDA(cudaMemcpy(pred.data(), sssp.pred, n * 8, cudaMemcpyDeviceToHost));
                ne = nedge_of(rs, col, pred);
            }
            inv += (b - a) / ne;
        }
        printf("%s[%llu, %.9g, %.0f]", i ? ", " : "", (unsigned long long)r, b - a, ne);
    }
    printf("], \"sssp_hmean_teps\": %.6g}\n", nsssp && count_edges ? 1.0 / (inv / nsssp) : 0.0);
    worker_finalize(&ws);
    return 0;
}
