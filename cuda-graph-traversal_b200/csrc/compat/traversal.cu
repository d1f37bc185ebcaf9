// traversal.cu -- the reference's src/traversal.h API over libg500b
// (replaces src/traversal.cu:342-721).  Same inputs, outputs and error
// behaviour; every call synchronises before returning, as the reference's
// do, so wall-clock timing around a call measures its work.
#include <cstring>
#include <vector>

#include "compat_internal.h"
#include "traversal.h"

using namespace g5compat;

static const float kLightDelta = 0.1f;  // the reference's SSSP delta (src/traversal.cu:645)

Oned_Graph oned_graph_from_tuple_graph(Worker_State *ws, Tuple_Graph *tg, u64 nglobalverts) {
    Oned_Graph g;
    memset(&g, 0, sizeof g);
    g.nglobalverts = nglobalverts;
    g.nlocalverts = nglobalverts;  // one rank owns every vertex
    u64 count = 0;
    g.rowstarts = worker_arena_push_array(ws, g.nlocalverts + 1, u64, &count);
    uint64_t wbytes = 0;
    check(ws, g5_csr_workspace_size(nglobalverts, tg->edges_size, &wbytes), "oned_graph_from_tuple_graph");
    const Arena before_count = ws->gpu_arena;
    void *work = gpu_push(ws, wbytes, "CSR workspace");
    check(ws,
          g5_csr_count((const uint64_t *)tg->edges, tg->edges_size, nglobalverts, g.rowstarts, work, wbytes,
                       &g.nlocaledges, 0),
          "oned_graph_from_tuple_graph");
    ws->gpu_arena = before_count;  // the count's scratch is free again (nothing else was pushed since)
    g.column = worker_arena_push_array(ws, g.nlocaledges, u64, &count);
    g.weights = worker_arena_push_array(ws, g.nlocaledges, f32, &count);
    GraphExt x;
    const uint64_t e = g.nlocaledges;
    x.col = (int32_t *)gpu_push(ws, e * sizeof(int32_t), "int32 column");
    x.bcol = (int32_t *)gpu_push(ws, e * sizeof(int32_t), "BFS column");
    x.srowstarts = (uint64_t *)gpu_push(ws, (nglobalverts + 1) * sizeof(uint64_t), "SSSP row starts");
    x.scol = (int32_t *)gpu_push(ws, e * sizeof(int32_t), "SSSP column");
    x.sw = (float *)gpu_push(ws, e * sizeof(float), "SSSP weights");
    x.light_deg = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "light degrees");
    x.tiny_deg = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "tiny degrees");
    x.perm = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "SSSP numbering");
    x.inv = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "SSSP numbering, inverse");
    x.light_delta = kLightDelta;
    x.main_host = nullptr;
    x.isolated = (uint32_t *)gpu_push(ws, (nglobalverts + 31) / 32 * sizeof(uint32_t), "isolated-vertex bitmap");
    x.btop = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "BFS first neighbours");
    // Rows in canonical order (sorted by neighbour, then weight), the SSSP
    // copy (split, then renumbered by decreasing degree) and the BFS copy;
    // the scratch (the split copy in the caller's numbering and the sorting
    // scratch, sized for the largest step) is the arena's last push, popped
    // after.
    uint64_t sbytes = 0, rbytes = 0;
    check(ws, g5_csr_degree_order_workspace_size(nglobalverts, e, &sbytes), "oned_graph_from_tuple_graph");
    check(ws, g5_csr_sssp_renumber_workspace_size(nglobalverts, &rbytes), "oned_graph_from_tuple_graph");
    sbytes = sbytes > rbytes ? sbytes : rbytes;
    const Arena before_sort = ws->gpu_arena;
    int32_t *tcol = (int32_t *)gpu_push(ws, e * sizeof(int32_t), "split SSSP column (scratch)");
    float *tw = (float *)gpu_push(ws, e * sizeof(float), "split SSSP weights (scratch)");
    uint32_t *tlight = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "light degrees (scratch)");
    uint32_t *ttiny = (uint32_t *)gpu_push(ws, nglobalverts * sizeof(uint32_t), "tiny degrees (scratch)");
    void *swork = gpu_push(ws, sbytes, "CSR sorting scratch");
    check(ws,
          g5_csr_fill_sorted((const uint64_t *)tg->edges, tg->weights, tg->edges_size, nglobalverts, g.rowstarts, e,
                             swork, sbytes, x.col, g.weights, g.column, 0),
          "oned_graph_from_tuple_graph");
    check(ws,
          g5_csr_split_light(g.rowstarts, x.col, g.weights, nglobalverts, e, kLightDelta, tcol, tw, tlight, ttiny,
                             swork, sbytes, 0),
          "oned_graph_from_tuple_graph");
    check(ws,
          g5_csr_sssp_renumber(g.rowstarts, tcol, tw, tlight, ttiny, nglobalverts, e, x.perm, x.inv, x.srowstarts,
                               x.scol, x.sw, x.light_deg, x.tiny_deg, swork, sbytes, 0),
          "oned_graph_from_tuple_graph");
    check(ws, g5_csr_degree_order(g.rowstarts, x.col, nglobalverts, e, x.bcol, swork, sbytes, 0),
          "oned_graph_from_tuple_graph");
    check(ws, g5_bfs_first_neighbours(g.rowstarts, x.bcol, nglobalverts, x.btop, 0), "oned_graph_from_tuple_graph");
    CHECK_CUDA(cudaDeviceSynchronize());
    ws->gpu_arena = before_sort;
    check(ws, g5_graph_isolated_bitmap(g.rowstarts, nglobalverts, x.isolated, 0), "oned_graph_from_tuple_graph");
    CHECK_CUDA(cudaDeviceSynchronize());
    put_graph(g.rowstarts, x);
    return g;
}

b32 oned_graph_is_vertex_isolated(Worker_State *ws, const Oned_Graph *g, u64 global_vertex) {
    if (global_vertex >= g->nglobalverts) {
        ERROR("Vertex %llu is outside graph vertex range [0, %llu)", (unsigned long long)global_vertex,
              (unsigned long long)g->nglobalverts);
        worker_abort(ws, 1);
    }
    u64 r[2];
    CHECK_CUDA(cudaMemcpy(r, g->rowstarts + global_vertex, sizeof r, cudaMemcpyDeviceToHost));
    return r[0] == r[1];
}

static void bfs_clear(Worker_State *ws, Bfs_State *bfs, bool first);
static void sssp_clear(Worker_State *ws, Sssp_State *sssp, bool first);

Bfs_State oned_graph_bfs_create(Worker_State *ws, const Oned_Graph *g) {
    Bfs_State bfs;
    memset(&bfs, 0, sizeof bfs);
    bfs.pred = worker_arena_push_array(ws, g->nlocalverts, i64, &bfs.max_nlocalverts);
    BfsExt x;
    x.isolated = get_graph(g, ws)->isolated;
    x.depth = (int32_t *)gpu_push(ws, g->nlocalverts * sizeof(int32_t), "BFS depth");
    check(ws, g5_bfs_workspace_size(g->nglobalverts, &x.work_bytes), "oned_graph_bfs_create");
    x.work = gpu_push(ws, x.work_bytes, "BFS workspace");
    check(ws, g5_validate_workspace_size(g->nglobalverts, &x.val_bytes), "oned_graph_bfs_create");
    x.val_work = gpu_push(ws, x.val_bytes, "BFS depth scratch");
    // Pinned root word followed by the statistics (g5_bfs_query reads and
    // writes both from the device when they are pinned).
    CHECK_CUDA(cudaMallocHost(&x.root_host, sizeof(uint64_t) + sizeof(g5_bfs_stats)));
    put_bfs(bfs.pred, x);
    GraphExt *gx = get_graph(g, ws);
    if (!gx->main_host && g->nlocaledges) {
        // The largest component: one search from a maximum-degree vertex.
        // Later searches from roots outside it run on a single block.
        std::vector<u64> rs(g->nglobalverts + 1);
        CHECK_CUDA(cudaMemcpy(rs.data(), g->rowstarts, rs.size() * sizeof(u64), cudaMemcpyDeviceToHost));
        u64 hub = 0;
        for (u64 v = 1; v < g->nglobalverts; ++v)
            if (rs[v + 1] - rs[v] > rs[hub + 1] - rs[hub]) hub = v;
        const u64 words = (g->nglobalverts + 31) / 32;
        check(ws, g5_bfs_reset(g->nglobalverts, bfs.pred, nullptr, nullptr, x.work, x.work_bytes, 0),
              "oned_graph_bfs_create");
        g5_bfs_params hp = {14.0f, 24.0f, 0, 0};
        hp.top = gx->btop;
        check(ws, g5_bfs_traverse(g->rowstarts, gx->bcol, g->nglobalverts, hub, bfs.pred, nullptr, x.work, x.work_bytes,
                                  &hp, 0),
              "oned_graph_bfs_create");
        uint32_t *bits = (uint32_t *)gpu_push(ws, words * sizeof(uint32_t), "component bitmap");
        check(ws, g5_bfs_visited_bitmap(x.work, x.work_bytes, g->nglobalverts, bits, 0), "oned_graph_bfs_create");
        gx->main_host = (uint32_t *)malloc(words * sizeof(uint32_t));
        CHECK_CUDA(cudaMemcpy(gx->main_host, bits, words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    bfs_clear(ws, &bfs, true);
    return bfs;
}

// The state's first clear (at creation) resets everything; later ones undo
// only what the last search wrote (O(reached) after a one-block search).
static void bfs_clear(Worker_State *ws, Bfs_State *bfs, bool first) {
    const BfsExt *bx = get_bfs(bfs->pred);
    if (!bx) {
        ERROR("Bfs_State was not created by oned_graph_bfs_create of this library");
        worker_abort(ws, 1);
    }
    auto reset = first ? g5_bfs_reset : g5_bfs_reset_touched;
    check(ws, reset(bfs->max_nlocalverts, bfs->pred, bx->depth, bx->isolated, bx->work, bx->work_bytes, 0),
          "oned_graph_bfs_clear");
    if (bfs->dist) CHECK_CUDA(cudaMemset(bfs->dist, 0xff, bfs->max_nlocalverts * sizeof(i64)));
    CHECK_CUDA(cudaDeviceSynchronize());
}

void oned_graph_bfs_clear(Worker_State *ws, Bfs_State *bfs) { bfs_clear(ws, bfs, false); }

void oned_graph_bfs_run(Worker_State *ws, const Oned_Graph *g, Bfs_State *bfs, u64 root) {
    if (root >= g->nglobalverts) {
        ERROR("BFS root %llu is outside graph vertex range [0, %llu)", (unsigned long long)root,
              (unsigned long long)g->nglobalverts);
        worker_abort(ws, 1);
    }
    const GraphExt *gx = get_graph(g, ws);
    BfsExt *bx = const_cast<BfsExt *>(get_bfs(bfs->pred));
    if (!bx) {
        ERROR("Bfs_State was not created by oned_graph_bfs_create of this library");
        worker_abort(ws, 1);
    }
    // The reset half ran in oned_graph_bfs_clear, which the reference's
    // protocol calls before every search (examples/graph500_runner.cu:309).
    *bx->root_host = root;
    g5_bfs_stats *st = (g5_bfs_stats *)(bx->root_host + 1);
    g5_bfs_params bp = {14.0f, 24.0f, 0, 0};  // the library's defaults, with the first-neighbour probe
    bp.top = gx->btop;
    check(ws, g5_bfs_query(g->rowstarts, gx->bcol, g->nglobalverts, bx->root_host, gx->main_host, bfs->pred, bx->depth,
                           bx->work, bx->work_bytes, &bp, st, 0),
          "oned_graph_bfs_run");
}

i64 *bfs_compute_dist_from_pred(Worker_State *ws, const Oned_Graph *g, Bfs_State *bfs, u64 root) {
    if (root >= g->nglobalverts) {
        ERROR("BFS root %llu is outside graph vertex range [0, %llu)", (unsigned long long)root,
              (unsigned long long)g->nglobalverts);
        worker_abort(ws, 1);
    }
    if (!bfs->dist) {
        u64 count = 0;
        bfs->dist = worker_arena_push_array(ws, g->nlocalverts, i64, &count);
    }
    const GraphExt *gx = get_graph(g, ws);
    const BfsExt *bx = get_bfs(bfs->pred);
    if (!bx) {
        ERROR("Bfs_State was not created by oned_graph_bfs_create of this library");
        worker_abort(ws, 1);
    }
    check(ws, g5_bfs_dist_from_pred(g->rowstarts, gx->col, g->nglobalverts, bfs->pred, root, bfs->dist, bx->val_work,
                                    bx->val_bytes, 0),
          "bfs_compute_dist_from_pred");
    CHECK_CUDA(cudaDeviceSynchronize());
    return bfs->dist;
}

void oned_graph_bfs_destroy(Bfs_State *bfs) {
    if (!bfs) return;
    drop_bfs(bfs->pred);
    memset(bfs, 0, sizeof *bfs);
}

Sssp_State oned_graph_sssp_create(Worker_State *ws, const Oned_Graph *g) {
    Sssp_State s;
    memset(&s, 0, sizeof s);
    s.pred = worker_arena_push_array(ws, g->nlocalverts, i64, &s.max_nlocalverts);
    u64 count = 0;
    s.dist = worker_arena_push_array(ws, g->nlocalverts, f32, &count);
    SsspExt x;
    check(ws, g5_sssp_workspace_size(g->nglobalverts, &x.work_bytes), "oned_graph_sssp_create");
    x.work = gpu_push(ws, x.work_bytes, "SSSP workspace");
    put_sssp(s.pred, x);
    sssp_clear(ws, &s, true);
    return s;
}

// pred = -1 and dist = -1.0f everywhere, the reference's "unreached"
// (src/traversal.cu:248-249); the search then writes reached vertices only.
// The first clear (at creation) resets everything; later ones undo only what
// the last search wrote.
static void sssp_clear(Worker_State *ws, Sssp_State *sssp, bool first) {
    const SsspExt *sx = get_sssp(sssp->pred);
    if (!sx) {
        ERROR("Sssp_State was not created by oned_graph_sssp_create of this library");
        worker_abort(ws, 1);
    }
    auto reset = first ? g5_sssp_reset : g5_sssp_reset_touched;
    check(ws, reset(sssp->max_nlocalverts, sssp->dist, sssp->pred, sx->work, sx->work_bytes, 0),
          "oned_graph_sssp_clear");
    CHECK_CUDA(cudaDeviceSynchronize());
}

void oned_graph_sssp_clear(Worker_State *ws, Sssp_State *sssp) { sssp_clear(ws, sssp, false); }

void oned_graph_sssp_run(Worker_State *ws, const Oned_Graph *g, Sssp_State *sssp, u64 root) {
    if (root >= g->nglobalverts) {
        ERROR("SSSP root %llu is outside graph vertex range [0, %llu)", (unsigned long long)root,
              (unsigned long long)g->nglobalverts);
        worker_abort(ws, 1);
    }
    const GraphExt *gx = get_graph(g, ws);
    const SsspExt *sx = get_sssp(sssp->pred);
    if (!sx) {
        ERROR("Sssp_State was not created by oned_graph_sssp_create of this library");
        worker_abort(ws, 1);
    }
    // A root outside the largest component (host bitmap from the first BFS
    // state) runs on one block: its search touches a handful of vertices.
    const bool small = gx->main_host && !((gx->main_host[root >> 5] >> (root & 31)) & 1u);
    g5_sssp_params p = {kLightDelta, small ? 1 : 0, 0.0f, 0, small ? 1 : 0, gx->tiny_deg, 0};
    p.perm = gx->perm;  // the SSSP copy is renumbered; root and outputs stay the caller's
    p.inv = gx->inv;
    check(ws, g5_sssp_traverse(gx->srowstarts, gx->scol, gx->sw, gx->light_deg, gx->light_delta, g->nglobalverts,
                               root, sssp->dist, sssp->pred, sx->work, sx->work_bytes, &p, 0),
          "oned_graph_sssp_run");
    check(ws, g5_sssp_last_status(sx->work, sx->work_bytes, nullptr, nullptr, 0), "oned_graph_sssp_run");
}

void oned_graph_sssp_destroy(Sssp_State *sssp) {
    if (!sssp) return;
    drop_sssp(sssp->pred);
    memset(sssp, 0, sizeof *sssp);
}

void oned_graph_free(Oned_Graph *g) {
    if (!g) return;
    drop_graph(g->rowstarts);
    memset(g, 0, sizeof *g);
}
