// visualization.cu -- Graphviz DOT dumps of the reference's
// src/visualization.h (its src/visualization.cu:149-334): the edge list
// (undirected), the CSR (directed, every entry) and one BFS state (vertices
// coloured by root / unreached / unresolved depth, parent edges drawn
// thick).  One rank, so the per-PE file and the global file carry the same
// lines; file names follow the reference's.
#include <errno.h>
#include <sys/stat.h>

#include <string>
#include <vector>

#include "compat_internal.h"
#include "visualization.h"

namespace {

void ensure_dir(Worker_State *ws, const char *dir) {
    if (mkdir(dir, 0777) != 0 && errno != EEXIST) {
        ERROR("Failed to create DOT output directory %s", dir);
        worker_abort(ws, 1);
    }
}

void write_file(Worker_State *ws, const char *dir, const std::string &name, const std::string &head,
                const std::string &body) {
    std::string path = std::string(dir) + "/" + name;
    FILE *f = fopen(path.c_str(), "w");
    if (!f) {
        ERROR("Rank %d: failed to open DOT file %s", ws->rank, path.c_str());
        worker_abort(ws, 1);
    }
    fputs(head.c_str(), f);
    fwrite(body.data(), 1, body.size(), f);
    fputs("}\n", f);
    fclose(f);
}

template <class T>
std::vector<T> fetch(const T *dev, u64 n) {
    std::vector<T> h(n);
    if (n) CHECK_CUDA(cudaMemcpy(h.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}

std::string vertex_line(u64 v) {
    char b[160];
    snprintf(b, sizeof b, "  %llu [label=\"v%llu\\npe=0 local=%llu\"];\n", (unsigned long long)v,
             (unsigned long long)v, (unsigned long long)v);
    return b;
}

std::string edge_line(u64 a, const char *op, u64 b, f32 w, const char *extra) {
    char s[200];
    snprintf(s, sizeof s, "  %llu %s %llu [label=\"%.6g\"%s];\n", (unsigned long long)a, op, (unsigned long long)b,
             (double)w, extra);
    return s;
}

std::string pe_name(const char *stem, i32 idx) {
    char b[96];
    if (idx >= 0) snprintf(b, sizeof b, "%s_%03d", stem, idx);
    else snprintf(b, sizeof b, "%s", stem);
    return b;
}

}  // namespace

void tuple_graph_write_dot_files(Worker_State *ws, const Tuple_Graph *tg, const char *dir) {
    ensure_dir(ws, dir);
    auto e = fetch(tg->edges, tg->edges_size);
    auto w = fetch(tg->weights, tg->edges_size);
    std::string body;
    for (u64 i = 0; i < tg->edges_size; ++i) {
        body += vertex_line(e[i].v0) + vertex_line(e[i].v1);
        body += edge_line(e[i].v0, "--", e[i].v1, w[i], "");
    }
    write_file(ws, dir, "tuple_pe_000.dot", "graph tuple_pe_0 {\n", body);
    write_file(ws, dir, "tuple_global.dot", "graph tuple_global {\n", body);
}

void oned_graph_write_dot_files(Worker_State *ws, const Oned_Graph *g, const char *dir) {
    ensure_dir(ws, dir);
    auto rs = fetch(g->rowstarts, g->nlocalverts + 1);
    auto col = fetch(g->column, g->nlocaledges);
    auto w = fetch(g->weights, g->nlocaledges);
    std::string body;
    for (u64 v = 0; v < g->nlocalverts; ++v) {
        body += vertex_line(v);
        for (u64 e = rs[v]; e < rs[v + 1]; ++e) body += vertex_line(col[e]) + edge_line(v, "->", col[e], w[e], "");
    }
    write_file(ws, dir, "oned_pe_000.dot", "digraph oned_pe_0 {\n", body);
    write_file(ws, dir, "oned_global.dot", "digraph oned_global {\n", body);
}

void bfs_write_dot_files_for_root(Worker_State *ws, const Oned_Graph *g, const Bfs_State *bfs, u64 root, i32 root_idx,
                                  const char *dir) {
    ensure_dir(ws, dir);
    auto rs = fetch(g->rowstarts, g->nlocalverts + 1);
    auto col = fetch(g->column, g->nlocaledges);
    auto w = fetch(g->weights, g->nlocaledges);
    auto pred = fetch(bfs->pred, g->nlocalverts);
    std::vector<i64> dist = bfs->dist ? fetch(bfs->dist, g->nlocalverts) : std::vector<i64>();
    std::string body;
    for (u64 v = 0; v < g->nlocalverts; ++v) {
        const char *style = "style=filled, fillcolor=\"#edf2f7\", color=\"#4a5568\"";
        if (v == root) style = "style=filled, fillcolor=\"#ffcc66\", color=\"#cc7a00\", penwidth=3";
        else if (pred[v] == -1) style = "style=filled, fillcolor=\"#eeeeee\", color=\"#999999\"";
        else if (!dist.empty() && dist[v] == INT64_MAX) style = "style=filled, fillcolor=\"#fed7d7\", color=\"#c53030\"";
        char b[400];
        if (!dist.empty())
            snprintf(b, sizeof b, "  %llu [label=\"v%llu\\npe=0 local=%llu\\npred=%lld\\ndist=%lld\", %s];\n",
                     (unsigned long long)v, (unsigned long long)v, (unsigned long long)v, (long long)pred[v],
                     (long long)dist[v], style);
        else
            snprintf(b, sizeof b, "  %llu [label=\"v%llu\\npe=0 local=%llu\\npred=%lld\\ndist=unset\", %s];\n",
                     (unsigned long long)v, (unsigned long long)v, (unsigned long long)v, (long long)pred[v], style);
        body += b;
        for (u64 e = rs[v]; e < rs[v + 1]; ++e) body += edge_line(v, "->", col[e], w[e], ", color=\"#a0aec0\"");
        if (pred[v] != -1) {
            snprintf(b, sizeof b, "  %lld -> %llu [label=\"pred\", color=\"#2b6cb0\", penwidth=3];\n",
                     (long long)pred[v], (unsigned long long)v);
            body += b;
        }
    }
    char head[200];
    snprintf(head, sizeof head, "  graph [label=\"BFS predecessor/dist state root=%llu\", labelloc=t];\n",
             (unsigned long long)root);
    write_file(ws, dir, pe_name("bfs", root_idx) + "_pe_000.dot", std::string("digraph bfs_pe_0 {\n") + head, body);
    write_file(ws, dir, pe_name("bfs", root_idx) + "_global.dot", std::string("digraph bfs_global {\n") + head, body);
}

void bfs_write_dot_files(Worker_State *ws, const Oned_Graph *g, const Bfs_State *bfs, u64 root, const char *dir) {
    bfs_write_dot_files_for_root(ws, g, bfs, root, -1, dir);
}
