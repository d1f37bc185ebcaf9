// compat_internal.h -- private state of the reference-compatible C++ API.
//
// The reference's structs cannot grow (code written against them touches
// their fields), so the library's extra per-object state -- the int32
// column and light counts of a graph, the workspaces of a BFS or SSSP
// state -- lives in side tables keyed by the object's first device pointer.
#pragma once

#include <stdint.h>

#include "g500b.h"
#include "traversal.h"

namespace g5compat {

struct GraphExt {
    int32_t *col;        // int32 neighbour ids, rows in canonical order (as Oned_Graph.column)
    int32_t *bcol;       // the BFS copy (g5_csr_degree_order): rows by decreasing neighbour degree
    uint32_t *btop;      // each row's first entry of bcol (g5_bfs_first_neighbours)
    // The SSSP copy: rows split tiny | light | heavy (g5_csr_split_light),
    // renumbered by decreasing degree (g5_csr_sssp_renumber).
    uint64_t *srowstarts;
    int32_t *scol;
    float *sw;           // its weights
    uint32_t *light_deg; // light entries per row
    uint32_t *tiny_deg;  // leading tiny entries of each light part
    uint32_t *perm, *inv;  // caller's vertex -> the copy's, and back
    uint32_t *isolated;  // bitmap of degree-0 vertices
    uint32_t *main_host; // host bitmap of the largest component (set by the first BFS state)
    float light_delta;
};

struct BfsExt {
    const uint32_t *isolated;  // the graph's isolated-vertex bitmap
    int32_t *depth;
    void *work;  // BFS kernel workspace (its statistics live at the front)
    uint64_t work_bytes;
    void *val_work;  // depth-from-parents scratch
    uint64_t val_bytes;
    uint64_t *root_host;  // pinned: the root of the next search, then its g5_bfs_stats
};

struct SsspExt {
    void *work;
    uint64_t work_bytes;
};

void put_graph(const u64 *rowstarts, const GraphExt &x);
GraphExt *get_graph(const Oned_Graph *g, Worker_State *ws);
void drop_graph(const u64 *rowstarts);
void put_bfs(const i64 *pred, const BfsExt &x);
const BfsExt *get_bfs(const i64 *pred);
void drop_bfs(const i64 *pred);
void put_sssp(const i64 *pred, const SsspExt &x);
const SsspExt *get_sssp(const i64 *pred);
void drop_sssp(const i64 *pred);

// Prints the library error and aborts the worker, the reference's
// convention for failed calls (src/base.h:48-54, src/worker.cu:64-67).
void die(Worker_State *ws, int rc, const char *what);
inline void check(Worker_State *ws, int rc, const char *what) {
    if (rc != G5_OK) die(ws, rc, what);
}

// Device memory for the library's private arrays, from the worker's GPU
// arena like everything else the reference allocates.
void *gpu_push(Worker_State *ws, uint64_t bytes, const char *what);

}  // namespace g5compat
