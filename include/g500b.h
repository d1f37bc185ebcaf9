/*
 * g500b.h -- C ABI of the B200 Graph500 hot path (libg500b.so).
 *
 * Plain pointers and sizes only.  Arrays named d_* live in device memory of
 * the calling thread's current CUDA device; `stream` is a cudaStream_t (NULL
 * = legacy default stream).  Every call is stream-ordered: it enqueues its
 * work and returns, except where it hands a value back through a host
 * pointer (those synchronise `stream` first).  Scratch memory is supplied
 * by the caller as (d_work, work_bytes); the matching *_workspace_size call
 * says how much, and nothing here calls cudaMalloc on the hot path.
 *
 * Every function returns G5_OK (0) or a negative G5_ERR_* code; the message
 * of the last failure on this host thread is g5_last_error().
 *
 * Each entry point names the function of RuanPetrus/cuda-graph-traversal it
 * replaces.  The reference's own C++ API (the src/ headers) is provided on top of
 * these calls by the compatibility layer (include/compat/).
 */
#ifndef G500B_H
#define G500B_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    G5_OK = 0,
    G5_ERR_INVALID = -1,   /* bad argument: range, null pointer, size        */
    G5_ERR_WORKSPACE = -2, /* work_bytes below the *_workspace_size answer   */
    G5_ERR_CUDA = -3,      /* a CUDA runtime call failed                     */
    G5_ERR_TIMEOUT = -4,   /* a bounded device-side wait gave up             */
    G5_ERR_DEVICE = -5,    /* a kernel reported an internal consistency error */
};

/* Message of the last error on this host thread ("" if none). */
const char *g5_last_error(void);
/* Library version string. */
const char *g5_version(void);

/* ---------------------------------------------------------------- MRG ---- */

/* make_mrg_seed, src/graph_generation.h:39 (src/graph_generation.cu:248-254). */
int g5_make_mrg_seed(uint64_t userseed1, uint64_t userseed2, uint32_t seed[5]);

/* make_random_numbers, src/graph_generation.h:40 (src/graph_generation.cu:256-266). */
int g5_make_random_numbers(int64_t nvalues, uint64_t userseed1, uint64_t userseed2, int64_t position,
                           double *result);

/* The two vertex-scrambling keys generate_kronecker_range derives from the
 * seed (src/graph_generation.cu:290-300). */
int g5_scramble_keys(const uint32_t seed[5], uint64_t *val0, uint64_t *val1);

/* ----------------------------------------------------------- generator --- */

/* generate_kronecker_range, src/graph_generation.h:33-37
 * (src/graph_generation.cu:269-310): Graph500 Kronecker edges
 * [start_edge, end_edge) of a 2^log_n-vertex graph.  d_edges receives
 * (v0, v1) u64 pairs (the Packed_Edge layout, 16 bytes per edge), d_weights
 * one float per edge.  Any sub-range reproduces the same edges. */
int g5_generate_kronecker_range(const uint32_t seed[5], uint32_t log_n, int64_t start_edge, int64_t end_edge,
                                uint64_t *d_edges, float *d_weights, void *stream);

/* ----------------------------------------------------------------- CSR --- */

/* Scratch bytes for g5_csr_count + g5_csr_fill on nverts vertices. */
int g5_csr_workspace_size(uint64_t nverts, uint64_t nedges, uint64_t *bytes);

/* First half of oned_graph_from_tuple_graph, src/traversal.h:43
 * (src/traversal.cu:342-368: compute_degrees_kernel + rowstarts scan):
 * d_rowstarts[0..nverts] = exclusive prefix of the non-self-loop degree of
 * every vertex.  *nentries (host) = d_rowstarts[nverts], the number of
 * directed CSR entries; the call synchronises `stream`. */
int g5_csr_count(const uint64_t *d_edges, uint64_t nedges, uint64_t nverts, uint64_t *d_rowstarts,
                 void *d_work, uint64_t work_bytes, uint64_t *nentries, void *stream);

/* Second half (src/traversal.cu:369-389, fill_csr_kernel): both directions
 * of every non-self-loop edge into its row, duplicates kept.  Within a row,
 * entries with weight < light_delta come first (their count per vertex goes
 * to d_light_deg, optional) and the rest after; d_col receives int32 vertex
 * ids, d_w the weights and d_col64 (optional) the same ids as u64, the
 * reference's Oned_Graph.column type.  Uses the workspace state left by
 * g5_csr_count. */
int g5_csr_fill(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                const uint64_t *d_rowstarts, float light_delta, void *d_work, uint64_t work_bytes,
                int32_t *d_col, float *d_w, uint64_t *d_col64, uint32_t *d_light_deg, void *stream);

/* The CSR of the Kronecker graph with edges [0, nedges) of seed `seed` on
 * 2^log_n vertices, without an edge list: both passes regenerate every edge
 * in registers (the generator fused into the build; 20 bytes per edge
 * neither written nor read twice).  Same results and workspace as
 * g5_csr_count + g5_csr_fill over g5_generate_kronecker_range's output. */
int g5_csr_count_kronecker(const uint32_t seed[5], uint32_t log_n, uint64_t nedges, uint64_t *d_rowstarts,
                           void *d_work, uint64_t work_bytes, uint64_t *nentries, void *stream);
int g5_csr_fill_kronecker(const uint32_t seed[5], uint32_t log_n, uint64_t nedges, const uint64_t *d_rowstarts,
                          float light_delta, void *d_work, uint64_t work_bytes, int32_t *d_col, float *d_w,
                          uint64_t *d_col64, uint32_t *d_light_deg, void *stream);

/* Light entries below light_delta / G5_TINY_DIV ("tiny") are the only ones
 * whose relaxation can stay inside an SSSP sub-bucket (width delta / 32 <=
 * light_delta / 32).  g5_csr_split_tiny reorders each row's light part
 * [rowstart, rowstart + light_deg) in place so that its tiny entries come
 * first (d_col, d_w and, when given, d_col64 move together; the multiset of
 * each row is unchanged) and writes their count per vertex to d_tiny_deg.
 * Idempotent; needs the light counts of g5_csr_fill.  No counterpart in the
 * reference (its rows are not split at all). */
#define G5_TINY_DIV 30
int g5_csr_split_tiny(const uint64_t *d_rowstarts, int32_t *d_col, float *d_w, uint64_t *d_col64,
                      const uint32_t *d_light_deg, uint64_t nverts, float light_delta, uint32_t *d_tiny_deg,
                      void *stream);

/* ------------------------------------------------- canonical CSR rows --- */

/* Rows in canonical order: every row sorted by (neighbour, weight bits) --
 * the order the reference's rows have once sorted (its fill leaves them in
 * atomic order, src/traversal.cu:48-73), so the CSR is the same on every
 * run.  After g5_csr_count (row starts, entry count), g5_csr_fill_sorted
 * scatters the edges by radix partitioning (256 source partitions, then
 * each partition's rows while they are L2-resident) and sorts every row;
 * d_col64 (optional) receives the u64 column of the reference's Oned_Graph.
 * Scratch: g5_csr_sorted_workspace_size(nverts, nentries) bytes (12 bytes
 * per entry, plus 12 per vertex). */
int g5_csr_sorted_workspace_size(uint64_t nverts, uint64_t nentries, uint64_t *bytes);
int g5_csr_fill_sorted(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                       const uint64_t *d_rowstarts, uint64_t nentries, void *d_work, uint64_t work_bytes,
                       int32_t *d_col, float *d_w, uint64_t *d_col64, void *stream);

/* The same canonical CSR by one LSD radix sort of every directed entry by
 * (source, neighbour), the reference's two steps (src/traversal.cu:342-389:
 * count_degrees + rowstarts scan, then fill_csr_kernel) recast:
 * g5_csr_radix_count counts, in one pass over the edges, the entries and
 * every sort pass's digit totals (kept in the workspace) and returns the
 * entry count (synchronises); the caller allocates the CSR and calls
 * g5_csr_radix_fill with the same edges, which sorts (8-bit digits,
 * ceil(2 * ceil(log2 nverts) / 8) one-sweep passes, the first reading the
 * edge list), then writes d_rowstarts (nverts + 1), d_col, d_w and d_col64
 * (optional), runs of one (row, neighbour) ordered by weight bits.  Output
 * identical to g5_csr_count + g5_csr_fill_sorted; no per-row atomics.
 * Self-loops are dropped, duplicates kept.  Scratch:
 * g5_csr_radix_workspace_size(nverts, nedges) bytes (24 bytes per possible
 * entry, 2 * nedges, plus 1 per edge and 12 per vertex).  Fails with
 * G5_ERR_INVALID when an endpoint is >= nverts or the edges changed between
 * the calls, G5_ERR_TIMEOUT when a pass's bounded look-back wait gives up. */
int g5_csr_radix_workspace_size(uint64_t nverts, uint64_t nedges, uint64_t *bytes);
int g5_csr_radix_count(const uint64_t *d_edges, uint64_t nedges, uint64_t nverts, void *d_work, uint64_t work_bytes,
                       uint64_t *nentries, void *stream);
int g5_csr_radix_fill(const uint64_t *d_edges, const float *d_weights, uint64_t nedges, uint64_t nverts,
                      uint64_t nentries, void *d_work, uint64_t work_bytes, uint64_t *d_rowstarts, int32_t *d_col,
                      float *d_w, uint64_t *d_col64, void *stream);

/* Sorts the rows of any CSR in place into canonical order (e.g. after
 * g5_csr_fill or g5_csr_fill_kronecker); same scratch as above. */
int g5_csr_sort_rows(const uint64_t *d_rowstarts, uint64_t nverts, uint64_t nentries, int32_t *d_col, float *d_w,
                     uint64_t *d_col64, void *d_work, uint64_t work_bytes, void *stream);

/* Opt-in dedupe of a canonical CSR (the reference keeps duplicates; this
 * changes the TEPS edge count): one entry per (row, neighbour), the one of
 * least weight.  g5_csr_dedupe_count writes the new row starts
 * (nverts + 1) and their entry count; g5_csr_dedupe_copy fills new arrays
 * of that size (d_col64_out optional).  No counterpart in the reference. */
int g5_csr_dedupe_count(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t nentries,
                        uint64_t *d_rowstarts_out, void *d_work, uint64_t work_bytes, uint64_t *nentries_out,
                        void *stream);
int g5_csr_dedupe_copy(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                       const uint64_t *d_rowstarts_out, int32_t *d_col_out, float *d_w_out, uint64_t *d_col64_out,
                       void *stream);

/* The SSSP copy of a CSR: each row stably partitioned into entries lighter
 * than light_delta / G5_TINY_DIV, the other ones lighter than light_delta,
 * then the rest (so a canonical CSR gives each part in canonical order),
 * with d_light_deg / d_tiny_deg = the first two parts' sizes per row -- the
 * layout g5_sssp_run reads (d_scol, d_sw as its column and weights).  Same
 * scratch as g5_csr_fill_sorted.  No counterpart in the reference. */
int g5_csr_split_light(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                       uint64_t nentries, float light_delta, int32_t *d_scol, float *d_sw, uint32_t *d_light_deg,
                       uint32_t *d_tiny_deg, void *d_work, uint64_t work_bytes, void *stream);

/* The BFS copy of a CSR's column: every row's neighbours ordered by
 * decreasing degree, ties by index (d_out_col, nentries entries, distinct
 * from d_col).  A bottom-up level then probes a vertex's best-connected
 * neighbours first, the ones most likely to be in the frontier.  Any
 * order of a row gives the same BFS depths; the parents chosen may differ
 * (every one is valid).  Scratch: g5_csr_degree_order_workspace_size.  No
 * counterpart in the reference. */
int g5_csr_degree_order_workspace_size(uint64_t nverts, uint64_t nentries, uint64_t *bytes);
int g5_csr_degree_order(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t nentries,
                        int32_t *d_out_col, void *d_work, uint64_t work_bytes, void *stream);

/* The SSSP copy renumbered for locality: vertices ordered by decreasing
 * degree (ties by index), so the few vertices most relaxations target have
 * their distances, stamps and bits side by side at the front of every
 * per-vertex array, where they stay in L2.  In: the split copy from
 * g5_csr_split_light with its row starts and counts.  Out: perm (caller's
 * vertex -> search's), inv (back), and the copy in the new numbering (rows
 * in the new order, each row's entries in the same order, neighbours
 * renamed); pass them to g5_sssp_* with g5_sssp_params.perm / inv.
 * Scratch: g5_csr_sssp_renumber_workspace_size(nverts).  No counterpart in
 * the reference. */
int g5_csr_sssp_renumber_workspace_size(uint64_t nverts, uint64_t *bytes);
int g5_csr_sssp_renumber(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                         const uint32_t *d_light_deg, const uint32_t *d_tiny_deg, uint64_t nverts, uint64_t nentries,
                         uint32_t *d_perm, uint32_t *d_inv, uint64_t *d_rowstarts_out, int32_t *d_col_out,
                         float *d_w_out, uint32_t *d_light_out, uint32_t *d_tiny_out, void *d_work,
                         uint64_t work_bytes, void *stream);

/* Packs disjoint graphs into one CSR (no counterpart in the reference, which
 * holds one graph): copies one graph's CSR into the destination at vertex
 * offset vbase and entry offset ebase, shifting its column by vbase.  Call
 * once per graph with increasing offsets; the last call also writes the
 * destination's final row start.  d_src_w / d_src_light_deg are optional,
 * together with their destinations. */
int g5_csr_pack_append(const uint64_t *d_src_rowstarts, const int32_t *d_src_col, const float *d_src_w,
                       const uint32_t *d_src_light_deg, uint64_t src_nverts, uint64_t src_nentries, uint64_t vbase,
                       uint64_t ebase, uint64_t *d_dst_rowstarts, int32_t *d_dst_col, float *d_dst_w,
                       uint32_t *d_dst_light_deg, void *stream);

/* ----------------------------------------------------------------- BFS --- */

typedef struct g5_bfs_params {
    float alpha;    /* top-down -> bottom-up when frontier edges > unvisited edges / alpha (default 14)  */
    float beta;     /* bottom-up -> top-down when frontier vertices < nverts / beta (default 24)         */
    int32_t mode;   /* 0 = direction-optimizing, 1 = top-down only, 2 = bottom-up after level 0,
                       3 = one lean block, top-down (a root in a small component; g5_bfs_query picks
                       it from the main-component bitmap)                                             */
    int32_t blocks; /* persistent grid size; 0 = fill the device                                          */
    /* Work tiles (0 = default; none changes a result, only the speed):                                  */
    int32_t big_deg;      /* queue entries with more edges are cut into chunks across the grid (1024)     */
    int32_t chunk;        /* edges per chunk, a multiple of 32 up to 65536 (256)                          */
    int32_t lane_entries; /* bottom-up: entries of a row one lane scans before its warp joins, a multiple
                             of 4 up to 1024 (8)                                                          */
    /* Optional (NULL = none): top[v] = col[rowstarts[v]], the first entry of v's row in the column the
       search is given (nverts for an empty row), from g5_bfs_first_neighbours.  A bottom-up level then
       probes each unvisited vertex's first neighbour from this dense array before reading its row: with
       rows by decreasing neighbour degree (g5_csr_degree_order) most hits are there.  Same parents. */
    const uint32_t *top;
} g5_bfs_params;

typedef struct g5_bfs_stats {
    int32_t levels;           /* BFS levels expanded                           */
    int32_t bottom_up_levels; /* of which bottom-up                            */
    uint64_t reached;         /* vertices with a parent (root included)        */
    uint32_t error_flags;     /* device-side error bits, 0 when none           */
    int32_t solo_levels;      /* levels run by one block before the grid       */
} g5_bfs_stats;

/* One reached vertex of a search, for the host (g5_bfs_export). */
typedef struct g5_bfs_reached {
    uint32_t vertex;
    int32_t depth;
    int64_t parent;
} g5_bfs_reached;

int g5_bfs_workspace_size(uint64_t nverts, uint64_t *bytes);

/* oned_graph_bfs_run, src/traversal.h:47 (src/traversal.cu:479-503): BFS
 * from root over the CSR (d_rowstarts u64[nverts+1], d_col int32).
 * d_pred[v] = parent (int64), -1 when unreached, root for the root;
 * d_depth[v] (optional, int32) = level, -1 when unreached.  One persistent
 * cooperative kernel runs every level; nothing returns to the host.
 * params NULL = defaults. */
int g5_bfs_run(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
               int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
               const g5_bfs_params *params, void *stream);

/* d_bits[ceil(nverts/32)]: bit v set when vertex v has no CSR entry. */
int g5_graph_isolated_bitmap(const uint64_t *d_rowstarts, uint64_t nverts, uint32_t *d_bits, void *stream);

/* g5_bfs_run in two steps, like the reference's oned_graph_bfs_clear
 * (src/traversal.cu:464-477) + oned_graph_bfs_run: g5_bfs_reset clears pred
 * (-1), depth (-1) and the workspace's visited bitmap (O(N) writes) -- to a
 * copy of d_visited_init when given (the isolated-vertex bitmap, so
 * bottom-up levels skip vertices no search can reach) -- and the control
 * block; g5_bfs_traverse runs the persistent kernel (on a reset state). */
int g5_bfs_reset(uint64_t nverts, int64_t *d_pred, int32_t *d_depth, const uint32_t *d_visited_init, void *d_work,
                 uint64_t work_bytes, void *stream);

/* g5_bfs_reset that undoes only what the last search on this workspace
 * wrote, for a workspace that has been reset (by either call) and searched
 * since: after a search that ran on one block (a root outside the main
 * component) it restores the vertices that search reached -- O(reached)
 * instead of O(N) -- in each of pred, depth and the visited bitmap that the
 * search wrote (the same arrays and initial bitmap as now); anything else
 * (another array, a grid search, a search that reported an error) is
 * cleared in full.  The decision is taken on the device, so the call stays
 * stream-ordered.  Not for a workspace fresh from the allocator: its first
 * reset must be g5_bfs_reset.  No counterpart in the reference (its clear is
 * always O(N)). */
int g5_bfs_reset_touched(uint64_t nverts, int64_t *d_pred, int32_t *d_depth, const uint32_t *d_visited_init,
                         void *d_work, uint64_t work_bytes, void *stream);
int g5_bfs_traverse(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                    int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                    const g5_bfs_params *params, void *stream);

/* g5_bfs_traverse from several roots at once (device array): every root is
 * at depth 0 and its own parent.  On disjoint graphs packed with
 * g5_csr_pack_append, one root per graph, this is every graph's own BFS in
 * one persistent launch (no counterpart in the reference).  Reset first with
 * g5_bfs_reset as for g5_bfs_traverse. */
int g5_bfs_traverse_multi(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, const uint64_t *d_roots,
                          uint32_t nroots, int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                          const g5_bfs_params *params, void *stream);

/* One search end to end from host memory, for callers that issue single
 * queries (the reference's synchronous oned_graph_bfs_run,
 * src/traversal.cu:479-503): reads *h_root, runs the traversal on a
 * workspace reset since its last search, stores the statistics in *h_stats
 * and returns once the search is complete.  When h_stats is pinned host
 * memory the kernel writes it itself (no copy call) and the host waits on
 * it rather than on the stream; otherwise it is copied on the stream, which
 * is then synchronised.  h_main_bits (host bitmap of the main component,
 * optional; see g5_bfs_visited_bitmap) lets a root outside it run on a
 * single block, which a small component needs and which avoids launching
 * and waiting for the whole grid. */
int g5_bfs_query(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, const uint64_t *h_root,
                 const uint32_t *h_main_bits, int64_t *d_pred, int32_t *d_depth, void *d_work, uint64_t work_bytes,
                 const g5_bfs_params *params, g5_bfs_stats *h_stats, void *stream);

/* g5_bfs_query prepared once for many queries on one graph, workspace and
 * set of outputs: the arguments are checked and resolved at creation, so
 * g5_bfs_query_plan_run(plan, root) costs one launch and the wait.  h_stats
 * must be pinned host memory the device can address; each run overwrites
 * it.  Reset the workspace before every run as for g5_bfs_query.  The plan
 * keeps pointers only; destroy it before freeing what they point to.  No
 * counterpart in the reference. */
typedef struct g5_bfs_query_plan g5_bfs_query_plan;
int g5_bfs_query_plan_create(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                             const uint32_t *h_main_bits, int64_t *d_pred, int32_t *d_depth, void *d_work,
                             uint64_t work_bytes, const g5_bfs_params *params, g5_bfs_stats *h_stats, void *stream,
                             g5_bfs_query_plan **plan);
int g5_bfs_query_plan_run(g5_bfs_query_plan *plan, uint64_t root);
/* g5_bfs_query_plan_run followed by g5_bfs_export of its result into `out`
 * (capacity records, *h_count the reached count), with one wait on the
 * host: the export kernel runs right behind the search in the stream (one
 * block after a search of a small component). */
int g5_bfs_query_plan_export(g5_bfs_query_plan *plan, uint64_t root, g5_bfs_reached *out, uint64_t capacity,
                             uint64_t *h_count);
void g5_bfs_query_plan_destroy(g5_bfs_query_plan *plan);

/* Copies the visited bitmap of the last search on this workspace (bit v set
 * when v was reached; ceil(nverts/32) words).  After a search from a
 * vertex of the largest component, reset without an initial bitmap, this
 * is the main-component bitmap g5_bfs_query takes. */
int g5_bfs_visited_bitmap(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint32_t *d_bits, void *stream);

/* The result of the last search on this workspace, for the host: one
 * record per reached vertex (root included) -- its index, depth (-1 when the
 * search kept no depth array) and parent -- written to `out` (device memory,
 * or pinned host memory mapped into the device: then the kernel writes it
 * over the bus itself, no copy call), with *h_count = the number of reached
 * vertices.  After a one-block search (a root in a small component) it reads
 * that search's list of touched vertices, records in the order reached, so
 * its cost follows the result, not nverts; otherwise it scans the parents,
 * records in no particular order.  Same d_pred / d_depth as the search.
 * More reached vertices than `capacity`: the first `capacity` records are
 * written, *h_count holds the full count and G5_ERR_INVALID is returned.
 * `out` must be 16-byte aligned.  Synchronises (returns once the records
 * are in place).  The reference
 * leaves Bfs_State.pred on the device (src/traversal.h:59-66). */
int g5_bfs_export(const int64_t *d_pred, const int32_t *d_depth, uint64_t nverts, void *d_work, uint64_t work_bytes,
                  g5_bfs_reached *out, uint64_t capacity, uint64_t *h_count, void *stream);

/* top[v] = d_col[d_rowstarts[v]] (nverts when row v is empty), for g5_bfs_params.top. */
int g5_bfs_first_neighbours(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint32_t *d_top,
                            void *stream);

/* Statistics of the last g5_bfs_run that used this workspace (synchronises). */
int g5_bfs_last_stats(const void *d_work, uint64_t work_bytes, g5_bfs_stats *stats, void *stream);

/* Per-level trace of the last g5_bfs_run on this workspace (synchronises):
 * direction (0 top-down, 1 bottom-up), frontier vertices and edges, and the
 * level's device time from the globaltimer, for up to max_levels levels
 * (64 recorded); *nlevels = levels expanded, *solo_levels = levels run by a
 * single block before the grid took over.  Any output pointer may be NULL
 * except nlevels. */
int g5_bfs_last_trace(const void *d_work, uint64_t work_bytes, int max_levels, int32_t *mode,
                      uint64_t *frontier_vertices, uint64_t *frontier_edges, double *level_ms, int32_t *nlevels,
                      int32_t *solo_levels, void *stream);

/* g5_bfs_run without a workspace, for callers that cannot allocate device
 * memory: a process whose device memory belongs entirely to another
 * allocator (an arena or caching pool) has none to give, and cudaMalloc /
 * cudaFree synchronise the whole device, which a query loop cannot stall
 * for.  The scratch is a fixed 5 MiB array inside the library, present on
 * every GPU that loads it until the process exits; graphs are limited to
 * 2^18 vertices (G5_ERR_INVALID beyond).  The caller still provides the
 * graph and the outputs.  Every call looks up the array's device address in
 * the current context (cheap; after cudaDeviceReset it finds the new
 * context's copy); make one call before any stream capture, so that the
 * library's device code is loaded.  All calls share the one array: calls
 * that overlap on the GPU (other streams, other host threads) race, so
 * serialise them.  Each call clears what must start at zero.  No
 * counterpart in the reference. */
int g5_bfs_run_static(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                      int64_t *d_pred, int32_t *d_depth, const g5_bfs_params *params, void *stream);

/* bfs_compute_dist_from_pred, src/traversal.h:48 (src/traversal.cu:505-563):
 * d_dist[v] = -1 where pred is -1, 0 at the root, the tree depth where the
 * parent chain reaches the root through CSR edges, INT64_MAX otherwise.
 * d_work needs g5_validate_workspace_size bytes (not the BFS workspace,
 * whose statistics it would overwrite).  Synchronises once per level. */
int g5_bfs_dist_from_pred(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts,
                          const int64_t *d_pred, uint64_t root, int64_t *d_dist, void *d_work,
                          uint64_t work_bytes, void *stream);

/* ---------------------------------------------------------------- SSSP --- */

typedef struct g5_sssp_params {
    float delta;    /* bucket width (default 0.1, the reference's fixed value) */
    int32_t blocks; /* persistent grid size; 0 = fill the device              */
    float pull;     /* a bucket's heavy phase pulls (each unsettled vertex scans
                       its own heavy entries) when the bucket's rows hold at
                       least pull x the entries of all unsettled vertices'
                       rows; 0 = default (1.0), < 0 = always push           */
    int32_t sub_min; /* once a bucket's light frontier holds this many light
                       CSR entries, the rest of the bucket runs in 32
                       sub-buckets in distance order; 0 = default (2^25),
                       < 0 = never                                           */
    int32_t small;   /* 1: the source's component is small (outside the main
                       component): one lean block, label-correcting rounds,
                       same distances and parents; 0 = the bucketed search  */
    const uint32_t *tiny_deg; /* per-vertex count of the leading light entries
                       below light_delta / G5_TINY_DIV, rows split by
                       g5_csr_split_tiny (optional, nullptr = not split).  A
                       sub-bucket then reads only that prefix of a row while
                       its distances are still dropping                      */
    int32_t check_opens; /* 1: bucket and sub-bucket opens exchange their list
                       stamps atomically and fail the search (G5_ERR_DEVICE,
                       "held a vertex twice") if a queue held a vertex twice;
                       a test aid, same results; 0 = plain stores (default) */
    int32_t big_deg; /* list entries with more edges to expand are cut into
                       chunks across the grid; 0 = default (256)            */
    int32_t chunk;   /* edges per chunk, a multiple of 64 up to 65536; 0 =
                       default (256).  Neither tile changes a result        */
    const uint32_t *perm; /* renumbered search (both set, from
                       g5_csr_sssp_renumber) or not (both NULL): the CSR
                       arguments (row starts, column, weights, light and
                       tiny counts) are the renumbered copy, the root(s) and
                       the outputs stay in the caller's numbering.  Same
                       distances; each parent is still a tight edge's
                       source (the smallest in the search's numbering)     */
    const uint32_t *inv;
} g5_sssp_params;

int g5_sssp_workspace_size(uint64_t nverts, uint64_t *bytes);

/* oned_graph_sssp_run, src/traversal.h:52 (src/traversal.cu:638-711):
 * delta-stepping with float32 relaxations.  d_dist[v] = distance, -1.0f when
 * unreached; d_pred[v] = a parent on a shortest path, -1 when unreached.
 * d_light_deg (optional) = per-vertex count of leading row entries lighter
 * than `light_delta` as produced by g5_csr_fill; it is used when
 * params->delta <= light_delta (light edges are then those below
 * light_delta), otherwise rows are filtered by weight against delta.
 * The bucket ring holds 31 buckets ahead, so delta must exceed
 * (largest weight) / 30 (G5_ERR_INVALID from the search otherwise). */
int g5_sssp_run(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, const uint32_t *d_light_deg,
                float light_delta, uint64_t nverts, uint64_t root, float *d_dist, int64_t *d_pred, void *d_work,
                uint64_t work_bytes, const g5_sssp_params *params, void *stream);

/* g5_sssp_run in two steps, like the reference's oned_graph_sssp_clear
 * (src/traversal.cu:625-636 with sssp_clear_kernel :242-253, which also
 * set pred to -1 and dist to -1.0f) +
 * oned_graph_sssp_run: g5_sssp_reset clears the workspace's O(N) arrays
 * (distances, stamps, settled bitmap) and its control block and, when given
 * d_dist and d_pred (both or neither), fills them with -1.0f / -1;
 * g5_sssp_traverse (on a state reset since its last search) runs the
 * persistent kernel and writes d_dist / d_pred.
 * When the traverse gets the same output arrays the reset pre-filled, it
 * writes only the reached vertices (O(reached) work); otherwise it writes
 * all nverts entries. */
int g5_sssp_reset(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes, void *stream);

/* g5_sssp_reset that undoes only what the last search on this workspace
 * wrote, for a workspace that has been reset (by either call) and searched
 * since: after a one-block search (a source outside the main component,
 * g5_sssp_params.small) it restores the packed distances, stamps and -- when
 * they are the arrays that search wrote sparsely -- the outputs of the
 * vertices it reached: O(reached) instead of O(N); after any other search
 * it is g5_sssp_reset.  Decided on the device (stream-ordered).  Not for a
 * workspace fresh from the allocator: its first reset must be g5_sssp_reset.
 * No counterpart in the reference (its clear is always O(N)). */
int g5_sssp_reset_touched(uint64_t nverts, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                          void *stream);
int g5_sssp_traverse(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, const uint32_t *d_light_deg,
                     float light_delta, uint64_t nverts, uint64_t root, float *d_dist, int64_t *d_pred, void *d_work,
                     uint64_t work_bytes, const g5_sssp_params *params, void *stream);

/* g5_sssp_traverse from several sources at once (device array), all at
 * distance 0: on packed disjoint graphs, one source per graph, every
 * graph's own SSSP in one persistent launch (no counterpart in the
 * reference). */
int g5_sssp_traverse_multi(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w,
                           const uint32_t *d_light_deg, float light_delta, uint64_t nverts, const uint64_t *d_roots,
                           uint32_t nroots, float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes,
                           const g5_sssp_params *params, void *stream);

/* Buckets and phases of the last g5_sssp_run that used this workspace, and
 * its device status (synchronises). */
int g5_sssp_last_status(const void *d_work, uint64_t work_bytes, uint64_t *buckets, uint64_t *phases, void *stream);

/* Counters and per-phase trace of the last g5_sssp_run on this workspace
 * (synchronises): counts[7] = edges looked at, edges into settled vertices,
 * atomicMin issued, distances lowered, bucket-queue pushes, same-bucket
 * frontier and sub-bucket pushes, heavy phases run as pulls; per phase (up
 * to 256) its kind (0 bucket open, 1 light, 2 heavy push, 3 heavy pull,
 * 4 sub-bucket open, 5 bucket split into sub-buckets), input list size,
 * device milliseconds and edges looked at.  Any output pointer may be NULL. */
int g5_sssp_last_trace(const void *d_work, uint64_t work_bytes, uint64_t counts[7], int max_phases, int32_t *kind,
                       uint64_t *size, double *phase_ms, uint64_t *phase_edges, int32_t *nphases, void *stream);

/* ---------------------------------------------------------- validation --- */

int g5_validate_workspace_size(uint64_t nverts, uint64_t *bytes);

/* oned_graph_edge_count, examples/graph500_runner.cu:171-201: number of CSR
 * entries col[e] <= v over rows of vertices with pred[v] != -1 (the TEPS
 * edge count).  Synchronises. */
int g5_edge_count(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, const int64_t *d_pred,
                  void *d_work, uint64_t work_bytes, uint64_t *count, void *stream);

/* oned_graph_bfs_validate, examples/graph500_runner.cu:203-255 (rules 1-7 of
 * :84-169): *errors = number of violations; 0 means the parent tree and the
 * depths (from g5_bfs_dist_from_pred) are a valid BFS.  Synchronises. */
int g5_bfs_validate(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                    const int64_t *d_pred, const int64_t *d_dist, void *d_work, uint64_t work_bytes,
                    uint64_t *errors, void *stream);

/* SSSP validation (the reference has none): root at 0 with itself as parent;
 * pred = -1 exactly where dist = -1; no edge from a reached vertex leads to
 * an unreached one or can still be relaxed (dist[u] + w < dist[v] in float);
 * every reached non-root v has an edge (pred[v], v, w) with
 * dist[pred[v]] + w == dist[v].  Synchronises. */
int g5_sssp_validate(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                     uint64_t root, const float *d_dist, const int64_t *d_pred, void *d_work, uint64_t work_bytes,
                     uint64_t *errors, void *stream);

/* The two validators on a renumbered CSR (perm: caller's vertex -> the CSR's,
 * inv back, e.g. the copy from g5_csr_sssp_renumber, whose rows hold every
 * entry of the graph): pred, dist and root stay in the caller's numbering;
 * the same error counts as on the graph in the caller's numbering.  The
 * records the rules read (a vertex's depth or distance and parent) then lie
 * in degree order, so the neighbours most entries point at share a few L2
 * lines.  NULL perm and inv: g5_bfs_validate / g5_sssp_validate. */
int g5_bfs_validate_renumbered(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t root,
                               const int64_t *d_pred, const int64_t *d_dist, const uint32_t *d_perm,
                               const uint32_t *d_inv, void *d_work, uint64_t work_bytes, uint64_t *errors,
                               void *stream);
int g5_sssp_validate_renumbered(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                                uint64_t root, const float *d_dist, const int64_t *d_pred, const uint32_t *d_perm,
                                const uint32_t *d_inv, void *d_work, uint64_t work_bytes, uint64_t *errors,
                                void *stream);

/* ------------------------------------------------------- batched BFS --- */
/*
 * Multi-source BFS: up to 256 roots searched together in one persistent
 * launch, one bit per root in a 256-bit row per vertex.  No counterpart in
 * the reference, which searches one root per oned_graph_bfs_run call
 * (src/traversal.cu:479-503); for every root the depth array equals that
 * search's depth (g5_bfs_run with d_depth).  Parents are not produced.
 *
 * A workspace is bound to one graph: size it with g5_msbfs_workspace_size,
 * fill its per-graph lists once with g5_msbfs_prepare, then run any number of
 * searches.  Depths are kept as `depth_bits` bit-planes, so a search whose
 * graph is deeper than 2^depth_bits - 1 levels fails with G5_ERR_INVALID.
 */
typedef struct g5_msbfs_params {
    float alpha;    /* top-down while frontier edges * alpha < CSR entries (<= 0: 32) */
    int mode;       /* 0 automatic, 1 top-down only, 2 pull only */
    int check_frontier; /* pull levels test the frontier bitmap before reading a neighbour's row:
                           0 when under half the entries lead into the frontier, 1 always, 2 never */
    int blocks;     /* persistent grid (0 = every co-resident block) */
} g5_msbfs_params;

typedef struct g5_msbfs_stats {
    int32_t levels;        /* levels expanded */
    int32_t pull_levels;   /* of which pull (bottom-up) levels */
    uint32_t error_flags;  /* nonzero: the search did not complete */
    uint32_t nroots;
    uint64_t pairs_reached; /* sum over roots of the vertices each reached */
    uint64_t frontier_edges; /* sum over levels of the frontier's CSR entries */
} g5_msbfs_stats;

/* Bytes of a workspace for a graph of nverts vertices and nentries CSR
 * entries with depth_bits planes (1..8; 0 = 6, depths up to 63). */
int g5_msbfs_workspace_size(uint64_t nverts, uint64_t nentries, int depth_bits, uint64_t *bytes);

/* Builds the workspace's copy of the graph: vertices renumbered by
 * decreasing degree (so the rows most CSR entries point at sit together and
 * stay in L2), the CSR in that order with its column in the new numbers,
 * and the longer rows (above 256 entries) cut into 1024-entry chunks.  Once
 * per graph and workspace; later searches read only the workspace.
 * Synchronises. */
int g5_msbfs_prepare(const uint64_t *d_rowstarts, const int32_t *d_col, uint64_t nverts, uint64_t nentries,
                     int depth_bits, void *d_work, uint64_t work_bytes, void *stream);

/* Searches from h_roots[0..nroots) (host array of vertex ids, 1 <= nroots
 * <= 256, repeats allowed) on the prepared graph.  Root i is bit i of every
 * row.  Stream-ordered; h_stats (may be NULL) makes the call synchronise
 * and report the search's status. */
int g5_msbfs_run(uint64_t nverts, uint64_t nentries, int depth_bits, const uint64_t *h_roots, uint32_t nroots,
                 void *d_work, uint64_t work_bytes, const g5_msbfs_params *params, g5_msbfs_stats *h_stats,
                 void *stream);

/* Depths of the last search as bytes, root-major: d_out[i * nverts + v] is
 * root i's depth of v, 255 where root i did not reach v. */
int g5_msbfs_depths_u8(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint64_t nentries, int depth_bits,
                       uint32_t nroots, uint8_t *d_out, void *stream);

/* Depth array of root i of the last search, -1 where unreached (the layout
 * of g5_bfs_run's d_depth). */
int g5_msbfs_depth(const void *d_work, uint64_t work_bytes, uint64_t nverts, uint64_t nentries, int depth_bits,
                   uint32_t root_index, int32_t *d_depth, void *stream);

/* Status and per-level trace of the last search (synchronises).  mode[i]:
 * 0 top-down, 1 pull. */
int g5_msbfs_last_stats(const void *d_work, uint64_t work_bytes, g5_msbfs_stats *stats, void *stream);
int g5_msbfs_last_trace(const void *d_work, uint64_t work_bytes, int max_levels, int32_t *mode,
                        uint64_t *frontier_vertices, uint64_t *frontier_edges, double *level_ms, int32_t *nlevels,
                        void *stream);

/* ------------------------------------------------------ batched SSSP --- */

/* SSSP from up to 32 sources of one graph in one persistent launch (the
 * reference runs one source at a time, src/traversal.cu:638-711): one warp
 * lane per source, each vertex's 32 packed (distance, parent) words side by
 * side, so an edge's column entry and weight are read once for every
 * source; label-correcting rounds over the vertices whose words dropped, in
 * buckets of width delta shared by the sources (0 = 0.1), as delta-stepping
 * takes them.
 * Distances and parents equal g5_sssp_run's for each source bit for bit.
 * Any row order of the CSR will do (the renumbered SSSP copy: pass its
 * perm / inv, sources and outputs stay in the caller's numbering).
 * d_dist / d_pred (optional, nsources x nverts, source-major: entry
 * s * nverts + v) receive -1.0f / -1 where unreached.  Synchronises when
 * h_stats is given.  Scratch: g5_sssp_multi_workspace_size (about 276 bytes
 * per vertex). */
typedef struct g5_sssp_multi_stats {
    int32_t rounds;            /* relaxation rounds                                   */
    uint32_t error_flags;      /* device-side error bits, 0 when none                 */
    uint64_t frontier_entries; /* queued vertices over all rounds                     */
    uint64_t entries_scanned;  /* CSR entries relaxed (each for every changed source) */
} g5_sssp_multi_stats;
int g5_sssp_multi_workspace_size(uint64_t nverts, uint64_t *bytes);
int g5_sssp_multi_run(const uint64_t *d_rowstarts, const int32_t *d_col, const float *d_w, uint64_t nverts,
                      const uint32_t *d_perm, const uint32_t *d_inv, const uint64_t *h_sources, uint32_t nsources,
                      float *d_dist, int64_t *d_pred, void *d_work, uint64_t work_bytes, float delta,
                      int32_t blocks, g5_sssp_multi_stats *h_stats, void *stream);
/* Statistics and status of the last g5_sssp_multi_run on this workspace
 * (synchronises `stream`); its grid: blocks for a graph of nverts vertices
 * and the largest co-resident grid. */
int g5_sssp_multi_last_stats(const void *d_work, uint64_t work_bytes, g5_sssp_multi_stats *stats, void *stream);
int g5_sssp_multi_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks);

/* ------------------------------------------------------------- grids ----- */
/* Grid (blocks) sized for a graph of nverts vertices -- what g5_bfs_* and
 * g5_sssp_* launch with params.blocks = 0 (g5_msbfs_run then takes every
 * co-resident block instead) -- and the most blocks of the kernel that fit
 * on the device at once.  A caller that runs searches on several streams at
 * the same time passes these grids in params.blocks and keeps their sum
 * within max_blocks, so every cooperative grid can be resident together. */
int g5_bfs_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks);
int g5_sssp_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks);
int g5_msbfs_grid(uint64_t nverts, int32_t *blocks, int32_t *max_blocks);

/* ------------------------------------------------------------- testing --- */

/* Launches a two-block cooperative kernel whose grid barrier can never
 * complete, so each block's bounded wait gives up after limit_ms: returns
 * G5_ERR_TIMEOUT and leaves the context usable.  It exercises the failure
 * path every persistent kernel here shares (no counterpart in the reference,
 * whose grid barrier spins without a bound, src/traversal.cu:126).
 * d_work needs 8 bytes. */
int g5_selftest_wait_timeout(unsigned limit_ms, void *d_work, uint64_t work_bytes, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* G500B_H */
