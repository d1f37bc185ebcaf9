/*
 * graph_generation.h -- drop-in for RuanPetrus/cuda-graph-traversal
 * src/graph_generation.h: same structs (:6-30) and functions (:33-43).
 * Edges and weights are bit-identical to the reference's for the same seed
 * and range; generation runs in libg500b's sm_100a kernel.
 */
#ifndef GRAPH_GENERATION_H
#define GRAPH_GENERATION_H
#include "base.h"
#include "worker.h"

typedef struct Packed_Edge Packed_Edge;
struct Packed_Edge {
    u64 v0;
    u64 v1;
};

typedef struct Tuple_Graph Tuple_Graph;
struct Tuple_Graph {
    Packed_Edge *edges;
    u64 edges_size;
    u64 max_edges_size;
    u64 nglobaledges;
    f32 *weights;
};

/* Kept for layout compatibility; the jump matrices are recomputed by the
 * library rather than read from a table of this type. */
typedef struct Mrg_Transition_Matrix Mrg_Transition_Matrix;
struct Mrg_Transition_Matrix {
    u32 s, t, u, v, w;
    u32 a, b, c, d;
};

typedef struct Mrg_State Mrg_State;
struct Mrg_State {
    u32 z1, z2, z3, z4, z5;
};

/* Edges [start_edge, end_edge) of a 2^logN-vertex Kronecker graph into
 * arena arrays of ws; seed words in [0, 2^31-1), not all zero. */
void generate_kronecker_range(Worker_State *st, u32 seed[5], u32 logN, i64 start_edge, i64 end_edge,
                              Tuple_Graph *tg);

void make_mrg_seed(u64 userseed1, u64 userseed2, u32 *seed);
void make_random_numbers(i64 nvalues, u64 userseed1, u64 userseed2, i64 position, f64 *result);

/* graph-refactor.bin (raw Packed_Edge) and graph-refactor.bin.weights (raw
 * f32) at offset start_edge, the reference's format; sizes are 64-bit here,
 * so dumps above 2 GiB stay whole. */
void tuple_graph_dump(const Tuple_Graph *tg, i64 start_edge);
void tuple_graph_load(Worker_State *ws, Tuple_Graph *tg, i64 start_edge, i64 edge_count);

#endif /* GRAPH_GENERATION_H */
