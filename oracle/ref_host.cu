// ref_host.cu -- the reference's host-side MRG code behind a C ABI, for
// pinning the oracle's recomputed jump tables (TEST INFRASTRUCTURE ONLY).
//
// It compiles the reference's src/graph_generation.cu into this translation
// unit from where it lies (oracle/ref.mk puts REF_ROOT/src on the include
// path), so its static __host__ __device__ helpers -- cuda_mrg_skip over the
// generated table of src/mrg_transitions.cu, and the MRG step -- can be
// called from the host.
#include "graph_generation.cu"

// generate_kronecker_range and tuple_graph_load in the included file refer to
// the worker arena; nothing here calls them, so the symbol only has to exist.
void *_worker_arena_push_array(Worker_State *, u64, u64, u64, u64 *) { return 0; }

extern "C" {

// state <- A^(high*2^128 + mid*2^64 + low) state  (cuda_mrg_skip, :209-223)
void ref_mrg_skip(u32 z[5], u64 high, u64 mid, u64 low) {
    Mrg_State s = {z[0], z[1], z[2], z[3], z[4]};
    cuda_mrg_skip(&s, high, mid, low);
    z[0] = s.z1; z[1] = s.z2; z[2] = s.z3; z[3] = s.z4; z[4] = s.z5;
}

// n successive outputs of cuda_mrg_get_uint_orig (:82-85) from state z.
void ref_mrg_draw(u32 z[5], int n, u32 *out) {
    Mrg_State s = {z[0], z[1], z[2], z[3], z[4]};
    for (int i = 0; i < n; ++i) out[i] = cuda_mrg_get_uint_orig(&s);
    z[0] = s.z1; z[1] = s.z2; z[2] = s.z3; z[3] = s.z4; z[4] = s.z5;
}

void ref_make_mrg_seed(u64 s1, u64 s2, u32 *seed) { make_mrg_seed(s1, s2, seed); }

void ref_make_random_numbers(i64 n, u64 s1, u64 s2, i64 pos, f64 *out) {
    make_random_numbers(n, s1, s2, pos, out);
}

}  // extern "C"
