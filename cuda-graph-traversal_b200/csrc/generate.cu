// generate.cu -- K1: Graph500 Kronecker edge generation (bit-exact with the
// reference's generate_kronecker_range, src/graph_generation.cu:225-310).
//
// Each edge ei is drawn from the MRG stream that starts at the seed jumped
// ahead by ei * 2^64 steps.  The reference jumps every edge from the seed
// (up to four table matrix products per edge).  Here thread t of T handles
// edges t, t+T, t+2T, ... and moves from one to the next with a single
// product by the fixed matrix A^(T * 2^64), computed on the host per
// launch; only each thread's first edge uses the byte tables.  Writes are
// coalesced: consecutive threads write consecutive 16-byte edges.
//
// Bound: integer ALU.  Per edge: SCALE (+ rare rejections) MRG steps, one
// 5x5 modular matrix-vector product, two scrambles, one float draw; output
// 20 bytes per edge (16-byte pair + 4-byte weight).
#include <mutex>

#include "g5_common.cuh"
#include "g5_mrg.cuh"

namespace g5 {

// ------------------------------------------------------- host MRG tables --

static MrgMatrix mat_mul(const MrgMatrix &a, const MrgMatrix &b) {
    MrgMatrix r;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) {
            uint64_t acc = 0;
            for (int k = 0; k < 5; ++k) acc = (acc + (uint64_t)a.m[5 * i + k] * b.m[5 * k + j]) % MRG_P;
            r.m[5 * i + j] = (uint32_t)acc;
        }
    return r;
}

static MrgMatrix identity() {
    MrgMatrix r{};
    for (int i = 0; i < 5; ++i) r.m[6 * i] = 1;
    return r;
}

// g_jump[b][v] = A^(v * 256^b): row b holds the powers of A^(256^b).
static MrgMatrix g_jump[24][256];
static std::once_flag g_jump_once;

static void build_jump_tables() {
    MrgMatrix a{};
    a.m[0] = MRG_X;  // z1' = X z1 + Y z5
    a.m[4] = MRG_Y;
    for (int i = 1; i < 5; ++i) a.m[5 * i + i - 1] = 1;  // z_{i+1}' = z_i
    MrgMatrix p = a;
    for (int b = 0; b < 24; ++b) {
        g_jump[b][0] = identity();
        for (int v = 1; v < 256; ++v) g_jump[b][v] = mat_mul(g_jump[b][v - 1], p);
        for (int k = 0; k < 8; ++k) p = mat_mul(p, p);
    }
}

const MrgMatrix &mrg_jump_matrix(int byte, int value) {
    std::call_once(g_jump_once, build_jump_tables);
    return g_jump[byte][value];
}

void mrg_skip_host(MrgState &s, uint64_t high, uint64_t mid, uint64_t low) {
    const uint64_t parts[3] = {low, mid, high};
    for (int w = 0; w < 3; ++w) {
        uint64_t x = parts[w];
        for (int b = 0; x; ++b, x >>= 8)
            if (x & 0xFF) mrg_apply(mrg_jump_matrix(8 * w + b, (int)(x & 0xFF)), s);
    }
}

MrgMatrix mrg_jump_mid(uint64_t n) {
    MrgMatrix r = identity();
    for (int b = 0; n; ++b, n >>= 8)
        if (n & 0xFF) r = mat_mul(r, mrg_jump_matrix(8 + b, (int)(n & 0xFF)));
    return r;
}

// Device copy of the byte tables for 2^64-step jumps (bytes 8..15 of the
// exponent): 8 * 256 matrices, 200 KiB per device.
__device__ MrgMatrix g5_mrg_mid_table[8 * 256];

int mrg_device_mid_table(const MrgMatrix **out) {
    static std::mutex mu;
    static bool loaded[64] = {};
    int dev = 0;
    G5_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(G5_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!loaded[dev]) {
        static MrgMatrix host[8 * 256];
        for (int b = 0; b < 8; ++b)
            for (int v = 0; v < 256; ++v) host[256 * b + v] = mrg_jump_matrix(8 + b, v);
        G5_CUDA_TRY(cudaMemcpyToSymbol(g5_mrg_mid_table, host, sizeof host));
        loaded[dev] = true;
    }
    void *p = nullptr;
    G5_CUDA_TRY(cudaGetSymbolAddress(&p, g5_mrg_mid_table));
    *out = (const MrgMatrix *)p;
    return G5_OK;
}

// ---------------------------------------------------------------- kernel --

__global__ void __launch_bounds__(256) kron_generate_kernel(MrgState base, MrgMatrix stride_jump, int log_n,
                                                            int64_t start, int64_t count, uint64_t val0,
                                                            uint64_t val1, const MrgMatrix *__restrict__ mid_table,
                                                            ulonglong2 *__restrict__ edges,
                                                            float *__restrict__ weights) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    if (t >= count) return;

    // Stream of the thread's first edge: seed * A^((start + t) * 2^64).
    MrgState z = base;
    uint64_t e = (uint64_t)(start + t);
    for (int b = 0; e; ++b, e >>= 8)
        if (e & 0xFF) mrg_apply(mid_table[256 * b + (e & 0xFF)], z);

    for (int64_t i = t; i < count; i += T) {
        MrgState s = z;
        uint64_t src = 0, dst = 0;
        // One quadrant per level, most significant bit first; on the
        // diagonal the lower-left quadrant folds onto the upper-right
        // (cuda_make_one_edge, src/graph_generation.cu:186-207).
        for (int lvl = log_n - 1; lvl >= 0; --lvl) {
            int q = kron_quadrant(s);
            uint64_t so = (uint64_t)(q >> 1), to = (uint64_t)(q & 1);
            if (src == dst && so > to) { so = 0; to = 1; }
            src |= so << lvl;
            dst |= to << lvl;
        }
        edges[i] = make_ulonglong2(kron_scramble(src, log_n, val0, val1), kron_scramble(dst, log_n, val0, val1));
        weights[i] = mrg_unit_float(mrg_next(s));
        mrg_apply(stride_jump, z);
    }
}

}  // namespace g5

using namespace g5;

extern "C" int g5_make_mrg_seed(uint64_t s1, uint64_t s2, uint32_t seed[5]) {
    G5_CHECK_ARG(seed, "g5_make_mrg_seed: seed is NULL");
    // make_mrg_seed, src/graph_generation.cu:248-254.
    seed[0] = (uint32_t)(s1 & 0x3FFFFFFFu) + 1;
    seed[1] = (uint32_t)((s1 >> 30) & 0x3FFFFFFFu) + 1;
    seed[2] = (uint32_t)(s2 & 0x3FFFFFFFu) + 1;
    seed[3] = (uint32_t)((s2 >> 30) & 0x3FFFFFFFu) + 1;
    seed[4] = (uint32_t)((s2 >> 60) << 4) + (uint32_t)(s1 >> 60) + 1;
    return G5_OK;
}

extern "C" int g5_make_random_numbers(int64_t n, uint64_t s1, uint64_t s2, int64_t position, double *out) {
    G5_CHECK_ARG(n >= 0 && (n == 0 || out), "g5_make_random_numbers: bad output");
    uint32_t seed[5];
    g5_make_mrg_seed(s1, s2, seed);
    MrgState s{{seed[0], seed[1], seed[2], seed[3], seed[4]}};
    // Jump by 2*2^128 + 2*position (src/graph_generation.cu:262).
    mrg_skip_host(s, 2, 0, 2 * (uint64_t)position);
    for (int64_t i = 0; i < n; ++i) out[i] = (double)mrg_next(s) * .0000000004656612875245796924106;
    return G5_OK;
}

extern "C" int g5_scramble_keys(const uint32_t seed[5], uint64_t *val0, uint64_t *val1) {
    G5_CHECK_ARG(seed && val0 && val1, "g5_scramble_keys: NULL argument");
    MrgState s{{seed[0], seed[1], seed[2], seed[3], seed[4]}};
    // src/graph_generation.cu:290-300: jump 50*2^128 + 7*2^64, then two
    // 62-bit keys built from pairs of draws.
    mrg_skip_host(s, 50, 7, 0);
    uint64_t a = mrg_next(s);
    a = a * 0xFFFFFFFFull + mrg_next(s);
    uint64_t b = mrg_next(s);
    b = b * 0xFFFFFFFFull + mrg_next(s);
    *val0 = a;
    *val1 = b;
    return G5_OK;
}

extern "C" int g5_generate_kronecker_range(const uint32_t seed[5], uint32_t log_n, int64_t start_edge,
                                           int64_t end_edge, uint64_t *d_edges, float *d_weights, void *stream) {
    clear_error();
    G5_CHECK_ARG(seed, "g5_generate_kronecker_range: seed is NULL");
    G5_CHECK_ARG(log_n >= 1 && log_n <= 62, "g5_generate_kronecker_range: log_n %u outside [1, 62]", log_n);
    G5_CHECK_ARG(start_edge >= 0, "g5_generate_kronecker_range: negative start edge");
    for (int i = 0; i < 5; ++i)
        G5_CHECK_ARG(seed[i] < MRG_P, "g5_generate_kronecker_range: seed word %d not below 2^31-1", i);
    G5_CHECK_ARG(seed[0] | seed[1] | seed[2] | seed[3] | seed[4], "g5_generate_kronecker_range: all-zero seed");
    if (end_edge <= start_edge) return G5_OK;
    G5_CHECK_ARG(d_edges && d_weights, "g5_generate_kronecker_range: NULL output");
    G5_CHECK_ARG(((uintptr_t)d_edges & 15) == 0, "g5_generate_kronecker_range: edges not 16-byte aligned");

    const int64_t count = end_edge - start_edge;
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    const MrgMatrix *table = nullptr;
    if ((rc = mrg_device_mid_table(&table))) return rc;

    const int threads = 256;
    int64_t blocks = (count + threads - 1) / threads;
    const int64_t cap = (int64_t)di.sms * (di.max_threads_per_sm / threads);
    if (blocks > cap) blocks = cap;
    const uint64_t T = (uint64_t)blocks * threads;

    uint64_t val0, val1;
    g5_scramble_keys(seed, &val0, &val1);
    MrgState base{{seed[0], seed[1], seed[2], seed[3], seed[4]}};
    MrgMatrix jump = mrg_jump_mid(T);
    kron_generate_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        base, jump, (int)log_n, start_edge, count, val0, val1, table, (ulonglong2 *)d_edges, d_weights);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}
