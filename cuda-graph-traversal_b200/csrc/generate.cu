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

__global__ void __launch_bounds__(256) kron_generate_kernel(KronLaunch k, ulonglong2 *__restrict__ edges,
                                                            float *__restrict__ weights) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    if (t >= k.count) return;
    MrgState z = kron_thread_start(k, t);
    for (int64_t i = t; i < k.count; i += T) {
        uint64_t src, dst;
        float w;
        kron_edge(z, k.log_n, k.val0, k.val1, src, dst, w);
        edges[i] = make_ulonglong2(src, dst);
        weights[i] = w;
        mrg_apply(k.stride_jump, z);
    }
}

int kron_prepare(const uint32_t seed[5], uint32_t log_n, int64_t start, int64_t end, int threads_per_block,
                 KronLaunch *k, int *blocks, const char *who) {
    G5_CHECK_ARG(seed, "%s: seed is NULL", who);
    G5_CHECK_ARG(log_n >= 1 && log_n <= 62, "%s: log_n %u outside [1, 62]", who, log_n);
    G5_CHECK_ARG(start >= 0 && end >= start, "%s: bad edge range", who);
    for (int i = 0; i < 5; ++i) G5_CHECK_ARG(seed[i] < MRG_P, "%s: seed word %d not below 2^31-1", who, i);
    G5_CHECK_ARG(seed[0] | seed[1] | seed[2] | seed[3] | seed[4], "%s: all-zero seed", who);
    const int64_t count = end - start;
    *blocks = 0;
    k->count = count;
    if (!count) return G5_OK;  // nothing to launch; no device work either
    DeviceInfo di;
    int rc = device_info(&di);
    if (rc) return rc;
    if ((rc = mrg_device_mid_table(&k->mid_table))) return rc;
    int64_t b = (count + threads_per_block - 1) / threads_per_block;
    const int64_t cap = (int64_t)di.sms * (di.max_threads_per_sm / threads_per_block);
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    *blocks = (int)b;
    k->base = MrgState{{seed[0], seed[1], seed[2], seed[3], seed[4]}};
    k->stride_jump = mrg_jump_mid((uint64_t)b * threads_per_block);
    k->log_n = (int)log_n;
    k->start = start;
    k->count = count;
    g5_scramble_keys(seed, &k->val0, &k->val1);
    return G5_OK;
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
    KronLaunch k;
    int blocks = 0;
    int rc = kron_prepare(seed, log_n, start_edge, end_edge < start_edge ? start_edge : end_edge, 256, &k, &blocks,
                          "g5_generate_kronecker_range");
    if (rc) return rc;
    if (end_edge <= start_edge) return G5_OK;
    G5_CHECK_ARG(d_edges && d_weights, "g5_generate_kronecker_range: NULL output");
    G5_CHECK_ARG(((uintptr_t)d_edges & 15) == 0, "g5_generate_kronecker_range: edges not 16-byte aligned");
    kron_generate_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(k, (ulonglong2 *)d_edges, d_weights);
    G5_CUDA_TRY(cudaGetLastError());
    return G5_OK;
}
