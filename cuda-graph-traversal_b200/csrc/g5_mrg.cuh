// g5_mrg.cuh -- the Graph500 multiple recursive generator (MRG) used by the
// Kronecker generator, as host+device inline code.
//
// The generator is z1' = 107374182*z1 + 104480*z5 (mod 2^31-1) with the
// other four words shifting down (src/graph_generation.cu:73-80 of the
// reference; its mul_x/mul_y helpers :38-50 compute the same products by
// Schrage's method).  Jumping n steps ahead multiplies the state by A^n,
// A the 5x5 companion matrix of that recurrence; the reference reads A^n
// from a byte-indexed table (src/mrg_transitions.cu:14,
// src/graph_generation.cu:209-223), which this library recomputes on the
// host instead of storing (generate.cu).  All arithmetic is exact mod p, so any
// correct evaluation order yields the reference's bits.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define G5_HD __host__ __device__ __forceinline__
#else
#define G5_HD inline
#endif

namespace g5 {

constexpr uint32_t MRG_P = 0x7FFFFFFFu;
constexpr uint32_t MRG_X = 107374182u;
constexpr uint32_t MRG_Y = 104480u;

// State, newest word first: z[0] = z1 ... z[4] = z5.
struct MrgState {
    uint32_t z[5];
};

// A full 5x5 matrix mod p, row-major.
struct MrgMatrix {
    uint32_t m[25];
};

// x mod p for any 64-bit x (two Mersenne folds and one conditional subtract).
G5_HD uint32_t mrg_fold(uint64_t x) {
    x = (x & MRG_P) + (x >> 31);
    x = (x & MRG_P) + (x >> 31);
    return (uint32_t)(x >= MRG_P ? x - MRG_P : x);
}

G5_HD uint32_t mrg_next(MrgState &s) {
    uint32_t n = mrg_fold((uint64_t)MRG_X * s.z[0] + (uint64_t)MRG_Y * s.z[4]);
    s.z[4] = s.z[3];
    s.z[3] = s.z[2];
    s.z[2] = s.z[1];
    s.z[1] = s.z[0];
    s.z[0] = n;
    return n;
}

// s <- M s.
G5_HD void mrg_apply(const MrgMatrix &M, MrgState &s) {
    uint32_t in[5] = {s.z[0], s.z[1], s.z[2], s.z[3], s.z[4]};
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int i = 0; i < 5; ++i) {
        const uint32_t *r = &M.m[5 * i];
        uint64_t acc = (uint64_t)r[0] * in[0] + (uint64_t)r[1] * in[1] + (uint64_t)r[2] * in[2];
        acc = (acc & MRG_P) + (acc >> 31);
        acc += (uint64_t)r[3] * in[3] + (uint64_t)r[4] * in[4];
        s.z[i] = mrg_fold(acc);
    }
}

// Quadrant of one Kronecker level with the reference's initiator
// (src/graph_generation.cu:114-143, SPK_NOISE_LEVEL 0): draws below
// (2^31-1) mod 10^4 are rejected, the rest reduced mod 10^4 and split at
// 1900 (quadrant 1), 3800 (2), 9500 (0), else 3.
G5_HD int kron_quadrant(MrgState &s) {
    uint32_t u = mrg_next(s);
    while (u < MRG_P % 10000u) u = mrg_next(s);
    u %= 10000u;
    return u < 1900u ? 1 : u < 3800u ? 2 : u < 9500u ? 0 : 3;
}

G5_HD uint64_t bit_reverse64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __brevll(x);
#else
    x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
    x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((x & 0x0F0F0F0F0F0F0F0Full) << 4);
    x = ((x >> 8) & 0x00FF00FF00FF00FFull) | ((x & 0x00FF00FF00FF00FFull) << 8);
    x = ((x >> 16) & 0x0000FFFF0000FFFFull) | ((x & 0x0000FFFF0000FFFFull) << 16);
    return (x >> 32) | (x << 32);
#endif
}

// Vertex permutation of the reference (cuda_scramble,
// src/graph_generation.cu:171-179); log_n in [1, 63].
G5_HD uint64_t kron_scramble(uint64_t v, int log_n, uint64_t val0, uint64_t val1) {
    v += val0 + val1;
    v *= (val0 | 0x4519840211493211ull);
    v = bit_reverse64(v) >> (64 - log_n);
    v *= (val1 | 0x3050852102C843A5ull);
    v = bit_reverse64(v) >> (64 - log_n);
    return v;
}

// Float draw of the reference (cuda_mrg_get_float_orig,
// src/graph_generation.cu:88-90): the integer rounded to binary32, times
// 4.65661287524579692e-10f, one rounding each.
G5_HD float mrg_unit_float(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(__uint2float_rn(u), 4.65661287524579692e-10f);
#else
    volatile float f = (float)u;
    return f * 4.65661287524579692e-10f;
#endif
}

// One Graph500 edge from the stream that starts at s: one quadrant per
// level, most significant bit first, folding the lower-left quadrant onto the
// upper-right while on the diagonal (cuda_make_one_edge,
// src/graph_generation.cu:186-207), both endpoints scrambled, then the
// weight drawn from the same stream (:225-238).
G5_HD void kron_edge(MrgState s, int log_n, uint64_t val0, uint64_t val1, uint64_t &src_out, uint64_t &dst_out,
                     float &w_out) {
    uint64_t src = 0, dst = 0;
    for (int lvl = log_n - 1; lvl >= 0; --lvl) {
        const int q = kron_quadrant(s);
        uint64_t so = (uint64_t)(q >> 1), to = (uint64_t)(q & 1);
        if (src == dst && so > to) {
            so = 0;
            to = 1;
        }
        src |= so << lvl;
        dst |= to << lvl;
    }
    src_out = kron_scramble(src, log_n, val0, val1);
    dst_out = kron_scramble(dst, log_n, val0, val1);
    w_out = mrg_unit_float(mrg_next(s));
}

// Everything a grid needs to walk edges [start, start + count): thread t of
// T starts at edge start + t (jump through the mid-byte tables) and steps by
// A^(T * 2^64).
struct KronLaunch {
    MrgState base;
    MrgMatrix stride_jump;
    int log_n;
    int64_t start, count;
    uint64_t val0, val1;
    const MrgMatrix *mid_table;
};

#ifdef __CUDACC__
__device__ __forceinline__ MrgState kron_thread_start(const KronLaunch &k, int64_t t) {
    MrgState z = k.base;
    uint64_t e = (uint64_t)(k.start + t);
    for (int b = 0; e; ++b, e >>= 8)
        if (e & 0xFF) mrg_apply(k.mid_table[256 * b + (e & 0xFF)], z);
    return z;
}
#endif

// ------------------------------------------------------------- host only --

// Host copy of A^(v * 256^b) for byte b in [0, 24) and value v.
const MrgMatrix &mrg_jump_matrix(int byte, int value);
// s <- A^(high*2^128 + mid*2^64 + low) s (the reference's cuda_mrg_skip).
void mrg_skip_host(MrgState &s, uint64_t high, uint64_t mid, uint64_t low);
// A^(n * 2^64) for a 64-bit n.
MrgMatrix mrg_jump_mid(uint64_t n);
// Uploads the byte tables for the 2^64-step jumps (bytes 8..15) to the
// current device once; returns their device address.
int mrg_device_mid_table(const MrgMatrix **out);
// Validates the seed and range and fills a KronLaunch for a grid of
// `threads` threads (capped by the device; *blocks gets the grid size).
int kron_prepare(const uint32_t seed[5], uint32_t log_n, int64_t start, int64_t end, int threads_per_block,
                 KronLaunch *k, int *blocks, const char *who);

}  // namespace g5
