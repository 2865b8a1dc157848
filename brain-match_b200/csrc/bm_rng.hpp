// bm_rng.hpp — the counter-based RNG and the exponential of the annealing
// chains, written so that host (gcc, -ffp-contract=off) and device (nvcc)
// produce bit-identical results, which makes a chain replayable on the CPU.
//
// Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11.  Ten rounds of two 32x32->64 multiplies with key bumps
// between rounds.
//
// bm_exp: exp(x) from the mathematics.  Cody-Waite reduction x = k ln2 + r,
// |r| <= ln2/2, with ln2 split into a 21-bit head (k*head is exact for
// |k| < 2^32) and a tail; e^r by its Taylor polynomial to degree 13 (the first
// omitted term is below 1e-17 relative), evaluated by Horner; the result
// scaled by 2^k through the exponent bits.  Every multiply and add is a
// separately rounded IEEE double operation (explicit __dmul_rn/__dadd_rn on the
// device, no contraction on the host), so host and device agree bit for bit.
// Results below 2^-1022 are returned as 0.
#pragma once

#include <stdint.h>
#include <string.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifndef BM_HD
#ifdef __CUDACC__
#define BM_HD __host__ __device__ __forceinline__
#elif defined(__cplusplus)
#define BM_HD inline
#else
#define BM_HD static inline
#endif
#endif

BM_HD void bm_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

BM_HD double bm_dmul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

BM_HD double bm_dadd(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}

BM_HD double bm_ddiv(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}

BM_HD double bm_from_bits(uint64_t b) {
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}

BM_HD double bm_exp(double x) {
    if (!(x < 709.0)) return bm_from_bits(0x7FF0000000000000ull);  // +inf (and NaN input)
    if (x < -708.0) return 0.0;
    const double inv_ln2 = bm_from_bits(0x3FF71547652B82FEull);  // 1/ln 2
    const double ln2_hi = bm_from_bits(0x3FE62E4200000000ull);   // ln 2, 21 significant bits
    const double ln2_lo = bm_from_bits(0x3E9FDF473DE6AF28ull);   // ln 2 - ln2_hi
    const double t = bm_dadd(bm_dmul(x, inv_ln2), 0.5);
    int32_t k = (int32_t)t;
    if ((double)k > t) k -= 1;  // floor
    const double kd = (double)k;
    const double r = bm_dadd(bm_dadd(x, -bm_dmul(kd, ln2_hi)), -bm_dmul(kd, ln2_lo));
    // 1/j! for j = 13..0, each the double nearest the exact fraction
    const uint64_t c[14] = {0x3DE6124613A86D09ull, 0x3E21EED8EFF8D898ull, 0x3E5AE64567F544E4ull,
                            0x3E927E4FB7789F5Cull, 0x3EC71DE3A556C734ull, 0x3EFA01A01A01A01Aull,
                            0x3F2A01A01A01A01Aull, 0x3F56C16C16C16C17ull, 0x3F81111111111111ull,
                            0x3FA5555555555555ull, 0x3FC5555555555555ull, 0x3FE0000000000000ull,
                            0x3FF0000000000000ull, 0x3FF0000000000000ull};
    double p = bm_from_bits(c[0]);
    for (int j = 1; j < 14; j++) p = bm_dadd(bm_dmul(p, r), bm_from_bits(c[j]));
    if (k < -1022) return 0.0;
    const double scale = bm_from_bits((uint64_t)(k + 1023) << 52);
    return bm_dmul(p, scale);
}

// Uniform double in [0, 1) from two 32-bit words (53 random bits).
BM_HD double bm_u01(uint32_t a, uint32_t b) {
    const uint64_t x = (((uint64_t)a << 32) | b) >> 11;
    return bm_dmul((double)x, bm_from_bits(0x3CA0000000000000ull));  // 2^-53
}

// One annealing proposal: Philox4x32-10 of counter (step lo, step hi, tag, 0)
// under the chain's key gives the two vertices (in 1..n, distinct, drawn like
// the reference's nodeM1/nodeM2 in src/best-swap/score-lookup.c:360-363) and
// the uniform of the acceptance test.
typedef struct bm_proposal {
    int32_t u, v;
    double uni;
} bm_proposal;

BM_HD bm_proposal bm_sa_proposal(uint64_t key, uint64_t step, int32_t n) {
    const uint32_t ctr[4] = {(uint32_t)step, (uint32_t)(step >> 32), 0x5A5A5A5Au, 0u};
    const uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    uint32_t o[4];
    bm_philox4x32_10(ctr, k, o);
    bm_proposal p;
    p.u = (int32_t)(o[0] % (uint32_t)(n - 1)) + 1;
    p.v = (int32_t)(o[1] % (uint32_t)n) + 1;
    if (p.u == p.v) p.u++;
    p.uni = bm_u01(o[2], o[3]);
    return p;
}

// Temperature of step s of a geometric schedule: t0 * exp(log_ratio * s / steps),
// with log_ratio = ln(t_end / t0) computed once by the caller.
BM_HD double bm_sa_temperature(double t0, double log_ratio, uint64_t s, uint64_t steps) {
    return bm_dmul(t0, bm_exp(bm_ddiv(bm_dmul(log_ratio, (double)s), (double)steps)));
}

// Metropolis acceptance: delta >= 0, or uni < exp(delta / T).
BM_HD bool bm_sa_accept(int64_t delta, double uni, double temperature) {
    if (delta >= 0) return true;
    return uni < bm_exp(bm_ddiv((double)delta, temperature));
}
