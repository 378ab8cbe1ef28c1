/*
 * Counter-based random streams for the XY update-and-measure path.
 *
 * The reference draws every random number from one serial SplitMix64 stream
 * (`FastRng`, src/types.rs:9-82), so its draw order depends on the traversal
 * order of the sweep (src/updates.rs:455-483) and of the Wolff DFS
 * (src/updates.rs:577-597).  A GPU sweep has no serial order, so every random
 * number here is a pure function of (task seed, sweep counter, purpose, unit):
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3", SC'11) with
 *
 *   key     = { seed[31:0], seed[63:32] }
 *   counter = { unit, sweep[31:0], (purpose << 24) | sub, sweep[63:32] }
 *
 * Purposes and units:
 *   METRO      unit = site_index >> 2, sub = colour.  The colour-c sites map
 *              one-to-one onto h = site_index >> 1 (all L_x are even), and
 *              the two colour-c sites with the same h >> 1 share one Philox
 *              block: lane h & 1 takes words {2*lane, 2*lane+1} as
 *              (u_proposal, u_accept).
 *   WOLFF_BOND unit = site_index, sub = Wolff step within the sweep; words
 *              x, y, z are the bond randoms of the +x, +y, +z bonds that start
 *              at the site, so a bond has one random whichever end tests it.
 *   WOLFF_PICK unit = 0, sub = Wolff step; word x gives the reflection axis
 *              phi, words y, z, w the seed site (multiply-shift range map).
 *   INIT       unit = site_index >> 2, sweep = 0, word (site_index & 3) gives
 *              the initial angle.
 *
 * The same header is compiled for the device (nvcc) and for the FP64 CPU
 * oracle (gcc), so both sides see bit-identical random words.
 */
#ifndef SLSF_XY_RNG_H
#define SLSF_XY_RNG_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SLSF_HD __host__ __device__ __forceinline__
#else
#define SLSF_HD static inline
#endif

#define SLSF_PHILOX_M0 0xD2511F53u
#define SLSF_PHILOX_M1 0xCD9E8D57u
#define SLSF_PHILOX_W0 0x9E3779B9u
#define SLSF_PHILOX_W1 0xBB67AE85u

#define SLSF_PURPOSE_METRO 1u
#define SLSF_PURPOSE_WOLFF_BOND 2u
#define SLSF_PURPOSE_WOLFF_PICK 3u
#define SLSF_PURPOSE_INIT 4u

/* 2*pi and pi rounded to FP32; the device keeps angles in [0, SLSF_TWO_PI_F). */
#define SLSF_TWO_PI_F 6.28318548202514648438f
#define SLSF_PI_F 3.14159274101257324219f

typedef struct {
    uint32_t x, y, z, w;
} slsf_u32x4;

SLSF_HD slsf_u32x4 slsf_philox4x32_10(slsf_u32x4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int round = 0; round < 10; ++round) {
#if defined(__CUDA_ARCH__)
        const uint32_t hi0 = __umulhi(SLSF_PHILOX_M0, c.x);
        const uint32_t lo0 = SLSF_PHILOX_M0 * c.x;
        const uint32_t hi1 = __umulhi(SLSF_PHILOX_M1, c.z);
        const uint32_t lo1 = SLSF_PHILOX_M1 * c.z;
#else
        const uint64_t p0 = (uint64_t)SLSF_PHILOX_M0 * c.x;
        const uint64_t p1 = (uint64_t)SLSF_PHILOX_M1 * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        slsf_u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += SLSF_PHILOX_W0;
        k1 += SLSF_PHILOX_W1;
    }
    return c;
}

/* Philox block for (seed, sweep, purpose, sub, unit). */
SLSF_HD slsf_u32x4 slsf_stream(uint64_t seed, uint64_t sweep, uint32_t purpose, uint32_t sub,
                               uint32_t unit) {
    slsf_u32x4 c;
    c.x = unit;
    c.y = (uint32_t)sweep;
    c.z = (purpose << 24) | (sub & 0x00FFFFFFu);
    c.w = (uint32_t)(sweep >> 32);
    return slsf_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

/* Top 24 bits of a word as a uniform in [0, 1); exact in FP32 and FP64. */
SLSF_HD float slsf_u24f(uint32_t w) { return (float)(w >> 8) * (1.0f / 16777216.0f); }
SLSF_HD double slsf_u24d(uint32_t w) { return (double)(w >> 8) * (1.0 / 16777216.0); }

/* floor(w * n / 2^32): the multiply-shift range map used for the Wolff seed site. */
SLSF_HD uint32_t slsf_range(uint32_t w, uint32_t n) {
    return (uint32_t)(((uint64_t)w * (uint64_t)n) >> 32);
}

/* Metropolis randoms of one colour-c site (see the header comment). */
SLSF_HD void slsf_metro_uniforms(slsf_u32x4 blk, uint32_t lane, float* u_prop, float* u_acc) {
    *u_prop = slsf_u24f(lane ? blk.z : blk.x);
    *u_acc = slsf_u24f(lane ? blk.w : blk.y);
}

#endif /* SLSF_XY_RNG_H */
