/*
 * FP32 angle arithmetic that must round identically on the device and in the
 * CPU oracle: the Metropolis proposal, the angle wrap, the Wolff reflection
 * and the reflection axis.  Every operation is a single IEEE-754 binary32
 * operation with round-to-nearest (explicit __fmaf_rn / __fadd_rn on the
 * device; fmaf and plain float arithmetic compiled with -ffp-contract=off on
 * the host), so a proposal that the device accepts produces the same FP32 bit
 * pattern as the oracle's emulation.
 *
 * Reference formulas:
 *   proposal   theta' = wrap(theta + w (2u - 1))      src/updates.rs:252
 *   wrap       one step into [0, 2 pi)                 src/types.rs:334-343
 *   reflection theta' = wrap(2 phi + pi - theta)       src/updates.rs:503-506
 *   axis       phi = 2 pi u                            src/updates.rs:564
 *
 * Two deliberate differences from the FP64 reference, both invisible to the
 * physics (they only choose which representative of the same spin direction
 * is stored):
 *   - wrap clamps the single FP32 case where t < 0 but t + 2 pi rounds up to
 *     exactly 2 pi, so stored angles are always in [0, 2 pi);
 *   - the reflection wraps up to twice.  2 phi + pi - theta lies in
 *     (-pi, 5 pi), and the reference's one-step wrap can leave a value in
 *     [2 pi, 3 pi); the device keeps every angle in [0, 2 pi) so that the
 *     fast sincos stays on its accurate range.
 */
#ifndef SLSF_XY_FP32_H
#define SLSF_XY_FP32_H

#include "xy_rng.h"

#if !defined(__CUDACC__)
#include <math.h>
#endif

SLSF_HD float slsf_fma_rn(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}

SLSF_HD float slsf_add_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    volatile float r = a + b;
    return r;
#endif
}

SLSF_HD float slsf_sub_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    volatile float r = a - b;
    return r;
#endif
}

SLSF_HD float slsf_mul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    volatile float r = a * b;
    return r;
#endif
}

/* One-step wrap into [0, 2 pi) with the FP32 round-up clamp. */
SLSF_HD float slsf_wrap_once(float t) {
    if (t >= SLSF_TWO_PI_F) {
        t = slsf_sub_rn(t, SLSF_TWO_PI_F);
    } else if (t < 0.0f) {
        t = slsf_add_rn(t, SLSF_TWO_PI_F);
        if (t >= SLSF_TWO_PI_F) t = 0.0f;
    }
    return t;
}

/* Metropolis proposal theta + w (2u - 1); 2u - 1 is exact for a 24-bit u. */
SLSF_HD float slsf_propose(float theta, float width, float u) {
    const float d = slsf_fma_rn(2.0f, u, -1.0f);
    return slsf_wrap_once(slsf_fma_rn(width, d, theta));
}

/* Reflection about the axis phi: 2 phi + pi - theta, wrapped into [0, 2 pi). */
SLSF_HD float slsf_reflect(float theta, float phi) {
    float t = slsf_sub_rn(slsf_fma_rn(2.0f, phi, SLSF_PI_F), theta);
    if (t >= SLSF_TWO_PI_F) {
        t = slsf_sub_rn(t, SLSF_TWO_PI_F);
        if (t >= SLSF_TWO_PI_F) t = slsf_sub_rn(t, SLSF_TWO_PI_F);
    } else if (t < 0.0f) {
        t = slsf_add_rn(t, SLSF_TWO_PI_F);
        if (t >= SLSF_TWO_PI_F) t = 0.0f;
    }
    return t;
}

/* 2 pi u for a 24-bit uniform; used for the Wolff axis and the initial angles. */
SLSF_HD float slsf_angle_from_word(uint32_t w) {
    float a = slsf_mul_rn(slsf_u24f(w), SLSF_TWO_PI_F);
    return a >= SLSF_TWO_PI_F ? 0.0f : a;
}

#endif /* SLSF_XY_FP32_H */
