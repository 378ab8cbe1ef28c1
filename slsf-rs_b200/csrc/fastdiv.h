/*
 * Division by a run-time constant d >= 1 for dividends n < 2^31, as a
 * multiply-high and a shift (the round-up method of Granlund and Montgomery,
 * "Division by invariant integers using multiplication", PLDI 1994):
 *   l = ceil(log2 d),  m = floor(2^32 (2^l - d) / d) + 1,
 *   n / d = (mulhi(n, m) + n) >> l.
 * The sum cannot overflow 32 bits because n < 2^31 and mulhi(n, m) < n.
 */
#ifndef SLSF_FASTDIV_H
#define SLSF_FASTDIV_H

#include <stdint.h>

#include "xy_rng.h"

typedef struct {
    uint32_t d, m, l;
} slsf_fastdiv;

SLSF_HD slsf_fastdiv slsf_fastdiv_make(uint32_t d) {
    slsf_fastdiv f;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.d = d;
    f.l = l;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    return f;
}

SLSF_HD uint32_t slsf_fastdiv_div(uint32_t n, slsf_fastdiv f) {
#if defined(__CUDA_ARCH__)
    const uint32_t hi = __umulhi(n, f.m);
#else
    const uint32_t hi = (uint32_t)(((uint64_t)n * f.m) >> 32);
#endif
    return (hi + n) >> f.l;
}

#endif /* SLSF_FASTDIV_H */
