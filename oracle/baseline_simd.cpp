/*
 * baseline_simd.cpp -- TEST INFRASTRUCTURE ONLY: the timed CPU baseline.
 *
 * The reference's Metropolis sweep evaluates each batch of 8 same-colour
 * sites (4 without AVX-512) with packed FP64 sincos and exp from sleef 0.3.3
 * (src/fast_math.rs:1-37, src/updates.rs:21-53, :300-408); its Wolff update
 * and measurements call sleef's scalar functions.  This file builds the
 * oracle's reference-order path a second time with the batches' sincos and
 * exp routed to glibc's vector math library (libmvec: 8-lane AVX-512 or
 * 4-lane AVX2 variants, called through their published vector-function ABI
 * names), compiled for the host's vector ISA.  sleef is not installed here;
 * libmvec is the vector library at hand, of the same kind and accuracy class
 * (<= 4 ulp).  The parity oracle stays the scalar build (oracle.cpp alone).
 *
 * Two builds (oracle/Makefile): libbaseline_v4.so for hosts with AVX-512F
 * (x86-64-v4; 8-lane batches, as the reference selects at run time by
 * has_avx512_f64_lanes) and libbaseline_v3.so for AVX2 hosts (x86-64-v3;
 * 4-lane batches only).
 */
#include <immintrin.h>

extern "C" {
__m256d _ZGVdN4v_sin(__m256d);
__m256d _ZGVdN4v_cos(__m256d);
__m256d _ZGVdN4v_exp(__m256d);
#if defined(__AVX512F__)
__m512d _ZGVeN8v_sin(__m512d);
__m512d _ZGVeN8v_cos(__m512d);
__m512d _ZGVeN8v_exp(__m512d);
#endif
}

#define OR_SIMD_BASELINE 1

namespace {

template <int LANES>
inline void batch_sincos(const double* x, double* s, double* c);
template <int LANES>
inline void batch_exp(const double* x, double* y);

template <>
inline void batch_sincos<4>(const double* x, double* s, double* c) {
    const __m256d v = _mm256_loadu_pd(x);
    _mm256_storeu_pd(s, _ZGVdN4v_sin(v));
    _mm256_storeu_pd(c, _ZGVdN4v_cos(v));
}

template <>
inline void batch_exp<4>(const double* x, double* y) {
    _mm256_storeu_pd(y, _ZGVdN4v_exp(_mm256_loadu_pd(x)));
}

#if defined(__AVX512F__)
template <>
inline void batch_sincos<8>(const double* x, double* s, double* c) {
    const __m512d v = _mm512_loadu_pd(x);
    _mm512_storeu_pd(s, _ZGVeN8v_sin(v));
    _mm512_storeu_pd(c, _ZGVeN8v_cos(v));
}

template <>
inline void batch_exp<8>(const double* x, double* y) {
    _mm512_storeu_pd(y, _ZGVeN8v_exp(_mm512_loadu_pd(x)));
}
#else
/* AVX2 build: the 8-lane batch runs only on AVX-512 hosts, which load the
 * other build; two 4-lane halves keep this one complete. */
template <>
inline void batch_sincos<8>(const double* x, double* s, double* c) {
    batch_sincos<4>(x, s, c);
    batch_sincos<4>(x + 4, s + 4, c + 4);
}

template <>
inline void batch_exp<8>(const double* x, double* y) {
    batch_exp<4>(x, y);
    batch_exp<4>(x + 4, y + 4);
}
#endif

}  // namespace

#include "oracle.cpp"
