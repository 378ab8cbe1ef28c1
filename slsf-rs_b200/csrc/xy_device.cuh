/*
 * Device building blocks shared by every kernel of the library, so that the
 * single-task kernels and the batched persistent kernel make bit-identical
 * decisions from identical inputs: lattice indexing, the local field, the
 * Metropolis decision, the Wolff bond test and FP64 block reductions.
 *
 * Lattice layout (src/types.rs:146-149): theta[x + Lx (y + Ly z)], FP32,
 * periodic in all three directions.  Bond z -> z+1 uses J_z[z]; the in-plane
 * bonds of layer z use J_xy[z] (src/updates.rs:131-167, :211-213).
 */
#ifndef SLSF_XY_DEVICE_CUH
#define SLSF_XY_DEVICE_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "xy_fp32.h"

namespace slsf {

/* Site index and colour-compact coordinates.  For colour c, the sites with
 * (x + y + z) & 1 == c map one-to-one onto h = idx >> 1 (L_x even). */
struct SiteXYZ {
    uint32_t x, y, z, idx;
};

/* Neighbour indices in the order +x, -x, +y, -y, +z, -z (the neighbors!
 * macro of src/updates.rs:131-167). */
__device__ __forceinline__ void neighbour_indices(const SiteXYZ& s, uint32_t lx, uint32_t ly,
                                                  uint32_t lz, uint32_t nb[6]) {
    const uint32_t plane = lx * ly;
    const uint32_t vol = plane * lz;
    nb[0] = (s.x + 1 == lx) ? s.idx + 1 - lx : s.idx + 1;
    nb[1] = (s.x == 0) ? s.idx + lx - 1 : s.idx - 1;
    nb[2] = (s.y + 1 == ly) ? s.idx + lx - plane : s.idx + lx;
    nb[3] = (s.y == 0) ? s.idx + plane - lx : s.idx - lx;
    nb[4] = (s.z + 1 == lz) ? s.idx + plane - vol : s.idx + plane;
    nb[5] = (s.z == 0) ? s.idx + vol - plane : s.idx - plane;
}

/* One component of the local field (src/updates.rs:215-228):
 * J_xy (a0 + a1 + a2 + a3) + J_z+ a4 + J_z- a5, with a fixed rounding order;
 * field_from_pairs takes the in-plane pairs a0 + a1 and a2 + a3 already
 * rounded, so a kernel can fold neighbours in as it loads them. */
__device__ __forceinline__ float field_from_pairs(float jxy, float jzp, float jzm, float a01, float a23,
                                                  float a4, float a5) {
    return __fmaf_rn(jzm, a5, __fmaf_rn(jzp, a4, __fmul_rn(jxy, __fadd_rn(a01, a23))));
}

__device__ __forceinline__ float field_component(float jxy, float jzp, float jzm, float a0,
                                                 float a1, float a2, float a3, float a4,
                                                 float a5) {
    return field_from_pairs(jxy, jzp, jzm, __fadd_rn(a0, a1), __fadd_rn(a2, a3), a4, a5);
}

/* The Metropolis decision of local_metropolis_step_at_unchecked
 * (src/updates.rs:251-270): propose theta' = wrap(theta + w (2u - 1)),
 * dE = -(cos' hx + sin' hy) + (cos hx + sin hy), accept iff dE <= 0 or
 * u_acc < exp(-beta dE).  Fast FP32 sincos / exp. */
__device__ __forceinline__ bool metro_decide(float theta, float ci, float si, float hx, float hy,
                                             float beta, float width, float u_prop, float u_acc,
                                             float* theta_new, float* s_new, float* c_new) {
    const float tn = slsf_propose(theta, width, u_prop);
    float sn, cn;
    __sincosf(tn, &sn, &cn);
    const float de = __fmaf_rn(__fsub_rn(ci, cn), hx, __fmul_rn(__fsub_rn(si, sn), hy));
    const bool acc = (de <= 0.0f) || (u_acc < __expf(__fmul_rn(-beta, de)));
    *theta_new = tn;
    *s_new = sn;
    *c_new = cn;
    return acc;
}

/* Projection of a spin on the Wolff axis from its cached trig,
 * r = cos(theta) cos(phi) + sin(theta) sin(phi) (src/updates.rs:579-582),
 * where (s, c) = __sincosf(theta) and (sphi, cphi) = __sincosf(phi). */
__device__ __forceinline__ float wolff_projection(float c, float s, float cphi, float sphi) {
    return __fmaf_rn(s, sphi, __fmul_rn(c, cphi));
}

/* Bond activation of try_add_wolff_neighbor (src/updates.rs:537-548) with a
 * per-bond random: active iff J r_i r_j > 0 and u < 1 - exp(-2 beta J r_i r_j). */
__device__ __forceinline__ bool wolff_bond_active(float coupling, float ri, float rj,
                                                  float minus_two_beta, uint32_t word) {
    const float prod = __fmul_rn(__fmul_rn(coupling, ri), rj);
    if (!(prod > 0.0f)) return false;
    const float p = __fsub_rn(1.0f, __expf(__fmul_rn(minus_two_beta, prod)));
    return slsf_u24f(word) < p;
}

/* Terms of one bond a -> b = a + mu of the observables
 * (src/observables.rs:108-137): J cos(theta_a - theta_b) and
 * J sin(theta_a - theta_b) from the two sites' trig, with a fixed rounding
 * order so that every kernel that measures (the single-task kernel, the
 * batched kernels' measurement pass and the measurement fused into their
 * Metropolis half-sweep) computes each bond's terms bit-identically. */
__device__ __forceinline__ float bond_cos(float j, float ca, float sa, float cb, float sb) {
    return __fmul_rn(j, __fmaf_rn(ca, cb, __fmul_rn(sa, sb)));
}

__device__ __forceinline__ float bond_sin(float j, float ca, float sa, float cb, float sb) {
    return __fmul_rn(j, __fmaf_rn(sa, cb, -__fmul_rn(ca, sb)));
}

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    }
}

/* Block-wide FP64 sum in a fixed order; the result is valid in thread 0.
 * scratch holds N * 32 doubles. */
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
    warp_sum(v);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) scratch[k * 32 + warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = lane < nwarps ? scratch[k * 32 + lane] : 0.0;
        warp_sum(v);
    }
    __syncthreads();
}

}  // namespace slsf

#endif /* SLSF_XY_DEVICE_CUH */
