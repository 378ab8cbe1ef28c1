/*
 * Bit-parallel closure of a Wolff cluster over active bonds, shared by the
 * batched one-CTA kernel (kernel_resident.cu, L = 32 cubes) and the
 * large-lattice growth (kernel_wolff_bits.cu): a block of 32 x 32 words --
 * 32 rows along y by 32 planes along z, one 32-bit word of 32 sites along x
 * per row -- closed in shared memory by warp scans.
 *
 * The cluster is the seed's connected component over the active bonds, the
 * set the reference's depth-first search collects (src/updates.rs:577-597)
 * when fed the same per-bond randoms.  Bits only ever get set, so every order
 * of the closure steps reaches the same fixed point.
 */
#ifndef SLSF_BITGROW_CUH
#define SLSF_BITGROW_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace slsf {

constexpr uint32_t kGrowEdge = 32; /* rows per plane and planes per block */

/* Periodic rotations of a 32-bit row word (L_x == 32: the row is one word). */
__device__ __forceinline__ uint32_t rotl32(uint32_t w, uint32_t s) { return __funnelshift_l(w, w, s); }
__device__ __forceinline__ uint32_t rotr32(uint32_t w, uint32_t s) { return __funnelshift_r(w, w, s); }

/* Closure of the cluster bits c of one word along x through its bonds b
 * (bit j: bond j -- j+1), by doubling in both directions.  periodic: the
 * word is a whole row (L_x == 32) and bit 31 bonds to bit 0; otherwise the
 * word is open at both ends (bits crossing words enter between passes). */
__device__ __forceinline__ uint32_t close_word(uint32_t c, uint32_t b, bool periodic) {
    if (periodic) {
        uint32_t gr = c, pr = b, gl = c, pl = rotl32(b, 1);
#pragma unroll
        for (uint32_t s = 1; s < 32; s <<= 1) {
            gr |= rotl32(gr & pr, s);
            pr &= rotr32(pr, s);
            gl |= rotr32(gl & pl, s);
            pl &= rotl32(pl, s);
        }
        return gr | gl;
    }
    /* open word: bond bit 31 leads out of the word and is not used here */
    const uint32_t bi = b & 0x7fffffffu;
    uint32_t gr = c, pr = bi, gl = c, pl = bi << 1;
#pragma unroll
    for (uint32_t s = 1; s < 32; s <<= 1) {
        gr |= (gr & pr) << s;
        pr &= pr >> s;
        gl |= (gl & pl) >> s;
        pl &= pl << s;
    }
    return gr | gl;
}

/* Closure along a line of 32 words held one per lane (lane = position):
 * bit x of lane i passes to lane i+1 when bit x of p (the lane's bond to the
 * next position) is set.  Doubling in both directions; periodic lines wrap
 * from lane 31 to lane 0. */
__device__ __forceinline__ uint32_t close_line(uint32_t c, uint32_t p, bool periodic) {
    const uint32_t lane = threadIdx.x & 31u;
    /* upward: G(i) |= P(i) & G(i - s), P(i) = bonds i-1 -> i over the span */
    uint32_t g = c;
    uint32_t q = __shfl_sync(0xffffffffu, p, (lane + 31u) & 31u);
    if (!periodic && lane == 0) q = 0;
#pragma unroll
    for (uint32_t s = 1; s < 32; s <<= 1) {
        const uint32_t src = (lane - s) & 31u;
        const uint32_t gs = __shfl_sync(0xffffffffu, g, src);
        const uint32_t qs = __shfl_sync(0xffffffffu, q, src);
        if (periodic || lane >= s) {
            g |= q & gs;
            q &= qs;
        }
    }
    /* downward: H(i) |= R(i) & H(i + s), R(i) = bonds i -> i+1 over the span */
    uint32_t h = c;
    uint32_t r = p;
    if (!periodic && lane == 31) r = 0;
#pragma unroll
    for (uint32_t s = 1; s < 32; s <<= 1) {
        const uint32_t src = (lane + s) & 31u;
        const uint32_t hs = __shfl_sync(0xffffffffu, h, src);
        const uint32_t rs = __shfl_sync(0xffffffffu, r, src);
        if (periodic || lane + s < 32) {
            h |= r & hs;
            r &= rs;
        }
    }
    return g | h;
}

/* Closes the block C[z][y] (cluster words, pitch kGrowEdge + 1) through its
 * bonds BX (along x inside the word), BY[z][y] (row y to y + 1) and BZ[z][y]
 * (plane z to z + 1), with px / py / pz telling whether the block spans the
 * whole period along x (one-word rows), y and z.  Needs 1024 threads (32
 * warps); C must already be closed along x.  Passes alternate a full warp
 * scan along y (lane = y, warp = z) or along z (lane = z, warp = y, the arrays
 * read transposed) with one step along the other axis and the closure along
 * x of the words that changed; a pass that changes nothing ends it.  Returns
 * the number of passes, or 0 if max_pass passes were not enough (every pass
 * that changes something sets a bit, so 32^3 + 1 always are). */
__device__ __forceinline__ uint32_t close_block(uint32_t (*C)[kGrowEdge + 1], const uint32_t (*BY)[kGrowEdge + 1],
                                                const uint32_t (*BZ)[kGrowEdge + 1], const uint32_t (*BX)[kGrowEdge + 1],
                                                bool px, bool py, bool pz,
                                                uint32_t max_pass = kGrowEdge * kGrowEdge * kGrowEdge + 1) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    constexpr uint32_t E = kGrowEdge;
    for (uint32_t pass = 0; pass < max_pass; ++pass) {
        int changed = 0;
        if ((pass & 1u) == 0) {
            const uint32_t z = warp, y = lane;
            const uint32_t old = C[z][y];
            const uint32_t by_ = BY[z][y];
            /* a warp scans only if some bit of it sits on a bond along the line */
            const uint32_t by_in = __shfl_sync(0xffffffffu, by_, (lane + 31u) & 31u);
            uint32_t v = __any_sync(0xffffffffu, (old & (by_ | by_in)) != 0u) ? close_line(old, by_, py) : old;
            if (z > 0) v |= C[z - 1][y] & BZ[z - 1][y];
            else if (pz) v |= C[E - 1][y] & BZ[E - 1][y];
            if (z + 1 < E) v |= C[z + 1][y] & BZ[z][y];
            else if (pz) v |= C[0][y] & BZ[z][y];
            if (__any_sync(0xffffffffu, v != old)) v = close_word(v, BX[z][y], px);
            if (v != old) {
                C[z][y] = v;
                changed = 1;
            }
        } else {
            const uint32_t z = lane, y = warp;
            const uint32_t old = C[z][y];
            const uint32_t bz_ = BZ[z][y];
            const uint32_t bz_in = __shfl_sync(0xffffffffu, bz_, (lane + 31u) & 31u);
            uint32_t v = __any_sync(0xffffffffu, (old & (bz_ | bz_in)) != 0u) ? close_line(old, bz_, pz) : old;
            if (y > 0) v |= C[z][y - 1] & BY[z][y - 1];
            else if (py) v |= C[z][E - 1] & BY[z][E - 1];
            if (y + 1 < E) v |= C[z][y + 1] & BY[z][y];
            else if (py) v |= C[z][0] & BY[z][y];
            if (__any_sync(0xffffffffu, v != old)) v = close_word(v, BX[z][y], px);
            if (v != old) {
                C[z][y] = v;
                changed = 1;
            }
        }
        if (!__syncthreads_or(changed)) return pass + 1;
    }
    return 0;
}

}  // namespace slsf

#endif /* SLSF_BITGROW_CUH */
