/*
 * Batched persistent kernel for replicas that fit in one CTA's shared
 * memory: many replicas of uneven size, one CTA per replica at a time, each
 * replica resident for all of its sweeps.  Replaces the carlo-mc Runner's
 * task-by-task loop over ThetaModel::sweep + ThetaModel::measure
 * (src/model.rs:379-442, src/results.rs:200-202) for every task of a batch.
 *
 * Per replica the CTA
 *   1. copies theta from HBM into a colour-split shared layout: the colour-c
 *      site with index idx sits at c * (V/2 + 16) + idx/2, so a warp reading
 *      one colour reads consecutive words, and the 64-byte pad puts the two
 *      colours of neighbouring sites in different bank halves;
 *   2. per sweep: two colour half-sweeps (the same decision code as the
 *      single-task kernel, xy_device.cuh) and `wolff_steps` Wolff updates;
 *      after thermalization each sweep's state is measured inside the next
 *      sweep's colour-0 half-sweep (the launch's last state by a separate
 *      pass) and added to the task's bins;
 *   3. copies theta back.
 * HBM traffic is 8 bytes per site per launch, independent of the sweep
 * count.  Trig values are recomputed with __sincosf where needed (a 32^3
 * replica leaves no room for a cos/sin cache next to theta).
 *
 * Wolff labelling is bit-parallel: the active +x/+y/+z bonds of a row of
 * L_x <= 32 sites are three 32-bit words; the cluster grows from the seed by
 * OR-ing neighbour rows through the bond words and closing every row that
 * gained bits along x, until a pass changes nothing.  (In one CTA a pass is
 * a single block barrier, which for replicas of this size beats the
 * column-scan rounds of kernel_cluster.cu.)  The result is the seed's
 * connected component over the active bonds -- the set the reference's DFS
 * (src/updates.rs:577-597) collects when fed the same per-bond randoms.
 * Growth is monotone, so the pass count is bounded by V.
 */
#include <algorithm>

#include "bins.cuh"
#include "bitgrow.cuh"
#include "engine.h"
#include "fastdiv.h"
#include "xy_device.cuh"

namespace slsf {

namespace {

constexpr int kBThreads = 1024;
constexpr uint32_t kPad = 16; /* floats: 64 bytes */
constexpr uint32_t kMaxRowBits = 32;

/* Optional per-phase cycle accounting (build with -DSLSF_PHASE_TIMING):
 * thread 0 of every CTA adds the clock64 cycles of each phase, measured
 * between block barriers, to g_phase_cycles; slot 6 counts cluster-growth
 * passes and slot 7 Wolff updates. */
#ifdef SLSF_PHASE_TIMING
__device__ unsigned long long g_res_phase_cycles[8];
__shared__ long long s_phase_mark;
#define SLSF_PHASE(k)                                                                     \
    do {                                                                                  \
        __syncthreads();                                                                  \
        if (threadIdx.x == 0) {                                                           \
            const long long now_ = clock64();                                             \
            atomicAdd(&g_res_phase_cycles[k], (unsigned long long)(now_ - s_phase_mark)); \
            s_phase_mark = now_;                                                          \
        }                                                                                 \
    } while (0)
#define SLSF_PHASE_COUNT(k, n)                                                              \
    do {                                                                                    \
        if (threadIdx.x == 0) atomicAdd(&g_res_phase_cycles[k], (unsigned long long)(n)); \
    } while (0)
#else
#define SLSF_PHASE(k) \
    do {              \
    } while (0)
#define SLSF_PHASE_COUNT(k, n) \
    do {                       \
    } while (0)
#endif

struct Geo {
    uint32_t lx, ly, lz, volume, half, rows, plane;
    uint32_t stride1; /* offset of the colour-1 array */
    uint32_t xmask;
    bool lx_tiles_warp;
    slsf_fastdiv div_hx, div_ly, div_lx;
};

__device__ __forceinline__ Geo make_geo(const TaskView& t) {
    Geo g;
    g.lx = t.lx;
    g.ly = t.ly;
    g.lz = t.lz;
    g.plane = t.lx * t.ly;
    g.volume = g.plane * t.lz;
    g.half = g.volume >> 1;
    g.rows = t.ly * t.lz;
    g.stride1 = g.half + kPad;
    g.xmask = t.lx >= 32 ? 0xffffffffu : ((1u << t.lx) - 1u);
    g.lx_tiles_warp = (32u % t.lx) == 0;
    g.div_hx = slsf_fastdiv_make(t.lx >> 1);
    g.div_ly = slsf_fastdiv_make(t.ly);
    g.div_lx = slsf_fastdiv_make(t.lx);
    return g;
}

/* Shared-memory slot of natural site index idx with colour c. */
__device__ __forceinline__ uint32_t slot(const Geo& g, uint32_t idx, uint32_t colour) {
    return colour * g.stride1 + (idx >> 1);
}

struct Coords {
    uint32_t x, y, z, row;
};

__device__ __forceinline__ Coords coords_of(const Geo& g, uint32_t idx) {
    Coords c;
    c.row = slsf_fastdiv_div(idx, g.div_lx);
    c.x = idx - c.row * g.lx;
    c.z = slsf_fastdiv_div(c.row, g.div_ly);
    c.y = c.row - c.z * g.ly;
    return c;
}

/* Forward neighbours of a site (+x, +y, +z) as natural indices. */
__device__ __forceinline__ void forward_neighbours(const Geo& g, uint32_t idx, const Coords& c, uint32_t& xp,
                                                   uint32_t& yp, uint32_t& zp) {
    xp = (c.x + 1 == g.lx) ? idx + 1 - g.lx : idx + 1;
    yp = (c.y + 1 == g.ly) ? idx + g.lx - g.plane : idx + g.lx;
    zp = (c.z + 1 == g.lz) ? idx + g.plane - g.volume : idx + g.plane;
}

/* Lane holding the +x neighbour when rows of lx sites tile the warp. */
__device__ __forceinline__ uint32_t xp_lane(uint32_t lane, uint32_t lx) {
    return (lane & ~(lx - 1u)) | ((lane + 1u) & (lx - 1u));
}

__device__ __forceinline__ uint32_t rotl_row(uint32_t w, uint32_t s, uint32_t lx, uint32_t mask) {
    return lx == 32 ? __funnelshift_l(w, w, s) : (((w << s) | (w >> (lx - s))) & mask);
}

__device__ __forceinline__ uint32_t rotr_row(uint32_t w, uint32_t s, uint32_t lx, uint32_t mask) {
    return lx == 32 ? __funnelshift_r(w, w, s) : (((w >> s) | (w << (lx - s))) & mask);
}

/* Closure of a periodic row's cluster bits c along x through the bond bits b
 * (bit x: bond x -- x+1).  Kogge-Stone doubling in both directions: after the
 * step with shift s, every site within 2s - 1 bond steps of a seed is set;
 * shifts 1..16 cover any row of L_x <= 32 sites. */
__device__ __forceinline__ uint32_t close_row(uint32_t c, uint32_t b, uint32_t lx, uint32_t mask) {
    uint32_t gr = c, pr = b;                        /* rightward: bond p -> p+1 */
    uint32_t gl = c, pl = rotl_row(b, 1, lx, mask); /* leftward: bond p-1 -> p */
#pragma unroll
    for (uint32_t s = 1; s < 32; s <<= 1) {
        if (s >= lx) break;
        gr |= rotl_row(gr & pr, s, lx, mask);
        pr &= rotr_row(pr, s, lx, mask);
        gl |= rotr_row(gl & pl, s, lx, mask);
        pl &= rotl_row(pl, s, lx, mask);
    }
    return gr | gl;
}

struct Smem {
    float* th; /* two colour arrays */
    uint32_t* bx;
    uint32_t* by;
    uint32_t* bz;
    uint32_t* cl;
    float* jxy;
    float* jz;
    uint32_t* blk; /* 32^3 replicas: cluster and bond words as [z][y] blocks of pitch 33 (cube32), else NULL */
    double* corr;  /* fused correlation scratch (resident_corr_doubles) */
};

/* Words of the padded blocks of a 32^3 replica's Wolff growth (C, BY, BZ, BX). */
constexpr uint32_t kBlockWords = 4 * kGrowEdge * (kGrowEdge + 1);

__device__ __forceinline__ Smem carve(unsigned char* base, uint32_t max_volume, uint32_t max_rows, uint32_t max_lz,
                                      uint32_t cube32) {
    Smem s;
    s.th = reinterpret_cast<float*>(base);
    uint32_t* w = reinterpret_cast<uint32_t*>(base + 4ull * (max_volume + 2 * kPad));
    s.bx = w;
    s.by = w + max_rows;
    s.bz = w + 2 * max_rows;
    s.cl = w + 3 * max_rows;
    s.jxy = reinterpret_cast<float*>(w + 4 * max_rows);
    s.jz = s.jxy + max_lz;
    uint32_t* after = reinterpret_cast<uint32_t*>(s.jz + max_lz);
    s.blk = cube32 ? after : nullptr;
    if (cube32) after += kBlockWords;
    /* 8-byte aligned: the volume is even, the other arrays are whole words */
    s.corr = reinterpret_cast<double*>(after);
    return s;
}

/* ---- phases ---- */

__device__ __forceinline__ void load_state(const TaskView& t, const Geo& g, Smem& s) {
    if (g.lx % 4) {
        /* L_x = 2 mod 4: four consecutive sites may span two rows; copy site by site */
        for (uint32_t i = threadIdx.x; i < g.volume; i += blockDim.x) {
            const Coords c = coords_of(g, i);
            s.th[slot(g, i, (c.x + c.y + c.z) & 1u)] = t.theta[i];
        }
    } else {
        const float4* src = reinterpret_cast<const float4*>(t.theta);
        for (uint32_t q = threadIdx.x; q < g.volume / 4; q += blockDim.x) {
            const float4 v = src[q];
            const Coords c = coords_of(g, 4 * q);
            const uint32_t p = (c.y + c.z) & 1u; /* colour of the even-x site */
            const uint32_t h = 2 * q;
            s.th[p * g.stride1 + h] = v.x;
            s.th[(p ^ 1u) * g.stride1 + h] = v.y;
            s.th[p * g.stride1 + h + 1] = v.z;
            s.th[(p ^ 1u) * g.stride1 + h + 1] = v.w;
        }
    }
    for (uint32_t z = threadIdx.x; z < g.lz; z += blockDim.x) {
        s.jxy[z] = t.jxy[z];
        s.jz[z] = t.jz[z];
    }
}

__device__ __forceinline__ void store_state(const TaskView& t, const Geo& g, const Smem& s) {
    if (g.lx % 4) {
        for (uint32_t i = threadIdx.x; i < g.volume; i += blockDim.x) {
            const Coords c = coords_of(g, i);
            t.theta[i] = s.th[slot(g, i, (c.x + c.y + c.z) & 1u)];
        }
        return;
    }
    float4* dst = reinterpret_cast<float4*>(t.theta);
    for (uint32_t q = threadIdx.x; q < g.volume / 4; q += blockDim.x) {
        const Coords c = coords_of(g, 4 * q);
        const uint32_t p = (c.y + c.z) & 1u;
        const uint32_t h = 2 * q;
        dst[q] = make_float4(s.th[p * g.stride1 + h], s.th[(p ^ 1u) * g.stride1 + h], s.th[p * g.stride1 + h + 1],
                             s.th[(p ^ 1u) * g.stride1 + h + 1]);
    }
}

/* One colour half-sweep.  A warp owns 32 consecutive Philox blocks (64
 * sites); lanes exchange words so that lane j updates colour-compact sites
 * 2*base + j and 2*base + 32 + j, i.e. consecutive shared words.
 *
 * With kMeasure (colour 0 only) it also measures the state the half-sweep
 * starts from, at no extra trig: every bond joins a colour-0 site to a
 * colour-1 site, and before its update a colour-0 site has the trig of
 * itself and of all six neighbours, so it adds the terms of its three
 * forward bonds and of the three backward bonds that end on it, and the
 * magnetisation of itself and of its +x neighbour (each colour-1 site is the
 * +x neighbour of exactly one colour-0 site).  Each term is the bond_cos /
 * bond_sin value the measurement pass computes; sums are FP64. */
template <bool kMeasure>
__device__ __forceinline__ uint32_t half_sweep(const TaskView& t, const Geo& g, Smem& s, uint64_t sweep,
                                               uint32_t colour, double (&acc)[8]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t npairs = (g.half + 1) >> 1;
    const uint32_t own = colour * g.stride1, other = (colour ^ 1u) * g.stride1;
    uint32_t accepted = 0;
    for (uint32_t base = warp * 32; base < npairs; base += nwarps * 32) {
        const uint32_t p = base + lane;
        slsf_u32x4 blk = {0, 0, 0, 0};
        if (p < npairs) blk = slsf_stream(t.seed, sweep, SLSF_PURPOSE_METRO, colour, p);
#pragma unroll
        for (uint32_t r = 0; r < 2; ++r) {
            const uint32_t src = 16 * r + (lane >> 1);
            const uint32_t wx = __shfl_sync(0xffffffffu, blk.x, src);
            const uint32_t wy = __shfl_sync(0xffffffffu, blk.y, src);
            const uint32_t wz = __shfl_sync(0xffffffffu, blk.z, src);
            const uint32_t ww = __shfl_sync(0xffffffffu, blk.w, src);
            const uint32_t h = 2 * base + 32 * r + lane;
            if (h >= g.half) continue;
            const float u_prop = slsf_u24f((lane & 1u) ? wz : wx);
            const float u_acc = slsf_u24f((lane & 1u) ? ww : wy);
            const uint32_t row = slsf_fastdiv_div(h, g.div_hx);
            const uint32_t k = h - row * (g.lx >> 1);
            const uint32_t z = slsf_fastdiv_div(row, g.div_ly);
            const uint32_t y = row - z * g.ly;
            SiteXYZ st;
            st.x = 2u * k + ((colour + y + z) & 1u);
            st.y = y;
            st.z = z;
            st.idx = st.x + g.lx * row;
            uint32_t nb[6];
            neighbour_indices(st, g.lx, g.ly, g.lz, nb);
            const float jx = s.jxy[z], jzp = s.jz[z], jzm = s.jz[z == 0 ? g.lz - 1 : z - 1];
            const float th = s.th[own + h];
            float si, ci;
            __sincosf(th, &si, &ci);
            /* neighbours in pairs, folded into the field as they come */
            float sa, ca, sb, cb;
            __sincosf(s.th[other + (nb[0] >> 1)], &sa, &ca);
            __sincosf(s.th[other + (nb[1] >> 1)], &sb, &cb);
            if (kMeasure) {
                /* forward bonds i -> i+mu, backward bonds i-mu -> i */
                acc[0] += (double)ci + (double)ca;
                acc[1] += (double)si + (double)sa;
                acc[2] += (double)bond_cos(jx, ci, si, ca, sa) + (double)bond_cos(jx, cb, sb, ci, si);
                acc[5] += (double)bond_sin(jx, ci, si, ca, sa) + (double)bond_sin(jx, cb, sb, ci, si);
            }
            const float hx01 = __fadd_rn(ca, cb), hy01 = __fadd_rn(sa, sb);
            __sincosf(s.th[other + (nb[2] >> 1)], &sa, &ca);
            __sincosf(s.th[other + (nb[3] >> 1)], &sb, &cb);
            if (kMeasure) {
                acc[3] += (double)bond_cos(jx, ci, si, ca, sa) + (double)bond_cos(jx, cb, sb, ci, si);
                acc[6] += (double)bond_sin(jx, ci, si, ca, sa) + (double)bond_sin(jx, cb, sb, ci, si);
            }
            const float hx23 = __fadd_rn(ca, cb), hy23 = __fadd_rn(sa, sb);
            __sincosf(s.th[other + (nb[4] >> 1)], &sa, &ca);
            __sincosf(s.th[other + (nb[5] >> 1)], &sb, &cb);
            if (kMeasure) {
                acc[4] += (double)bond_cos(jzp, ci, si, ca, sa) + (double)bond_cos(jzm, cb, sb, ci, si);
                acc[7] += (double)bond_sin(jzp, ci, si, ca, sa) + (double)bond_sin(jzm, cb, sb, ci, si);
            }
            const float hx = field_from_pairs(jx, jzp, jzm, hx01, hx23, ca, cb);
            const float hy = field_from_pairs(jx, jzp, jzm, hy01, hy23, sa, sb);
            float tn, sn, cn;
            if (metro_decide(th, ci, si, hx, hy, t.beta, t.width, u_prop, u_acc, &tn, &sn, &cn)) {
                s.th[own + h] = tn;
                ++accepted;
            }
        }
    }
    return accepted;
}

/* The same colour half-sweep for L_x = 32, walking along z.  A warp owns a
 * pair of rows (y0, y0 + 1) for a run of planes: lanes 0-15 hold row y0 and
 * lanes 16-31 row y0 + 1, lane k of a group updating the colour-c site of
 * compact index k (x = 2k + parity).  At every plane the lane keeps the trig
 * of the other colour's site of the same compact index on the planes below,
 * at and above (the z neighbours; a window that takes one sincos per plane);
 * the x neighbours are that value of lanes k and k -/+ 1, the y neighbour
 * inside the pair the other group's, and only the y neighbour outside the
 * pair is loaded: four sincos per update instead of eight, and no per-site
 * index division.  Operands, rounding order and randoms are those of
 * half_sweep, so decisions and new angles are bit-identical.  The lane pair
 * (2m, 2m + 1) shares one Philox block per plane: the even lane computes the
 * block of plane z and the odd lane that of plane z + 1, and each passes the
 * other the two words it needs. */
template <bool kMeasure>
__device__ __forceinline__ uint32_t half_sweep_walk32(const TaskView& t, const Geo& g, Smem& s, uint64_t sweep,
                                                      uint32_t colour, double (&acc)[8]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t grp = lane >> 4, k = lane & 15u, odd = k & 1u;
    const uint32_t own = colour * g.stride1, other = (colour ^ 1u) * g.stride1;
    const uint32_t pairs = g.ly >> 1;
    /* planes per unit: every warp gets work when there are fewer pairs than warps */
    const uint32_t nseg = max(1u, min(g.lz / 2, nwarps / max(1u, pairs)));
    const uint32_t seglen = (g.lz + nseg - 1) / nseg;
    const uint32_t lk = grp * 16u + ((k + 15u) & 15u), rk = grp * 16u + ((k + 1u) & 15u);
    uint32_t accepted = 0;
    for (uint32_t u = warp; u < pairs * nseg; u += nwarps) {
        const uint32_t m = u / nseg, sgi = u - m * nseg;
        const uint32_t z_lo = sgi * seglen, z_hi = min(g.lz, z_lo + seglen);
        if (z_lo >= z_hi) continue;
        const uint32_t yr = 2u * m + grp;
        const uint32_t yext = grp ? (yr + 1 == g.ly ? 0u : yr + 1) : (yr == 0 ? g.ly - 1 : yr - 1);
        auto trig_other = [&](uint32_t y, uint32_t z) {
            float sn, cn;
            __sincosf(s.th[other + (y + g.ly * z) * 16u + k], &sn, &cn);
            return make_float2(cn, sn);
        };
        float2 om = trig_other(yr, z_lo == 0 ? g.lz - 1 : z_lo - 1);
        float2 o0 = trig_other(yr, z_lo);
        slsf_u32x4 blk = {0, 0, 0, 0};
        uint32_t w0 = 0, w1 = 0;
        for (uint32_t z = z_lo; z < z_hi; ++z) {
            const uint32_t zi = z - z_lo;
            if ((zi & 1u) == 0) {
                /* the pair's blocks for planes z and z + 1 */
                const uint32_t unit = ((yr + g.ly * (z + odd)) * 16u + k) >> 1;
                blk = slsf_stream(t.seed, sweep, SLSF_PURPOSE_METRO, colour, unit);
                w0 = __shfl_xor_sync(0xffffffffu, odd ? blk.x : blk.z, 1);
                w1 = __shfl_xor_sync(0xffffffffu, odd ? blk.y : blk.w, 1);
            }
            /* plane z: the even lane's own block (x, y), the odd lane the even
             * lane's (z, w); plane z + 1: the even lane the odd lane's (x, y),
             * the odd lane its own (z, w) */
            const bool first = (zi & 1u) == 0;
            const uint32_t wp = first ? (odd ? w0 : blk.x) : (odd ? blk.z : w0);
            const uint32_t wa = first ? (odd ? w1 : blk.y) : (odd ? blk.w : w1);
            const float u_prop = slsf_u24f(wp), u_acc = slsf_u24f(wa);
            const float2 op = trig_other(yr, z + 1 == g.lz ? 0u : z + 1);
            const float2 oy = trig_other(yext, z);
            /* neighbours: x from this group's window, y inside the pair from the other group */
            const float lc = __shfl_sync(0xffffffffu, o0.x, lk), ls = __shfl_sync(0xffffffffu, o0.y, lk);
            const float rc = __shfl_sync(0xffffffffu, o0.x, rk), rs = __shfl_sync(0xffffffffu, o0.y, rk);
            const float pc = __shfl_xor_sync(0xffffffffu, o0.x, 16), ps = __shfl_xor_sync(0xffffffffu, o0.y, 16);
            const uint32_t parity = (colour + yr + z) & 1u;
            /* parity 0: +x is this lane's other-colour site, -x lane k - 1's; parity 1: -x own, +x lane k + 1's */
            const float cxp = parity ? rc : o0.x, sxp = parity ? rs : o0.y;
            const float cxm = parity ? o0.x : lc, sxm = parity ? o0.y : ls;
            const float cyp = grp ? oy.x : pc, syp = grp ? oy.y : ps;
            const float cym = grp ? pc : oy.x, sym = grp ? ps : oy.y;
            const uint32_t q = (yr + g.ly * z) * 16u + k;
            const float jx = s.jxy[z], jzp = s.jz[z], jzm = s.jz[z == 0 ? g.lz - 1 : z - 1];
            const float th = s.th[own + q];
            float si, ci;
            __sincosf(th, &si, &ci);
            if (kMeasure) {
                acc[0] += (double)ci + (double)cxp;
                acc[1] += (double)si + (double)sxp;
                acc[2] += (double)bond_cos(jx, ci, si, cxp, sxp) + (double)bond_cos(jx, cxm, sxm, ci, si);
                acc[5] += (double)bond_sin(jx, ci, si, cxp, sxp) + (double)bond_sin(jx, cxm, sxm, ci, si);
                acc[3] += (double)bond_cos(jx, ci, si, cyp, syp) + (double)bond_cos(jx, cym, sym, ci, si);
                acc[6] += (double)bond_sin(jx, ci, si, cyp, syp) + (double)bond_sin(jx, cym, sym, ci, si);
                acc[4] += (double)bond_cos(jzp, ci, si, op.x, op.y) + (double)bond_cos(jzm, om.x, om.y, ci, si);
                acc[7] += (double)bond_sin(jzp, ci, si, op.x, op.y) + (double)bond_sin(jzm, om.x, om.y, ci, si);
            }
            const float hx01 = __fadd_rn(cxp, cxm), hy01 = __fadd_rn(sxp, sxm);
            const float hx23 = __fadd_rn(cyp, cym), hy23 = __fadd_rn(syp, sym);
            const float hx = field_from_pairs(jx, jzp, jzm, hx01, hx23, op.x, om.x);
            const float hy = field_from_pairs(jx, jzp, jzm, hy01, hy23, op.y, om.y);
            float tn, sn, cn;
            if (metro_decide(th, ci, si, hx, hy, t.beta, t.width, u_prop, u_acc, &tn, &sn, &cn)) {
                s.th[own + q] = tn;
                ++accepted;
            }
            om = o0;
            o0 = op;
        }
    }
    return accepted;
}

/* One colour half-sweep: the z walk for L_x = 32, the general form otherwise. */
template <bool kMeasure>
__device__ __forceinline__ uint32_t sweep_colour(const TaskView& t, const Geo& g, Smem& s, uint64_t sweep,
                                                 uint32_t colour, double (&acc)[8]) {
    if (g.lx == 32) return half_sweep_walk32<kMeasure>(t, g, s, sweep, colour, acc);
    return half_sweep<kMeasure>(t, g, s, sweep, colour, acc);
}

__device__ __forceinline__ float site_theta(const Geo& g, const Smem& s, uint32_t idx, const Coords& c) {
    return s.th[slot(g, idx, (c.x + c.y + c.z) & 1u)];
}

__device__ __forceinline__ float proj_of(float theta, float cphi, float sphi) {
    float sn, cn;
    __sincosf(theta, &sn, &cn);
    return wolff_projection(cn, sn, cphi, sphi);
}

/* One growth pass: every row takes the cluster bits that reach it through
 * its y and z bonds; a row that gained bits is closed along x (stored rows
 * are always closed).  Returns nonzero if any row changed.  Rows updated
 * earlier in the same pass are seen by later ones, so bits can travel more
 * than one row per pass. */
__device__ __forceinline__ int grow_pass(const Geo& g, Smem& s) {
    int changed = 0;
    for (uint32_t r = threadIdx.x; r < g.rows; r += blockDim.x) {
        const uint32_t old = s.cl[r];
        const uint32_t z = slsf_fastdiv_div(r, g.div_ly);
        const uint32_t y = r - z * g.ly;
        const uint32_t r_yp = (y + 1 == g.ly) ? r + 1 - g.ly : r + 1;
        const uint32_t r_ym = (y == 0) ? r + g.ly - 1 : r - 1;
        const uint32_t r_zp = (z + 1 == g.lz) ? r + g.ly - g.rows : r + g.ly;
        const uint32_t r_zm = (z == 0) ? r + g.rows - g.ly : r - g.ly;
        const uint32_t in = (s.cl[r_ym] & s.by[r_ym]) | (s.cl[r_yp] & s.by[r]) | (s.cl[r_zm] & s.bz[r_zm]) |
                            (s.cl[r_zp] & s.bz[r]);
        const uint32_t c = old | in;
        if (c != old) {
            s.cl[r] = close_row(c, s.bx[r], g.lx, g.xmask);
            changed = 1;
        }
    }
    return changed;
}

/* One Wolff update (src/updates.rs:551-620); adds the cluster size to *count. */
__device__ __forceinline__ void wolff_update(const TaskView& t, const Geo& g, Smem& s, uint64_t counter,
                                             uint32_t* s_count) {
    const uint32_t lane = threadIdx.x & 31u;
    const slsf_u32x4 pick = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_PICK, 0, 0);
    const float phi = slsf_angle_from_word(pick.x);
    const uint32_t x0 = slsf_range(pick.y, g.lx), y0 = slsf_range(pick.z, g.ly), z0 = slsf_range(pick.w, g.lz);
    float sphi, cphi;
    __sincosf(phi, &sphi, &cphi);
    const float m2b = __fmul_rn(-2.0f, t.beta);

    if (!g.lx_tiles_warp && g.lx < 24) { /* the general path below ORs into the rows */
        for (uint32_t r = threadIdx.x; r < g.rows; r += blockDim.x) {
            s.bx[r] = 0;
            s.by[r] = 0;
            s.bz[r] = 0;
        }
        __syncthreads();
    }
    if (g.lx == 32) {
        /* A row is a warp (lane = x).  Each warp walks columns of rows along
         * y -- (z, y segment) units, round robin -- so the projection of the
         * +y row is the next row's own: two sincos per site instead of three,
         * and no per-site index division. */
        const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        const uint32_t nseg = (nwarps + g.lz - 1) / g.lz;
        const uint32_t seg = (g.ly + nseg - 1) / nseg;
        for (uint32_t u = warp; u < g.lz * nseg; u += nwarps) {
            const uint32_t z = u / nseg, y_lo = (u % nseg) * seg, y_hi = min(g.ly, y_lo + seg);
            if (y_lo >= y_hi) continue;
            const uint32_t zp_off = (z + 1 == g.lz) ? 0u : (z + 1) * g.plane; /* base of the +z plane */
            const float jx = s.jxy[z], jzz = s.jz[z];
            const uint32_t zbase = z * g.plane;
            float ri = proj_of(s.th[slot(g, zbase + y_lo * 32u + lane, (lane + y_lo + z) & 1u)], cphi, sphi);
            for (uint32_t y = y_lo; y < y_hi; ++y) {
                const uint32_t idx = zbase + y * 32u + lane;
                const uint32_t y1 = (y + 1 == g.ly) ? 0u : y + 1;
                const float ryp = proj_of(s.th[slot(g, zbase + y1 * 32u + lane, (lane + y1 + z) & 1u)], cphi, sphi);
                const float rzp = proj_of(s.th[slot(g, zp_off + y * 32u + lane, (lane + y + z + 1) & 1u)], cphi, sphi);
                const float rxp = __shfl_sync(0xffffffffu, ri, (lane + 1) & 31u);
                const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, idx);
                const uint32_t bal_x = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, rxp, m2b, b.x));
                const uint32_t bal_y = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, ryp, m2b, b.y));
                const uint32_t bal_z = __ballot_sync(0xffffffffu, wolff_bond_active(jzz, ri, rzp, m2b, b.z));
                if (lane == 0) {
                    const uint32_t row = y + g.ly * z;
                    s.bx[row] = bal_x;
                    s.by[row] = bal_y;
                    s.bz[row] = bal_z;
                }
                ri = ryp;
            }
        }
    } else if (g.lx >= 24) {
        /* 24 <= L_x < 32: a row is a warp (lane = x; lanes past the row read
         * the row's first site and keep no bits).  Each warp walks an equal run
         * of the replica's rows in order (y fastest), so the projection of the
         * +y row is the next row's own -- two sincos per site instead of
         * three, and no per-site index division -- except at the first row of
         * its run and of each plane.  (Narrower rows would leave too many
         * lanes idle: they take the general path below.) */
        const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        const uint32_t nrows = g.rows;
        const uint32_t r_lo = (uint32_t)((uint64_t)warp * nrows / nwarps);
        const uint32_t r_hi = (uint32_t)((uint64_t)(warp + 1) * nrows / nwarps);
        const uint32_t xl = lane < g.lx ? lane : 0u;
        const uint32_t xsrc = lane + 1u < g.lx ? lane + 1u : 0u;
        uint32_t z = slsf_fastdiv_div(r_lo, g.div_ly), y = r_lo - z * g.ly;
        uint32_t zbase = 0, zp_off = 0;
        float ri = 0.0f, jx = 0.0f, jzz = 0.0f;
        for (uint32_t row = r_lo; row < r_hi; ++row) {
            if (row == r_lo || y == 0) { /* a new plane: its couplings, offsets and first row */
                zbase = z * g.plane;
                zp_off = (z + 1 == g.lz) ? 0u : (z + 1) * g.plane; /* base of the +z plane */
                jx = s.jxy[z];
                jzz = s.jz[z];
                ri = proj_of(s.th[slot(g, zbase + y * g.lx + xl, (xl + y + z) & 1u)], cphi, sphi);
            }
            const uint32_t idx = zbase + y * g.lx + xl;
            const uint32_t y1 = (y + 1 == g.ly) ? 0u : y + 1;
            const float ryp = proj_of(s.th[slot(g, zbase + y1 * g.lx + xl, (xl + y1 + z) & 1u)], cphi, sphi);
            const float rzp = proj_of(s.th[slot(g, zp_off + y * g.lx + xl, (xl + y + z + 1) & 1u)], cphi, sphi);
            const float rxp = __shfl_sync(0xffffffffu, ri, xsrc);
            const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, idx);
            const uint32_t bal_x = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, rxp, m2b, b.x));
            const uint32_t bal_y = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, ryp, m2b, b.y));
            const uint32_t bal_z = __ballot_sync(0xffffffffu, wolff_bond_active(jzz, ri, rzp, m2b, b.z));
            if (lane == 0) {
                s.bx[row] = bal_x & g.xmask;
                s.by[row] = bal_y & g.xmask;
                s.bz[row] = bal_z & g.xmask;
            }
            ri = ryp;
            if (++y == g.ly) {
                y = 0;
                ++z;
            }
        }
    } else if (g.lx_tiles_warp) {
        /* L_x = 4, 8, 16: a warp holds G = 32 / L_x rows (lane = x + L_x sub), sub-group sub
         * in plane z = G zb + sub; each warp walks columns of rows along y --
         * (zb, y segment) units, round robin -- so the projection of the +y
         * row is the next row's own: two sincos per site instead of three,
         * and no per-site index division.  Sub-groups past the last plane
         * (L_z not a multiple of G) compute on the last plane and keep
         * nothing. */
        const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        const uint32_t gsz = 32u / g.lx, sub = lane / g.lx, x = lane - sub * g.lx;
        const uint32_t nzb = (g.lz + gsz - 1) / gsz;
        const uint32_t nseg = (nwarps + nzb - 1) / nzb;
        const uint32_t seg = (g.ly + nseg - 1) / nseg;
        const uint32_t xsrc = sub * g.lx + (x + 1 == g.lx ? 0u : x + 1);
        for (uint32_t u = warp; u < nzb * nseg; u += nwarps) {
            const uint32_t zb = u / nseg, y_lo = (u % nseg) * seg, y_hi = min(g.ly, y_lo + seg);
            if (y_lo >= y_hi) continue;
            const uint32_t zq = zb * gsz + sub;
            const bool zvalid = zq < g.lz;
            const uint32_t z = zvalid ? zq : g.lz - 1;
            const uint32_t zp_off = (z + 1 == g.lz) ? 0u : (z + 1) * g.plane; /* base of the +z plane */
            const float jx = s.jxy[z], jzz = s.jz[z];
            const uint32_t zbase = z * g.plane;
            float ri = proj_of(s.th[slot(g, zbase + y_lo * g.lx + x, (x + y_lo + z) & 1u)], cphi, sphi);
            for (uint32_t y = y_lo; y < y_hi; ++y) {
                const uint32_t idx = zbase + y * g.lx + x;
                const uint32_t y1 = (y + 1 == g.ly) ? 0u : y + 1;
                const float ryp = proj_of(s.th[slot(g, zbase + y1 * g.lx + x, (x + y1 + z) & 1u)], cphi, sphi);
                const float rzp = proj_of(s.th[slot(g, zp_off + y * g.lx + x, (x + y + z + 1) & 1u)], cphi, sphi);
                const float rxp = __shfl_sync(0xffffffffu, ri, xsrc);
                const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, idx);
                const uint32_t bal_x = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, rxp, m2b, b.x));
                const uint32_t bal_y = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ri, ryp, m2b, b.y));
                const uint32_t bal_z = __ballot_sync(0xffffffffu, wolff_bond_active(jzz, ri, rzp, m2b, b.z));
                if (x == 0 && zvalid) {
                    const uint32_t row = y + g.ly * z;
                    s.bx[row] = (bal_x >> lane) & g.xmask;
                    s.by[row] = (bal_y >> lane) & g.xmask;
                    s.bz[row] = (bal_z >> lane) & g.xmask;
                }
                ri = ryp;
            }
        }
    } else
    /* Bond activation, one thread per site, warp-aligned site ranges. */
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.volume; i0 += blockDim.x) {
        const uint32_t idx = i0 + lane;
        const bool valid = idx < g.volume;
        const uint32_t ii = valid ? idx : 0;
        const Coords c = coords_of(g, ii);
        uint32_t xp, yp, zp;
        forward_neighbours(g, ii, c, xp, yp, zp);
        const float ri = proj_of(site_theta(g, s, ii, c), cphi, sphi);
        float rxp;
        if (g.lx_tiles_warp) {
            rxp = __shfl_sync(0xffffffffu, ri, xp_lane(lane, g.lx));
        } else {
            /* the +x neighbour is the next lane unless the row or the warp ends */
            rxp = __shfl_down_sync(0xffffffffu, ri, 1);
            if (lane == 31 || c.x + 1 == g.lx) {
                const Coords cx = {c.x + 1 == g.lx ? 0 : c.x + 1, c.y, c.z, c.row};
                rxp = proj_of(site_theta(g, s, xp, cx), cphi, sphi);
            }
        }
        const Coords cy = {c.x, c.y + 1 == g.ly ? 0 : c.y + 1, c.z, 0};
        const Coords cz = {c.x, c.y, c.z + 1 == g.lz ? 0 : c.z + 1, 0};
        const float ryp = proj_of(site_theta(g, s, yp, cy), cphi, sphi);
        const float rzp = proj_of(site_theta(g, s, zp, cz), cphi, sphi);
        const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, ii);
        const float jx = s.jxy[c.z], jzz = s.jz[c.z];
        const bool ax = valid && wolff_bond_active(jx, ri, rxp, m2b, b.x);
        const bool ay = valid && wolff_bond_active(jx, ri, ryp, m2b, b.y);
        const bool az = valid && wolff_bond_active(jzz, ri, rzp, m2b, b.z);
        if (g.lx_tiles_warp) {
            const uint32_t bal_x = __ballot_sync(0xffffffffu, ax);
            const uint32_t bal_y = __ballot_sync(0xffffffffu, ay);
            const uint32_t bal_z = __ballot_sync(0xffffffffu, az);
            if (valid && c.x == 0) {
                s.bx[c.row] = (bal_x >> lane) & g.xmask;
                s.by[c.row] = (bal_y >> lane) & g.xmask;
                s.bz[c.row] = (bal_z >> lane) & g.xmask;
            }
        } else {
            /* The warp's 32 consecutive sites cover pieces of a few rows; the
             * first lane of each piece ORs the piece's ballot bits into its
             * row (rows shared with another warp need the atomic). */
            const uint32_t bal_x = __ballot_sync(0xffffffffu, ax);
            const uint32_t bal_y = __ballot_sync(0xffffffffu, ay);
            const uint32_t bal_z = __ballot_sync(0xffffffffu, az);
            if (valid && (lane == 0 || c.x == 0)) {
                const uint32_t len = min(g.lx - c.x, 32u - lane);
                const uint32_t m = len >= 32 ? 0xffffffffu : ((1u << len) - 1u);
                const uint32_t px = ((bal_x >> lane) & m) << c.x;
                const uint32_t py = ((bal_y >> lane) & m) << c.x;
                const uint32_t pz = ((bal_z >> lane) & m) << c.x;
                if (px) atomicOr(&s.bx[c.row], px);
                if (py) atomicOr(&s.by[c.row], py);
                if (pz) atomicOr(&s.bz[c.row], pz);
            }
        }
    }
    const uint32_t seed_row = y0 + g.ly * z0;
    for (uint32_t r = threadIdx.x; r < g.rows; r += blockDim.x) s.cl[r] = (r == seed_row) ? (1u << x0) : 0u;
    __syncthreads();
    if (threadIdx.x == 0) s.cl[seed_row] = close_row(s.cl[seed_row], s.bx[seed_row], g.lx, g.xmask);
    __syncthreads();
    SLSF_PHASE(2);

    /* Grow the seed's component; every pass that goes on adds at least one
     * site, so the count is bounded by V (or the context's loop limit). */
    const uint32_t bound = t.loop_limit ? min(t.loop_limit, g.volume) : g.volume;
    uint32_t pass = 0;
    bool converged = false;
    if (s.blk && g.lx == 32 && g.ly == 32 && g.lz == 32 && blockDim.x == 1024) {
        /* a 32^3 replica is one block of the shared bit-parallel closure: warp
         * scans along y and z, a few passes instead of one row step per pass */
        typedef uint32_t Row[kGrowEdge + 1];
        Row* C = reinterpret_cast<Row*>(s.blk);
        Row* BY = C + kGrowEdge;
        Row* BZ = BY + kGrowEdge;
        Row* BX = BZ + kGrowEdge;
        const uint32_t z = threadIdx.x >> 5, y = threadIdx.x & 31u, r = y + 32u * z;
        C[z][y] = s.cl[r];
        BY[z][y] = s.by[r];
        BZ[z][y] = s.bz[r];
        BX[z][y] = s.bx[r];
        __syncthreads();
        const uint32_t used = close_block(C, BY, BZ, BX, true, true, true, bound + 1);
        converged = used != 0;
        pass = used ? used - 1 : bound;
        s.cl[r] = C[z][y];
        __syncthreads();
    } else if (g.rows <= blockDim.x) {
        /* one row per thread: its neighbour rows and bond masks stay fixed
         * during the growth, so they are read once */
        const uint32_t r = threadIdx.x;
        const bool has = r < g.rows;
        uint32_t r_yp = 0, r_ym = 0, r_zp = 0, r_zm = 0, b_ym = 0, b_yp = 0, b_zm = 0, b_zp = 0, b_x = 0;
        if (has) {
            const uint32_t z = slsf_fastdiv_div(r, g.div_ly);
            const uint32_t y = r - z * g.ly;
            r_yp = (y + 1 == g.ly) ? r + 1 - g.ly : r + 1;
            r_ym = (y == 0) ? r + g.ly - 1 : r - 1;
            r_zp = (z + 1 == g.lz) ? r + g.ly - g.rows : r + g.ly;
            r_zm = (z == 0) ? r + g.rows - g.ly : r - g.ly;
            b_ym = s.by[r_ym];
            b_yp = s.by[r];
            b_zm = s.bz[r_zm];
            b_zp = s.bz[r];
            b_x = s.bx[r];
        }
        for (; pass <= bound; ++pass) {
            int changed = 0;
            if (has) {
                const uint32_t old = s.cl[r];
                const uint32_t c = old | (s.cl[r_ym] & b_ym) | (s.cl[r_yp] & b_yp) | (s.cl[r_zm] & b_zm) |
                                   (s.cl[r_zp] & b_zp);
                if (c != old) {
                    s.cl[r] = close_row(c, b_x, g.lx, g.xmask);
                    changed = 1;
                }
            }
            if (!__syncthreads_or(changed)) {
                converged = true;
                break;
            }
        }
    } else {
        for (; pass <= bound; ++pass)
            if (!__syncthreads_or(grow_pass(g, s))) {
                converged = true;
                break;
            }
    }
    if (!converged && threadIdx.x == 0) atomicOr(&t.stats[kStatError], kErrGrowthLimit);
    SLSF_PHASE(3);
    SLSF_PHASE_COUNT(6, pass + 1);
    SLSF_PHASE_COUNT(7, 1);

    /* Reflect the cluster (src/updates.rs:602-617) and count it. */
    uint32_t members = 0;
    for (uint32_t r = threadIdx.x; r < g.rows; r += blockDim.x) members += __popc(s.cl[r]);
    for (uint32_t idx = threadIdx.x; idx < g.volume; idx += blockDim.x) {
        const Coords c = coords_of(g, idx);
        if ((s.cl[c.row] >> c.x) & 1u) {
            const uint32_t sl = slot(g, idx, (c.x + c.y + c.z) & 1u);
            s.th[sl] = slsf_reflect(s.th[sl], phi);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) members += __shfl_down_sync(0xffffffffu, members, off);
    if (lane == 0 && members) atomicAdd(s_count, members);
    __syncthreads();
    SLSF_PHASE(4);
}

/* (cos, sin) of the site (x, y, z) of the resident state. */
__device__ __forceinline__ float2 trig_at(const Geo& g, const Smem& s, uint32_t x, uint32_t y, uint32_t z) {
    float sn, cn;
    __sincosf(s.th[slot(g, x + g.lx * (y + g.ly * z), (x + y + z) & 1u)], &sn, &cn);
    return make_float2(cn, sn);
}

/* FP64 sum over the warp's lanes (the same shuffle tree everywhere). */
__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

/* Correlation functions of the resident state (measure_theta_correlations_with_scratch,
 * src/observables.rs:165-270), measured between sweeps and added into row
 * count / binsize of the task's correlation bins in ThetaModel::measure's
 * order (C_x, C_y, C_xy, C_xy(z, r), C_z).  Per layer z a warp takes the x
 * lines (lane = x; partners at x + r by shuffle within the row) and the y
 * lines (lane = x; a register window of 8 partners slides along y); per row
 * y a warp takes the z lines the same way along z.  Products are FP32 fused
 * multiply-adds summed per lane over one line length (<= 32), lanes and
 * layers in FP64 in a fixed order.  Scratch (shared): sx, sy [L_z][R] and the
 * per-row z sums [L_y][R_z]. */
__device__ __noinline__ void corr_measure(const ResidentCorr& c, const Geo& g, const Smem& s) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t R = c.rxy, Rz = c.rz, lx = g.lx, ly = g.ly, lz = g.lz;
    double* sx = s.corr;
    double* sy = sx + lz * R;
    double* szr = sy + lz * R;
    const bool xv = lane < lx;
    const uint32_t x = xv ? lane : 0u;
    for (uint32_t u = warp; u < lz + ly; u += nwarps) {
        if (u < lz) {
            const uint32_t z = u;
            for (uint32_t r0 = 1; r0 <= R; r0 += 8) {
                /* x lines: the partner of x at lag r is lane (x + r) mod L_x of the row */
                uint32_t src[8];
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) src[j] = (x + r0 + j) % lx;
                float ax[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                float ay[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                /* y lines: w[j] = partner (x, k + r0 + j) of the current k */
                float2 w[8];
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) w[j] = trig_at(g, s, x, (r0 + j) % ly, z);
                uint32_t nxt = (r0 + 8) % ly; /* y of the partner entering the window after k */
                for (uint32_t k = 0; k < ly; ++k) {
                    float2 a = trig_at(g, s, x, k, z);
                    if (!xv) a = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) {
                        const float pc = __shfl_sync(0xffffffffu, a.x, src[j]);
                        const float ps = __shfl_sync(0xffffffffu, a.y, src[j]);
                        ax[j] = __fmaf_rn(a.y, ps, __fmaf_rn(a.x, pc, ax[j]));
                        ay[j] = __fmaf_rn(a.y, w[j].y, __fmaf_rn(a.x, w[j].x, ay[j]));
                    }
#pragma unroll
                    for (uint32_t j = 0; j + 1 < 8; ++j) w[j] = w[j + 1];
                    w[7] = trig_at(g, s, x, nxt, z);
                    nxt = nxt + 1 == ly ? 0u : nxt + 1;
                }
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) {
                    const double vx = warp_total((double)ax[j]), vy = warp_total((double)ay[j]);
                    if (lane == 0 && r0 + j <= R) {
                        sx[z * R + r0 + j - 1] = vx;
                        sy[z * R + r0 + j - 1] = vy;
                    }
                }
            }
        } else {
            const uint32_t y = u - lz;
            for (uint32_t r0 = 1; r0 <= Rz; r0 += 8) {
                /* z lines of row y: w[j] = partner (x, y, k + r0 + j) */
                float az[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                float2 w[8];
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) w[j] = trig_at(g, s, x, y, (r0 + j) % lz);
                uint32_t nxt = (r0 + 8) % lz;
                for (uint32_t k = 0; k < lz; ++k) {
                    float2 a = trig_at(g, s, x, y, k);
                    if (!xv) a = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) az[j] = __fmaf_rn(a.y, w[j].y, __fmaf_rn(a.x, w[j].x, az[j]));
#pragma unroll
                    for (uint32_t j = 0; j + 1 < 8; ++j) w[j] = w[j + 1];
                    w[7] = trig_at(g, s, x, y, nxt);
                    nxt = nxt + 1 == lz ? 0u : nxt + 1;
                }
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) {
                    const double v = warp_total((double)az[j]);
                    if (lane == 0 && r0 + j <= Rz) szr[y * Rz + r0 + j - 1] = v;
                }
            }
        }
    }
    __shared__ unsigned long long s_row;
    if (threadIdx.x == 0) s_row = *c.count / c.binsize;
    __syncthreads();
    if (s_row < c.n_bins) {
        const uint32_t nv = 3 * R + lz * R + Rz;
        double* bin = c.bins + s_row * nv;
        const double volume = (double)g.volume, area = (double)g.plane;
        for (uint32_t j = threadIdx.x; j < lz * R; j += blockDim.x) bin[3 * R + j] += (sx[j] + sy[j]) / (2.0 * area);
        for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) {
            double a = 0.0, b = 0.0;
            for (uint32_t z = 0; z < lz; ++z) {
                a += sx[z * R + r];
                b += sy[z * R + r];
            }
            const double cx = a / volume, cy = b / volume;
            bin[r] += cx;
            bin[R + r] += cy;
            bin[2 * R + r] += (cx + cy) / 2.0;
        }
        for (uint32_t r = threadIdx.x; r < Rz; r += blockDim.x) {
            double a = 0.0;
            for (uint32_t y = 0; y < ly; ++y) a += szr[y * Rz + r];
            bin[3 * R + lz * R + r] += a / volume;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *c.count += 1;
}

/* Fused observables of the resident state (src/observables.rs:99-141): mx,
 * my, cos xyz, sin xyz; FP64 sums of the FP32 bond terms, block total valid
 * in thread 0. */
__device__ __forceinline__ void measure(const Geo& g, const Smem& s, double (&acc)[8], double* red) {
    const uint32_t lane = threadIdx.x & 31u;
    double f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.volume; i0 += blockDim.x) {
        const uint32_t idx = i0 + lane;
        const bool valid = idx < g.volume;
        const uint32_t ii = valid ? idx : 0;
        const Coords c = coords_of(g, ii);
        uint32_t xp, yp, zp;
        forward_neighbours(g, ii, c, xp, yp, zp);
        float si, ci, sx, cx, sy, cy, sz, cz;
        __sincosf(site_theta(g, s, ii, c), &si, &ci);
        if (g.lx_tiles_warp) {
            const uint32_t src = xp_lane(lane, g.lx);
            sx = __shfl_sync(0xffffffffu, si, src);
            cx = __shfl_sync(0xffffffffu, ci, src);
        } else {
            const Coords cxp = {c.x + 1 == g.lx ? 0 : c.x + 1, c.y, c.z, c.row};
            __sincosf(site_theta(g, s, xp, cxp), &sx, &cx);
        }
        const Coords cyp = {c.x, c.y + 1 == g.ly ? 0 : c.y + 1, c.z, 0};
        const Coords czp = {c.x, c.y, c.z + 1 == g.lz ? 0 : c.z + 1, 0};
        __sincosf(site_theta(g, s, yp, cyp), &sy, &cy);
        __sincosf(site_theta(g, s, zp, czp), &sz, &cz);
        if (!valid) continue;
        const float jx = s.jxy[c.z], jzz = s.jz[c.z];
        f[0] += ci;
        f[1] += si;
        f[2] += bond_cos(jx, ci, si, cx, sx);
        f[3] += bond_cos(jx, ci, si, cy, sy);
        f[4] += bond_cos(jzz, ci, si, cz, sz);
        f[5] += bond_sin(jx, ci, si, cx, sx);
        f[6] += bond_sin(jx, ci, si, cy, sy);
        f[7] += bond_sin(jzz, ci, si, cz, sz);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = f[k];
    block_sum<8>(acc, red);
}


template <bool kCorr>
__global__ void __launch_bounds__(kBThreads, 1)
    k_resident(const TaskView* __restrict__ views, uint32_t n, uint32_t n_sweeps, unsigned int* __restrict__ queue,
               uint32_t max_volume, uint32_t max_rows, uint32_t max_lz, unsigned long long* __restrict__ counters,
               const ResidentCorr* __restrict__ corr, uint32_t cube32) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[8 * 32];
    __shared__ double bin_acc[kBinCols];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_cluster;
    __shared__ uint32_t s_accepted;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n) return;
        TaskView t = views[item];
        if (counters) { /* a replayed launch: the counters live in their own array */
            t.metro_sweeps = counters[2 * item];
            t.wolff_done = counters[2 * item + 1];
        }
        const Geo g = make_geo(t);
        Smem s = carve(smem_raw, max_volume, max_rows, max_lz, cube32);
        if (threadIdx.x == 0) {
            s_cluster = 0;
            s_accepted = 0;
        }
        load_state(t, g, s);
        __syncthreads();
#ifdef SLSF_PHASE_TIMING
        if (threadIdx.x == 0) s_phase_mark = clock64();
#endif
        const uint32_t sweeps = t.sweeps ? t.sweeps : n_sweeps;
        uint32_t accepted = 0;
        int64_t bin_cur = -1;
        /* ThetaModel::measure after every sweep past thermalization: the state
         * after sweep k is measured inside sweep k+1's colour-0 half-sweep,
         * the launch's last state by the measurement pass below. */
        const bool measuring = t.n_bins > 0;
        for (uint32_t sw = 0; sw < sweeps; ++sw) {
            const uint64_t sweep = t.metro_sweeps + sw;
            double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (measuring && sw > 0 && sweep > t.thermalization) {
                accepted += sweep_colour<true>(t, g, s, sweep, 0, acc);
                double tot[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) tot[k] = acc[k];
                block_sum<8>(tot, red);
                if (threadIdx.x == 0) bin_measurement(t, g.volume, sweep, tot, bin_acc, bin_cur);
            } else {
                accepted += sweep_colour<false>(t, g, s, sweep, 0, acc);
            }
            __syncthreads();
            SLSF_PHASE(0);
            accepted += sweep_colour<false>(t, g, s, sweep, 1, acc);
            __syncthreads();
            SLSF_PHASE(1);
            for (uint32_t k = 0; k < t.wolff_steps; ++k)
                wolff_update(t, g, s, t.wolff_done + (uint64_t)sw * t.wolff_steps + k, &s_cluster);
            /* ThetaModel::measure's correlations of the state after this sweep:
             * measurement m = sweep - thermalization, every corr_interval-th */
            if constexpr (kCorr) {
                const ResidentCorr& c = corr[item];
                if (c.bins && sweep >= t.thermalization && (sweep - t.thermalization) % c.interval == 0) {
                    __syncthreads();
                    corr_measure(c, g, s);
                    __syncthreads();
                }
            }
        }
        const uint64_t last = t.metro_sweeps + sweeps;
        /* the counters advance on the device, so that a replayed launch
         * (slsf_batch_open / slsf_batch_step) continues the streams; every
         * thread read them before the first barrier of the item */
        if (counters && threadIdx.x == 0) {
            counters[2 * item] = last;
            counters[2 * item + 1] = t.wolff_done + (uint64_t)sweeps * t.wolff_steps;
        }
        if (measuring && sweeps > 0 && last > t.thermalization) {
            double acc[8];
            measure(g, s, acc, red);
            SLSF_PHASE(5);
            if (threadIdx.x == 0) bin_measurement(t, g.volume, last, acc, bin_acc, bin_cur);
        }
        if (threadIdx.x == 0) flush_bin(t, bin_acc, bin_cur);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) accepted += __shfl_down_sync(0xffffffffu, accepted, off);
        if ((threadIdx.x & 31u) == 0 && accepted) atomicAdd(&s_accepted, accepted);
        __syncthreads();
        store_state(t, g, s);
        if (threadIdx.x == 0) {
            atomicAdd(&t.stats[kStatAccepted], (unsigned long long)s_accepted);
            atomicAdd(&t.stats[kStatClusterSites], (unsigned long long)s_cluster);
            atomicAdd(&t.stats[kStatClusters], (unsigned long long)sweeps * t.wolff_steps);
        }
    }
}

size_t smem_bytes(uint32_t max_volume, uint32_t max_rows, uint32_t max_lz, uint32_t corr_doubles = 0,
                  bool cube32 = false) {
    return 4ull * (max_volume + 2 * kPad) + 16ull * max_rows + 8ull * max_lz + (cube32 ? 4ull * kBlockWords : 0ull) +
           8ull * corr_doubles;
}

template <bool kCorr>
cudaError_t launch_resident_t(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                              int device, cudaStream_t s, uint32_t max_volume, uint32_t max_rows, uint32_t max_lz,
                              uint32_t threads, unsigned long long* counters, const ResidentCorr* corr,
                              uint32_t corr_doubles, bool cube32) {
    const size_t smem = smem_bytes(max_volume, max_rows, max_lz, corr_doubles, cube32);
    cudaError_t e = cudaFuncSetAttribute(k_resident<kCorr>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int sms = 0, per_sm = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resident<kCorr>, (int)threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const uint32_t grid = std::min<uint32_t>(n, (uint32_t)(sms * per_sm));
    k_resident<kCorr><<<grid, threads, smem, s>>>(views_dev, n, n_sweeps, queue, max_volume, max_rows, max_lz,
                                                  counters, corr, cube32 ? 1u : 0u);
    return cudaGetLastError();
}

int max_dynamic_smem(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    /* leave room for the kernel's static shared arrays */
    return v - 4096;
}

}  // namespace

bool resident_supports(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    /* Row words hold L_x <= 32 bits; the colour-split layout needs even
     * dimensions (L_x = 2 mod 4 copies the state site by site). */
    if (lx > kMaxRowBits || lx < 4 || lx % 2 || ly < 2 || ly % 2 || lz < 2 || lz % 2) return false;
    const uint64_t v = (uint64_t)lx * ly * lz;
    return smem_bytes((uint32_t)v, ly * lz, lz) <= (size_t)max_dynamic_smem(device);
}

uint32_t resident_corr_doubles(uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    return (rxy || rz) ? 2 * lz * rxy + ly * rz : 0;
}

cudaError_t launch_resident(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                            int device, cudaStream_t s, uint32_t max_volume, uint32_t max_rows, uint32_t max_lz,
                            uint32_t threads, unsigned long long* counters, const ResidentCorr* corr_dev,
                            uint32_t corr_doubles, bool cube32) {
    if (threads < 32 || threads > (uint32_t)kBThreads || threads % 32) return cudaErrorInvalidConfiguration;
    /* the padded growth blocks of 32^3 replicas, when they fit beside the largest replica */
    if (cube32 && smem_bytes(max_volume, max_rows, max_lz, corr_doubles, true) > (size_t)max_dynamic_smem(device))
        cube32 = false;
    /* the fused correlation measurement is compiled into its own instance, so
     * groups without it run the kernel unchanged */
    if (corr_dev && corr_doubles)
        return launch_resident_t<true>(views_dev, n, n_sweeps, queue, device, s, max_volume, max_rows, max_lz,
                                       threads, counters, corr_dev, corr_doubles, cube32);
    return launch_resident_t<false>(views_dev, n, n_sweeps, queue, device, s, max_volume, max_rows, max_lz,
                                    threads, counters, nullptr, 0, cube32);
}

}  // namespace slsf

#ifdef SLSF_PHASE_TIMING
extern "C" int slsf_debug_resident_phase_cycles(unsigned long long out[8], int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out, slsf::g_res_phase_cycles, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess && reset) {
        const unsigned long long zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        e = cudaMemcpyToSymbol(slsf::g_res_phase_cycles, zero, sizeof(zero));
    }
    return e == cudaSuccess ? 0 : 1;
}
#endif
