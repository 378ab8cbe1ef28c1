/*
 * Batched persistent kernel: many replicas of uneven size, each resident in
 * the distributed shared memory of a thread-block cluster for all of its
 * sweeps.  Replaces the carlo-mc Runner's task-by-task loop over
 * ThetaModel::sweep + ThetaModel::measure (src/model.rs:379-442,
 * src/results.rs:200-202) for every task of a batch at once.
 *
 * A replica is split into C z-slabs (C = cluster size, 1, 2, 4 or 8), one
 * per CTA.  Each CTA keeps, for its slab,
 *   theta   FP32, colour-split layout: the colour-c site with slab index li
 *           sits at c * (Vs/2 + 16) + li/2, so a warp reading one colour
 *           reads consecutive words, and the 64-byte pad puts the two colours
 *           of neighbouring sites in different bank halves;
 *   trig    (cos theta, sin theta) FP32 pairs in the same layout (pad 8
 *           pairs = 64 bytes), always equal to __sincosf(theta), like the
 *           reference's ThetaScratch (src/types.rs:163-214);
 *   bonds   Wolff +x/+y/+z active-bond words and cluster words, one 32-bit
 *           word per row of L_x <= 32 sites;
 *   halo    trig of the partner planes just above and below the slab, copied
 *           from the partners' shared memory (DSMEM) before each phase that
 *           needs it, so that the update loops only touch local memory.
 * Cluster barriers separate the phases.  HBM traffic is one read and one
 * write of theta per launch, independent of the sweep count.
 *
 * Per sweep: two colour half-sweeps with the decision code shared with the
 * single-task kernel (xy_device.cuh), `wolff_steps` Wolff updates, and, after
 * thermalization, the fused measurement accumulated into the task's bins.
 *
 * Wolff labelling is bit-parallel: the cluster grows from the seed by OR-ing
 * neighbour rows through the bond words and closing each changed row along
 * x, until a pass changes nothing in the whole cluster.  The result is the
 * seed's connected component over the active bonds -- the set the
 * reference's DFS (src/updates.rs:577-597) collects when fed the same
 * per-bond randoms.  Growth is monotone, so the pass count is bounded by the
 * site count.
 */
#include <cooperative_groups.h>

#include <algorithm>

#include "engine.h"
#include "fastdiv.h"
#include "xy_device.cuh"

namespace cg = cooperative_groups;

namespace slsf {

namespace {

constexpr int kBThreads = 1024;
constexpr uint32_t kPadTheta = 16; /* floats: 64 bytes */
constexpr uint32_t kPadTrig = 8;   /* float2: 64 bytes */
constexpr uint32_t kMaxRowBits = 32;
constexpr uint32_t kMaxCluster = 8;

/* Optional per-phase cycle accounting (build with -DSLSF_PHASE_TIMING):
 * thread 0 of every CTA adds the clock64 cycles of each phase, measured
 * between block barriers, to g_phase_cycles; slot 6 counts cluster-growth
 * passes and slot 7 Wolff updates. */
#ifdef SLSF_PHASE_TIMING
__device__ unsigned long long g_phase_cycles[8];
__shared__ long long s_phase_mark;
#define SLSF_PHASE(k)                                                                 \
    do {                                                                              \
        __syncthreads();                                                              \
        if (threadIdx.x == 0) {                                                       \
            const long long now_ = clock64();                                         \
            atomicAdd(&g_phase_cycles[k], (unsigned long long)(now_ - s_phase_mark)); \
            s_phase_mark = now_;                                                      \
        }                                                                             \
    } while (0)
#define SLSF_PHASE_COUNT(k, n)                                                          \
    do {                                                                                \
        if (threadIdx.x == 0) atomicAdd(&g_phase_cycles[k], (unsigned long long)(n)); \
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
    uint32_t lx, ly, lz, volume, plane;
    uint32_t nz, z0, rank, csize; /* slab: planes z0 .. z0 + nz - 1 */
    uint32_t vs, half_s, rows_s;  /* slab sites, per colour, rows */
    uint32_t tstride, cstride;    /* colour-1 offsets of theta and trig */
    uint32_t hp;                  /* sites of one colour in one plane */
    uint32_t xmask;
    bool lx_tiles_warp;
    slsf_fastdiv div_hx, div_ly, div_lx;
};

__device__ __forceinline__ Geo make_geo(const TaskView& t, uint32_t rank, uint32_t csize) {
    Geo g;
    g.lx = t.lx;
    g.ly = t.ly;
    g.lz = t.lz;
    g.plane = t.lx * t.ly;
    g.volume = g.plane * t.lz;
    g.csize = csize;
    g.rank = rank;
    g.nz = t.lz / csize;
    g.z0 = rank * g.nz;
    g.vs = g.plane * g.nz;
    g.half_s = g.vs >> 1;
    g.rows_s = t.ly * g.nz;
    g.tstride = g.half_s + kPadTheta;
    g.cstride = g.half_s + kPadTrig;
    g.hp = g.plane >> 1;
    g.xmask = t.lx >= 32 ? 0xffffffffu : ((1u << t.lx) - 1u);
    g.lx_tiles_warp = (32u % t.lx) == 0;
    g.div_hx = slsf_fastdiv_make(t.lx >> 1);
    g.div_ly = slsf_fastdiv_make(t.ly);
    g.div_lx = slsf_fastdiv_make(t.lx);
    return g;
}

struct Coords {
    uint32_t x, y, zl, row; /* zl: plane within the slab; row = y + ly zl */
};

__device__ __forceinline__ Coords coords_of(const Geo& g, uint32_t li) {
    Coords c;
    c.row = slsf_fastdiv_div(li, g.div_lx);
    c.x = li - c.row * g.lx;
    c.zl = slsf_fastdiv_div(c.row, g.div_ly);
    c.y = c.row - c.zl * g.ly;
    return c;
}

__device__ __forceinline__ uint32_t colour_of(const Geo& g, uint32_t x, uint32_t y, uint32_t zl) {
    return (x + y + g.z0 + zl) & 1u;
}

/* Lane holding the next site of a periodic segment of n lanes (n divides 32). */
__device__ __forceinline__ uint32_t seg_next(uint32_t lane, uint32_t n) {
    return (lane & ~(n - 1u)) | ((lane + 1u) & (n - 1u));
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
 * shifts 1..16 cover any row of L_x <= 32 sites.  A shift of L_x or more is
 * skipped (the row is already closed by then). */
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
    float2* cs;   /* [2][cstride] (cos, sin) */
    float* th;    /* [2][tstride] */
    float2* halo; /* [2][hp] partner-plane trig */
    uint32_t* bx;
    uint32_t* by;
    uint32_t* bz;
    uint32_t* cl;
    float* jxy;
    float* jz;
};

/* Per-CTA layout for the largest slab of the launch. */
struct Limits {
    uint32_t vs, rows, lz, hp;
};

__device__ __forceinline__ Smem carve(unsigned char* base, const Limits& m) {
    Smem s;
    unsigned char* p = base;
    s.cs = reinterpret_cast<float2*>(p);
    p += 8ull * (m.vs + 2 * kPadTrig);
    s.halo = reinterpret_cast<float2*>(p);
    p += 16ull * m.hp;
    s.th = reinterpret_cast<float*>(p);
    p += 4ull * (m.vs + 2 * kPadTheta);
    uint32_t* w = reinterpret_cast<uint32_t*>(p);
    s.bx = w;
    s.by = w + m.rows;
    s.bz = w + 2 * m.rows;
    s.cl = w + 3 * m.rows;
    s.jxy = reinterpret_cast<float*>(w + 4 * m.rows);
    s.jz = s.jxy + m.lz;
    return s;
}

/* The partner CTAs holding the planes above (up) and below (dn) this slab;
 * with C = 1 both are this CTA. */
struct Remote {
    const float2* cs_up;
    const float2* cs_dn;
    const uint32_t* cl_up;
    const uint32_t* cl_dn;
    const uint32_t* bz_dn;
};

__device__ __forceinline__ void cluster_barrier(const Geo& g, cg::cluster_group& cluster) {
    if (g.csize == 1)
        __syncthreads();
    else
        cluster.sync();
}

/* halo[0][i] <- up plane 0, colour a; halo[1][i] <- (b_from_up ? up plane 0
 * : dn plane nz-1), colour b.  i is the plane-compact index (x + Lx y) / 2.
 * Ends with a block barrier. */
__device__ __forceinline__ void fill_halo(const Geo& g, Smem& s, const Remote& rm, uint32_t a, uint32_t b,
                                          bool b_from_up) {
    const float2* src_a = rm.cs_up + a * g.cstride;
    const float2* src_b = b_from_up ? rm.cs_up + b * g.cstride
                                    : rm.cs_dn + b * g.cstride + ((g.plane * (g.nz - 1)) >> 1);
    for (uint32_t i = threadIdx.x; i < g.hp; i += blockDim.x) {
        s.halo[i] = src_a[i];
        s.halo[g.hp + i] = src_b[i];
    }
    __syncthreads();
}

/* ---- load / store ---- */

__device__ __forceinline__ void load_slab(const TaskView& t, const Geo& g, Smem& s) {
    const float4* src = reinterpret_cast<const float4*>(t.theta + (size_t)g.plane * g.z0);
    for (uint32_t q = threadIdx.x; q < g.vs / 4; q += blockDim.x) {
        const float4 v = src[q];
        const Coords c = coords_of(g, 4 * q);
        const uint32_t p = colour_of(g, 0, c.y, c.zl); /* x = 4q mod lx is even */
        const uint32_t h = 2 * q;
        const uint32_t ta = p * g.tstride + h, tb = (p ^ 1u) * g.tstride + h;
        const uint32_t ca = p * g.cstride + h, cb = (p ^ 1u) * g.cstride + h;
        float sn, cn;
        s.th[ta] = v.x;
        __sincosf(v.x, &sn, &cn);
        s.cs[ca] = make_float2(cn, sn);
        s.th[tb] = v.y;
        __sincosf(v.y, &sn, &cn);
        s.cs[cb] = make_float2(cn, sn);
        s.th[ta + 1] = v.z;
        __sincosf(v.z, &sn, &cn);
        s.cs[ca + 1] = make_float2(cn, sn);
        s.th[tb + 1] = v.w;
        __sincosf(v.w, &sn, &cn);
        s.cs[cb + 1] = make_float2(cn, sn);
    }
    for (uint32_t z = threadIdx.x; z < g.lz; z += blockDim.x) {
        s.jxy[z] = t.jxy[z];
        s.jz[z] = t.jz[z];
    }
}

__device__ __forceinline__ void store_slab(const TaskView& t, const Geo& g, const Smem& s) {
    float4* dst = reinterpret_cast<float4*>(t.theta + (size_t)g.plane * g.z0);
    for (uint32_t q = threadIdx.x; q < g.vs / 4; q += blockDim.x) {
        const Coords c = coords_of(g, 4 * q);
        const uint32_t p = colour_of(g, 0, c.y, c.zl);
        const uint32_t h = 2 * q;
        const uint32_t ta = p * g.tstride + h, tb = (p ^ 1u) * g.tstride + h;
        dst[q] = make_float4(s.th[ta], s.th[tb], s.th[ta + 1], s.th[tb + 1]);
    }
}

/* ---- Metropolis ---- */

/* One colour half-sweep of the slab; the halo holds the colour-(1-c) trig of
 * the partner planes (halo[0]: above, halo[1]: below).  A warp owns 32
 * consecutive Philox blocks (64 sites); lanes exchange words so that lane j
 * updates colour-compact sites 2*base + j and 2*base + 32 + j. */
__device__ __forceinline__ uint32_t half_sweep(const TaskView& t, const Geo& g, Smem& s, uint64_t sweep,
                                               uint32_t colour) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t npairs = g.half_s >> 1;
    const uint32_t pair0 = (g.plane * g.z0) >> 2; /* global Philox block of the slab's first pair */
    const uint32_t own_t = colour * g.tstride, own_c = colour * g.cstride;
    const uint32_t oth = (colour ^ 1u) * g.cstride;
    const uint32_t hx = g.lx >> 1;
    uint32_t accepted = 0;
    for (uint32_t base = warp * 32; base < npairs; base += nwarps * 32) {
        const uint32_t p = base + lane;
        slsf_u32x4 blk = {0, 0, 0, 0};
        if (p < npairs) blk = slsf_stream(t.seed, sweep, SLSF_PURPOSE_METRO, colour, pair0 + p);
#pragma unroll
        for (uint32_t r = 0; r < 2; ++r) {
            const uint32_t src = 16 * r + (lane >> 1);
            const uint32_t wx = __shfl_sync(0xffffffffu, blk.x, src);
            const uint32_t wy = __shfl_sync(0xffffffffu, blk.y, src);
            const uint32_t wz = __shfl_sync(0xffffffffu, blk.z, src);
            const uint32_t ww = __shfl_sync(0xffffffffu, blk.w, src);
            const uint32_t h = 2 * base + 32 * r + lane;
            if (h >= g.half_s) continue;
            const float u_prop = slsf_u24f((lane & 1u) ? wz : wx);
            const float u_acc = slsf_u24f((lane & 1u) ? ww : wy);
            const uint32_t row = slsf_fastdiv_div(h, g.div_hx);
            const uint32_t k = h - row * hx;
            const uint32_t zl = slsf_fastdiv_div(row, g.div_ly);
            const uint32_t y = row - zl * g.ly;
            const uint32_t z = g.z0 + zl;
            const uint32_t x = 2u * k + ((colour + y + z) & 1u);
            const uint32_t li = x + g.lx * row;
            const uint32_t pc = (x + g.lx * y) >> 1; /* plane-compact index */
            /* in-plane neighbours (slab-local indices) */
            const uint32_t xp = (x + 1 == g.lx) ? li + 1 - g.lx : li + 1;
            const uint32_t xm = (x == 0) ? li + g.lx - 1 : li - 1;
            const uint32_t yp = (y + 1 == g.ly) ? li + g.lx - g.plane : li + g.lx;
            const uint32_t ym = (y == 0) ? li + g.plane - g.lx : li - g.lx;
            const float2 n0 = s.cs[oth + (xp >> 1)];
            const float2 n1 = s.cs[oth + (xm >> 1)];
            const float2 n2 = s.cs[oth + (yp >> 1)];
            const float2 n3 = s.cs[oth + (ym >> 1)];
            const float2 n4 = (zl + 1 < g.nz) ? s.cs[oth + ((li + g.plane) >> 1)] : s.halo[pc];
            const float2 n5 = (zl > 0) ? s.cs[oth + ((li - g.plane) >> 1)] : s.halo[g.hp + pc];
            const float jx = s.jxy[z], jzp = s.jz[z], jzm = s.jz[z == 0 ? g.lz - 1 : z - 1];
            const float hxf = field_component(jx, jzp, jzm, n0.x, n1.x, n2.x, n3.x, n4.x, n5.x);
            const float hyf = field_component(jx, jzp, jzm, n0.y, n1.y, n2.y, n3.y, n4.y, n5.y);
            const float th = s.th[own_t + h];
            const float2 cur = s.cs[own_c + h];
            float tn, sn, cn;
            if (metro_decide(th, cur.x, cur.y, hxf, hyf, t.beta, t.width, u_prop, u_acc, &tn, &sn, &cn)) {
                s.th[own_t + h] = tn;
                s.cs[own_c + h] = make_float2(cn, sn);
                ++accepted;
            }
        }
    }
    return accepted;
}

/* ---- Wolff ---- */

__device__ __forceinline__ float proj(float2 v, float cphi, float sphi) {
    return wolff_projection(v.x, v.y, cphi, sphi);
}

/* Bond activation for every slab site; fills bx/by/bz and seeds cl.  The
 * halo holds both colours of the plane above the slab. */
__device__ __forceinline__ void wolff_bonds(const TaskView& t, const Geo& g, Smem& s, uint64_t counter,
                                            float cphi, float sphi, uint32_t seed_idx) {
    const uint32_t lane = threadIdx.x & 31u;
    const float m2b = __fmul_rn(-2.0f, t.beta);
    if (!g.lx_tiles_warp) {
        for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) {
            s.bx[r] = 0;
            s.by[r] = 0;
            s.bz[r] = 0;
        }
        __syncthreads();
    }
    const uint32_t base_idx = g.plane * g.z0;
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.vs; i0 += blockDim.x) {
        const uint32_t li = i0 + lane;
        const bool valid = li < g.vs;
        const uint32_t ll = valid ? li : 0;
        const Coords c = coords_of(g, ll);
        const uint32_t col = colour_of(g, c.x, c.y, c.zl), oth = (col ^ 1u) * g.cstride;
        const float ri = proj(s.cs[col * g.cstride + (ll >> 1)], cphi, sphi);
        float rxp;
        if (g.lx_tiles_warp) {
            rxp = __shfl_sync(0xffffffffu, ri, seg_next(lane, g.lx));
        } else {
            const uint32_t xp = (c.x + 1 == g.lx) ? ll + 1 - g.lx : ll + 1;
            rxp = proj(s.cs[oth + (xp >> 1)], cphi, sphi);
        }
        const uint32_t yp = (c.y + 1 == g.ly) ? ll + g.lx - g.plane : ll + g.lx;
        const float ryp = proj(s.cs[oth + (yp >> 1)], cphi, sphi);
        const float2 vz = (c.zl + 1 < g.nz) ? s.cs[oth + ((ll + g.plane) >> 1)]
                                            : s.halo[(col ^ 1u) * g.hp + ((c.x + g.lx * c.y) >> 1)];
        const float rzp = proj(vz, cphi, sphi);
        const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, base_idx + ll);
        const float jx = s.jxy[g.z0 + c.zl], jzz = s.jz[g.z0 + c.zl];
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
        } else if (valid) {
            if (ax) atomicOr(&s.bx[c.row], 1u << c.x);
            if (ay) atomicOr(&s.by[c.row], 1u << c.x);
            if (az) atomicOr(&s.bz[c.row], 1u << c.x);
        }
    }
    /* seed the cluster */
    const uint32_t sx = seed_idx % g.lx, srow = seed_idx / g.lx;
    const uint32_t sz = srow / g.ly, sy = srow - sz * g.ly;
    const bool mine = sz >= g.z0 && sz < g.z0 + g.nz;
    const uint32_t seed_row = sy + g.ly * (sz - g.z0);
    for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x)
        s.cl[r] = (mine && r == seed_row) ? (1u << sx) : 0u;
}

/* One growth pass: every row takes the cluster bits that reach it through
 * its y and z bonds; a row that gained bits is closed along x.  Returns
 * nonzero if any row of this CTA changed. */
__device__ __forceinline__ int grow_pass(const Geo& g, Smem& s, const Remote& rm) {
    int changed = 0;
    for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) {
        const uint32_t zl = slsf_fastdiv_div(r, g.div_ly);
        const uint32_t y = r - zl * g.ly;
        const uint32_t old = s.cl[r];
        const uint32_t r_yp = (y + 1 == g.ly) ? r + 1 - g.ly : r + 1;
        const uint32_t r_ym = (y == 0) ? r + g.ly - 1 : r - 1;
        uint32_t in = (s.cl[r_ym] & s.by[r_ym]) | (s.cl[r_yp] & s.by[r]);
        if (zl > 0) {
            in |= s.cl[r - g.ly] & s.bz[r - g.ly];
        } else {
            const uint32_t rr = y + g.ly * (g.nz - 1);
            in |= rm.cl_dn[rr] & rm.bz_dn[rr];
        }
        in |= ((zl + 1 < g.nz) ? s.cl[r + g.ly] : rm.cl_up[y]) & s.bz[r];
        const uint32_t c = old | in;
        if (c != old) {
            s.cl[r] = close_row(c, s.bx[r], g.lx, g.xmask);
            changed = 1;
        }
    }
    return changed;
}

/* One Wolff update (src/updates.rs:551-620); adds the cluster size to *count. */
__device__ __forceinline__ void wolff_update(const TaskView& t, const Geo& g, Smem& s, const Remote& rm,
                                             cg::cluster_group& cluster, uint64_t counter, uint32_t* count,
                                             int* flags) {
    const slsf_u32x4 pick = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_PICK, 0, 0);
    const float phi = slsf_angle_from_word(pick.x);
    const uint32_t x0 = slsf_range(pick.y, g.lx), y0 = slsf_range(pick.z, g.ly), z0 = slsf_range(pick.w, g.lz);
    float sphi, cphi;
    __sincosf(phi, &sphi, &cphi);
    fill_halo(g, s, rm, 0, 1, true);
    wolff_bonds(t, g, s, counter, cphi, sphi, x0 + g.lx * (y0 + g.ly * z0));
    /* the seed row is closed before the first pass */
    __syncthreads();
    if (z0 >= g.z0 && z0 < g.z0 + g.nz && threadIdx.x == 0) {
        const uint32_t r = y0 + g.ly * (z0 - g.z0);
        s.cl[r] = close_row(s.cl[r], s.bx[r], g.lx, g.xmask);
    }
    cluster_barrier(g, cluster);
    SLSF_PHASE(2);

    uint32_t pass = 0;
    for (; pass <= g.volume; ++pass) {
        int any = __syncthreads_or(grow_pass(g, s, rm));
        if (g.csize > 1) {
            if (threadIdx.x == 0) flags[pass & 1] = any;
            cluster.sync();
            any = 0;
            for (uint32_t q = 0; q < g.csize; ++q) any |= *cluster.map_shared_rank(&flags[pass & 1], q);
        }
        if (!any) break;
    }
    SLSF_PHASE(3);
    SLSF_PHASE_COUNT(6, pass + 1);
    SLSF_PHASE_COUNT(7, 1);

    /* Reflect the cluster (src/updates.rs:602-617), refresh its trig. */
    uint32_t members = 0;
    for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) members += __popc(s.cl[r]);
    for (uint32_t li = threadIdx.x; li < g.vs; li += blockDim.x) {
        const Coords c = coords_of(g, li);
        if ((s.cl[c.row] >> c.x) & 1u) {
            const uint32_t col = colour_of(g, c.x, c.y, c.zl);
            const uint32_t st = col * g.tstride + (li >> 1), sc = col * g.cstride + (li >> 1);
            const float nt = slsf_reflect(s.th[st], phi);
            float sn, cn;
            __sincosf(nt, &sn, &cn);
            s.th[st] = nt;
            s.cs[sc] = make_float2(cn, sn);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) members += __shfl_down_sync(0xffffffffu, members, off);
    if ((threadIdx.x & 31u) == 0 && members) atomicAdd(count, members);
    cluster_barrier(g, cluster);
    SLSF_PHASE(4);
}

/* ---- measurement ---- */

/* Slab sums of mx, my, cos xyz, sin xyz (src/observables.rs:99-141): FP32
 * per thread over its sites, FP64 across the block (valid in thread 0).  The
 * halo holds both colours of the plane above the slab. */
__device__ __forceinline__ void measure_slab(const Geo& g, const Smem& s, double (&acc)[8], double* red) {
    const uint32_t lane = threadIdx.x & 31u;
    float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.vs; i0 += blockDim.x) {
        const uint32_t li = i0 + lane;
        const bool valid = li < g.vs;
        const uint32_t ll = valid ? li : 0;
        const Coords c = coords_of(g, ll);
        const uint32_t col = colour_of(g, c.x, c.y, c.zl), oth = (col ^ 1u) * g.cstride;
        const float2 me = s.cs[col * g.cstride + (ll >> 1)];
        float2 nx;
        if (g.lx_tiles_warp) {
            const uint32_t src = seg_next(lane, g.lx);
            nx.x = __shfl_sync(0xffffffffu, me.x, src);
            nx.y = __shfl_sync(0xffffffffu, me.y, src);
        } else {
            const uint32_t xp = (c.x + 1 == g.lx) ? ll + 1 - g.lx : ll + 1;
            nx = s.cs[oth + (xp >> 1)];
        }
        const uint32_t yp = (c.y + 1 == g.ly) ? ll + g.lx - g.plane : ll + g.lx;
        const float2 ny = s.cs[oth + (yp >> 1)];
        const float2 nz = (c.zl + 1 < g.nz) ? s.cs[oth + ((ll + g.plane) >> 1)]
                                            : s.halo[(col ^ 1u) * g.hp + ((c.x + g.lx * c.y) >> 1)];
        if (!valid) continue;
        const float jx = s.jxy[g.z0 + c.zl], jzz = s.jz[g.z0 + c.zl];
        /* diff_cos_sin (src/observables.rs:9-11) */
        f[0] += me.x;
        f[1] += me.y;
        f[2] += jx * (me.x * nx.x + me.y * nx.y);
        f[3] += jx * (me.x * ny.x + me.y * ny.y);
        f[4] += jzz * (me.x * nz.x + me.y * nz.y);
        f[5] += jx * (me.y * nx.x - me.x * nx.y);
        f[6] += jx * (me.y * ny.x - me.x * ny.y);
        f[7] += jzz * (me.y * nz.x - me.x * nz.y);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = (double)f[k];
    block_sum<8>(acc, red);
}

__global__ void __launch_bounds__(kBThreads, 1)
    k_batched(const TaskView* __restrict__ views, uint32_t n, uint32_t n_sweeps, unsigned int* __restrict__ queue,
              Limits lim) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[8 * 32];
    __shared__ double cred[kMaxCluster][8]; /* slab sums gathered in rank 0 */
    __shared__ double bin_acc[kBinCols];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_cluster;
    __shared__ int s_flags[2];
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank(), csize = cluster.num_blocks();
    Smem s = carve(smem_raw, lim);
    Remote rm;
    {
        const uint32_t up = (rank + 1) % csize, dn = (rank + csize - 1) % csize;
        rm.cs_up = cluster.map_shared_rank(s.cs, up);
        rm.cs_dn = cluster.map_shared_rank(s.cs, dn);
        rm.cl_up = cluster.map_shared_rank(s.cl, up);
        rm.cl_dn = cluster.map_shared_rank(s.cl, dn);
        rm.bz_dn = cluster.map_shared_rank(s.bz, dn);
    }
    for (;;) {
        /* rank 0 takes the next replica and tells its partners */
        if (rank == 0 && threadIdx.x == 0) {
            const uint32_t item = atomicAdd(queue, 1u);
            for (uint32_t q = 0; q < csize; ++q) *cluster.map_shared_rank(&s_item, q) = item;
        }
        cluster.sync();
        const uint32_t item = s_item;
        if (item >= n) return;
        const TaskView t = views[item];
        const Geo g = make_geo(t, rank, csize);
        if (threadIdx.x == 0) s_cluster = 0;
        load_slab(t, g, s);
        cluster.sync();
#ifdef SLSF_PHASE_TIMING
        if (threadIdx.x == 0) s_phase_mark = clock64();
#endif
        uint32_t accepted = 0;
        int64_t bin_cur = -1;
        for (uint32_t sw = 0; sw < n_sweeps; ++sw) {
            const uint64_t sweep = t.metro_sweeps + sw;
            fill_halo(g, s, rm, 1, 1, false);
            accepted += half_sweep(t, g, s, sweep, 0);
            cluster_barrier(g, cluster);
            SLSF_PHASE(0);
            fill_halo(g, s, rm, 0, 0, false);
            accepted += half_sweep(t, g, s, sweep, 1);
            cluster_barrier(g, cluster);
            SLSF_PHASE(1);
            for (uint32_t k = 0; k < t.wolff_steps; ++k)
                wolff_update(t, g, s, rm, cluster, t.wolff_done + (uint64_t)sw * t.wolff_steps + k, &s_cluster,
                             s_flags);
            /* ThetaModel::measure after the sweep, once thermalized. */
            const uint64_t done = sweep + 1;
            if (done > t.thermalization && t.n_bins > 0) {
                double acc[8];
                fill_halo(g, s, rm, 0, 1, true);
                measure_slab(g, s, acc, red);
                if (threadIdx.x == 0)
                    for (int k = 0; k < 8; ++k) *cluster.map_shared_rank(&cred[rank][k], 0) = acc[k];
                cluster_barrier(g, cluster);
                SLSF_PHASE(5);
                if (rank == 0 && threadIdx.x == 0) {
                    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    for (uint32_t q = 0; q < csize; ++q)
                        for (int k = 0; k < 8; ++k) a[k] += cred[q][k];
                    const int64_t b = (int64_t)((done - t.thermalization - 1) / t.binsize);
                    if (b != bin_cur) {
                        if (bin_cur >= 0 && bin_cur < (int64_t)t.n_bins)
                            for (int q = 0; q < kBinCols; ++q) t.bins[bin_cur * kBinCols + q] += bin_acc[q];
                        for (int q = 0; q < kBinCols; ++q) bin_acc[q] = 0.0;
                        bin_cur = b;
                    }
                    const double v = (double)g.volume;
                    const double e = -(a[2] + a[3] + a[4]) / v;
                    const double vals[kBinCols] = {e,    e * e, (a[0] * a[0] + a[1] * a[1]) / (v * v),
                                                   a[2], a[3],  a[4],
                                                   a[5], a[6],  a[7],
                                                   a[5] * a[5], a[6] * a[6], a[7] * a[7]};
                    for (int q = 0; q < kBinCols; ++q) bin_acc[q] += vals[q];
                }
                /* partners must not overwrite cred or trig before rank 0 is done */
                cluster_barrier(g, cluster);
            }
        }
        if (rank == 0 && threadIdx.x == 0 && bin_cur >= 0 && bin_cur < (int64_t)t.n_bins)
            for (int q = 0; q < kBinCols; ++q) t.bins[bin_cur * kBinCols + q] += bin_acc[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) accepted += __shfl_down_sync(0xffffffffu, accepted, off);
        if ((threadIdx.x & 31u) == 0 && accepted) atomicAdd(&t.stats[kStatAccepted], (unsigned long long)accepted);
        store_slab(t, g, s);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_cluster) atomicAdd(&t.stats[kStatClusterSites], (unsigned long long)s_cluster);
            if (rank == 0) atomicAdd(&t.stats[kStatClusters], (unsigned long long)n_sweeps * t.wolff_steps);
        }
        /* no CTA may start the next replica while a partner still reads its slab */
        cluster.sync();
    }
}

size_t smem_bytes(const Limits& m) {
    return 8ull * (m.vs + 2 * kPadTrig) + 16ull * m.hp + 4ull * (m.vs + 2 * kPadTheta) + 16ull * m.rows +
           8ull * m.lz;
}

int max_dynamic_smem(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    /* leave room for the kernel's static shared arrays */
    return v - 4096;
}

}  // namespace

uint32_t batched_cluster_size(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    /* Row words hold L_x <= 32 bits; the float4 colour-split copy needs
     * L_x % 4 == 0 so that four consecutive sites never span two rows. */
    if (lx > kMaxRowBits || lx < 4 || lx % 4 || ly < 2 || ly % 2 || lz < 2 || lz % 2) return 0;
    for (uint32_t c = 1; c <= kMaxCluster; c <<= 1) {
        if (lz % c) continue;
        const uint32_t nz = lz / c;
        const Limits m = {lx * ly * nz, ly * nz, lz, (lx * ly) / 2};
        if (smem_bytes(m) <= (size_t)max_dynamic_smem(device)) return c;
    }
    return 0;
}

bool batched_supports(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    return batched_cluster_size(lx, ly, lz, device) != 0;
}

cudaError_t launch_batched(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                           int device, cudaStream_t s, uint32_t cluster, uint32_t max_vs, uint32_t max_rows,
                           uint32_t max_lz, uint32_t max_plane) {
    (void)device;
    const Limits lim = {max_vs, max_rows, max_lz, max_plane / 2};
    const size_t smem = smem_bytes(lim);
    cudaError_t e = cudaFuncSetAttribute(k_batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kBThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cluster, 1, 1);
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, k_batched, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorInvalidConfiguration;
    const uint32_t grid_clusters = std::min<uint32_t>(n, (uint32_t)clusters);
    cfg.gridDim = dim3(grid_clusters * cluster, 1, 1);
    return cudaLaunchKernelEx(&cfg, k_batched, views_dev, n, n_sweeps, queue, lim);
}

}  // namespace slsf

#ifdef SLSF_PHASE_TIMING
extern "C" int slsf_debug_phase_cycles(unsigned long long out[8], int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out, slsf::g_phase_cycles, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess && reset) {
        const unsigned long long zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        e = cudaMemcpyToSymbol(slsf::g_phase_cycles, zero, sizeof(zero));
    }
    return e == cudaSuccess ? 0 : 1;
}
#endif
