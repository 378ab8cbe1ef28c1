/*
 * Batched persistent kernel for replicas too large for one CTA: each replica
 * is split into C z-slabs (C = 1, 2, 4 or 8) held in the distributed shared
 * memory of a thread-block cluster for all of its sweeps.  Same role as
 * kernel_resident.cu -- the carlo-mc Runner's task-by-task loop over
 * ThetaModel::sweep + ThetaModel::measure (src/model.rs:379-442,
 * src/results.rs:200-202) for every task of a batch -- for L_x up to 64
 * (L = 48 and 64 cubes: 4 and 8 CTAs of about 110 and 130 KiB).
 *
 * Each CTA keeps, for its slab (planes z0 .. z0 + nz - 1),
 *   theta   FP32, colour-split layout: the colour-c site with slab index li
 *           at c * (Vs/2 + 16) + li/2 (consecutive words per warp access; the
 *           64-byte pad puts the colours of neighbouring sites in different
 *           bank halves);
 *   halo    theta of the partner planes just above (z0 + nz) and below
 *           (z0 - 1), copied from the partners' shared memory through DSMEM
 *           before every phase that needs them, so the update loops read only
 *           local shared memory;
 *   bonds   Wolff +x/+y/+z active-bond words and cluster words, one W-bit
 *           word per row (W = 32 for L_x <= 32, 64 for L_x <= 64).
 * Trig values are recomputed with __sincosf from theta where needed, exactly
 * as in the single-task kernels, so results are bit-identical to them.
 * Cluster barriers separate the phases.  HBM traffic is one read and one
 * write of theta per launch, independent of the sweep count.
 *
 * Wolff labelling is bit-parallel: the cluster grows from the seed in
 * rounds; a round closes every column along z (sequentially per column,
 * across the slab faces through the partners' rows), then every row along y
 * (a segmented scan over the lanes of a warp) and along x (a doubling scan
 * inside the row word), until a round changes nothing in the whole cluster.
 * The result is the seed's connected component over the active bonds -- the
 * set the reference's DFS (src/updates.rs:577-597) collects when fed the
 * same per-bond randoms.  Growth is monotone, so the round count is bounded
 * by V.
 */
#include <cooperative_groups.h>

#include <algorithm>

#include "bins.cuh"
#include "engine.h"
#include "fastdiv.h"
#include "xy_device.cuh"

namespace cg = cooperative_groups;

namespace slsf {

namespace {

constexpr int kBThreads = 1024;
constexpr uint32_t kPad = 16; /* floats: 64 bytes */
constexpr uint32_t kMaxRowBits = 64;
constexpr uint32_t kMaxCluster = 16; /* 16 needs the non-portable cluster size opt-in */

/* Optional per-phase cycle accounting (build with -DSLSF_PHASE_TIMING). */
#ifdef SLSF_PHASE_TIMING
__device__ unsigned long long g_cl_phase_cycles[8];
__shared__ long long s_phase_mark;
#define SLSF_PHASE(k)                                                                    \
    do {                                                                                 \
        __syncthreads();                                                                 \
        if (threadIdx.x == 0) {                                                          \
            const long long now_ = clock64();                                            \
            atomicAdd(&g_cl_phase_cycles[k], (unsigned long long)(now_ - s_phase_mark)); \
            s_phase_mark = now_;                                                         \
        }                                                                                \
    } while (0)
#define SLSF_PHASE_COUNT(k, n)                                                             \
    do {                                                                                   \
        if (threadIdx.x == 0) atomicAdd(&g_cl_phase_cycles[k], (unsigned long long)(n)); \
    } while (0)
#else
#define SLSF_PHASE(k) \
    do {              \
    } while (0)
#define SLSF_PHASE_COUNT(k, n) \
    do {                       \
    } while (0)
#endif

/* ---- row words ---- */

template <typename W>
struct RowOps;

template <>
struct RowOps<uint32_t> {
    static __device__ __forceinline__ uint32_t rotl(uint32_t w, uint32_t s, uint32_t lx, uint32_t mask) {
        return lx == 32 ? __funnelshift_l(w, w, s) : (((w << s) | (w >> (lx - s))) & mask);
    }
    static __device__ __forceinline__ uint32_t rotr(uint32_t w, uint32_t s, uint32_t lx, uint32_t mask) {
        return lx == 32 ? __funnelshift_r(w, w, s) : (((w >> s) | (w << (lx - s))) & mask);
    }
    static __device__ __forceinline__ uint32_t popc(uint32_t w) { return __popc(w); }
};

template <>
struct RowOps<uint64_t> {
    static __device__ __forceinline__ uint64_t rotl(uint64_t w, uint32_t s, uint32_t lx, uint64_t mask) {
        return lx == 64 ? ((w << s) | (w >> (64 - s))) : (((w << s) | (w >> (lx - s))) & mask);
    }
    static __device__ __forceinline__ uint64_t rotr(uint64_t w, uint32_t s, uint32_t lx, uint64_t mask) {
        return lx == 64 ? ((w >> s) | (w << (64 - s))) : (((w >> s) | (w << (lx - s))) & mask);
    }
    static __device__ __forceinline__ uint32_t popc(uint64_t w) { return __popcll(w); }
};

__device__ __forceinline__ void atomic_or_row(uint32_t* p, uint32_t v) { atomicOr(p, v); }
__device__ __forceinline__ void atomic_or_row(uint64_t* p, uint64_t v) {
    atomicOr(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

/* Closure of a periodic row's cluster bits c along x through the bond bits b
 * (bit x: bond x -- x+1).  Kogge-Stone doubling in both directions: after the
 * step with shift s, every site within 2s - 1 bond steps of a seed is set;
 * shifts up to 32 cover any row of L_x <= 64 sites. */
template <typename W>
__device__ __forceinline__ W close_row(W c, W b, uint32_t lx, W mask) {
    using R = RowOps<W>;
    W gr = c, pr = b;                   /* rightward: bond p -> p+1 */
    W gl = c, pl = R::rotl(b, 1, lx, mask); /* leftward: bond p-1 -> p */
#pragma unroll
    for (uint32_t s = 1; s < 8 * sizeof(W); s <<= 1) {
        if (s >= lx) break;
        gr |= R::rotl(gr & pr, s, lx, mask);
        pr &= R::rotr(pr, s, lx, mask);
        gl |= R::rotr(gl & pl, s, lx, mask);
        pl &= R::rotl(pl, s, lx, mask);
    }
    return gr | gl;
}

/* ---- geometry ---- */

struct Geo {
    uint32_t lx, ly, lz, volume, plane;
    uint32_t nz, z0, rank, csize; /* slab: planes z0 .. z0 + nz - 1 */
    uint32_t vs, half_s, rows_s;  /* slab sites, per colour, rows */
    uint32_t tstride;             /* colour-1 offset of theta */
    uint32_t hp;                  /* sites of one colour in one plane */
    bool lx_tiles_warp;           /* 32 % lx == 0 */
    bool lx_two_warps;            /* 32 < lx <= 64: a warp holds a row, lanes j and j + 32 */
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
    g.tstride = g.half_s + kPad;
    g.hp = g.plane >> 1;
    g.lx_tiles_warp = t.lx <= 32 && (32u % t.lx) == 0;
    g.lx_two_warps = t.lx > 32 && t.lx <= 64;
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

/* ---- shared memory ---- */

template <typename W>
struct Smem {
    float* th;   /* [2][tstride] */
    float* halo; /* [0..1]: plane above, colours 0/1; [2..3]: plane below, colours 0/1; each [hp] */
    W* bx;
    W* by;
    W* bz;
    W* cl;
    float* jxy;
    float* jz;
    uint8_t* dirty; /* per row: changed by growth stage Z, not yet x-closed */
    W* zc;          /* stage Z: carry out of each column segment */
    W* zp;          /* stage Z: product of each column segment's links */
};

struct Limits {
    uint32_t vs, rows, lz, hp;
};

template <typename W>
__device__ __forceinline__ Smem<W> carve(unsigned char* base, const Limits& m) {
    Smem<W> s;
    unsigned char* p = base;
    W* w = reinterpret_cast<W*>(p); /* 8-byte aligned first */
    s.bx = w;
    s.by = w + m.rows;
    s.bz = w + 2 * m.rows;
    s.cl = w + 3 * m.rows;
    s.zc = w + 4 * m.rows;
    s.zp = w + 5 * m.rows;
    p += 6ull * m.rows * sizeof(W);
    s.th = reinterpret_cast<float*>(p);
    p += 4ull * (m.vs + 2 * kPad);
    s.halo = reinterpret_cast<float*>(p);
    p += 16ull * m.hp;
    s.jxy = reinterpret_cast<float*>(p);
    s.jz = s.jxy + m.lz;
    s.dirty = reinterpret_cast<uint8_t*>(s.jz + m.lz);
    return s;
}

template <typename W>
struct Remote {
    const float* th_up; /* partner holding plane z0 + nz */
    const float* th_dn; /* partner holding plane z0 - 1 */
    const W* cl_up;
    const W* cl_dn;
    const W* bz_dn;
};

__device__ __forceinline__ void cluster_barrier(const Geo& g, cg::cluster_group& cluster) {
    if (g.csize == 1)
        __syncthreads();
    else
        cluster.sync();
}

/* Copy colour `col` (or both colours when col > 1) of the partner planes
 * above and below the slab into the halo; ends with a block barrier. */
template <typename W>
__device__ __forceinline__ void fill_halo(const Geo& g, Smem<W>& s, const Remote<W>& rm, uint32_t col) {
    const uint32_t c0 = col > 1 ? 0 : col, c1 = col > 1 ? 1 : col;
    const uint32_t below = (g.plane * (g.nz - 1)) >> 1; /* compact offset of the partner's last plane */
    for (uint32_t c = c0; c <= c1; ++c) {
        const float* up = rm.th_up + c * g.tstride;
        const float* dn = rm.th_dn + c * g.tstride + below;
        for (uint32_t i = threadIdx.x; i < g.hp; i += blockDim.x) {
            s.halo[c * g.hp + i] = up[i];
            s.halo[(2 + c) * g.hp + i] = dn[i];
        }
    }
    __syncthreads();
}

/* theta of the site at plane-compact index pc, colour col, one plane above
 * (up = true) or below the slab. */
template <typename W>
__device__ __forceinline__ float halo_theta(const Geo& g, const Smem<W>& s, bool up, uint32_t col, uint32_t pc) {
    return s.halo[(up ? 0u : 2u) * g.hp + col * g.hp + pc];
}

/* ---- load / store ---- */

template <typename W>
__device__ __forceinline__ void load_slab(const TaskView& t, const Geo& g, Smem<W>& s) {
    if (g.lx % 4) {
        /* L_x = 2 mod 4: four consecutive sites may span two rows; copy site by site */
        const float* src = t.theta + (size_t)g.plane * g.z0;
        for (uint32_t li = threadIdx.x; li < g.vs; li += blockDim.x) {
            const Coords c = coords_of(g, li);
            s.th[colour_of(g, c.x, c.y, c.zl) * g.tstride + (li >> 1)] = src[li];
        }
    } else {
        const float4* src = reinterpret_cast<const float4*>(t.theta + (size_t)g.plane * g.z0);
        for (uint32_t q = threadIdx.x; q < g.vs / 4; q += blockDim.x) {
            const float4 v = src[q];
            const Coords c = coords_of(g, 4 * q);
            const uint32_t p = colour_of(g, 0, c.y, c.zl); /* x = 4q mod lx is even */
            const uint32_t h = 2 * q;
            s.th[p * g.tstride + h] = v.x;
            s.th[(p ^ 1u) * g.tstride + h] = v.y;
            s.th[p * g.tstride + h + 1] = v.z;
            s.th[(p ^ 1u) * g.tstride + h + 1] = v.w;
        }
    }
    for (uint32_t z = threadIdx.x; z < g.lz; z += blockDim.x) {
        s.jxy[z] = t.jxy[z];
        s.jz[z] = t.jz[z];
    }
}

template <typename W>
__device__ __forceinline__ void store_slab(const TaskView& t, const Geo& g, const Smem<W>& s) {
    if (g.lx % 4) {
        float* dst = t.theta + (size_t)g.plane * g.z0;
        for (uint32_t li = threadIdx.x; li < g.vs; li += blockDim.x) {
            const Coords c = coords_of(g, li);
            dst[li] = s.th[colour_of(g, c.x, c.y, c.zl) * g.tstride + (li >> 1)];
        }
        return;
    }
    float4* dst = reinterpret_cast<float4*>(t.theta + (size_t)g.plane * g.z0);
    for (uint32_t q = threadIdx.x; q < g.vs / 4; q += blockDim.x) {
        const Coords c = coords_of(g, 4 * q);
        const uint32_t p = colour_of(g, 0, c.y, c.zl);
        const uint32_t h = 2 * q;
        dst[q] = make_float4(s.th[p * g.tstride + h], s.th[(p ^ 1u) * g.tstride + h],
                             s.th[p * g.tstride + h + 1], s.th[(p ^ 1u) * g.tstride + h + 1]);
    }
}

/* ---- Metropolis ---- */

/* One colour half-sweep of the slab; the halo holds colour 1-c of the
 * partner planes.  A warp owns 32 consecutive Philox blocks (64 sites);
 * lanes exchange words so that lane j updates colour-compact sites
 * 2*base + j and 2*base + 32 + j.  With kMeasure (colour 0) it also adds the
 * slab's share of the observables of the state it starts from: the three
 * forward and three backward bonds of every colour-0 site (every bond has
 * exactly one colour-0 end) and the magnetisation of the site and of its +x
 * neighbour, with the bond_cos / bond_sin terms of the measurement pass. */
template <bool kMeasure, typename W>
__device__ __forceinline__ uint32_t half_sweep(const TaskView& t, const Geo& g, Smem<W>& s, uint64_t sweep,
                                               uint32_t colour, double (&acc)[8]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t npairs = g.half_s >> 1;
    const uint32_t pair0 = (g.plane * g.z0) >> 2;
    const uint32_t own = colour * g.tstride, oth = (colour ^ 1u) * g.tstride, ocol = colour ^ 1u;
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
            const uint32_t pc = (x + g.lx * y) >> 1;
            const uint32_t xp = (x + 1 == g.lx) ? li + 1 - g.lx : li + 1;
            const uint32_t xm = (x == 0) ? li + g.lx - 1 : li - 1;
            const uint32_t yp = (y + 1 == g.ly) ? li + g.lx - g.plane : li + g.lx;
            const uint32_t ym = (y == 0) ? li + g.plane - g.lx : li - g.lx;
            const float jx = s.jxy[z], jzp = s.jz[z], jzm = s.jz[z == 0 ? g.lz - 1 : z - 1];
            const float th = s.th[own + h];
            float si, ci;
            __sincosf(th, &si, &ci);
            /* neighbours in pairs (+x -x, +y -y, +z -z), folded into the field as they come */
            float sa, ca, sb, cb;
            __sincosf(s.th[oth + (xp >> 1)], &sa, &ca);
            __sincosf(s.th[oth + (xm >> 1)], &sb, &cb);
            if (kMeasure) {
                acc[0] += (double)ci + (double)ca;
                acc[1] += (double)si + (double)sa;
                acc[2] += (double)bond_cos(jx, ci, si, ca, sa) + (double)bond_cos(jx, cb, sb, ci, si);
                acc[5] += (double)bond_sin(jx, ci, si, ca, sa) + (double)bond_sin(jx, cb, sb, ci, si);
            }
            const float hx01 = __fadd_rn(ca, cb), hy01 = __fadd_rn(sa, sb);
            __sincosf(s.th[oth + (yp >> 1)], &sa, &ca);
            __sincosf(s.th[oth + (ym >> 1)], &sb, &cb);
            if (kMeasure) {
                acc[3] += (double)bond_cos(jx, ci, si, ca, sa) + (double)bond_cos(jx, cb, sb, ci, si);
                acc[6] += (double)bond_sin(jx, ci, si, ca, sa) + (double)bond_sin(jx, cb, sb, ci, si);
            }
            const float hx23 = __fadd_rn(ca, cb), hy23 = __fadd_rn(sa, sb);
            const float t4 = (zl + 1 < g.nz) ? s.th[oth + ((li + g.plane) >> 1)] : halo_theta(g, s, true, ocol, pc);
            const float t5 = (zl > 0) ? s.th[oth + ((li - g.plane) >> 1)] : halo_theta(g, s, false, ocol, pc);
            __sincosf(t4, &sa, &ca);
            __sincosf(t5, &sb, &cb);
            if (kMeasure) {
                acc[4] += (double)bond_cos(jzp, ci, si, ca, sa) + (double)bond_cos(jzm, cb, sb, ci, si);
                acc[7] += (double)bond_sin(jzp, ci, si, ca, sa) + (double)bond_sin(jzm, cb, sb, ci, si);
            }
            const float hxf = field_from_pairs(jx, jzp, jzm, hx01, hx23, ca, cb);
            const float hyf = field_from_pairs(jx, jzp, jzm, hy01, hy23, sa, sb);
            float tn, sn, cn;
            if (metro_decide(th, ci, si, hxf, hyf, t.beta, t.width, u_prop, u_acc, &tn, &sn, &cn)) {
                s.th[own + h] = tn;
                ++accepted;
            }
        }
    }
    return accepted;
}

/* ---- Wolff ---- */

__device__ __forceinline__ float proj_of(float theta, float cphi, float sphi) {
    float sn, cn;
    __sincosf(theta, &sn, &cn);
    return wolff_projection(cn, sn, cphi, sphi);
}

/* Bond activation for every slab site (the halo holds both colours of the
 * partner planes); fills bx/by/bz and seeds cl with the closed seed row. */
template <typename W>
__device__ __forceinline__ void wolff_bonds(const TaskView& t, const Geo& g, Smem<W>& s, uint64_t counter,
                                            float cphi, float sphi, uint32_t seed_idx) {
    const uint32_t lane = threadIdx.x & 31u;
    const float m2b = __fmul_rn(-2.0f, t.beta);
    const bool ballots = g.lx_tiles_warp || g.lx_two_warps;
    if (!ballots) {
        for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) {
            s.bx[r] = 0;
            s.by[r] = 0;
            s.bz[r] = 0;
        }
        __syncthreads();
    }
    const uint32_t base_idx = g.plane * g.z0;
    bool walked = false;
    if constexpr (sizeof(W) == 8) {
      if (g.lx_two_warps) {
        walked = true;
        /* 32 < L_x <= 64: a warp holds a whole row, lane j the sites x = j and
         * x = j + 32 (lanes past the row's end repeat x = j, whose colour is the
         * same, and keep no bits).  Each warp walks an equal run of the slab's
         * rows in order (y fastest), so the projections of the +y row are the
         * next row's own -- two sincos per site instead of three -- except at
         * the first row of its run and of each plane. */
        const uint32_t warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
        const uint32_t nrows = g.nz * g.ly;
        const uint32_t r_lo = (uint32_t)((uint64_t)warp * nrows / nwarps);
        const uint32_t r_hi = (uint32_t)((uint64_t)(warp + 1) * nrows / nwarps);
        const uint32_t nxt = (lane + 1u) & 31u;
        const uint32_t lx = g.lx;
        const uint32_t xb = lane + 32u < lx ? lane + 32u : lane; /* this lane's site of half 1 */
        const uint32_t mb = lx == 64u ? 0xffffffffu : ((1u << (lx - 32u)) - 1u);
        const bool wrap_b = lane + 33u >= lx; /* half 1's +x partner is x = 0 */
        uint32_t* hx32 = reinterpret_cast<uint32_t*>(s.bx);
        uint32_t* hy32 = reinterpret_cast<uint32_t*>(s.by);
        uint32_t* hz32 = reinterpret_cast<uint32_t*>(s.bz);
        uint32_t zl = slsf_fastdiv_div(r_lo, g.div_ly), y = r_lo - zl * g.ly;
        uint32_t col = 0;
        float ra = 0.0f, rb = 0.0f;
        for (uint32_t row = r_lo; row < r_hi; ++row) {
            const float jx = s.jxy[g.z0 + zl], jzz = s.jz[g.z0 + zl];
            const uint32_t pbase = zl * g.plane;
            if (row == r_lo || y == 0) {
                /* colour of (x = lane, y, zl); x + 32 has the same colour */
                col = colour_of(g, lane, y, zl);
                ra = proj_of(s.th[col * g.tstride + ((pbase + y * lx + lane) >> 1)], cphi, sphi);
                rb = proj_of(s.th[col * g.tstride + ((pbase + y * lx + xb) >> 1)], cphi, sphi);
            }
            {
                const uint32_t li = pbase + y * lx + lane, lib = pbase + y * lx + xb;
                const uint32_t y1 = (y + 1 == g.ly) ? 0u : y + 1;
                const uint32_t ocol = col ^ 1u; /* colour of the +y and +z partners */
                const uint32_t li_y = pbase + y1 * lx + lane, lib_y = pbase + y1 * lx + xb;
                const bool top = zl + 1 == g.nz;
                /* +x partners: x + 1 in the same half, across the halves at x = 31 and x = L_x - 1 */
                const float b0 = __shfl_sync(0xffffffffu, rb, 0), a0 = __shfl_sync(0xffffffffu, ra, 0);
                const float na = __shfl_sync(0xffffffffu, ra, nxt), nb = __shfl_sync(0xffffffffu, rb, nxt);
                /* half 0: x = lane; each half is finished (bonds, ballots, 32-bit row-word half) in turn */
                const float rya = proj_of(s.th[ocol * g.tstride + (li_y >> 1)], cphi, sphi);
                {
                    const float tz = top ? halo_theta(g, s, true, ocol, (lane + lx * y) >> 1)
                                         : s.th[ocol * g.tstride + ((li + g.plane) >> 1)];
                    const float rz = proj_of(tz, cphi, sphi);
                    const slsf_u32x4 bw = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, base_idx + li);
                    const uint32_t bx = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ra, lane < 31u ? na : b0, m2b, bw.x));
                    const uint32_t by = __ballot_sync(0xffffffffu, wolff_bond_active(jx, ra, rya, m2b, bw.y));
                    const uint32_t bz = __ballot_sync(0xffffffffu, wolff_bond_active(jzz, ra, rz, m2b, bw.z));
                    if (lane == 0) {
                        hx32[2 * row] = bx;
                        hy32[2 * row] = by;
                        hz32[2 * row] = bz;
                    }
                }
                /* half 1: x = lane + 32 */
                const float ryb = proj_of(s.th[ocol * g.tstride + (lib_y >> 1)], cphi, sphi);
                {
                    const float tz = top ? halo_theta(g, s, true, ocol, (xb + lx * y) >> 1)
                                         : s.th[ocol * g.tstride + ((lib + g.plane) >> 1)];
                    const float rz = proj_of(tz, cphi, sphi);
                    const slsf_u32x4 bw = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, base_idx + lib);
                    const uint32_t bx = __ballot_sync(0xffffffffu, wolff_bond_active(jx, rb, wrap_b ? a0 : nb, m2b, bw.x));
                    const uint32_t by = __ballot_sync(0xffffffffu, wolff_bond_active(jx, rb, ryb, m2b, bw.y));
                    const uint32_t bz = __ballot_sync(0xffffffffu, wolff_bond_active(jzz, rb, rz, m2b, bw.z));
                    if (lane == 0) {
                        hx32[2 * row + 1] = bx & mb;
                        hy32[2 * row + 1] = by & mb;
                        hz32[2 * row + 1] = bz & mb;
                    }
                }
                ra = rya;
                rb = ryb;
                col = ocol;
            }
            if (++y == g.ly) {
                y = 0;
                ++zl;
            }
        }
      }
    }
    if (!walked)
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.vs; i0 += blockDim.x) {
        const uint32_t li = i0 + lane;
        const bool valid = li < g.vs;
        const uint32_t ll = valid ? li : 0;
        const Coords c = coords_of(g, ll);
        const uint32_t col = colour_of(g, c.x, c.y, c.zl), oth = (col ^ 1u) * g.tstride;
        const float ri = proj_of(s.th[col * g.tstride + (ll >> 1)], cphi, sphi);
        float rxp;
        if (g.lx_tiles_warp) {
            rxp = __shfl_sync(0xffffffffu, ri, seg_next(lane, g.lx));
        } else {
            /* the +x neighbour is the next lane unless the row or the warp ends */
            rxp = __shfl_down_sync(0xffffffffu, ri, 1);
            if (lane == 31 || c.x + 1 == g.lx) {
                const uint32_t xp = (c.x + 1 == g.lx) ? ll + 1 - g.lx : ll + 1;
                rxp = proj_of(s.th[oth + (xp >> 1)], cphi, sphi);
            }
        }
        const uint32_t yp = (c.y + 1 == g.ly) ? ll + g.lx - g.plane : ll + g.lx;
        const float ryp = proj_of(s.th[oth + (yp >> 1)], cphi, sphi);
        const float tz = (c.zl + 1 < g.nz) ? s.th[oth + ((ll + g.plane) >> 1)]
                                           : halo_theta(g, s, true, col ^ 1u, (c.x + g.lx * c.y) >> 1);
        const float rzp = proj_of(tz, cphi, sphi);
        const slsf_u32x4 b = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, base_idx + ll);
        const float jx = s.jxy[g.z0 + c.zl], jzz = s.jz[g.z0 + c.zl];
        const bool ax = valid && wolff_bond_active(jx, ri, rxp, m2b, b.x);
        const bool ay = valid && wolff_bond_active(jx, ri, ryp, m2b, b.y);
        const bool az = valid && wolff_bond_active(jzz, ri, rzp, m2b, b.z);
        if (ballots) {
            const uint32_t bal_x = __ballot_sync(0xffffffffu, ax);
            const uint32_t bal_y = __ballot_sync(0xffffffffu, ay);
            const uint32_t bal_z = __ballot_sync(0xffffffffu, az);
            /* L_x dividing 32 (rows of 32 < L_x <= 64 are walked above) */
            if (valid && c.x == 0) {
                const W m = (W)((g.lx >= 32) ? 0xffffffffu : ((1u << g.lx) - 1u));
                s.bx[c.row] = (W)(bal_x >> lane) & m;
                s.by[c.row] = (W)(bal_y >> lane) & m;
                s.bz[c.row] = (W)(bal_z >> lane) & m;
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
                const W px = (W)((bal_x >> lane) & m) << c.x;
                const W py = (W)((bal_y >> lane) & m) << c.x;
                const W pz = (W)((bal_z >> lane) & m) << c.x;
                if (px) atomic_or_row(&s.bx[c.row], px);
                if (py) atomic_or_row(&s.by[c.row], py);
                if (pz) atomic_or_row(&s.bz[c.row], pz);
            }
        }
    }
    /* seed the cluster */
    const uint32_t sx = seed_idx % g.lx, srow = seed_idx / g.lx;
    const uint32_t sz = srow / g.ly, sy = srow - sz * g.ly;
    const bool mine = sz >= g.z0 && sz < g.z0 + g.nz;
    const uint32_t seed_row = sy + g.ly * (sz - g.z0);
    for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) {
        s.cl[r] = (mine && r == seed_row) ? ((W)1 << sx) : (W)0;
        s.dirty[r] = 0;
    }
    __syncthreads();
    if (mine && threadIdx.x == 0) {
        const W mask = g.lx >= 8 * sizeof(W) ? ~(W)0 : (((W)1 << g.lx) - 1);
        s.cl[seed_row] = close_row<W>(s.cl[seed_row], s.bx[seed_row], g.lx, mask);
    }
}

constexpr uint32_t kZSeg = 4;    /* planes per column segment in growth stage Z */
constexpr uint32_t kZChain = 8;  /* slabs up to this many planes run stage Z as one chain per column */

/* Growth stage Z: every column of the slab (the rows of one y) carries its
 * cluster bits along z through its bz words, forward and backward, fed
 * across the slab faces by the partner rows (for a one-CTA cluster the
 * partner is this CTA: the periodic wrap).  A slab of up to kZChain planes
 * runs one chain per column; a deeper one is cut into segments of kZSeg
 * planes, one thread each (lanes over consecutive columns, so shared
 * accesses are conflict-free): each segment runs its chain with no carry in,
 * publishes its carry out and the product of its links, then runs again
 * from the carry that the segments before it deliver, stopping where the
 * carry adds nothing.  Changed rows are stored unclosed along x and marked
 * dirty.  Returns nonzero if any row changed. */
template <typename W>
__device__ __forceinline__ int grow_z(const Geo& g, Smem<W>& s, const Remote<W>& rm) {
    const uint32_t top = g.ly * (g.nz - 1);
    int changed = 0;
    if (g.nz <= kZChain) {
        /* A short slab: one thread runs its column's whole chain forward,
         * then backward, with no barrier inside the stage. */
        for (uint32_t y = threadIdx.x; y < g.ly; y += blockDim.x) {
            W acc = rm.cl_dn[top + y] & rm.bz_dn[top + y];
            for (uint32_t zl = 0; zl < g.nz; ++zl) {
                const uint32_t r = y + g.ly * zl;
                const W c = s.cl[r];
                const W v = c | acc;
                if (v != c) {
                    s.cl[r] = v;
                    s.dirty[r] = 1;
                    changed = 1;
                }
                acc = v & s.bz[r];
            }
            acc = rm.cl_up[y] & s.bz[top + y];
            for (uint32_t zl = g.nz; zl-- > 0;) {
                const uint32_t r = y + g.ly * zl;
                const W c = s.cl[r];
                const W v = c | acc;
                if (v != c) {
                    s.cl[r] = v;
                    s.dirty[r] = 1;
                    changed = 1;
                }
                acc = zl > 0 ? (v & s.bz[r - g.ly]) : (W)0;
            }
        }
        return changed;
    }
    const uint32_t nseg = (g.nz + kZSeg - 1) / kZSeg;
    const uint32_t n = nseg * g.ly;
    /* forward: plane zl feeds plane zl + 1 through bz[zl] */
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        const uint32_t j = slsf_fastdiv_div(t, g.div_ly), y = t - j * g.ly;
        const uint32_t z0 = j * kZSeg, z1 = min(z0 + kZSeg, g.nz);
        W acc = j == 0 ? (rm.cl_dn[top + y] & rm.bz_dn[top + y]) : (W)0, prod = ~(W)0;
        for (uint32_t zl = z0; zl < z1; ++zl) {
            const uint32_t r = y + g.ly * zl;
            const W c = s.cl[r], b = s.bz[r];
            const W v = c | acc;
            if (v != c) {
                s.cl[r] = v;
                s.dirty[r] = 1;
                changed = 1;
            }
            acc = v & b;
            prod &= b;
        }
        s.zc[t] = acc;
        s.zp[t] = prod;
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        const uint32_t j = slsf_fastdiv_div(t, g.div_ly), y = t - j * g.ly;
        if (j == 0) continue;
        W acc = s.zc[y];
        for (uint32_t q = 1; q < j; ++q) acc = (acc & s.zp[q * g.ly + y]) | s.zc[q * g.ly + y];
        const uint32_t z1 = min(j * kZSeg + kZSeg, g.nz);
        for (uint32_t zl = j * kZSeg; zl < z1 && acc; ++zl) {
            const uint32_t r = y + g.ly * zl;
            const W c = s.cl[r];
            const W v = c | acc;
            if (v == c) break; /* from here on the first run's chain stands */
            s.cl[r] = v;
            s.dirty[r] = 1;
            changed = 1;
            acc = v & s.bz[r];
        }
    }
    __syncthreads();
    /* backward: plane zl feeds plane zl - 1 through bz[zl - 1] */
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        const uint32_t j = slsf_fastdiv_div(t, g.div_ly), y = t - j * g.ly;
        const uint32_t z0 = j * kZSeg, z1 = min(z0 + kZSeg, g.nz);
        W acc = j == nseg - 1 ? (rm.cl_up[y] & s.bz[top + y]) : (W)0, prod = ~(W)0;
        for (uint32_t zl = z1; zl-- > z0;) {
            const uint32_t r = y + g.ly * zl;
            const W c = s.cl[r], b = zl > 0 ? s.bz[r - g.ly] : (W)0;
            const W v = c | acc;
            if (v != c) {
                s.cl[r] = v;
                s.dirty[r] = 1;
                changed = 1;
            }
            acc = v & b;
            prod &= b;
        }
        s.zc[t] = acc;
        s.zp[t] = prod;
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
        const uint32_t j = slsf_fastdiv_div(t, g.div_ly), y = t - j * g.ly;
        if (j == nseg - 1) continue;
        W acc = s.zc[(nseg - 1) * g.ly + y];
        for (uint32_t q = nseg - 2; q > j; --q) acc = (acc & s.zp[q * g.ly + y]) | s.zc[q * g.ly + y];
        const uint32_t z0 = j * kZSeg, z1 = min(z0 + kZSeg, g.nz);
        for (uint32_t zl = z1; zl-- > z0 && acc;) {
            const uint32_t r = y + g.ly * zl;
            const W c = s.cl[r];
            const W v = c | acc;
            if (v == c) break;
            s.cl[r] = v;
            s.dirty[r] = 1;
            changed = 1;
            acc = zl > 0 ? (v & s.bz[r - g.ly]) : (W)0;
        }
    }
    return changed;
}

/* Growth stage XY: one thread per row, warps over consecutive rows.  A row
 * takes the bits of its y neighbours through their by words, then each warp
 * closes its rows along x (a doubling scan in the row word) and along y (a
 * segmented Kogge-Stone scan, forward and backward over the lanes that hold
 * consecutive y of one plane), and along x again where the y scan added
 * bits.  A warp whose rows are all x-closed (none dirty from stage Z) and
 * gain nothing from their neighbours is skipped: its rows are closed along
 * x and along the y bonds inside the warp.  Returns nonzero if any row
 * changed. */
template <typename W>
__device__ __forceinline__ int grow_xy(const Geo& g, Smem<W>& s, W mask) {
    const uint32_t lane = threadIdx.x & 31u;
    int changed = 0;
    for (uint32_t r0 = threadIdx.x & ~31u; r0 < g.rows_s; r0 += blockDim.x) {
        const uint32_t r = r0 + lane;
        const bool valid = r < g.rows_s;
        const uint32_t rr = valid ? r : 0;
        const uint32_t zl = slsf_fastdiv_div(rr, g.div_ly);
        const uint32_t y = rr - zl * g.ly;
        const uint32_t r_yp = (y + 1 == g.ly) ? rr + 1 - g.ly : rr + 1;
        const uint32_t r_ym = (y == 0) ? rr + g.ly - 1 : rr - 1;
        const W old = s.cl[rr], by_r = s.by[rr];
        W c = old | (s.cl[r_ym] & s.by[r_ym]) | (s.cl[r_yp] & by_r);
        const bool is_dirty = valid && s.dirty[rr];
        if (__all_sync(0xffffffffu, !is_dirty && (!valid || c == old))) continue;
        if (is_dirty) s.dirty[rr] = 0;
        if (is_dirty || c != old) c = close_row<W>(c, s.bx[rr], g.lx, mask);
        /* forward: lane - 1 holds row rr - 1 of the same plane when y > 0 */
        W gsum = c;
        W link = (lane > 0 && y > 0) ? s.by[rr - 1] : (W)0;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const W up = __shfl_up_sync(0xffffffffu, gsum, d);
            const W lk = __shfl_up_sync(0xffffffffu, link, d);
            if (lane >= d) {
                gsum |= up & link;
                link &= lk;
            }
        }
        /* backward: lane + 1 holds row rr + 1 of the same plane */
        link = (lane < 31 && y + 1 < g.ly && rr + 1 < g.rows_s) ? by_r : (W)0;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const W dn = __shfl_down_sync(0xffffffffu, gsum, d);
            const W lk = __shfl_down_sync(0xffffffffu, link, d);
            if (lane + d < 32) {
                gsum |= dn & link;
                link &= lk;
            }
        }
        if (gsum != c) gsum = close_row<W>(gsum, s.bx[rr], g.lx, mask);
        if (valid && gsum != old) {
            s.cl[rr] = gsum;
            changed = 1;
        }
    }
    return changed;
}

/* One Wolff update (src/updates.rs:551-620); adds the cluster size to *count. */
template <typename W>
__device__ __forceinline__ void wolff_update(const TaskView& t, const Geo& g, Smem<W>& s, const Remote<W>& rm,
                                             cg::cluster_group& cluster, uint64_t counter, uint32_t* count,
                                             int* flags) {
    const slsf_u32x4 pick = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_PICK, 0, 0);
    const float phi = slsf_angle_from_word(pick.x);
    const uint32_t x0 = slsf_range(pick.y, g.lx), y0 = slsf_range(pick.z, g.ly), z0 = slsf_range(pick.w, g.lz);
    float sphi, cphi;
    __sincosf(phi, &sphi, &cphi);
    const W mask = g.lx >= 8 * sizeof(W) ? ~(W)0 : (((W)1 << g.lx) - 1);
    fill_halo(g, s, rm, 2);
    wolff_bonds(t, g, s, counter, cphi, sphi, x0 + g.lx * (y0 + g.ly * z0));
    cluster_barrier(g, cluster);
    SLSF_PHASE(2);

    /* Rounds of stage Z then stage XY until a round changes nothing in the
     * whole cluster; every round that goes on adds at least one site. */
    const uint32_t bound = t.loop_limit ? min(t.loop_limit, g.volume) : g.volume;
    uint32_t pass = 0;
    bool converged = false;
    for (; pass <= bound; ++pass) {
        int any = grow_z(g, s, rm);
        __syncthreads();
        any = __syncthreads_or(grow_xy(g, s, mask) | any);
        if (g.csize > 1) {
            /* lane q of warp 0 reads rank q's flag; one block barrier spreads the OR */
            if (threadIdx.x == 0) flags[pass & 1] = any;
            cluster.sync();
            const int mine = threadIdx.x < g.csize ? *cluster.map_shared_rank(&flags[pass & 1], threadIdx.x) : 0;
            any = __syncthreads_or(mine);
        }
        if (!any) {
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
    for (uint32_t r = threadIdx.x; r < g.rows_s; r += blockDim.x) members += RowOps<W>::popc(s.cl[r]);
    for (uint32_t li = threadIdx.x; li < g.vs; li += blockDim.x) {
        const Coords c = coords_of(g, li);
        if ((s.cl[c.row] >> c.x) & (W)1) {
            const uint32_t sl = colour_of(g, c.x, c.y, c.zl) * g.tstride + (li >> 1);
            s.th[sl] = slsf_reflect(s.th[sl], phi);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) members += __shfl_down_sync(0xffffffffu, members, off);
    if ((threadIdx.x & 31u) == 0 && members) atomicAdd(count, members);
    cluster_barrier(g, cluster);
    SLSF_PHASE(4);
}

/* ---- measurement ---- */

/* Slab sums of mx, my, cos xyz, sin xyz (src/observables.rs:99-141): FP64
 * sums of the FP32 bond terms, block total valid in thread 0.  The halo
 * holds both colours of the partner planes. */
template <typename W>
__device__ __forceinline__ void measure_slab(const Geo& g, const Smem<W>& s, double (&acc)[8], double* red) {
    const uint32_t lane = threadIdx.x & 31u;
    double f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i0 = (threadIdx.x & ~31u); i0 < g.vs; i0 += blockDim.x) {
        const uint32_t li = i0 + lane;
        const bool valid = li < g.vs;
        const uint32_t ll = valid ? li : 0;
        const Coords c = coords_of(g, ll);
        const uint32_t col = colour_of(g, c.x, c.y, c.zl), oth = (col ^ 1u) * g.tstride;
        float si, ci, sx, cx, sy, cy, sz, cz;
        __sincosf(s.th[col * g.tstride + (ll >> 1)], &si, &ci);
        if (g.lx_tiles_warp) {
            const uint32_t src = seg_next(lane, g.lx);
            sx = __shfl_sync(0xffffffffu, si, src);
            cx = __shfl_sync(0xffffffffu, ci, src);
        } else {
            const uint32_t xp = (c.x + 1 == g.lx) ? ll + 1 - g.lx : ll + 1;
            __sincosf(s.th[oth + (xp >> 1)], &sx, &cx);
        }
        const uint32_t yp = (c.y + 1 == g.ly) ? ll + g.lx - g.plane : ll + g.lx;
        __sincosf(s.th[oth + (yp >> 1)], &sy, &cy);
        const float tz = (c.zl + 1 < g.nz) ? s.th[oth + ((ll + g.plane) >> 1)]
                                           : halo_theta(g, s, true, col ^ 1u, (c.x + g.lx * c.y) >> 1);
        __sincosf(tz, &sz, &cz);
        if (!valid) continue;
        const float jx = s.jxy[g.z0 + c.zl], jzz = s.jz[g.z0 + c.zl];
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

/* Rank 0, thread 0: totals of the slab sums and their bin entry. */
__device__ __forceinline__ void bin_cluster_sums(const TaskView& t, const Geo& g, uint64_t done,
                                                 const double (*cred)[8], double* bin_acc, int64_t& bin_cur) {
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = 0; q < g.csize; ++q)
        for (int k = 0; k < 8; ++k) a[k] += cred[q][k];
    bin_measurement(t, g.volume, done, a, bin_acc, bin_cur);
}

template <typename W>
__global__ void __launch_bounds__(kBThreads, 1)
    k_cluster(const TaskView* __restrict__ views, uint32_t n, uint32_t n_sweeps, unsigned int* __restrict__ queue,
              Limits lim, unsigned long long* __restrict__ counters) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[8 * 32];
    __shared__ double cred[kMaxCluster][8]; /* slab sums gathered in rank 0 */
    __shared__ double bin_acc[kBinCols];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_cluster;
    __shared__ int s_flags[2];
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank(), csize = cluster.num_blocks();
    Smem<W> s = carve<W>(smem_raw, lim);
    Remote<W> rm;
    {
        const uint32_t up = (rank + 1) % csize, dn = (rank + csize - 1) % csize;
        rm.th_up = cluster.map_shared_rank(s.th, up);
        rm.th_dn = cluster.map_shared_rank(s.th, dn);
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
        TaskView t = views[item];
        if (counters) { /* a replayed launch: the counters live in their own array */
            t.metro_sweeps = counters[2 * item];
            t.wolff_done = counters[2 * item + 1];
        }
        const Geo g = make_geo(t, rank, csize);
        const uint32_t sweeps = t.sweeps ? t.sweeps : n_sweeps;
        if (threadIdx.x == 0) s_cluster = 0;
        load_slab(t, g, s);
        cluster.sync();
#ifdef SLSF_PHASE_TIMING
        if (threadIdx.x == 0) s_phase_mark = clock64();
#endif
        uint32_t accepted = 0;
        int64_t bin_cur = -1;
        /* ThetaModel::measure after every sweep past thermalization: the state
         * after sweep k is measured inside sweep k+1's colour-0 half-sweep,
         * the launch's last state by the measurement pass below; each CTA
         * sends its slab sums to rank 0, which bins them. */
        const bool measuring = t.n_bins > 0;
        for (uint32_t sw = 0; sw < sweeps; ++sw) {
            const uint64_t sweep = t.metro_sweeps + sw;
            const bool meas = measuring && sw > 0 && sweep > t.thermalization;
            double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            fill_halo(g, s, rm, 1);
            if (meas) {
                accepted += half_sweep<true>(t, g, s, sweep, 0, acc);
                double tot[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) tot[k] = acc[k];
                block_sum<8>(tot, red);
                if (threadIdx.x == 0)
                    for (int k = 0; k < 8; ++k) *cluster.map_shared_rank(&cred[rank][k], 0) = tot[k];
            } else {
                accepted += half_sweep<false>(t, g, s, sweep, 0, acc);
            }
            cluster_barrier(g, cluster);
            SLSF_PHASE(0);
            /* cred is written again only after two more cluster barriers */
            if (meas && rank == 0 && threadIdx.x == 0) bin_cluster_sums(t, g, sweep, cred, bin_acc, bin_cur);
            fill_halo(g, s, rm, 0);
            accepted += half_sweep<false>(t, g, s, sweep, 1, acc);
            cluster_barrier(g, cluster);
            SLSF_PHASE(1);
            for (uint32_t k = 0; k < t.wolff_steps; ++k)
                wolff_update(t, g, s, rm, cluster, t.wolff_done + (uint64_t)sw * t.wolff_steps + k, &s_cluster,
                             s_flags);
        }
        const uint64_t last = t.metro_sweeps + sweeps;
        /* the counters advance on the device, so that a replayed launch
         * (slsf_batch_open / slsf_batch_step) continues the streams; every
         * CTA of the cluster read them before the first barrier of the item */
        if (counters && rank == 0 && threadIdx.x == 0) {
            counters[2 * item] = last;
            counters[2 * item + 1] = t.wolff_done + (uint64_t)sweeps * t.wolff_steps;
        }
        if (measuring && sweeps > 0 && last > t.thermalization) {
            double acc[8];
            fill_halo(g, s, rm, 2);
            measure_slab(g, s, acc, red);
            if (threadIdx.x == 0)
                for (int k = 0; k < 8; ++k) *cluster.map_shared_rank(&cred[rank][k], 0) = acc[k];
            cluster_barrier(g, cluster);
            SLSF_PHASE(5);
            if (rank == 0 && threadIdx.x == 0) bin_cluster_sums(t, g, last, cred, bin_acc, bin_cur);
        }
        if (rank == 0 && threadIdx.x == 0) flush_bin(t, bin_acc, bin_cur);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) accepted += __shfl_down_sync(0xffffffffu, accepted, off);
        if ((threadIdx.x & 31u) == 0 && accepted) atomicAdd(&t.stats[kStatAccepted], (unsigned long long)accepted);
        store_slab(t, g, s);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_cluster) atomicAdd(&t.stats[kStatClusterSites], (unsigned long long)s_cluster);
            if (rank == 0) atomicAdd(&t.stats[kStatClusters], (unsigned long long)sweeps * t.wolff_steps);
        }
        /* no CTA may start the next replica while a partner still reads its slab */
        cluster.sync();
    }
}

size_t smem_bytes(const Limits& m, size_t word) {
    return 6ull * m.rows * word + 4ull * (m.vs + 2 * kPad) + 16ull * m.hp + 8ull * m.lz + m.rows;
}

int max_dynamic_smem(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    /* leave room for the kernel's static shared arrays */
    return v - 4096;
}

template <typename W>
cudaError_t launch_w(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                     cudaStream_t s, uint32_t cluster, uint32_t threads, const Limits& lim,
                     unsigned long long* counters) {
    const size_t smem = smem_bytes(lim, sizeof(W));
    cudaError_t e = cudaFuncSetAttribute(k_cluster<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(k_cluster<W>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cluster, 1, 1);
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, k_cluster<W>, &cfg);
    if (e != cudaSuccess) return e;
    if (clusters < 1) return cudaErrorInvalidConfiguration;
    const uint32_t grid_clusters = std::min<uint32_t>(n, (uint32_t)clusters);
    cfg.gridDim = dim3(grid_clusters * cluster, 1, 1);
    return cudaLaunchKernelEx(&cfg, k_cluster<W>, views_dev, n, n_sweeps, queue, lim, counters);
}

}  // namespace

bool cluster_feasible(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t c, int device) {
    /* Row words hold L_x <= 64 bits; the colour-split layout needs even
     * dimensions (L_x = 2 mod 4 copies the state site by site). */
    if (lx > kMaxRowBits || lx < 4 || lx % 2 || ly < 2 || ly % 2 || lz < 2 || lz % 2) return false;
    if (c < 1 || c > kMaxCluster || (c & (c - 1)) || lz % c) return false;
    const size_t word = lx > 32 ? 8 : 4;
    const uint32_t nz = lz / c;
    const Limits m = {lx * ly * nz, ly * nz, lz, (lx * ly) / 2};
    return smem_bytes(m, word) <= (size_t)max_dynamic_smem(device);
}

uint32_t batched_cluster_size(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    for (uint32_t c = 1; c <= 8; c <<= 1)
        if (cluster_feasible(lx, ly, lz, c, device)) return c;
    return 0;
}

bool batched_supports(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    return batched_cluster_size(lx, ly, lz, device) != 0;
}

cudaError_t launch_batched(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                           int device, cudaStream_t s, uint32_t cluster, uint32_t threads, uint32_t max_vs,
                           uint32_t max_rows, uint32_t max_lz, uint32_t max_plane, uint32_t max_lx,
                           unsigned long long* counters) {
    (void)device;
    if (threads < 64 || threads > (uint32_t)kBThreads || threads % 32) return cudaErrorInvalidConfiguration;
    const Limits lim = {max_vs, max_rows, max_lz, max_plane / 2};
    if (max_lx > 32) return launch_w<uint64_t>(views_dev, n, n_sweeps, queue, s, cluster, threads, lim, counters);
    return launch_w<uint32_t>(views_dev, n, n_sweeps, queue, s, cluster, threads, lim, counters);
}

}  // namespace slsf

#ifdef SLSF_PHASE_TIMING
extern "C" int slsf_debug_phase_cycles(unsigned long long out[8], int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out, slsf::g_cl_phase_cycles, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess && reset) {
        const unsigned long long zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        e = cudaMemcpyToSymbol(slsf::g_cl_phase_cycles, zero, sizeof(zero));
    }
    return e == cudaSuccess ? 0 : 1;
}
#endif
