/*
 * Single-task Wolff update on bit-packed bonds: grows the seed's cluster
 * only, for lattices whose three sides are multiples of 32 (the large
 * single-replica lattices: L = 64 ... 256 and more).
 *
 * Replaces, for those shapes, the whole-lattice union-find labelling of
 * kernels_plain.cu.  The reference grows one cluster from a random seed by
 * depth-first search (wolff_cluster_step_with_theta_scratch,
 * src/updates.rs:551-620); with one counter-based random per bond, that
 * cluster is the seed's connected component over the active bonds, and only
 * it is needed.
 *
 *   k_wb_bonds   per-site +x/+y/+z bond activation (try_add_wolff_neighbor,
 *                src/updates.rs:537-548) into three bit planes: bit i of the
 *                flat bitmap is site i (site index x + Lx (y + Ly z), so a
 *                32-bit word is 32 consecutive sites of one row); clears the
 *                cluster bitmap and queues the seed's region, whose first
 *                processing adds the seed's bit.
 *   k_wb_grow    the cluster over the active bonds.  The lattice is cut into
 *                regions of 32 x 32 x 32 sites (one word wide, 32 rows, 32
 *                planes).  A CTA takes a region from a work queue, reads its
 *                cluster and bond words into shared memory with the bits that
 *                enter through the region's faces, closes the region in
 *                passes (each pass a full warp scan along y -- lane = y -- or
 *                along z -- lane = z, the shared array read transposed --
 *                one step along the other axis, and the closure along x
 *                inside each word), ORs the result back and queues every
 *                neighbour region its bits can enter.  Regions are processed
 *                as they are queued, with no grid-wide barrier: CTAs only
 *                wait for work that running CTAs hold, so the kernel needs
 *                no co-residency.  Bits only ever get set, so the fixed point
 *                is the seed's component whatever the order.
 *   k_wb_flip    reflection of the cluster's sites (src/updates.rs:602-617)
 *                and its size.
 *
 * Every wait and loop is bounded; past a bound the kernel sets
 * kErrGrowthLimit in the task's error word and returns.
 */
#include <algorithm>

#include "bitgrow.cuh"
#include "engine.h"
#include "xy_device.cuh"

namespace slsf {

namespace {

constexpr uint32_t kRegion = kGrowEdge; /* region edge in sites along y and z; one word along x */
constexpr uint32_t kGrowThreads = kRegion * kRegion;
constexpr int kBondThreads = 256;
constexpr int kFlipThreads = 256;
constexpr uint32_t kEmpty = 0;
constexpr uint32_t kNoRegion = 0xffffffffu;

/* Optional counters (build with -DSLSF_WB_STATS): regions processed, growth
 * passes, grow launches, and region loads that changed nothing. */
#ifdef SLSF_WB_STATS
/* [0] regions processed, [1] passes, [2] grow launches, [3] loads without new
 * bits, [4..7] cycles of thread 0 in: waiting for work, loading, closing,
 * writing back and queueing neighbours */
__device__ unsigned long long g_wb_stats[8];
#define SLSF_WB_CLOCK(k, t0)                                                                     \
    do {                                                                                         \
        if (threadIdx.x == 0) {                                                                  \
            const long long t1_ = clock64();                                                     \
            atomicAdd(&g_wb_stats[k], (unsigned long long)(t1_ - (t0)));                         \
            (t0) = t1_;                                                                          \
        }                                                                                        \
    } while (0)
#define SLSF_WB_COUNT(k, n)                                                          \
    do {                                                                             \
        if (threadIdx.x == 0) atomicAdd(&g_wb_stats[k], (unsigned long long)(n));    \
    } while (0)
#else
#define SLSF_WB_COUNT(k, n) \
    do {                    \
    } while (0)
#define SLSF_WB_CLOCK(k, t0) \
    do {                     \
    } while (0)
#endif

/* Scratch of one update, carved from the task's union-find array. */
struct WolffBits {
    uint32_t* bx;      /* bond bit planes, one bit per site */
    uint32_t* by;
    uint32_t* bz;
    uint32_t* cl;      /* cluster bitmap */
    uint32_t* queued;  /* [regions] 1 while the region is in the queue */
    uint32_t* ring;    /* [cap] region + 1, or 0 */
    uint32_t* ctl;     /* head, tail, pending (queued or in flight), abort, seed site + 1 */
    uint32_t regions, cap;
};

__host__ __device__ inline uint64_t round256(uint64_t b) { return (b + 255) & ~255ull; }

__device__ __forceinline__ float proj_at(const float* __restrict__ theta, uint32_t i, float cphi, float sphi) {
    float sn, cn;
    __sincosf(theta[i], &sn, &cn);
    return wolff_projection(cn, sn, cphi, sphi);
}

/* Bond activation.  A warp owns word k of plane z for a run of rows y
 * (lane = bit = x - 32 k) and walks it along y, so the projection of the +y
 * row is the next row's own: two sincos per site.  The seed word gets its
 * bit; the seed's region is queued. */
__global__ void __launch_bounds__(kBondThreads)
    k_wb_bonds(const float* __restrict__ theta, const float* __restrict__ jxy, const float* __restrict__ jz,
               uint32_t lx, uint32_t ly, uint32_t lz, float minus_two_beta, float phi, uint64_t seed,
               uint64_t counter, WolffBits wb, uint32_t seed_idx, uint32_t seg, uint8_t* __restrict__ bond_bytes) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t words = lx >> 5, nseg = ly / seg;
    const uint32_t k = wid % words, rest = wid / words;
    const uint32_t sg = rest % nseg, z = rest / nseg;
    if (z >= lz) return; /* whole warps */
    float sphi, cphi;
    __sincosf(phi, &sphi, &cphi);
    const uint32_t plane = lx * ly;
    const uint32_t x = 32u * k + lane;
    const uint32_t xn = (k + 1 == words) ? 0u : 32u * (k + 1); /* first site of the next word, periodic */
    const uint32_t zbase = z * plane, zp_base = (z + 1 == lz) ? 0u : (z + 1) * plane;
    const float jx = jxy[z], jzz = jz[z];
    const uint32_t y0 = sg * seg;
    float ri = proj_at(theta, zbase + y0 * lx + x, cphi, sphi);
    /* lane j < seg (seg <= 32): the projection of the first site of the next
     * word in row y0 + j, the +x partner of lane 31 in that row */
    const float r_next_word = proj_at(theta, zbase + (y0 + (lane < seg ? lane : 0u)) * lx + xn, cphi, sphi);
    /* the angles of the next row's loads, one row ahead */
    auto yrow = [&](uint32_t y) { return (y + 1 == ly) ? 0u : y + 1; };
    float t_yp = theta[zbase + yrow(y0) * lx + x], t_zp = theta[zp_base + y0 * lx + x];
    for (uint32_t y = y0; y < y0 + seg; ++y) {
        const uint32_t row = zbase + y * lx;
        const uint32_t i = row + x;
        const float a_yp = t_yp, a_zp = t_zp;
        if (y + 1 < y0 + seg) {
            t_yp = theta[zbase + yrow(y + 1) * lx + x];
            t_zp = theta[zp_base + (y + 1) * lx + x];
        }
        float sn, cn;
        __sincosf(a_yp, &sn, &cn);
        const float ryp = wolff_projection(cn, sn, cphi, sphi);
        __sincosf(a_zp, &sn, &cn);
        const float rzp = wolff_projection(cn, sn, cphi, sphi);
        const float rnext = __shfl_sync(0xffffffffu, r_next_word, y - y0);
        float rxp = __shfl_sync(0xffffffffu, ri, (lane + 1u) & 31u);
        if (lane == 31) rxp = rnext;
        const slsf_u32x4 b = slsf_stream(seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, i);
        const bool ax = wolff_bond_active(jx, ri, rxp, minus_two_beta, b.x);
        const bool ay = wolff_bond_active(jx, ri, ryp, minus_two_beta, b.y);
        const bool az = wolff_bond_active(jzz, ri, rzp, minus_two_beta, b.z);
        const uint32_t wx = __ballot_sync(0xffffffffu, ax);
        const uint32_t wy = __ballot_sync(0xffffffffu, ay);
        const uint32_t wz = __ballot_sync(0xffffffffu, az);
        const uint32_t w = i >> 5;
        if (lane == 0) wb.bx[w] = wx;
        if (lane == 1) wb.by[w] = wy;
        if (lane == 2) wb.bz[w] = wz;
        if (lane == 3) wb.cl[w] = 0u;
        if (bond_bytes) bond_bytes[i] = (uint8_t)((ax ? 1u : 0u) | (ay ? 2u : 0u) | (az ? 4u : 0u));
        ri = ryp;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        /* the seed's region is the first queue entry (the scratch was zeroed) */
        const uint32_t sx = seed_idx % lx, srow = seed_idx / lx, sy = srow % ly, sz = srow / ly;
        const uint32_t r = (sx >> 5) + words * ((sy / kRegion) + (ly / kRegion) * (sz / kRegion));
        wb.queued[r] = 1;
        wb.ring[0] = r + 1;
        wb.ctl[1] = 1; /* tail */
        wb.ctl[2] = 1; /* pending */
        wb.ctl[4] = seed_idx + 1; /* the seed's bit enters its region like a face bit */
    }
}

struct GrowGeo {
    uint32_t lx, ly, lz, words, ry_n, rz_n;
    bool px, py, pz; /* the region spans the whole period along x (one-word rows), y, z */
};

/* Claims region r for processing unless it is claimed already (queued or
 * kept): the first neighbour a CTA claims it keeps in *keep and processes
 * next itself, the others go to the queue. */
__device__ __forceinline__ void push_region(const WolffBits& wb, uint32_t r, uint32_t* keep) {
    if (atomicExch(&wb.queued[r], 1u) != 0u) return;
    atomicAdd(&wb.ctl[2], 1u); /* pending before the region can be taken */
    if (atomicCAS(keep, kNoRegion, r) == kNoRegion) return;
    const uint32_t slot = atomicAdd(&wb.ctl[1], 1u);
    __threadfence();
    atomicExch(&wb.ring[slot & (wb.cap - 1)], r + 1);
}

__device__ __forceinline__ uint32_t region_of(const GrowGeo& g, uint32_t k, uint32_t ry, uint32_t rz) {
    return k + g.words * (ry + g.ry_n * rz);
}

/* One region: load with the bits entering through its faces, close in
 * shared memory, OR back, queue the neighbours its bits can enter.  Returns
 * false if a pass bound was hit. */
__device__ bool grow_region(const WolffBits& wb, const GrowGeo& g, uint32_t r, uint32_t seed_site,
                            uint32_t (*C)[kRegion + 1], uint32_t (*BY)[kRegion + 1], uint32_t (*BZ)[kRegion + 1],
                            uint32_t (*BX)[kRegion + 1], uint32_t* keep, uint32_t* s_want) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t k = r % g.words, rest = r / g.words, ry = rest % g.ry_n, rz = rest / g.ry_n;
    const uint32_t rowlen = g.words; /* words per row */
    const uint32_t gy = ry * kRegion + lane, gz = rz * kRegion + warp;
    auto word = [&](uint32_t kk, uint32_t yy, uint32_t zz) { return kk + rowlen * (yy + g.ly * zz); };
#ifdef SLSF_WB_STATS
    long long tclk = clock64();
#endif
    const uint32_t w = word(k, gy, gz);
    /* the region's own words (written only by processings of this region) */
    const uint32_t c0 = __ldcg(&wb.cl[w]);
    const uint32_t bxw = wb.bx[w], byw = wb.by[w], bzw = wb.bz[w];
    /* claimable again from here on: the reset is visible before the
     * neighbours' words are read, so a neighbour that adds face bits later
     * finds the region unqueued and queues it */
    if (threadIdx.x == 0) {
        wb.queued[r] = 0u;
        __threadfence();
    }
    __syncthreads();
    uint32_t c = c0;
    /* bits entering through the faces */
    const uint32_t kl = k == 0 ? g.words - 1 : k - 1, kr = k + 1 == g.words ? 0 : k + 1;
    const uint32_t ym = gy == 0 ? g.ly - 1 : gy - 1, yp = gy + 1 == g.ly ? 0 : gy + 1;
    const uint32_t zm = gz == 0 ? g.lz - 1 : gz - 1, zp = gz + 1 == g.lz ? 0 : gz + 1;
    /* the faces' neighbour words as loaded here also decide, at the end,
     * which neighbours to queue: a neighbour word only ever gains bits, so a
     * stale copy can queue a region that needs nothing, never miss one */
    uint32_t cl_l = ~0u, bx_l = 0, cl_r = ~0u, cl_ym = ~0u, by_ym = 0, cl_yp = ~0u, cl_zm = ~0u, bz_zm = 0, cl_zp = ~0u;
    if (!g.px) {
        const uint32_t wl = word(kl, gy, gz), wr = word(kr, gy, gz);
        cl_l = __ldcg(&wb.cl[wl]);
        bx_l = wb.bx[wl];
        cl_r = __ldcg(&wb.cl[wr]);
        c |= (cl_l >> 31) & (bx_l >> 31);
        c |= ((cl_r & 1u) & (bxw >> 31)) << 31;
    }
    if (!g.py) {
        if (lane == 0) {
            const uint32_t wm = word(k, ym, gz);
            cl_ym = __ldcg(&wb.cl[wm]);
            by_ym = wb.by[wm];
            c |= cl_ym & by_ym;
        }
        if (lane == kRegion - 1) {
            cl_yp = __ldcg(&wb.cl[word(k, yp, gz)]);
            c |= cl_yp & byw;
        }
    }
    if (!g.pz) {
        if (warp == 0) {
            const uint32_t wm = word(k, gy, zm);
            cl_zm = __ldcg(&wb.cl[wm]);
            bz_zm = wb.bz[wm];
            c |= cl_zm & bz_zm;
        }
        if (warp == kRegion - 1) {
            cl_zp = __ldcg(&wb.cl[word(k, gy, zp)]);
            c |= cl_zp & bzw;
        }
    }
    if (w == seed_site >> 5) c |= 1u << (seed_site & 31u);
    c = close_word(c, bxw, g.px);
    /* the stored region is closed already: without new bits nothing changes */
    const int any_new = __syncthreads_or(c != c0);
    SLSF_WB_CLOCK(5, tclk);
    if (!any_new) {
        SLSF_WB_COUNT(3, 1);
        return true;
    }
    C[warp][lane] = c;
    BX[warp][lane] = bxw;
    BY[warp][lane] = byw;
    BZ[warp][lane] = bzw;
    __syncthreads();
    const uint32_t passes = close_block(C, BY, BZ, BX, g.px, g.py, g.pz);
    SLSF_WB_COUNT(1, passes);
    SLSF_WB_CLOCK(6, tclk);
    const bool ok = passes != 0;
    c = C[warp][lane];
    if (c != c0) atomicOr(&wb.cl[w], c);
    /* neighbours that the region's bits can enter: bit 0/1 -x/+x, 2/3 -y/+y, 4/5 -z/+z */
    uint32_t want = 0;
    if (!g.px) {
        if ((c & 1u) && (bx_l >> 31) && !(cl_l >> 31)) want |= 1u;
        if ((c >> 31) && (bxw >> 31) && !(cl_r & 1u)) want |= 2u;
    }
    if (!g.py) {
        if (lane == 0 && (c & by_ym & ~cl_ym)) want |= 4u;
        if (lane == kRegion - 1 && (c & byw & ~cl_yp)) want |= 8u;
    }
    if (!g.pz) {
        if (warp == 0 && (c & bz_zm & ~cl_zm)) want |= 16u;
        if (warp == kRegion - 1 && (c & bzw & ~cl_zp)) want |= 32u;
    }
    want = __reduce_or_sync(0xffffffffu, want);
    if (lane == 0 && want) atomicOr(s_want, want);
    __syncthreads();
    /* thread d queues the neighbour in direction d, so that the six queue
     * operations (each a few dependent atomics) overlap; the block's cluster
     * words are written (barrier above) and each pushing thread's fence
     * orders them before its neighbour can be taken */
    const uint32_t m = *s_want;
    if (threadIdx.x < 6 && ((m >> threadIdx.x) & 1u)) {
        uint32_t nb;
        switch (threadIdx.x) {
            case 0: nb = region_of(g, k == 0 ? g.words - 1 : k - 1, ry, rz); break;
            case 1: nb = region_of(g, k + 1 == g.words ? 0 : k + 1, ry, rz); break;
            case 2: nb = region_of(g, k, ry == 0 ? g.ry_n - 1 : ry - 1, rz); break;
            case 3: nb = region_of(g, k, ry + 1 == g.ry_n ? 0 : ry + 1, rz); break;
            case 4: nb = region_of(g, k, ry, rz == 0 ? g.rz_n - 1 : rz - 1); break;
            default: nb = region_of(g, k, ry, rz + 1 == g.rz_n ? 0 : rz + 1); break;
        }
        __threadfence();
        push_region(wb, nb, keep);
    }
    __syncthreads(); /* every thread has read the mask before it is cleared */
    if (threadIdx.x == 0) *s_want = 0;
    return ok;
}

__global__ void __launch_bounds__(kGrowThreads, 1)
    k_wb_grow(WolffBits wb, GrowGeo g, uint32_t max_items, unsigned long long* __restrict__ stats) {
    __shared__ uint32_t C[kRegion][kRegion + 1];
    __shared__ uint32_t BY[kRegion][kRegion + 1];
    __shared__ uint32_t BZ[kRegion][kRegion + 1];
    __shared__ uint32_t BX[kRegion][kRegion + 1];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_keep;
    __shared__ uint32_t s_want;
    /* Each CTA takes regions until nothing is queued or in flight: the
     * neighbour it claimed while processing the last one (no queue round
     * trip), else the queue entry of its ticket (one atomic; the producer
     * may not have filled it yet, the CTA waits for it, bounded).  A ticket
     * whose entry never comes is given up when nothing is pending. */
    constexpr uint32_t kSpin = 1u << 24;
    const uint32_t seed_site = __ldcg(&wb.ctl[4]) - 1;
    bool ok = true;
    if (threadIdx.x == 0) {
        s_keep = kNoRegion;
        s_want = 0;
    }
    __syncthreads();
#ifdef SLSF_WB_STATS
    long long tq = clock64();
#endif
    for (uint32_t item = 0; item < max_items; ++item) {
        if (threadIdx.x == 0) {
#ifdef SLSF_WB_STATS
            tq = clock64();
#endif
            uint32_t got = s_keep;
            if (got == kNoRegion) {
                got = 0xfffffffeu; /* gave up, unless set below */
                const uint32_t ticket = atomicAdd(&wb.ctl[0], 1u);
                volatile uint32_t* slot = &wb.ring[ticket & (wb.cap - 1)];
                volatile uint32_t* ctl = wb.ctl;
                for (uint32_t spin = 0; spin < kSpin; ++spin) {
                    const uint32_t v = *slot;
                    if (v != kEmpty) {
                        *slot = kEmpty;
                        got = v - 1;
                        break;
                    }
                    if (ctl[2] == 0 || ctl[3] != 0) { /* nothing queued or in flight, or aborted */
                        got = 0xffffffffu;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            s_keep = kNoRegion;
            s_item = got;
        }
        __syncthreads();
        SLSF_WB_CLOCK(4, tq);
        const uint32_t r = s_item;
        if (r == 0xffffffffu) break;
        if (r >= wb.regions) {
            ok = false;
            break;
        }
        ok &= grow_region(wb, g, r, seed_site, C, BY, BZ, BX, &s_keep, &s_want);
        SLSF_WB_COUNT(0, 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicSub(&wb.ctl[2], 1u);
        }
        SLSF_WB_CLOCK(7, tq);
        if (item + 1 == max_items) ok = false;
    }
    if (!ok && threadIdx.x == 0) {
        atomicOr(&stats[kStatError], kErrGrowthLimit);
        atomicExch(&wb.ctl[3], 1u); /* the other CTAs stop at their next pop */
    }
}

/* Reflect the cluster's sites, count them; optional byte mask. */
__global__ void __launch_bounds__(kFlipThreads)
    k_wb_flip(float* __restrict__ theta, uint32_t volume, const uint32_t* __restrict__ cl, float phi,
              unsigned long long* __restrict__ stats, uint8_t* __restrict__ cluster_out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; /* four sites */
    uint32_t n = 0;
    if (4ull * q < volume) {
        const uint32_t i = 4 * q;
        const uint32_t m = (__ldcg(&cl[i >> 5]) >> (i & 31u)) & 0xfu;
        if (m) {
            float4 v = reinterpret_cast<float4*>(theta)[q];
            if (m & 1u) v.x = slsf_reflect(v.x, phi);
            if (m & 2u) v.y = slsf_reflect(v.y, phi);
            if (m & 4u) v.z = slsf_reflect(v.z, phi);
            if (m & 8u) v.w = slsf_reflect(v.w, phi);
            reinterpret_cast<float4*>(theta)[q] = v;
        }
        n = __popc(m);
        if (cluster_out) {
            uchar4 o = make_uchar4(m & 1u, (m >> 1) & 1u, (m >> 2) & 1u, (m >> 3) & 1u);
            reinterpret_cast<uchar4*>(cluster_out)[q] = o;
        }
    }
    __shared__ unsigned int s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) n += __shfl_down_sync(0xffffffffu, n, off);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(&s_sum, n);
    __syncthreads();
    if (threadIdx.x == 0 && s_sum) atomicAdd(&stats[kStatClusterSites], (unsigned long long)s_sum);
}

uint32_t pow2_at_least(uint32_t n) {
    uint32_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

}  // namespace

bool wolff_bits_supports(uint32_t lx, uint32_t ly, uint32_t lz) {
    return lx % 32 == 0 && ly % kRegion == 0 && lz % kRegion == 0 && lx > 0 && ly > 0 && lz > 0 &&
           (uint64_t)lx * ly * lz < (1ull << 31);
}

uint64_t wolff_bits_scratch_bytes(uint32_t lx, uint32_t ly, uint32_t lz) {
    const uint64_t words = (uint64_t)lx * ly * lz / 32;
    const uint64_t regions = words / (kRegion * kRegion);
    const uint64_t cap = pow2_at_least((uint32_t)(2 * regions + 2));
    return 4 * round256(4 * words) + round256(4 * regions) + round256(4 * cap) + 256;
}

int launch_wolff_bits(const TaskView& t, uint64_t counter, void* scratch, uint8_t* bond_bytes, uint8_t* cluster_out,
                      cudaStream_t s, float* phi_out, uint32_t seed_site[3]) {
    /* The reflection axis and seed site (src/updates.rs:564-568) from the
     * WOLFF_PICK block, computed on the host from the shared header. */
    const slsf_u32x4 pick = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_PICK, 0, 0);
    const float phi = slsf_angle_from_word(pick.x);
    const uint32_t x0 = slsf_range(pick.y, t.lx), y0 = slsf_range(pick.z, t.ly), z0 = slsf_range(pick.w, t.lz);
    const uint32_t volume = t.lx * t.ly * t.lz;
    const uint32_t seed_idx = x0 + t.lx * (y0 + t.ly * z0);
    const uint64_t words = volume / 32;
    WolffBits wb;
    unsigned char* p = static_cast<unsigned char*>(scratch);
    wb.bx = reinterpret_cast<uint32_t*>(p);
    p += round256(4 * words);
    wb.by = reinterpret_cast<uint32_t*>(p);
    p += round256(4 * words);
    wb.bz = reinterpret_cast<uint32_t*>(p);
    p += round256(4 * words);
    wb.cl = reinterpret_cast<uint32_t*>(p);
    p += round256(4 * words);
    wb.regions = (uint32_t)(words / (kRegion * kRegion));
    wb.cap = pow2_at_least(2 * wb.regions + 2);
    unsigned char* control = p;
    wb.queued = reinterpret_cast<uint32_t*>(p);
    p += round256(4ull * wb.regions);
    wb.ring = reinterpret_cast<uint32_t*>(p);
    p += round256(4ull * wb.cap);
    wb.ctl = reinterpret_cast<uint32_t*>(p);
    p += 256;
    cudaMemsetAsync(control, 0, (size_t)(p - control), s);
    /* bond kernel: warps walk runs of `seg` rows */
    const uint32_t seg = 16; /* L_y is a multiple of 32 */
    const uint64_t warps = (uint64_t)(t.lx / 32) * (t.ly / seg) * t.lz;
    const uint32_t bond_blocks = (uint32_t)((warps * 32 + kBondThreads - 1) / kBondThreads);
    k_wb_bonds<<<bond_blocks, kBondThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, -2.0f * t.beta, phi,
                                                    t.seed, counter, wb, seed_idx, seg, bond_bytes);
    GrowGeo g;
    g.lx = t.lx;
    g.ly = t.ly;
    g.lz = t.lz;
    g.words = t.lx / 32;
    g.ry_n = t.ly / kRegion;
    g.rz_n = t.lz / kRegion;
    g.px = g.words == 1;
    g.py = g.ry_n == 1;
    g.pz = g.rz_n == 1;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const uint32_t grid = std::min<uint32_t>(wb.regions, (uint32_t)sms);
    /* every region is processed at most once per bit it gains */
    const uint32_t max_items = t.loop_limit ? t.loop_limit : std::max<uint32_t>(64, volume / 32);
    k_wb_grow<<<grid, kGrowThreads, 0, s>>>(wb, g, max_items, t.stats);
    const uint32_t quads = volume / 4;
    k_wb_flip<<<(quads + kFlipThreads - 1) / kFlipThreads, kFlipThreads, 0, s>>>(t.theta, volume, wb.cl, phi,
                                                                                 t.stats, cluster_out);
    if (phi_out) *phi_out = phi;
    if (seed_site) {
        seed_site[0] = x0;
        seed_site[1] = y0;
        seed_site[2] = z0;
    }
    return 3;
}

}  // namespace slsf

#ifdef SLSF_WB_STATS
extern "C" int slsf_debug_wb_stats(unsigned long long out[8], int reset) {
    cudaError_t e = cudaMemcpyFromSymbol(out, slsf::g_wb_stats, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess && reset) {
        const unsigned long long zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        e = cudaMemcpyToSymbol(slsf::g_wb_stats, zero, sizeof(zero));
    }
    return e == cudaSuccess ? 0 : 1;
}
#endif
