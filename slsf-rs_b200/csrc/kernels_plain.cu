/*
 * Single-task kernels: the plain GPU path behind slsf_task_*.
 *
 *   k_init_random        ThetaModel::init (src/model.rs:373-377)
 *   k_metro_colour       one colour of metropolis_sweep_with_scratch
 *                        (src/updates.rs:440-486), one thread per Philox block
 *                        (two same-colour sites)
 *   k_metro_colour0_measure  colour 0 fused with the measurement of the state
 *                        it starts from (the batched grid path)
 *   k_wolff_tiles        per-site +x/+y/+z bond activation of
 *   k_wolff_boundary     wolff_cluster_step_with_theta_scratch
 *   k_wolff_compress     (src/updates.rs:551-620): components inside
 *   k_wolff_flip         32x8x4 tiles by union-find in shared memory, the
 *                        bonds between tiles by a lock-free global
 *                        union-find over the tile roots, the tile roots
 *                        pointed at their component's root, then reflect
 *                        the seed's component
 *   k_measure            measure_theta_observables_with_scratch
 *                        (src/observables.rs:80-154), FP64 block sums, fixed
 *                        summation order (last block reduces the partials);
 *   k_measure_rows       the same with warps walking rows (L_x a multiple of
 *                        32): two sincos per site instead of four
 *
 * (The correlation functions are in kernel_corr.cu, batched over tasks.)
 */
#include <algorithm>

#include "engine.h"
#include "fastdiv.h"
#include "xy_device.cuh"

namespace slsf {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_init_random(float* __restrict__ theta, uint32_t volume,
                                                          uint64_t seed) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (4ull * q >= volume) return;
    const slsf_u32x4 b = slsf_stream(seed, 0, SLSF_PURPOSE_INIT, 0, q);
    const uint32_t w[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = 4 * q + k;
        if (i < volume) theta[i] = slsf_angle_from_word(w[k]);
    }
}

/* Adds a per-thread count to stats[slot] with one global atomic per block
 * (warp sums, then a shared-memory sum): grid-wide kernels have tens of
 * thousands of warps, and one same-address atomic per warp serialises. */
__device__ __forceinline__ void block_count(uint32_t v, unsigned long long* stats, int slot) {
    __shared__ unsigned int s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_sum, v);
    __syncthreads();
    if (threadIdx.x == 0 && s_sum) atomicAdd(&stats[slot], (unsigned long long)s_sum);
}

/* Sums of the measurement (mx, my, J cos and J sin per axis) and where they
 * go: per-block partials, a block counter, the totals and an optional bin
 * row -- the last block adds the partials in block order. */
struct MeasureSink {
    double* partials;
    unsigned int* done;
    double* result;
    double* bin_row;
};

/* The last block's reduction of the per-block measurement partials into the
 * totals and the bin row (ThetaModel::measure's stream, src/model.rs:406-409,
 * in the batched kernels' column order). */
__device__ __forceinline__ void finish_measure(double (&acc)[8], double* scratch, const MeasureSink& m,
                                               uint32_t volume) {
    __shared__ bool last;
    block_sum<8>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) m.partials[blockIdx.x * 8 + k] = acc[k];
        __threadfence();
        last = (atomicAdd(m.done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        for (int k = 0; k < 8; ++k) tot[k] += ((volatile double*)m.partials)[b * 8 + k];
    block_sum<8>(tot, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) m.result[k] = tot[k];
        if (m.bin_row) {
            const double v = (double)volume;
            const double e = -(tot[2] + tot[3] + tot[4]) / v;
            const double vals[kBinCols] = {e,      e * e,  (tot[0] * tot[0] + tot[1] * tot[1]) / (v * v),
                                           tot[2], tot[3], tot[4],
                                           tot[5], tot[6], tot[7],
                                           tot[5] * tot[5], tot[6] * tot[6], tot[7] * tot[7]};
            for (int q = 0; q < kBinCols; ++q) m.bin_row[q] += vals[q];
        }
        *m.done = 0;
    }
}

/* Colour 0 of a sweep, grid-stride blocks, measuring the state it starts
 * from as the batched kernels do: every
 * bond has exactly one colour-0 end, so the three forward and three backward
 * bonds of the colour-0 sites and the magnetisation of each colour-0 site and
 * of its +x neighbour cover the lattice once; the FP32 bond terms are the
 * measurement kernels' (bond_cos / bond_sin), summed in FP64. */
template <bool kRecord>
__global__ void __launch_bounds__(kThreads)
    k_metro_colour(float* __restrict__ theta, const float* __restrict__ jxy,
                   const float* __restrict__ jz, uint32_t lx, uint32_t ly, uint32_t lz, float beta,
                   float width, uint64_t seed, uint64_t sweep, uint32_t colour, slsf_fastdiv div_hx,
                   slsf_fastdiv div_ly, unsigned long long* __restrict__ stats, uint8_t* __restrict__ record) {
    const uint32_t volume = lx * ly * lz;
    const uint32_t half = volume >> 1;
    const uint32_t npairs = (half + 1) >> 1;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t accepted = 0;
    if (p < npairs) {
        const slsf_u32x4 blk = slsf_stream(seed, sweep, SLSF_PURPOSE_METRO, colour, p);
#pragma unroll
        for (uint32_t lane = 0; lane < 2; ++lane) {
            const uint32_t h = 2 * p + lane;
            if (h >= half) break;
            /* the h-th site of this colour: row = h / (L_x / 2) (x + L_x row = site index),
             * x = 2 (h mod L_x / 2) + (colour + y + z) mod 2; divisions as multiply-shifts */
            SiteXYZ s;
            const uint32_t row = slsf_fastdiv_div(h, div_hx), k = h - row * div_hx.d;
            s.z = slsf_fastdiv_div(row, div_ly);
            s.y = row - s.z * ly;
            s.x = 2u * k + ((colour + s.y + s.z) & 1u);
            s.idx = s.x + lx * row;
            uint32_t nb[6];
            neighbour_indices(s, lx, ly, lz, nb);
            float ns[6], nc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) __sincosf(theta[nb[k]], &ns[k], &nc[k]);
            const float jx = jxy[s.z], jzp = jz[s.z], jzm = jz[s.z == 0 ? lz - 1 : s.z - 1];
            const float hx = field_component(jx, jzp, jzm, nc[0], nc[1], nc[2], nc[3], nc[4], nc[5]);
            const float hy = field_component(jx, jzp, jzm, ns[0], ns[1], ns[2], ns[3], ns[4], ns[5]);
            const float th = theta[s.idx];
            float si, ci;
            __sincosf(th, &si, &ci);
            float u_prop, u_acc;
            slsf_metro_uniforms(blk, lane, &u_prop, &u_acc);
            float tn, sn, cn;
            const bool acc = metro_decide(th, ci, si, hx, hy, beta, width, u_prop, u_acc, &tn, &sn, &cn);
            if (acc) {
                theta[s.idx] = tn;
                ++accepted;
            }
            if (kRecord) record[s.idx] = acc ? 1 : 0;
        }
    }
    block_count(accepted, stats, kStatAccepted);
}

__global__ void __launch_bounds__(kThreads, 3)
    k_metro_colour0_measure(float* __restrict__ theta, const float* __restrict__ jxy,
                   const float* __restrict__ jz, uint32_t lx, uint32_t ly, uint32_t lz, float beta,
                   float width, uint64_t seed, uint64_t sweep, uint32_t colour, slsf_fastdiv div_hx,
                   slsf_fastdiv div_ly, unsigned long long* __restrict__ stats, MeasureSink sink) {
    const uint32_t volume = lx * ly * lz;
    const uint32_t half = volume >> 1;
    const uint32_t npairs = (half + 1) >> 1;
    uint32_t accepted = 0;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    auto pair = [&](uint32_t p) {
        const slsf_u32x4 blk = slsf_stream(seed, sweep, SLSF_PURPOSE_METRO, colour, p);
#pragma unroll
        for (uint32_t lane = 0; lane < 2; ++lane) {
            const uint32_t h = 2 * p + lane;
            if (h >= half) break;
            /* the h-th site of this colour: row = h / (L_x / 2) (x + L_x row = site index),
             * x = 2 (h mod L_x / 2) + (colour + y + z) mod 2; divisions as multiply-shifts */
            SiteXYZ s;
            const uint32_t row = slsf_fastdiv_div(h, div_hx), k = h - row * div_hx.d;
            s.z = slsf_fastdiv_div(row, div_ly);
            s.y = row - s.z * ly;
            s.x = 2u * k + ((colour + s.y + s.z) & 1u);
            s.idx = s.x + lx * row;
            uint32_t nb[6];
            neighbour_indices(s, lx, ly, lz, nb);
            float ns[6], nc[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) __sincosf(theta[nb[k]], &ns[k], &nc[k]);
            const float jx = jxy[s.z], jzp = jz[s.z], jzm = jz[s.z == 0 ? lz - 1 : s.z - 1];
            const float hx = field_component(jx, jzp, jzm, nc[0], nc[1], nc[2], nc[3], nc[4], nc[5]);
            const float hy = field_component(jx, jzp, jzm, ns[0], ns[1], ns[2], ns[3], ns[4], ns[5]);
            const float th = theta[s.idx];
            float si, ci;
            __sincosf(th, &si, &ci);
            {
                /* neighbours in the order +x -x +y -y +z -z; a backward bond
                 * starts at the neighbour (its layer's coupling for z) */
                acc[0] += (double)ci + (double)nc[0];
                acc[1] += (double)si + (double)ns[0];
                acc[2] += (double)bond_cos(jx, ci, si, nc[0], ns[0]) + (double)bond_cos(jx, nc[1], ns[1], ci, si);
                acc[3] += (double)bond_cos(jx, ci, si, nc[2], ns[2]) + (double)bond_cos(jx, nc[3], ns[3], ci, si);
                acc[4] += (double)bond_cos(jzp, ci, si, nc[4], ns[4]) + (double)bond_cos(jzm, nc[5], ns[5], ci, si);
                acc[5] += (double)bond_sin(jx, ci, si, nc[0], ns[0]) + (double)bond_sin(jx, nc[1], ns[1], ci, si);
                acc[6] += (double)bond_sin(jx, ci, si, nc[2], ns[2]) + (double)bond_sin(jx, nc[3], ns[3], ci, si);
                acc[7] += (double)bond_sin(jzp, ci, si, nc[4], ns[4]) + (double)bond_sin(jzm, nc[5], ns[5], ci, si);
            }
            float u_prop, u_acc;
            slsf_metro_uniforms(blk, lane, &u_prop, &u_acc);
            float tn, sn, cn;
            const bool ok = metro_decide(th, ci, si, hx, hy, beta, width, u_prop, u_acc, &tn, &sn, &cn);
            if (ok) {
                theta[s.idx] = tn;
                ++accepted;
            }
        }
    };
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npairs; p += gridDim.x * blockDim.x) pair(p);
    block_count(accepted, stats, kStatAccepted);
    __shared__ double scratch[8 * 32];
    finish_measure(acc, scratch, sink, volume);
}

/* Smallest lattice whose Wolff update grows the seed's cluster on bit-packed
 * bonds instead of labelling 32x8x4 tiles (measured crossover on B200). */
#ifndef SLSF_WOLFF_BITS_MIN_SITES
#define SLSF_WOLFF_BITS_MIN_SITES (1u << 22)
#endif
constexpr uint64_t kWolffBitsMinSites = SLSF_WOLFF_BITS_MIN_SITES;

/* ---- Wolff: union-find with links from larger to smaller roots ---- */

/* Loop bounds of the union-find: a path is strictly decreasing, so at most
 * `volume` long; a union retries at most 2^22 times.  A nonzero `limit`
 * (slsf_ctx_set_loop_limit) lowers both, to exercise the error path. */
struct UfBounds {
    uint32_t find, uni;
};

__device__ __forceinline__ UfBounds uf_bounds(uint32_t volume, uint32_t limit) {
    const uint32_t u = 1u << 22;
    return {limit ? min(limit, volume) : volume, limit ? min(limit, u) : u};
}

/* Root of x with path splitting.  parent[i] <= i always holds, so every path
 * is strictly decreasing; the loop is bounded by b.find. */
__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x, UfBounds b, bool* ok) {
    volatile uint32_t* par = parent;
    for (uint32_t it = 0; it <= b.find; ++it) {
        const uint32_t p = par[x];
        if (p == x) return x;
        const uint32_t gp = par[p];
        if (gp != p) par[x] = gp;
        x = p;
    }
    *ok = false;
    return x;
}

/* Lock-free union: hook the larger root under the smaller with a CAS.  A
 * failed CAS means another thread linked that root; every retry follows some
 * other thread's progress, and the retry count is bounded. */
__device__ __forceinline__ bool uf_union(uint32_t* parent, uint32_t a, uint32_t b, UfBounds bd) {
    bool ok = true;
    for (uint32_t it = 0; it < bd.uni; ++it) {
        a = uf_find(parent, a, bd, &ok);
        b = uf_find(parent, b, bd, &ok);
        if (!ok) return false;
        if (a == b) return true;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicCAS(&parent[b], b, a);
        if (old == b) return true;
    }
    return false;
}

/* Wolff tiles: a CTA labels one tile of kTileX x kTileY x kTileZ sites. */
constexpr uint32_t kTileX = 32, kTileY = 8, kTileZ = 4;
constexpr uint32_t kTileSites = kTileX * kTileY * kTileZ;
static_assert(kTileX == 32, "a tile row is one warp");
/* Bit 3 of a site's bond byte: the site is the root of its component inside
 * its tile (bits 0-2 are the +x/+y/+z bonds). */
constexpr uint8_t kTileRoot = 8;

/* Local union-find in shared memory: hook the larger root under the smaller
 * with a CAS; bounded like the global one. */
__device__ __forceinline__ uint32_t tile_find(uint32_t* lpar, uint32_t x, UfBounds bd, bool* ok) {
    volatile uint32_t* par = lpar;
    for (uint32_t it = 0; it <= bd.find; ++it) {
        const uint32_t p = par[x];
        if (p == x) return x;
        const uint32_t gp = par[p];
        if (gp != p) par[x] = gp;
        x = p;
    }
    *ok = false;
    return x;
}

__device__ __forceinline__ bool tile_union(uint32_t* lpar, uint32_t a, uint32_t b, UfBounds bd) {
    bool ok = true;
    for (uint32_t it = 0; it < bd.uni; ++it) {
        a = tile_find(lpar, a, bd, &ok);
        b = tile_find(lpar, b, bd, &ok);
        if (!ok) return false;
        if (a == b) return true;
        if (a > b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&lpar[b], b, a) == b) return true;
    }
    return false;
}

/* Bond activation (try_add_wolff_neighbor, src/updates.rs:537-548) for every
 * site of a tile, then the tile's components over its inner bonds: each site
 * gets parent = the smallest site of its component inside the tile (local
 * order is global order inside a tile, so parent[i] <= i holds).  Bonds that
 * leave the tile are joined by k_wolff_boundary. */
__global__ void __launch_bounds__(kThreads)
    k_wolff_tiles(const float* __restrict__ theta, const float* __restrict__ jxy,
                  const float* __restrict__ jz, uint32_t lx, uint32_t ly, uint32_t lz,
                  float minus_two_beta, float phi, uint64_t seed, uint64_t counter,
                  uint8_t* __restrict__ bonds, uint32_t* __restrict__ parent,
                  unsigned long long* __restrict__ stats, uint32_t limit) {
    __shared__ uint32_t lpar[kTileSites];
    const UfBounds bd = uf_bounds(kTileSites, limit);
    const UfBounds bu = {bd.find, limit ? min(limit, 4 * kTileSites) : 4 * kTileSites};
    __shared__ uint8_t lbits[kTileSites];
    const uint32_t ntx = (lx + kTileX - 1) / kTileX, nty = (ly + kTileY - 1) / kTileY;
    const uint32_t tx = blockIdx.x % ntx, rest = blockIdx.x / ntx;
    const uint32_t ty = rest % nty, tz = rest / nty;
    const uint32_t x0 = tx * kTileX, y0 = ty * kTileY, z0 = tz * kTileZ;
    const uint32_t ex = min(kTileX, lx - x0), ey = min(kTileY, ly - y0), ez = min(kTileZ, lz - z0);
    const uint32_t plane = lx * ly, volume = plane * lz;
    float sphi, cphi;
    __sincosf(phi, &sphi, &cphi);
    auto proj = [&](uint32_t site) {
        float sn, cn;
        __sincosf(theta[site], &sn, &cn);
        return wolff_projection(cn, sn, cphi, sphi);
    };
    for (uint32_t l = threadIdx.x; l < kTileSites; l += blockDim.x) {
        const uint32_t ax = l % kTileX, ay = (l / kTileX) % kTileY, az = l / (kTileX * kTileY);
        uint32_t bits = 0;
        if (ax < ex && ay < ey && az < ez) {
            const uint32_t x = x0 + ax, y = y0 + ay, z = z0 + az;
            const uint32_t i = x + lx * (y + ly * z);
            const uint32_t xp = (x + 1 == lx) ? i + 1 - lx : i + 1;
            const uint32_t yp = (y + 1 == ly) ? i + lx - plane : i + lx;
            const uint32_t zp = (z + 1 == lz) ? i + plane - volume : i + plane;
            const float ri = proj(i);
            const slsf_u32x4 b = slsf_stream(seed, counter, SLSF_PURPOSE_WOLFF_BOND, 0, i);
            if (wolff_bond_active(jxy[z], ri, proj(xp), minus_two_beta, b.x)) bits |= 1u;
            if (wolff_bond_active(jxy[z], ri, proj(yp), minus_two_beta, b.y)) bits |= 2u;
            if (wolff_bond_active(jz[z], ri, proj(zp), minus_two_beta, b.z)) bits |= 4u;
            bonds[i] = (uint8_t)bits;
        }
        lbits[l] = (uint8_t)bits;
        /* A warp holds one row of the tile (kTileX == 32 sites, lane = x):
         * the sites joined along x form runs, and every site's parent is the
         * first site of its run (the highest run start at or below its lane),
         * so the x bonds inside the tile need no union. */
        const unsigned xb = __ballot_sync(0xffffffffu, (bits & 1u) && ax + 1 < ex);
        const unsigned starts = ~(xb << 1);
        const uint32_t lane = l % kTileX;
        const unsigned upto = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
        lpar[l] = l - lane + (31u - __clz(starts & upto));
    }
    __syncthreads();
    bool ok = true;
    for (uint32_t l = threadIdx.x; l < kTileSites; l += blockDim.x) {
        /* a warp holds one row (lane = x); a y or z bond whose left neighbour's
         * bond joins the same two x-runs adds nothing, so only the first bond of
         * each such stretch unions */
        const uint32_t lane = l % kTileX, bits = lbits[l];
        const uint32_t ay = (l / kTileX) % kTileY, az = l / (kTileX * kTileY);
        const bool yin = ay + 1 < ey, zin = az + 1 < ez; /* warp-uniform */
        const bool xin = lane + 1 < ex;
        const unsigned own = __ballot_sync(0xffffffffu, (bits & 1u) && xin);
        const unsigned yb = __ballot_sync(0xffffffffu, (bits & 2u) && yin);
        const unsigned zb = __ballot_sync(0xffffffffu, (bits & 4u) && zin);
        const unsigned yrow = yin ? __ballot_sync(0xffffffffu, (lbits[l + kTileX] & 1u) && xin) : 0u;
        const unsigned zrow = zin ? __ballot_sync(0xffffffffu, (lbits[l + kTileX * kTileY] & 1u) && xin) : 0u;
        const unsigned ylead = yb & ~((yb & own & yrow) << 1), zlead = zb & ~((zb & own & zrow) << 1);
        if ((ylead >> lane) & 1u) ok &= tile_union(lpar, l, l + kTileX, bu);
        if ((zlead >> lane) & 1u) ok &= tile_union(lpar, l, l + kTileX * kTileY, bu);
    }
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < kTileSites; l += blockDim.x) {
        const uint32_t ax = l % kTileX, ay = (l / kTileX) % kTileY, az = l / (kTileX * kTileY);
        if (ax >= ex || ay >= ey || az >= ez) continue;
        const uint32_t r = tile_find(lpar, l, bd, &ok);
        const uint32_t rx = r % kTileX, ry = (r / kTileX) % kTileY, rz = r / (kTileX * kTileY);
        const uint32_t i = (x0 + ax) + lx * ((y0 + ay) + ly * (z0 + az));
        parent[i] = (x0 + rx) + lx * ((y0 + ry) + ly * (z0 + rz));
        if (r == l) bonds[i] = (uint8_t)(lbits[l] | kTileRoot); /* marks the tile's roots for k_wolff_compress */
    }
    if (!ok) atomicOr(&stats[kStatError], kErrUnionFindLimit);
}

/* The active bonds that leave a tile (its last x, y or z; periodic wraps
 * included), joined in the global union-find over the tile roots.  A warp
 * takes one face row of one tile: the 8 x 4 bonds of the +x face (lane =
 * y + 8 z), one of the 4 rows of the +y face or one of the 8 rows of the +z
 * face (lane = x).  The bonds of a face row mostly join the same few pairs of
 * tile roots, so the lanes group them by (root, root) pair and one lane per
 * pair joins. */
constexpr uint32_t kFaceRows = 1 + kTileZ + kTileY;
static_assert(kTileY * kTileZ == 32, "an x face is one warp");

__global__ void __launch_bounds__(kThreads)
    k_wolff_boundary(const uint8_t* __restrict__ bonds, uint32_t lx, uint32_t ly, uint32_t lz, uint32_t n_tiles,
                     uint32_t* parent, unsigned long long* stats, uint32_t limit) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t tile = w / kFaceRows, item = w - tile * kFaceRows;
    if (tile >= n_tiles) return; /* whole warps */
    const uint32_t ntx = (lx + kTileX - 1) / kTileX, nty = (ly + kTileY - 1) / kTileY;
    const uint32_t tx = tile % ntx, rest = tile / ntx, ty = rest % nty, tz = rest / nty;
    const uint32_t x0 = tx * kTileX, y0 = ty * kTileY, z0 = tz * kTileZ;
    const uint32_t ex = min(kTileX, lx - x0), ey = min(kTileY, ly - y0), ez = min(kTileZ, lz - z0);
    const uint32_t plane = lx * ly, volume = plane * lz;
    uint32_t ax, ay, az, d;
    if (item == 0) {
        d = 0, ax = ex - 1, ay = lane % kTileY, az = lane / kTileY;
    } else if (item <= kTileZ) {
        d = 1, ax = lane, ay = ey - 1, az = item - 1;
    } else {
        d = 2, ax = lane, ay = item - 1 - kTileZ, az = ez - 1;
    }
    const bool in = ax < ex && ay < ey && az < ez;
    const uint32_t x = x0 + ax, y = y0 + ay, z = z0 + az;
    const uint32_t i = in ? x + lx * (y + ly * z) : 0u;
    const bool act = in && (bonds[i] & (1u << d));
    uint32_t a = 0, b = 0;
    if (act) {
        const uint32_t nb = d == 0   ? ((x + 1 == lx) ? i + 1 - lx : i + 1)
                            : d == 1 ? ((y + 1 == ly) ? i + lx - plane : i + lx)
                                     : ((z + 1 == lz) ? i + plane - volume : i + plane);
        a = parent[i];
        b = parent[nb];
    }
    const unsigned long long key = act ? (((unsigned long long)a << 32) | b) : ~0ull;
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    bool ok = true;
    if (act && lane == (uint32_t)(__ffs(grp) - 1) && a != b) ok = uf_union(parent, a, b, uf_bounds(volume, limit));
    if (!ok) atomicOr(&stats[kStatError], kErrUnionFindLimit);
}

/* After the joins between tiles, every tile root points at its component's
 * root (path compression from the roots only: the other sites point at a
 * tile root, and nobody points at them). */
__global__ void __launch_bounds__(kThreads)
    k_wolff_compress(const uint8_t* __restrict__ bonds, uint32_t volume, uint32_t* parent,
                     unsigned long long* stats, uint32_t limit) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= volume || !(bonds[i] & kTileRoot)) return;
    /* A find without path splitting: the only writes in this kernel set a
     * tile root's parent to its component's root, so every parent a thread
     * reads leads to the same root (a split could write back a stale
     * ancestor over a root already written). */
    const volatile uint32_t* par = parent;
    const uint32_t bound = uf_bounds(volume, limit).find;
    uint32_t x = i;
    for (uint32_t it = 0;; ++it) {
        const uint32_t p = par[x];
        if (p == x) break;
        if (it >= bound) {
            atomicOr(&stats[kStatError], kErrUnionFindLimit);
            return;
        }
        x = p;
    }
    parent[i] = x;
}

/* Reflect the seed's component (src/updates.rs:602-617).  A site's parent is
 * a tile root whose parent is the component's root, so two loads find it. */
__global__ void __launch_bounds__(kThreads)
    k_wolff_flip(float* __restrict__ theta, uint32_t volume, const uint32_t* __restrict__ parent, uint32_t seed_idx,
                 float phi, unsigned long long* stats, uint8_t* __restrict__ cluster_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t in = 0;
    if (i < volume) {
        const uint32_t root = parent[parent[seed_idx]];
        in = (parent[parent[i]] == root) ? 1u : 0u;
        if (in) theta[i] = slsf_reflect(theta[i], phi);
        if (cluster_out) cluster_out[i] = (uint8_t)in;
    }
    block_count(in, stats, kStatClusterSites);
}

/* ---- fused observables ---- */
constexpr int kMeasureThreads = 256;

__global__ void __launch_bounds__(kMeasureThreads)
    k_measure(const float* __restrict__ theta, const float* __restrict__ jxy,
              const float* __restrict__ jz, uint32_t lx, uint32_t ly, uint32_t lz, slsf_fastdiv div_lx,
              slsf_fastdiv div_ly, double* __restrict__ partials, unsigned int* __restrict__ done,
              double* __restrict__ result, double* __restrict__ bin_row) {
    __shared__ double scratch[8 * 32];
    __shared__ bool last;
    const uint32_t volume = lx * ly * lz, plane = lx * ly;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < volume; i += stride) {
        const uint32_t row = slsf_fastdiv_div(i, div_lx), z = slsf_fastdiv_div(row, div_ly);
        const uint32_t x = i - row * lx, y = row - z * ly;
        const uint32_t ix = (x + 1 == lx) ? i + 1 - lx : i + 1;
        const uint32_t iy = (y + 1 == ly) ? i + lx - plane : i + lx;
        const uint32_t iz = (z + 1 == lz) ? i + plane - volume : i + plane;
        float si, ci, sx, cx, sy, cy, sz, cz;
        __sincosf(theta[i], &si, &ci);
        __sincosf(theta[ix], &sx, &cx);
        __sincosf(theta[iy], &sy, &cy);
        __sincosf(theta[iz], &sz, &cz);
        const float jx = jxy[z], jzz = jz[z];
        /* diff_cos_sin (src/observables.rs:9-11): cos(a-b), sin(a-b) from trig. */
        acc[0] += ci;
        acc[1] += si;
        acc[2] += bond_cos(jx, ci, si, cx, sx);
        acc[3] += bond_cos(jx, ci, si, cy, sy);
        acc[4] += bond_cos(jzz, ci, si, cz, sz);
        acc[5] += bond_sin(jx, ci, si, cx, sx);
        acc[6] += bond_sin(jx, ci, si, cy, sy);
        acc[7] += bond_sin(jzz, ci, si, cz, sz);
    }
    block_sum<8>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) partials[blockIdx.x * 8 + k] = acc[k];
        __threadfence();
        last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    /* Last block: sum the per-block partials in block order. */
    __threadfence();
    double tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        for (int k = 0; k < 8; ++k) tot[k] += ((volatile double*)partials)[b * 8 + k];
    block_sum<8>(tot, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) result[k] = tot[k];
        if (bin_row) {
            /* ThetaModel::measure's stream (src/model.rs:406-409) added to
             * the bin's sums, in the batched kernels' column order. */
            const double v = (double)volume;
            const double e = -(tot[2] + tot[3] + tot[4]) / v;
            const double vals[kBinCols] = {e,      e * e,  (tot[0] * tot[0] + tot[1] * tot[1]) / (v * v),
                                           tot[2], tot[3], tot[4],
                                           tot[5], tot[6], tot[7],
                                           tot[5] * tot[5], tot[6] * tot[6], tot[7] * tot[7]};
            for (int q = 0; q < kBinCols; ++q) bin_row[q] += vals[q];
        }
        *done = 0;
    }
}

/* The same measurement for L_x a multiple of 32 and L_y a multiple of 16:
 * a warp owns word k (lane = x - 32 k) of plane z for a run of 16 rows and
 * walks it along y, so each site's own trig is the previous row's +y trig:
 * two sincos per site (+y, +z) instead of four, the +x neighbour by shuffle.
 * Identical FP32 bond terms; FP64 sums in another order. */
constexpr uint32_t kMeasureSeg = 16;

__global__ void __launch_bounds__(kMeasureThreads)
    k_measure_rows(const float* __restrict__ theta, const float* __restrict__ jxy,
                   const float* __restrict__ jz, uint32_t lx, uint32_t ly, uint32_t lz,
                   double* __restrict__ partials, unsigned int* __restrict__ done,
                   double* __restrict__ result, double* __restrict__ bin_row) {
    __shared__ double scratch[8 * 32];
    __shared__ bool last;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t words = lx >> 5, nseg = ly / kMeasureSeg, plane = lx * ly, volume = plane * lz;
    const uint32_t units = words * nseg * lz;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += nwarps) {
        const uint32_t k = u % words, rest = u / words, sg = rest % nseg, z = rest / nseg;
        const uint32_t x = 32u * k + lane, xn = (k + 1 == words) ? 0u : 32u * (k + 1);
        const uint32_t zbase = z * plane, zp_base = (z + 1 == lz) ? 0u : (z + 1) * plane;
        const float jx = jxy[z], jzz = jz[z];
        const uint32_t y0 = sg * kMeasureSeg;
        float si, ci;
        __sincosf(theta[zbase + y0 * lx + x], &si, &ci);
        /* the angles of the next row's loads, one row ahead */
        auto yrow = [&](uint32_t y) { return (y + 1 == ly) ? 0u : y + 1; };
        float t_yp = theta[zbase + yrow(y0) * lx + x], t_zp = theta[zp_base + y0 * lx + x];
        float t_xn = theta[zbase + y0 * lx + xn];
        for (uint32_t y = y0; y < y0 + kMeasureSeg; ++y) {
            const uint32_t row = zbase + y * lx;
            const float a_yp = t_yp, a_zp = t_zp, a_xn = t_xn;
            if (y + 1 < y0 + kMeasureSeg) {
                t_yp = theta[zbase + yrow(y + 1) * lx + x];
                t_zp = theta[zp_base + (y + 1) * lx + x];
                t_xn = theta[row + lx + xn];
            }
            float sx, cx, sy, cy, sz, cz, sn, cn;
            __sincosf(a_yp, &sy, &cy);
            __sincosf(a_zp, &sz, &cz);
            __sincosf(a_xn, &sn, &cn);
            sx = __shfl_sync(0xffffffffu, si, (lane + 1u) & 31u);
            cx = __shfl_sync(0xffffffffu, ci, (lane + 1u) & 31u);
            if (lane == 31) {
                sx = sn;
                cx = cn;
            }
            acc[0] += ci;
            acc[1] += si;
            acc[2] += bond_cos(jx, ci, si, cx, sx);
            acc[3] += bond_cos(jx, ci, si, cy, sy);
            acc[4] += bond_cos(jzz, ci, si, cz, sz);
            acc[5] += bond_sin(jx, ci, si, cx, sx);
            acc[6] += bond_sin(jx, ci, si, cy, sy);
            acc[7] += bond_sin(jzz, ci, si, cz, sz);
            si = sy;
            ci = cy;
        }
    }
    block_sum<8>(acc, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) partials[blockIdx.x * 8 + k] = acc[k];
        __threadfence();
        last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        for (int k = 0; k < 8; ++k) tot[k] += ((volatile double*)partials)[b * 8 + k];
    block_sum<8>(tot, scratch);
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) result[k] = tot[k];
        if (bin_row) {
            const double v = (double)volume;
            const double e = -(tot[2] + tot[3] + tot[4]) / v;
            const double vals[kBinCols] = {e,      e * e,  (tot[0] * tot[0] + tot[1] * tot[1]) / (v * v),
                                           tot[2], tot[3], tot[4],
                                           tot[5], tot[6], tot[7],
                                           tot[5] * tot[5], tot[6] * tot[6], tot[7] * tot[7]};
            for (int q = 0; q < kBinCols; ++q) bin_row[q] += vals[q];
        }
        *done = 0;
    }
}

inline bool measure_rows_supported(uint32_t lx, uint32_t ly) { return lx % 32 == 0 && ly % kMeasureSeg == 0; }

inline uint32_t blocks_for(uint64_t n, int threads) { return (uint32_t)((n + threads - 1) / threads); }

}  // namespace

namespace {

/* One block per source array; coalesced copy into the contiguous output. */
__global__ void k_gather(const double* const* __restrict__ src, uint32_t per, double* __restrict__ dst) {
    const double* s = src[blockIdx.x];
    double* d = dst + (size_t)blockIdx.x * per;
    for (uint32_t k = threadIdx.x; k < per; k += blockDim.x) d[k] = s[k];
}

}  // namespace

void launch_gather(const double* const* src, uint32_t n, uint32_t per, double* dst, cudaStream_t s) {
    k_gather<<<n, 128, 0, s>>>(src, per, dst);
}

void launch_init_random(float* theta, uint32_t volume, uint64_t seed, cudaStream_t s) {
    const uint32_t quads = (volume + 3) / 4;
    k_init_random<<<blocks_for(quads, kThreads), kThreads, 0, s>>>(theta, volume, seed);
}

void launch_metro_colour(const TaskView& t, uint64_t sweep, uint32_t colour, uint8_t* record,
                         cudaStream_t s) {
    const uint32_t volume = t.lx * t.ly * t.lz;
    const uint32_t npairs = ((volume >> 1) + 1) >> 1;
    const uint32_t grid = blocks_for(npairs, kThreads);
    const slsf_fastdiv dhx = slsf_fastdiv_make(t.lx / 2), dly = slsf_fastdiv_make(t.ly);
    if (record)
        k_metro_colour<true><<<grid, kThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, t.beta, t.width,
                                                       t.seed, sweep, colour, dhx, dly, t.stats, record);
    else
        k_metro_colour<false><<<grid, kThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, t.beta, t.width,
                                                        t.seed, sweep, colour, dhx, dly, t.stats, nullptr);
}

void launch_metro_colour0_measure(const TaskView& t, uint64_t sweep, double* partials, unsigned int* done,
                                  double* result, double* bin_row, cudaStream_t s) {
    const uint32_t volume = t.lx * t.ly * t.lz;
    const uint32_t npairs = ((volume >> 1) + 1) >> 1;
    /* grid-stride blocks, as many as stay resident (at most kMeasureMaxBlocks,
     * the partials' rows); a fixed count per device keeps the sums' order */
    static int per_sm = 0;
    if (per_sm == 0 &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_metro_colour0_measure, kThreads, 0) !=
            cudaSuccess)
        per_sm = 1;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t cap = (uint32_t)std::max(1, std::min(per_sm * sms, kMeasureMaxBlocks));
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(blocks_for(npairs, kThreads), cap));
    const slsf_fastdiv dhx = slsf_fastdiv_make(t.lx / 2), dly = slsf_fastdiv_make(t.ly);
    const MeasureSink sink = {partials, done, result, bin_row};
    k_metro_colour0_measure<<<grid, kThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, t.beta, t.width,
                                                      t.seed, sweep, 0, dhx, dly, t.stats, sink);
}

int launch_wolff(const TaskView& t, uint64_t counter, uint8_t* bonds, uint32_t* parent,
                 uint8_t* cluster_out, cudaStream_t s, float* phi_out, uint32_t seed_site[3], bool record_bonds) {
    /* Large lattices with sides that are multiples of 32 grow the seed's
     * cluster on bit-packed bonds (kernel_wolff_bits.cu), in the union-find
     * array; below kWolffBitsMinSites the tile labelling is faster. */
    if ((uint64_t)t.lx * t.ly * t.lz >= kWolffBitsMinSites && wolff_bits_supports(t.lx, t.ly, t.lz) &&
        wolff_bits_scratch_bytes(t.lx, t.ly, t.lz) <= 4ull * t.lx * t.ly * t.lz)
        return launch_wolff_bits(t, counter, parent, record_bonds ? bonds : nullptr, cluster_out, s, phi_out,
                                 seed_site);
    /* The reflection axis and seed site (src/updates.rs:564-568) come from
     * the WOLFF_PICK block, computed here on the host from the same header. */
    const slsf_u32x4 pick = slsf_stream(t.seed, counter, SLSF_PURPOSE_WOLFF_PICK, 0, 0);
    const float phi = slsf_angle_from_word(pick.x);
    const uint32_t x0 = slsf_range(pick.y, t.lx), y0 = slsf_range(pick.z, t.ly), z0 = slsf_range(pick.w, t.lz);
    const uint32_t volume = t.lx * t.ly * t.lz;
    const uint32_t seed_idx = x0 + t.lx * (y0 + t.ly * z0);
    const uint32_t grid = blocks_for(volume, kThreads);
    const uint32_t tiles = ((t.lx + kTileX - 1) / kTileX) * ((t.ly + kTileY - 1) / kTileY) *
                           ((t.lz + kTileZ - 1) / kTileZ);
    k_wolff_tiles<<<tiles, kThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, -2.0f * t.beta, phi,
                                             t.seed, counter, bonds, parent, t.stats, t.loop_limit);
    k_wolff_boundary<<<blocks_for((uint64_t)tiles * kFaceRows * 32, kThreads), kThreads, 0, s>>>(
        bonds, t.lx, t.ly, t.lz, tiles, parent, t.stats, t.loop_limit);
    k_wolff_compress<<<grid, kThreads, 0, s>>>(bonds, volume, parent, t.stats, t.loop_limit);
    k_wolff_flip<<<grid, kThreads, 0, s>>>(t.theta, volume, parent, seed_idx, phi, t.stats, cluster_out);
    if (phi_out) *phi_out = phi;
    if (seed_site) {
        seed_site[0] = x0;
        seed_site[1] = y0;
        seed_site[2] = z0;
    }
    return 4;
}

int measure_partial_blocks(uint32_t volume) {
    return (int)std::max<uint32_t>(1, std::min<uint32_t>(blocks_for(volume, kMeasureThreads), kMeasureMaxBlocks));
}

void launch_measure(const TaskView& t, double* partials, unsigned int* done, double* result,
                    cudaStream_t s) {
    const uint32_t volume = t.lx * t.ly * t.lz;
    if (measure_rows_supported(t.lx, t.ly)) {
        k_measure_rows<<<measure_partial_blocks(volume), kMeasureThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly,
                                                                                  t.lz, partials, done, result, nullptr);
        return;
    }
    k_measure<<<measure_partial_blocks(volume), kMeasureThreads, 0, s>>>(
        t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, slsf_fastdiv_make(t.lx), slsf_fastdiv_make(t.ly), partials, done,
        result, nullptr);
}

void launch_measure_into_bin(const TaskView& t, double* partials, unsigned int* done, double* result,
                             double* bin_row, cudaStream_t s) {
    const uint32_t volume = t.lx * t.ly * t.lz;
    if (measure_rows_supported(t.lx, t.ly)) {
        k_measure_rows<<<measure_partial_blocks(volume), kMeasureThreads, 0, s>>>(t.theta, t.jxy, t.jz, t.lx, t.ly,
                                                                                  t.lz, partials, done, result, bin_row);
        return;
    }
    k_measure<<<measure_partial_blocks(volume), kMeasureThreads, 0, s>>>(
        t.theta, t.jxy, t.jz, t.lx, t.ly, t.lz, slsf_fastdiv_make(t.lx), slsf_fastdiv_make(t.ly), partials, done,
        result, bin_row);
}

}  // namespace slsf
