/*
 * Correlation functions of many tasks in two launches
 * (measure_theta_correlations_with_scratch, src/observables.rs:165-270):
 *
 *   C_x(r)     = sum_{x,y,z} s(x,y,z) . s(x+r,y,z) / V
 *   C_y(r)     = sum s(x,y,z) . s(x,y+r,z) / V
 *   C_xy(r)    = (C_x(r) + C_y(r)) / 2
 *   C_xy(z, r) = sum_{x,y} [s . s(x+r) + s . s(y+r)] / (2 Lx Ly)
 *   C_z(r)     = sum s(x,y,z) . s(x,y,z+r) / V
 *
 * with periodic shifts, r = 1..R (R = rmax_xy clamped to Lx/2, Ly/2) and
 * r = 1..R_z (R_z = rmax_z clamped to Lz/2); s . s' = cos cos' + sin sin'.
 *
 * k_corr_lines: one block per work item of all tasks (the hardware balances
 * items of different lengths across the SMs).  An
 * item is up to 32 parallel lines of one task along one axis -- x lines: 32
 * consecutive rows y of one layer; y lines: 32 consecutive x of one layer;
 * z lines: 32 consecutive x of one row y -- staged as (cos, sin) pairs in a
 * shared tile [n + R][pitch] (the first R entries of each line repeated
 * after its end, so k + r needs no modulo).  y and z lines fill the tile
 * row-wise with a 32-pair pitch (a warp's row read is two aligned 128-byte
 * wavefronts); x lines fill it transposed with a 33-pair pitch, which keeps
 * that fill free of bank conflicts.  Lane c owns
 * line c; warp w owns 8 consecutive lags and keeps their partners in a
 * register ring along k, one shared load per k for 8 products.  Products
 * are FP32 (fused multiply-add), summed in FP32 over runs of 32 k and the
 * runs in FP64; the item's per-lag sums (FP64, over its lines) go to the
 * task's scratch.
 *
 * z lines whose length is 32, 64, 128 or 256 take a shorter route
 * (k_corr_zfft, launched beside k_corr_lines, which skips those items):
 * the circular correlation of a line is the inverse transform of its power
 * spectrum, sum_k s_k . s_{k+r} = Re (1/n) sum_q |A(q)|^2 e^{2 pi i q r / n}
 * with A the discrete Fourier transform of cos + i sin along the line.  A
 * block takes a unit of four consecutive z items of a task (128 lines); a
 * warp transforms one line at a time in FP32 (lane t holds elements t + 32 j:
 * a radix-(n/32) DFT in registers, twiddles, then a 32-point decimation-in-
 * frequency FFT across the lanes) from the raw angles staged in shared
 * memory, adds |A|^2 into its FP64 sums in shared memory, and the unit's
 * spectrum (the warps' sums in warp order) is stored folded.  O(n log n) per
 * line instead of O(n R).
 *
 * k_corr_finalize: one block per task sums the item partials in a fixed
 * order (per layer for x and y, over everything for z; on the spectral route
 * the units' spectra, inverted once with tabulated cosines), forms the values in
 * ThetaModel::measure's order (src/model.rs:420-437) -- C_x, C_y, C_xy,
 * C_xy(z, r) z-major, C_z -- and writes them out and/or adds them into row
 * count / binsize of the task's correlation bin sums.  Everything is
 * deterministic: a task's values do not depend on the other tasks of the
 * launch or on the grid size.
 */
#include <algorithm>

#include "engine.h"

namespace slsf {

namespace {

constexpr int kCorrThreads = 256;
constexpr uint32_t kCorrCols = 32;  /* lines per item */
constexpr uint32_t kCorrPitch = 33; /* (cos, sin) pairs per tile row, at most */
constexpr uint32_t kCorrLags = 8;   /* lags per warp pass */
constexpr uint32_t kCorrRun = 32;   /* k per FP32 run */
constexpr size_t kCorrMaxTile = 200 * 1024;

constexpr uint32_t kFftMax = 256; /* longest z line of the spectral route */
constexpr uint32_t kFftMaxN1 = kFftMax / 32;

/* z lines of length n = 32 N1 (N1 = 1, 2, 4, 8) take the spectral route. */
__host__ __device__ inline bool corr_fft_len(uint32_t n) { return n == 32 || n == 64 || n == 128 || n == 256; }

struct CorrShape {
    uint32_t cx, cy;     /* items per layer: x lines (chunks of rows), y or z lines (chunks of x) */
    uint32_t nx, ny, nz; /* items along x, y, z */
    uint32_t rp;         /* partial row pitch: max(R, R_z), and L_z / 2 + 1 on the spectral route */
    bool spectral;       /* z items store folded power spectra */
};

__host__ __device__ inline CorrShape corr_shape(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    CorrShape s;
    s.cx = (ly + kCorrCols - 1) / kCorrCols;
    s.cy = (lx + kCorrCols - 1) / kCorrCols;
    s.nx = rxy ? lz * s.cx : 0;
    s.ny = rxy ? lz * s.cy : 0;
    s.nz = rz ? ly * s.cy : 0;
    s.rp = rxy > rz ? rxy : rz;
    s.spectral = rz > 0 && corr_fft_len(lz);
    if (s.spectral && s.rp < lz / 2 + 1) s.rp = lz / 2 + 1;
    return s;
}



/* Spectral route: one block sums the power spectra of kZGroup consecutive z
 * items of a task (a unit) and writes one folded spectrum per unit, which
 * cuts the rows the finalize adds by kZGroup; the units are fixed by the
 * task's own item numbering, so the sums do not depend on the launch. */
constexpr uint32_t kZGroup = 4;

__host__ __device__ inline uint32_t corr_zunits_of(const CorrShape& sh) {
    return sh.spectral ? (sh.nz + kZGroup - 1) / kZGroup : 0;
}

/* Twiddles of the spectral route (FP32), laid out so that a warp reads 32
 * consecutive entries: stage[k][t] = w_(2h)^(t mod h) for the lane stage of
 * half-size h = 16 >> k, slot[j][t] = w_n^(t bitrev(j)) for register slot j,
 * reg[q] = w_n^q for q < n (the register stages), with w_N = exp(-2 pi i / N)
 * evaluated in FP64 and rounded. */
struct FftTables {
    float2 stage[5][32];
    float2 slot[kFftMaxN1][32];
    float2 reg[kFftMax];
};

__device__ __forceinline__ uint32_t bitrev_bits(uint32_t j, uint32_t bits) {
    return bits ? (__brev(j) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ void fft_tables(FftTables& T, uint32_t n) {
    const uint32_t n1 = n / 32, bits = __ffs(n1) - 1;
    auto w = [&](uint32_t q) {
        double sn, cn;
        sincospi(-2.0 * (double)(q & (n - 1)) / (double)n, &sn, &cn);
        return make_float2((float)cn, (float)sn);
    };
    for (uint32_t q = threadIdx.x; q < n; q += blockDim.x) T.reg[q] = w(q);
    for (uint32_t e = threadIdx.x; e < 5 * 32; e += blockDim.x) {
        const uint32_t k = e / 32, t = e % 32, h = 16u >> k;
        T.stage[k][t] = w((t & (h - 1)) * (n / (2 * h)));
    }
    for (uint32_t e = threadIdx.x; e < n1 * 32; e += blockDim.x) {
        const uint32_t j = e / 32, t = e % 32;
        T.slot[j][t] = w(t * bitrev_bits(j, bits));
    }
}

/* Stages n rows of `cols` consecutive angles (row k at base + k * stride) as
 * (cos, sin) pairs into tile[k * pitch + c], zero past `cols`.  Eight loads
 * per thread are issued before their trig, so the block keeps many loads in
 * flight. */
__device__ __forceinline__ void stage_rows(float2* __restrict__ tile, uint32_t pitch, const float* __restrict__ theta,
                                           uint32_t base, uint32_t stride, uint32_t n, uint32_t cols) {
    constexpr uint32_t kU = 8;
    const uint32_t total = n * kCorrCols;
    for (uint32_t e0 = threadIdx.x; e0 < total; e0 += kU * blockDim.x) {
        float v[kU];
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            const uint32_t e = e0 + u * blockDim.x, k = e / kCorrCols, c = e % kCorrCols;
            v[u] = (e < total && c < cols) ? theta[base + k * stride + c] : 0.0f;
        }
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            const uint32_t e = e0 + u * blockDim.x, k = e / kCorrCols, c = e % kCorrCols;
            if (e >= total) break;
            float sn = 0.0f, cn = 0.0f;
            if (c < cols) __sincosf(v[u], &sn, &cn);
            tile[k * pitch + c] = make_float2(cn, sn);
        }
    }
}

/* Stages n rows of `cols` consecutive angles (row k at base + k * stride)
 * into raw[k * kCorrPitch + c] as they are, zero past `cols`; eight loads
 * per thread in flight. */
__device__ __forceinline__ void stage_raw(float* __restrict__ raw, const float* __restrict__ theta, uint32_t base,
                                          uint32_t stride, uint32_t n, uint32_t cols) {
    constexpr uint32_t kU = 8;
    const uint32_t total = n * kCorrCols;
    for (uint32_t e0 = threadIdx.x; e0 < total; e0 += kU * blockDim.x) {
        float v[kU];
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            const uint32_t e = e0 + u * blockDim.x, k = e / kCorrCols, c = e % kCorrCols;
            v[u] = (e < total && c < cols) ? theta[base + k * stride + c] : 0.0f;
        }
#pragma unroll
        for (uint32_t u = 0; u < kU; ++u) {
            const uint32_t e = e0 + u * blockDim.x, k = e / kCorrCols, c = e % kCorrCols;
            if (e < total) raw[k * kCorrPitch + c] = v[u];
        }
    }
}

/* The spectral route for unit g of task T: for each of its z items (32
 * lines of one row y), the tile [n][kCorrPitch] receives the lines' (cos,
 * sin) and each warp transforms its lines, adding their power spectra into
 * its per-lane sums (FP64); the warps' sums are added in warp order into P[n]
 * (FP64) and out[0 .. n/2] receives the folded form.  The transforms run in
 * FP32: their rounding moves C_z by about 1e-8 on ordered-phase lines,
 * against the 2e-6 agreement held with the FP64 oracle. */
template <uint32_t N1>
__device__ void corr_z_unit(const CorrTask& Tk, const CorrShape& sh, uint32_t g, float* raw, double* rows,
                            const FftTables& T, double* __restrict__ out) {
    constexpr uint32_t n = 32 * N1;
    constexpr uint32_t bits = N1 == 1 ? 0 : (N1 == 2 ? 1 : (N1 == 4 ? 2 : 3));
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t plane = Tk.lx * Tk.ly, q1 = min(sh.nz, (g + 1) * kZGroup);
    /* the warp's power sums, slot j of lane t at rows[warp][j][t] */
    double* pw = rows + warp * n;
#pragma unroll
    for (uint32_t j = 0; j < N1; ++j) pw[j * 32 + lane] = 0.0;
    for (uint32_t item = g * kZGroup; item < q1; ++item) {
        const uint32_t y = item / sh.cy, x0 = (item % sh.cy) * kCorrCols;
        const uint32_t cols = min(kCorrCols, Tk.lx - x0);
        __syncthreads(); /* the previous item's angles are no longer read */
        stage_raw(raw, Tk.theta, y * Tk.lx + x0, plane, n, cols);
        __syncthreads();
        for (uint32_t c = warp; c < cols; c += nwarps) {
            float2 X[N1];
#pragma unroll
            for (uint32_t j = 0; j < N1; ++j) {
                float sn, cn;
                __sincosf(raw[(lane + 32 * j) * kCorrPitch + c], &sn, &cn);
                X[j] = make_float2(cn, sn);
            }
            /* radix-2 decimation in frequency over j in registers (N1-point DFT
             * of the elements lane + 32 j); slot j ends with frequency bitrev(j) */
#pragma unroll
            for (uint32_t h = N1 / 2; h > 0; h >>= 1) {
#pragma unroll
                for (uint32_t j = 0; j < N1; ++j) {
                    if (j & h) continue;
                    const float2 a = X[j], b = X[j + h];
                    const float2 w = T.reg[(j & (h - 1)) * (n / (2 * h))]; /* same entry across the warp */
                    X[j] = make_float2(a.x + b.x, a.y + b.y);
                    X[j + h] = cmulf(make_float2(a.x - b.x, a.y - b.y), w);
                }
            }
#pragma unroll
            for (uint32_t j = 1; j < N1; ++j) X[j] = cmulf(X[j], T.slot[j][lane]);
            /* 32-point decimation-in-frequency FFT across the lanes; lane t
             * ends with frequency index bitrev5(t) */
#pragma unroll
            for (uint32_t k = 0; k < 5; ++k) {
                const uint32_t h = 16u >> k;
                const bool upper = lane & h;
                const float2 w = T.stage[k][lane];
#pragma unroll
                for (uint32_t j = 0; j < N1; ++j) {
                    const float yx = __shfl_xor_sync(0xffffffffu, X[j].x, h);
                    const float yy = __shfl_xor_sync(0xffffffffu, X[j].y, h);
                    const float2 sum = make_float2(X[j].x + yx, X[j].y + yy);
                    const float2 dif = cmulf(make_float2(yx - X[j].x, yy - X[j].y), w);
                    X[j] = upper ? dif : sum;
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < N1; ++j) {
                const double re = (double)X[j].x, im = (double)X[j].y;
                pw[j * 32 + lane] += re * re + im * im;
            }
        }
    }
    /* the unit's spectrum: the warps' sums added in warp order; slot j of
     * lane t is frequency bitrev(j) + N1 bitrev5(t); P takes the angle
     * area, read by no warp any more */
    double* P = reinterpret_cast<double*>(raw);
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < n; q += blockDim.x) {
        const uint32_t j = bitrev_bits(q & (N1 - 1), bits), t = __brev(q / N1) >> 27;
        double a = 0.0;
        for (uint32_t w = 0; w < nwarps; ++w) a += rows[w * n + j * 32 + t];
        P[q] = a;
    }
    __syncthreads();
    /* the folded spectrum F(0) = P(0), F(q) = P(q) + P(n - q), F(n/2) = P(n/2):
     * the lag sums are (1/n) sum_q F(q) cos(2 pi q r / n), formed once per
     * task by the finalize from the units' summed F */
    for (uint32_t q = threadIdx.x; q <= n / 2; q += blockDim.x)
        out[q] = (q == 0 || q == n / 2) ? P[q] : P[q] + P[n - q];
}

/* The task of a spectral unit: the last one whose first unit is at or
 * before it (tasks without units share the next task's zunit0). */
__device__ __forceinline__ const CorrTask& unit_task(const CorrTask* __restrict__ tasks, const CorrTask& one,
                                                    uint32_t n_tasks, uint32_t unit) {
    uint32_t lo = 0, hi = n_tasks;
    while (tasks && hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tasks[mid].zunit0 <= unit) lo = mid;
        else hi = mid;
    }
    return tasks ? tasks[lo] : one;
}

/* The spectral route: blocks loop over the units of all tasks. */
__global__ void __launch_bounds__(kCorrThreads, 3)
    k_corr_zfft(const CorrTask* __restrict__ tasks, CorrTask one, uint32_t n_tasks, uint32_t n_units) {
    extern __shared__ double zsm[]; /* power sums [warps][n], then angles [n][kCorrPitch] */
    __shared__ FftTables tabs;
    double* rows = zsm;
    float* raw = reinterpret_cast<float*>(zsm + (kCorrThreads / 32) * kFftMax);
    uint32_t tab_n = 0; /* the line length the tables hold */
    for (uint32_t unit = blockIdx.x; unit < n_units; unit += gridDim.x) {
        const CorrTask& T = unit_task(tasks, one, n_tasks, unit);
        const CorrShape sh = corr_shape(T.lx, T.ly, T.lz, T.rxy, T.rz);
        const uint32_t n = T.lz, g = unit - T.zunit0;
        if (!sh.spectral || g >= corr_zunits_of(sh)) continue; /* block-uniform; not reached for valid launches */
        if (n != tab_n) {
            __syncthreads(); /* the previous unit's tables are no longer read */
            fft_tables(tabs, n);
            tab_n = n;
        }
        double* out = T.partial + (size_t)(sh.nx + sh.ny + g) * sh.rp;
        switch (n) {
            case 32: corr_z_unit<1>(T, sh, g, raw, rows, tabs, out); break;
            case 64: corr_z_unit<2>(T, sh, g, raw, rows, tabs, out); break;
            case 128: corr_z_unit<4>(T, sh, g, raw, rows, tabs, out); break;
            default: corr_z_unit<8>(T, sh, g, raw, rows, tabs, out); break;
        }
    }
}

/* `tasks` in device memory, or NULL and the single task `one` by value. */
__global__ void __launch_bounds__(kCorrThreads)
    k_corr_lines(const CorrTask* __restrict__ tasks, CorrTask one, uint32_t n_tasks, uint32_t n_items) {
    extern __shared__ float2 tile[]; /* [n][pitch]: one period of each line */
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t item = blockIdx.x; item < n_items; item += gridDim.x) {
        /* the task: the last one whose first item is at or before `item` */
        uint32_t lo = 0, hi = n_tasks;
        while (tasks && hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (tasks[mid].item0 <= item) lo = mid;
            else hi = mid;
        }
        const CorrTask& T = tasks ? tasks[lo] : one;
        const uint32_t lx = T.lx, ly = T.ly, lz = T.lz, plane = lx * ly;
        const CorrShape sh = corr_shape(lx, ly, lz, T.rxy, T.rz);
        const uint32_t local = item - T.item0;
        /* line geometry: n sites per line, `stride` between sites of a line,
         * `cstride` between lines, `cols` lines, first site `base` */
        uint32_t n, stride, cstride, cols, base, rmax;
        if (local < sh.nx) {
            const uint32_t z = local / sh.cx, y0 = (local % sh.cx) * kCorrCols;
            n = lx, stride = 1, cstride = lx, cols = min(kCorrCols, ly - y0), base = z * plane + y0 * lx;
            rmax = T.rxy;
        } else if (local < sh.nx + sh.ny) {
            const uint32_t q = local - sh.nx, z = q / sh.cy, x0 = (q % sh.cy) * kCorrCols;
            n = ly, stride = lx, cstride = 1, cols = min(kCorrCols, lx - x0), base = z * plane + x0;
            rmax = T.rxy;
        } else {
            const uint32_t q = local - sh.nx - sh.ny, y = q / sh.cy, x0 = (q % sh.cy) * kCorrCols;
            n = lz, stride = plane, cstride = 1, cols = min(kCorrCols, lx - x0), base = y * lx + x0;
            rmax = T.rz;
        }
        const float* __restrict__ theta = T.theta;
        if (local >= sh.nx + sh.ny && corr_fft_len(n)) continue; /* k_corr_zfft's item (block-uniform) */
        __syncthreads(); /* the previous item's tile is no longer read */
        const uint32_t pitch = cstride == 1 ? kCorrCols : kCorrPitch;
        if (cstride == 1) {
            stage_rows(tile, pitch, theta, base, stride, n, cols);
        } else {
            /* x lines: consecutive threads take consecutive sites of a row */
            for (uint32_t e = threadIdx.x; e < n * kCorrCols; e += blockDim.x) {
                const uint32_t c = e / n, k = e % n;
                float sn = 0.0f, cn = 0.0f;
                if (c < cols) __sincosf(theta[base + c * cstride + k], &sn, &cn);
                tile[k * pitch + c] = make_float2(cn, sn);
            }
        }
        __syncthreads();
        double* out = T.partial + (size_t)local * sh.rp;
        /* The tile holds one period of each line: the partner of site k at lag
         * r is row (k + r) mod n.  Lags past R in the last group of 8 are
         * computed and dropped. */
        for (uint32_t r0 = 1 + warp * kCorrLags; r0 <= rmax; r0 += nwarps * kCorrLags) {
            /* w[j]: partner of lag r0 + j at the current k */
            float2 w[kCorrLags];
#pragma unroll
            for (uint32_t j = 0; j < kCorrLags; ++j) w[j] = tile[((r0 + j) % n) * pitch + lane];
            /* row of the next partner to load, (k + r0 + 8) mod n, advanced by one per k */
            uint32_t q = (r0 + kCorrLags) % n;
            double tot[kCorrLags];
            float part[kCorrLags];
#pragma unroll
            for (uint32_t j = 0; j < kCorrLags; ++j) {
                tot[j] = 0.0;
                part[j] = 0.0f;
            }
            /* k in groups of 8: the partner of lag r0 + j at k = k0 + kk sits
             * in slot (kk + j) % 8, and slot kk takes the next partner after
             * k, so the ring needs no register moves */
            const uint32_t n8 = n - n % kCorrLags;
            for (uint32_t k0 = 0; k0 < n8; k0 += kCorrLags) {
#pragma unroll
                for (uint32_t kk = 0; kk < kCorrLags; ++kk) {
                    const float2 a = tile[(k0 + kk) * pitch + lane];
#pragma unroll
                    for (uint32_t j = 0; j < kCorrLags; ++j) {
                        const float2 wj = w[(kk + j) % kCorrLags];
                        part[j] = __fmaf_rn(a.y, wj.y, __fmaf_rn(a.x, wj.x, part[j]));
                    }
                    w[kk] = tile[q * pitch + lane];
                    q = q + 1 == n ? 0u : q + 1;
                }
                if ((k0 + kCorrLags) % kCorrRun == 0) {
#pragma unroll
                    for (uint32_t j = 0; j < kCorrLags; ++j) {
                        tot[j] += (double)part[j];
                        part[j] = 0.0f;
                    }
                }
            }
            /* the ring is aligned again (slot j = lag r0 + j); the last n % 8
             * values of k slide it */
            for (uint32_t k = n8; k < n; ++k) {
                const float2 a = tile[k * pitch + lane];
#pragma unroll
                for (uint32_t j = 0; j < kCorrLags; ++j)
                    part[j] = __fmaf_rn(a.y, w[j].y, __fmaf_rn(a.x, w[j].x, part[j]));
#pragma unroll
                for (uint32_t j = 0; j + 1 < kCorrLags; ++j) w[j] = w[j + 1];
                w[kCorrLags - 1] = tile[q * pitch + lane];
                q = q + 1 == n ? 0u : q + 1;
            }
#pragma unroll
            for (uint32_t j = 0; j < kCorrLags; ++j) {
                double v = tot[j] + (double)part[j];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
                if (lane == 0 && r0 + j <= rmax) out[r0 + j - 1] = v;
            }
        }
    }
}

constexpr int kFinThreads = 1024;
constexpr uint32_t kZParts = 8;     /* interleaved partial sums per C_z lag */
constexpr uint32_t kMaxZLags = 400; /* R_z <= corr_ext - L_z < 775 / 2 */

__global__ void __launch_bounds__(kFinThreads) k_corr_finalize(const CorrTask* __restrict__ tasks, CorrTask one) {
    const CorrTask& T = tasks ? tasks[blockIdx.x] : one;
    const uint32_t R = T.rxy, Rz = T.rz, lz = T.lz;
    if (R == 0 && Rz == 0) return;
    const CorrShape sh = corr_shape(T.lx, T.ly, lz, R, Rz);
    const uint32_t items = sh.nx + sh.ny + sh.nz;
    const uint32_t nv = 3 * R + lz * R + Rz;
    const double volume = (double)T.lx * T.ly * lz, area = (double)T.lx * T.ly;
    const double* __restrict__ part = T.partial;
    double* lsx = T.partial + (size_t)items * sh.rp; /* [lz][R] layer sums */
    double* lsy = lsx + (size_t)lz * R;
    __shared__ unsigned long long row_s;
    if (threadIdx.x == 0) row_s = T.count ? *T.count / (T.binsize ? T.binsize : 1) : 0;
    __syncthreads();
    const unsigned long long row = row_s;
    double* bin = (T.bins && row < T.n_bins) ? T.bins + row * nv : nullptr;
    auto emit = [&](uint32_t j, double v) {
        if (T.values) T.values[j] = v;
        if (bin) bin[j] += v;
    };
    for (uint32_t j = threadIdx.x; j < lz * R; j += blockDim.x) {
        const uint32_t z = j / R, r = j % R;
        double a = 0.0, b = 0.0;
        for (uint32_t c = 0; c < sh.cx; ++c) a += part[(size_t)(z * sh.cx + c) * sh.rp + r];
        for (uint32_t c = 0; c < sh.cy; ++c) b += part[(size_t)(sh.nx + z * sh.cy + c) * sh.rp + r];
        lsx[j] = a;
        lsy[j] = b;
        emit(3 * R + j, (a + b) / (2.0 * area));
    }
    __syncthreads(); /* the layer sums are visible to the whole block */
    for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) {
        double sx = 0.0, sy = 0.0;
        for (uint32_t z = 0; z < lz; ++z) {
            sx += lsx[(size_t)z * R + r];
            sy += lsy[(size_t)z * R + r];
        }
        const double cx = sx / volume, cy = sy / volume;
        emit(r, cx);
        emit(R + r, cy);
        emit(2 * R + r, (cx + cy) / 2.0);
    }
    /* C_z: each column of the z items' rows (a lag, or on the spectral route
     * a frequency of the folded spectrum) summed over the items in kZParts
     * interleaved partial sums (items p = q mod kZParts, in order), then the
     * partial sums in order -- the same order whatever the block size, so
     * every launch of a task gives the same bits */
    __shared__ double zpart[kZParts * kMaxZLags];
    const uint32_t zc = sh.spectral ? lz / 2 + 1 : Rz; /* columns */
    const uint32_t zrows = sh.spectral ? corr_zunits_of(sh) : sh.nz; /* rows: units, or items */
    for (uint32_t idx = threadIdx.x; idx < zc * kZParts; idx += blockDim.x) {
        const uint32_t r = idx % zc, q = idx / zc;
        const double* col = part + (size_t)(sh.nx + sh.ny) * sh.rp + r;
        /* in item order; 16 loads in flight before their adds */
        double a = 0.0;
        uint32_t p = q;
        for (; p + 15 * kZParts < zrows; p += 16 * kZParts) {
            double v[16];
#pragma unroll
            for (uint32_t j = 0; j < 16; ++j) v[j] = col[(size_t)(p + j * kZParts) * sh.rp];
#pragma unroll
            for (uint32_t j = 0; j < 16; ++j) a += v[j];
        }
        for (; p < zrows; p += kZParts) a += col[(size_t)p * sh.rp];
        zpart[idx] = a;
    }
    __syncthreads();
    __shared__ double zcol[kMaxZLags];
    for (uint32_t r = threadIdx.x; r < zc; r += blockDim.x) {
        double sz = 0.0;
        for (uint32_t q = 0; q < kZParts; ++q) sz += zpart[q * zc + r];
        zcol[r] = sz;
    }
    /* cos(2 pi m / n) for the n residues m of q * lag, evaluated once each */
    __shared__ double ctab[kFftMax];
    if (sh.spectral)
        for (uint32_t m = threadIdx.x; m < lz; m += blockDim.x) ctab[m] = cospi(2.0 * (double)m / (double)lz);
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < Rz; r += blockDim.x) {
        double sz = zcol[r];
        if (sh.spectral) {
            /* lag r + 1 from the summed folded spectrum, in frequency order */
            const uint32_t n = lz, lag = r + 1;
            sz = 0.0;
            for (uint32_t q = 0; q <= n / 2; ++q) sz += zcol[q] * ctab[(q * lag) % n];
            sz /= (double)n;
        }
        emit(3 * R + lz * R + r, sz / volume);
    }
    __syncthreads();
    if (threadIdx.x == 0 && T.count) *T.count += 1;
}

}  // namespace

uint32_t corr_items(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    const CorrShape s = corr_shape(lx, ly, lz, rxy, rz);
    return s.nx + s.ny + s.nz;
}

size_t corr_partial_doubles(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    const CorrShape s = corr_shape(lx, ly, lz, rxy, rz);
    return (size_t)(s.nx + s.ny + s.nz) * s.rp + 2ull * lz * rxy;
}

uint32_t corr_values(uint32_t lz, uint32_t rxy, uint32_t rz) { return 3 * rxy + lz * rxy + rz; }

uint32_t corr_z_items(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    return corr_shape(lx, ly, lz, rxy, rz).nz;
}

uint32_t corr_z_units(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    return corr_zunits_of(corr_shape(lx, ly, lz, rxy, rz));
}

uint32_t corr_len(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    uint32_t n = 0;
    if (rxy) n = std::max(lx, ly);
    if (rz) n = std::max(n, lz);
    return n;
}

uint32_t corr_ext(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    uint32_t e = 0;
    if (rxy) e = std::max(lx, ly) + rxy;
    if (rz) e = std::max(e, lz + rz);
    return e;
}

bool corr_supports(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz) {
    return (size_t)corr_ext(lx, ly, lz, rxy, rz) * kCorrPitch * sizeof(float2) <= kCorrMaxTile;
}

cudaError_t launch_corr(const CorrTask* tasks_dev, const CorrTask* one, uint32_t n_tasks, uint32_t n_items,
                        uint32_t n_zunits, uint32_t max_len, uint32_t max_r, uint32_t max_nz, int sm_count,
                        cudaStream_t s) {
    /* a warp takes 8 lags per pass: blocks of one or two warps for small
     * radii, so that short lines do not hold idle warps */
    const int line_threads = max_r <= 16 ? 64 : (max_r <= 32 ? 128 : kCorrThreads);
    /* the finalize splits each C_z sum over its z items only when there are
     * many; each lag needs a thread of its own (R_z <= 258 < kFinThreads) */
    const int fin_threads = (max_nz > 64 || max_r > 128) ? kFinThreads : 128;
    if (n_tasks == 0 || (!tasks_dev && (!one || n_tasks != 1))) return cudaErrorInvalidValue;
    const CorrTask by_value = one ? *one : CorrTask{};
    if (n_items > 0) {
        const size_t smem = (size_t)max_len * kCorrPitch * sizeof(float2);
        cudaError_t e = cudaSuccess;
        if (smem > 48 * 1024)
            e = cudaFuncSetAttribute(k_corr_lines, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        const uint32_t grid = std::min<uint32_t>(n_items, 1u << 30);
        k_corr_lines<<<grid, line_threads, smem, s>>>(one ? nullptr : tasks_dev, by_value, n_tasks, n_items);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (n_zunits > 0) {
            /* z items of lines of 32..256 sites: the spectral route */
            const size_t zsmem = (size_t)(kCorrThreads / 32) * kFftMax * sizeof(double) +
                                 (size_t)kFftMax * kCorrPitch * sizeof(float);
            e = cudaFuncSetAttribute(k_corr_zfft, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem);
            if (e != cudaSuccess) return e;
            /* blocks loop over the units, so each computes its twiddle tables
             * once: four per SM (the kernel's occupancy) */
            const uint32_t zgrid = sm_count > 0 ? std::min<uint32_t>(n_zunits, 3u * (uint32_t)sm_count) : n_zunits;
            k_corr_zfft<<<zgrid, kCorrThreads, zsmem, s>>>(one ? nullptr : tasks_dev, by_value, n_tasks, n_zunits);
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    k_corr_finalize<<<n_tasks, fin_threads, 0, s>>>(one ? nullptr : tasks_dev, by_value);
    return cudaGetLastError();
}

}  // namespace slsf
