/*
 * oracle.cpp -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * CPU FP64 restatement of SLSF-rs's update-and-measure path, the checker for
 * the CUDA library and the timed CPU baseline.  Compiled with
 * -ffp-contract=off so that the FP32 emulation in the counter-based forms
 * rounds exactly like the device's explicit round-to-nearest intrinsics.
 */
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../slsf-rs_b200/csrc/xy_fp32.h"

namespace {

thread_local std::string g_error;

int fail(const std::string& message) {
    g_error = message;
    return 1;
}

constexpr double kTwoPi = 2.0 * M_PI;
constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

/* ---------------------------------------------------------------------------
 * FastRng (src/types.rs:16-82) and rand's sampling of it.
 * ------------------------------------------------------------------------- */
inline uint64_t splitmix_next(or_rng* r) {
    r->state += kGamma;
    uint64_t z = r->state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    r->draws += 1;
    return z ^ (z >> 31);
}

/* rand StandardUniform for f64: 53 high bits times 2^-53. */
inline double rng_f64(or_rng* r) { return (double)(splitmix_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* FastRng::try_next_u32 keeps the low 32 bits of the 64-bit word (types.rs:60-62). */
inline uint32_t rng_u32(or_rng* r) { return (uint32_t)splitmix_next(r); }

/* rand's Canon's-method range sampling (random_range(0..n)); ranges that fit in
 * 32 bits are sampled as u32, as rand does for usize. */
uint64_t rng_range(or_rng* r, uint64_t n) {
    if (n - 1 <= 0xFFFFFFFFull) {
        const uint32_t range = (uint32_t)n; /* n == 2^32 wraps to 0: full range */
        if (range == 0) return rng_u32(r);
        const uint64_t m = (uint64_t)rng_u32(r) * range;
        uint32_t result = (uint32_t)(m >> 32);
        const uint32_t lo = (uint32_t)m;
        if (lo > (uint32_t)(0u - range)) {
            const uint64_t m2 = (uint64_t)rng_u32(r) * range;
            const uint32_t new_hi = (uint32_t)(m2 >> 32);
            if ((uint64_t)lo + new_hi > 0xFFFFFFFFull) result += 1;
        }
        return result;
    }
    const uint64_t range = n;
    unsigned __int128 m = (unsigned __int128)splitmix_next(r) * range;
    uint64_t result = (uint64_t)(m >> 64);
    const uint64_t lo = (uint64_t)m;
    if (lo > (0ull - range)) {
        unsigned __int128 m2 = (unsigned __int128)splitmix_next(r) * range;
        const uint64_t new_hi = (uint64_t)(m2 >> 64);
        if (lo + new_hi < lo) result += 1;
    }
    return result;
}

inline double wrap_angle(double t) {
    if (t >= kTwoPi) return t - kTwoPi;
    if (t < 0.0) return t + kTwoPi;
    return t;
}

inline size_t plus(size_t i, size_t l) { return i + 1 < l ? i + 1 : 0; }
inline size_t minus(size_t i, size_t l) { return i > 0 ? i - 1 : l - 1; }

const char* kErrTemperature = "temperature T must be positive and finite";
const char* kErrWidth = "proposal_width must be nonnegative and finite";
const char* kErrEven = "red-black Metropolis sweep requires even lattice dimensions";

bool temperature_ok(double t) { return t > 0.0 && std::isfinite(t); }

/* has_avx512_f64_lanes (src/fast_math.rs:27-37): the reference switches its
 * Metropolis draw order to 8-lane batches when AVX-512F is present. */
int host_batch8() { return __builtin_cpu_supports("avx512f") ? 1 : 0; }
bool width_ok(double w) { return w >= 0.0 && std::isfinite(w); }

}  // namespace

/* ---------------------------------------------------------------------------
 * The model state: ThetaLattice + ThetaScratch + WolffScratch + FastRng
 * (src/types.rs:109-251, src/model.rs:255-271).
 * ------------------------------------------------------------------------- */
struct or_model {
    size_t lx, ly, lz;
    std::vector<double> theta, jxy, jz;
    std::vector<double> sin_t, cos_t;
    std::vector<uint8_t> in_cluster;
    std::vector<size_t> stack_x, stack_y, stack_z;
    std::vector<size_t> cluster_sites;
    or_rng rng;
    double temperature;
    double width;
    size_t wolff_steps;

    size_t volume() const { return lx * ly * lz; }
    size_t idx(size_t x, size_t y, size_t z) const { return x + lx * (y + ly * z); }
    void refresh() {
        for (size_t i = 0; i < theta.size(); ++i) {
            sin_t[i] = std::sin(theta[i]);
            cos_t[i] = std::cos(theta[i]);
        }
    }
};

namespace {

/* local_field (src/updates.rs:169-231). */
inline void local_field(const or_model& m, size_t idx, size_t x, size_t y, size_t z, double& hx,
                        double& hy) {
    const size_t plane = m.lx * m.ly;
    const size_t vol = m.volume();
    const size_t xp = (x + 1 == m.lx) ? idx + 1 - m.lx : idx + 1;
    const size_t xm = (x == 0) ? idx + m.lx - 1 : idx - 1;
    const size_t yp = (y + 1 == m.ly) ? idx + m.lx - plane : idx + m.lx;
    const size_t ym = (y == 0) ? idx + plane - m.lx : idx - m.lx;
    const size_t zp = (z + 1 == m.lz) ? idx + plane - vol : idx + plane;
    const size_t zm_layer = (z == 0) ? m.lz - 1 : z - 1;
    const size_t zm = (z == 0) ? idx + vol - plane : idx - plane;
    const double j_xy = m.jxy[z], j_zp = m.jz[z], j_zm = m.jz[zm_layer];
    hx = j_xy * (m.cos_t[xp] + m.cos_t[xm] + m.cos_t[yp] + m.cos_t[ym]) + j_zp * m.cos_t[zp] +
         j_zm * m.cos_t[zm];
    hy = j_xy * (m.sin_t[xp] + m.sin_t[xm] + m.sin_t[yp] + m.sin_t[ym]) + j_zp * m.sin_t[zp] +
         j_zm * m.sin_t[zm];
}

/* local_metropolis_step_at_unchecked (src/updates.rs:238-271). */
bool step_at(or_model& m, double width, double beta, size_t idx, size_t x, size_t y, size_t z) {
    const double old = m.theta[idx];
    const double nw = wrap_angle(old + width * (2.0 * rng_f64(&m.rng) - 1.0));
    const double ns = std::sin(nw), nc = std::cos(nw);
    double hx, hy;
    local_field(m, idx, x, y, z, hx, hy);
    const double old_e = -(m.cos_t[idx] * hx + m.sin_t[idx] * hy);
    const double de = -(nc * hx + ns * hy) - old_e;
    if (de <= 0.0 || rng_f64(&m.rng) < std::exp(-de * beta)) {
        m.theta[idx] = nw;
        m.sin_t[idx] = ns;
        m.cos_t[idx] = nc;
        return true;
    }
    return false;
}

/* The batched transcendental functions of the 8- and 4-lane Metropolis
 * batches (src/fast_math.rs:3-25).  The oracle evaluates them lane by lane
 * with glibc's scalar sin, cos and exp.  The timed CPU baseline compiles this
 * file a second time with OR_SIMD_BASELINE (baseline_simd.cpp), which
 * supplies the same three functions on glibc's vector math library, as the
 * reference calls sleef's vector functions there. */
#ifndef OR_SIMD_BASELINE
template <int LANES>
inline void batch_sincos(const double* x, double* s, double* c) {
    for (int lane = 0; lane < LANES; ++lane) {
        s[lane] = std::sin(x[lane]);
        c[lane] = std::cos(x[lane]);
    }
}
template <int LANES>
inline void batch_exp(const double* x, double* y) {
    for (int lane = 0; lane < LANES; ++lane) y[lane] = std::exp(x[lane]);
}
#endif

/* metropolis_accept_probabilities (src/updates.rs:21-53): the uphill lanes'
 * arguments are packed; with at least 3 of 8 (2 of 4) uphill lanes the packed
 * exp runs, otherwise the scalar exp per uphill lane. */
template <int LANES>
inline void accept_probabilities(const double* de, double beta, double* prob) {
    double arg[LANES] = {0};
    int lane_of[LANES];
    int uphill = 0;
    for (int lane = 0; lane < LANES; ++lane) {
        prob[lane] = 1.0;
        if (de[lane] > 0.0) {
            arg[uphill] = -de[lane] * beta;
            lane_of[uphill] = lane;
            ++uphill;
        }
    }
    const int min_uphill = LANES == 8 ? 3 : (LANES == 4 ? 2 : LANES);
    if (uphill >= min_uphill) {
        double packed[LANES];
        batch_exp<LANES>(arg, packed);
        for (int k = 0; k < uphill; ++k) prob[lane_of[k]] = packed[k];
    } else {
        for (int k = 0; k < uphill; ++k) prob[lane_of[k]] = std::exp(arg[k]);
    }
}

/* local_metropolis_step_x_batch (src/updates.rs:302-356): proposals for all
 * lanes first, then the accept draws in lane order, each only when the lane
 * is uphill (the `||` short-circuit at :349). */
template <int LANES>
size_t step_batch(or_model& m, double width, double beta, size_t x0, size_t y, size_t z) {
    size_t idxs[LANES];
    double nw[LANES], hx[LANES], hy[LANES], old_e[LANES], ns[LANES], nc[LANES], de[LANES];
    for (int lane = 0; lane < LANES; ++lane) {
        const size_t x = x0 + 2 * lane;
        const size_t idx = m.idx(x, y, z);
        idxs[lane] = idx;
        nw[lane] = wrap_angle(m.theta[idx] + width * (2.0 * rng_f64(&m.rng) - 1.0));
        local_field(m, idx, x, y, z, hx[lane], hy[lane]);
        old_e[lane] = -(m.cos_t[idx] * hx[lane] + m.sin_t[idx] * hy[lane]);
    }
    batch_sincos<LANES>(nw, ns, nc);
    for (int lane = 0; lane < LANES; ++lane) de[lane] = -(nc[lane] * hx[lane] + ns[lane] * hy[lane]) - old_e[lane];
    double prob[LANES];
    accept_probabilities<LANES>(de, beta, prob);
    size_t accepted = 0;
    for (int lane = 0; lane < LANES; ++lane) {
        if (de[lane] <= 0.0 || rng_f64(&m.rng) < prob[lane]) {
            m.theta[idxs[lane]] = nw[lane];
            m.sin_t[idxs[lane]] = ns[lane];
            m.cos_t[idxs[lane]] = nc[lane];
            ++accepted;
        }
    }
    return accepted;
}

/* metropolis_sweep_with_scratch (src/updates.rs:440-486). */
int metropolis_sweep(or_model& m, int use_batch8, double* acceptance) {
    if (!temperature_ok(m.temperature)) return fail(kErrTemperature);
    if (!width_ok(m.width)) return fail(kErrWidth);
    if (m.lx % 2 || m.ly % 2 || m.lz % 2) return fail(kErrEven);
    const double beta = 1.0 / m.temperature;
    size_t accepted = 0;
    for (size_t parity = 0; parity < 2; ++parity) {
        for (size_t z = 0; z < m.lz; ++z) {
            for (size_t y = 0; y < m.ly; ++y) {
                size_t x = (parity + y + z) & 1;
                if (use_batch8) {
                    while (x + 14 < m.lx) {
                        accepted += step_batch<8>(m, m.width, beta, x, y, z);
                        x += 16;
                    }
                }
                while (x + 6 < m.lx) {
                    accepted += step_batch<4>(m, m.width, beta, x, y, z);
                    x += 8;
                }
                while (x < m.lx) {
                    accepted += step_at(m, m.width, beta, m.idx(x, y, z), x, y, z) ? 1 : 0;
                    x += 2;
                }
            }
        }
    }
    if (acceptance) *acceptance = (double)accepted / (double)m.volume();
    return 0;
}

/* wolff_cluster_step_with_theta_scratch (src/updates.rs:551-620) with the
 * neighbour order of the neighbors! macro (:131-167). */
int wolff_step(or_model& m, size_t* cluster_size) {
    if (!temperature_ok(m.temperature)) return fail(kErrTemperature);
    const double beta = 1.0 / m.temperature;
    const double phi = kTwoPi * rng_f64(&m.rng);
    const double sin_phi = std::sin(phi), cos_phi = std::cos(phi);
    const size_t x0 = rng_range(&m.rng, m.lx);
    const size_t y0 = rng_range(&m.rng, m.ly);
    const size_t z0 = rng_range(&m.rng, m.lz);
    m.stack_x.clear();
    m.stack_y.clear();
    m.stack_z.clear();
    const size_t seed_idx = m.idx(x0, y0, z0);
    m.in_cluster[seed_idx] = 1;
    m.stack_x.push_back(x0);
    m.stack_y.push_back(y0);
    m.stack_z.push_back(z0);
    m.cluster_sites.push_back(seed_idx);
    while (!m.stack_x.empty()) {
        const size_t x = m.stack_x.back(), y = m.stack_y.back(), z = m.stack_z.back();
        m.stack_x.pop_back();
        m.stack_y.pop_back();
        m.stack_z.pop_back();
        const size_t idx = m.idx(x, y, z);
        const double ri = m.cos_t[idx] * cos_phi + m.sin_t[idx] * sin_phi;
        const size_t xp = plus(x, m.lx), xm = minus(x, m.lx);
        const size_t yp = plus(y, m.ly), ym = minus(y, m.ly);
        const size_t zp = plus(z, m.lz), zm = minus(z, m.lz);
        const size_t nx[6] = {xp, xm, x, x, x, x};
        const size_t ny[6] = {y, y, yp, ym, y, y};
        const size_t nz[6] = {z, z, z, z, zp, zm};
        const double coupling[6] = {m.jxy[z], m.jxy[z], m.jxy[z], m.jxy[z], m.jz[z], m.jz[zm]};
        for (int k = 0; k < 6; ++k) {
            const size_t n = m.idx(nx[k], ny[k], nz[k]);
            if (m.in_cluster[n]) continue;
            const double rj = m.cos_t[n] * cos_phi + m.sin_t[n] * sin_phi;
            if (coupling[k] * ri * rj <= 0.0) continue;
            const double p = 1.0 - std::exp(std::min(0.0, -2.0 * beta * coupling[k] * ri * rj));
            if (rng_f64(&m.rng) < p) {
                m.in_cluster[n] = 1;
                m.stack_x.push_back(nx[k]);
                m.stack_y.push_back(ny[k]);
                m.stack_z.push_back(nz[k]);
                m.cluster_sites.push_back(n);
            }
        }
    }
    const size_t size = m.cluster_sites.size();
    for (size_t idx : m.cluster_sites) {
        const double nt = wrap_angle(2.0 * phi + M_PI - m.theta[idx]);
        m.theta[idx] = nt;
        m.sin_t[idx] = std::sin(nt);
        m.cos_t[idx] = std::cos(nt);
        m.in_cluster[idx] = 0;
    }
    m.cluster_sites.clear();
    if (cluster_size) *cluster_size = size;
    return 0;
}

/* measure_theta_observables_with_scratch (src/observables.rs:80-154) over
 * cached trig arrays. */
void observables_from_trig(size_t lx, size_t ly, size_t lz, const double* s, const double* c,
                           const double* jxy, const double* jz, or_obs* out) {
    double e = 0, mx = 0, my = 0, cx = 0, cy = 0, cz = 0, sx = 0, sy = 0, sz = 0;
    for (size_t z = 0; z < lz; ++z) {
        for (size_t y = 0; y < ly; ++y) {
            for (size_t x = 0; x < lx; ++x) {
                const size_t i = x + lx * (y + ly * z);
                const double ci = c[i], si = s[i];
                mx += ci;
                my += si;
                const size_t ix = plus(x, lx) + lx * (y + ly * z);
                const size_t iy = x + lx * (plus(y, ly) + ly * z);
                const size_t iz = x + lx * (y + ly * plus(z, lz));
                const double dxc = ci * c[ix] + si * s[ix], dxs = si * c[ix] - ci * s[ix];
                const double dyc = ci * c[iy] + si * s[iy], dys = si * c[iy] - ci * s[iy];
                const double dzc = ci * c[iz] + si * s[iz], dzs = si * c[iz] - ci * s[iz];
                const double jcx = jxy[z] * dxc, jcy = jxy[z] * dyc, jcz = jz[z] * dzc;
                cx += jcx;
                cy += jcy;
                cz += jcz;
                sx += jxy[z] * dxs;
                sy += jxy[z] * dys;
                sz += jz[z] * dzs;
                e -= jcx + jcy + jcz;
            }
        }
    }
    const double v = (double)(lx * ly * lz);
    out->energy = e / v;
    out->magnetization_squared = (mx * mx + my * my) / (v * v);
    out->cos_x = cx;
    out->cos_y = cy;
    out->cos_z = cz;
    out->sin_x = sx;
    out->sin_y = sy;
    out->sin_z = sz;
}

/* measure_theta_correlations_with_scratch (src/observables.rs:166-265);
 * the 8-lane SIMD dot of :13-43 is a plain loop here. */
void correlations_from_trig(size_t lx, size_t ly, size_t lz, const double* s, const double* c,
                            size_t rxy, size_t rz, double* corr_x, double* corr_y,
                            double* corr_xy, double* corr_xy_by_z, double* corr_z) {
    const double volume = (double)(lx * ly * lz);
    const double area = (double)(lx * ly);
    auto dot = [&](size_t a, size_t b, size_t len) {
        double sum = 0.0;
        for (size_t i = 0; i < len; ++i) sum += c[a + i] * c[b + i] + s[a + i] * s[b + i];
        return sum;
    };
    for (size_t r = 1; r <= rxy; ++r) {
        double sx = 0, sy = 0;
        for (size_t z = 0; z < lz; ++z) {
            const size_t zb = lx * ly * z;
            double lsx = 0, lsy = 0;
            for (size_t y = 0; y < ly; ++y) {
                const size_t row = zb + lx * y;
                lsx += dot(row, row + r, lx - r);
                lsx += dot(row + lx - r, row, r);
                lsy += dot(row, zb + lx * ((y + r) % ly), lx);
            }
            sx += lsx;
            sy += lsy;
            if (corr_xy_by_z) corr_xy_by_z[z * rxy + (r - 1)] = (lsx + lsy) / (2.0 * area);
        }
        if (corr_x) corr_x[r - 1] = sx / volume;
        if (corr_y) corr_y[r - 1] = sy / volume;
        if (corr_xy) corr_xy[r - 1] = (sx / volume + sy / volume) / 2.0;
    }
    for (size_t r = 1; r <= rz; ++r) {
        double sz = 0;
        for (size_t z = 0; z < lz; ++z) {
            const size_t zb = lx * ly * z, zs = lx * ly * ((z + r) % lz);
            for (size_t y = 0; y < ly; ++y) sz += dot(zb + lx * y, zs + lx * y, lx);
        }
        if (corr_z) corr_z[r - 1] = sz / volume;
    }
}

void trig_of(size_t n, const double* theta, std::vector<double>& s, std::vector<double>& c) {
    s.resize(n);
    c.resize(n);
    for (size_t i = 0; i < n; ++i) {
        s[i] = std::sin(theta[i]);
        c[i] = std::cos(theta[i]);
    }
}

double mean_of(const std::vector<double>& x) {
    double s = 0;
    for (double v : x) s += v;
    return s / (double)x.size();
}

double mean_square_of(const std::vector<double>& x) {
    double s = 0;
    for (double v : x) s += v * v;
    return s / (double)x.size();
}

double sample_std(const std::vector<double>& x) {
    if (x.size() <= 1) return 0.0;
    const double avg = mean_of(x);
    double v = 0;
    for (double e : x) v += (e - avg) * (e - avg);
    return std::sqrt(v / (double)(x.size() - 1));
}

}  // namespace

extern "C" {

/* ---- FastRng ---- */
void or_rng_seed(or_rng* rng, uint64_t seed) {
    rng->seed = seed;
    rng->state = seed;
    rng->draws = 0;
}

void or_rng_set_position(or_rng* rng, uint64_t position) {
    rng->state = rng->seed + kGamma * position;
    rng->draws = position;
}

uint64_t or_rng_next_u64(or_rng* rng) { return splitmix_next(rng); }
double or_rng_f64(or_rng* rng) { return rng_f64(rng); }
int or_rng_bool(or_rng* rng) { return (int32_t)rng_u32(rng) < 0 ? 1 : 0; }
uint64_t or_rng_range(or_rng* rng, uint64_t n) { return rng_range(rng, n); }

const char* or_last_error(void) { return g_error.c_str(); }

/* ---- scalar helpers ---- */
double or_wrap_angle(double theta) { return wrap_angle(theta); }

double or_wolff_add_probability(double beta, double coupling, double ri, double rj) {
    return 1.0 - std::exp(std::min(0.0, -2.0 * beta * coupling * ri * rj));
}

double or_wolff_reflect_angle(double theta, double phi) { return wrap_angle(2.0 * phi + M_PI - theta); }

int or_validate_temperature(double temperature) {
    return temperature_ok(temperature) ? 0 : fail(kErrTemperature);
}

int or_validate_proposal_width(double width) { return width_ok(width) ? 0 : fail(kErrWidth); }

/* ---- initialisation (src/initialization.rs:5-62) ---- */
int or_two_point_disorder(double* values, size_t n, double mean, double delta, or_rng* rng,
                          const char* name) {
    if (delta < 0.0) return fail(std::string("\xce\xb4") + name + " must be nonnegative");
    const double lower = mean - delta, upper = mean + delta;
    if (lower < 0.0)
        return fail(std::string("two-point layer disorder requires ") + name + "_mean - \xce\xb4" +
                    name + " >= 0");
    if (delta == 0.0) {
        for (size_t i = 0; i < n; ++i) values[i] = mean;
    } else {
        for (size_t i = 0; i < n; ++i) values[i] = or_rng_bool(rng) ? upper : lower;
    }
    return 0;
}

/* Uniform layer disorder lo + (hi - lo) u, u from FastRng(seed) in layer
 * order: the "J_z(z) uniform [0.5, 1.5] per layer from seed" workloads. */
void or_uniform_disorder(double* values, size_t n, double lo, double hi, uint64_t seed) {
    or_rng r;
    or_rng_seed(&r, seed);
    for (size_t i = 0; i < n; ++i) values[i] = lo + (hi - lo) * rng_f64(&r);
}

void or_init_angles(double* theta, size_t n, int cold, or_rng* rng) {
    for (size_t i = 0; i < n; ++i) theta[i] = cold ? 0.0 : kTwoPi * rng_f64(rng);
}

/* ---- observables on an FP64 lattice ---- */
double or_measure_energy(size_t lx, size_t ly, size_t lz, const double* th, const double* jxy,
                         const double* jz) {
    double e = 0;
    for (size_t z = 0; z < lz; ++z)
        for (size_t y = 0; y < ly; ++y)
            for (size_t x = 0; x < lx; ++x) {
                const double t = th[x + lx * (y + ly * z)];
                e -= jxy[z] * std::cos(t - th[plus(x, lx) + lx * (y + ly * z)]);
                e -= jxy[z] * std::cos(t - th[x + lx * (plus(y, ly) + ly * z)]);
                e -= jz[z] * std::cos(t - th[x + lx * (y + ly * plus(z, lz))]);
            }
    return e / (double)(lx * ly * lz);
}

double or_magnetization_squared(size_t n, const double* theta) {
    double mx = 0, my = 0;
    for (size_t i = 0; i < n; ++i) {
        mx += std::cos(theta[i]);
        my += std::sin(theta[i]);
    }
    return (mx * mx + my * my) / ((double)n * (double)n);
}

void or_helicity_sums(size_t lx, size_t ly, size_t lz, const double* th, const double* jxy,
                      const double* jz, double out[6]) {
    double cx = 0, cy = 0, cz = 0, sx = 0, sy = 0, sz = 0;
    for (size_t z = 0; z < lz; ++z)
        for (size_t y = 0; y < ly; ++y)
            for (size_t x = 0; x < lx; ++x) {
                const double t = th[x + lx * (y + ly * z)];
                const double dx = t - th[plus(x, lx) + lx * (y + ly * z)];
                const double dy = t - th[x + lx * (plus(y, ly) + ly * z)];
                const double dz = t - th[x + lx * (y + ly * plus(z, lz))];
                cx += jxy[z] * std::cos(dx);
                cy += jxy[z] * std::cos(dy);
                cz += jz[z] * std::cos(dz);
                sx += jxy[z] * std::sin(dx);
                sy += jxy[z] * std::sin(dy);
                sz += jz[z] * std::sin(dz);
            }
    out[0] = cx;
    out[1] = cy;
    out[2] = cz;
    out[3] = sx;
    out[4] = sy;
    out[5] = sz;
}

int or_helicity_modulus(size_t lx, size_t ly, size_t lz, const double* th, const double* jxy,
                        const double* jz, double temperature, double out[3]) {
    if (!temperature_ok(temperature)) return fail(kErrTemperature);
    const double v = (double)(lx * ly * lz), beta = 1.0 / temperature;
    double h[6];
    or_helicity_sums(lx, ly, lz, th, jxy, jz, h);
    for (int k = 0; k < 3; ++k) out[k] = h[k] / v - beta * h[k + 3] * h[k + 3] / v;
    return 0;
}

void or_measure_observables(size_t lx, size_t ly, size_t lz, const double* theta,
                            const double* jxy, const double* jz, or_obs* out) {
    std::vector<double> s, c;
    trig_of(lx * ly * lz, theta, s, c);
    observables_from_trig(lx, ly, lz, s.data(), c.data(), jxy, jz, out);
}

void or_measure_correlations(size_t lx, size_t ly, size_t lz, const double* theta, long rmax,
                             long rmax_xy, long rmax_z, double* corr_x, double* corr_y,
                             double* corr_xy, double* corr_xy_by_z, double* corr_z,
                             size_t eff[2]) {
    const size_t req_xy = rmax_xy >= 0 ? (size_t)rmax_xy
                          : rmax >= 0  ? (size_t)rmax
                                       : std::min(lx / 2, ly / 2);
    const size_t req_z = rmax_z >= 0 ? (size_t)rmax_z : rmax >= 0 ? (size_t)rmax : lz / 2;
    const size_t rxy = std::min(std::min(req_xy, lx / 2), ly / 2);
    const size_t rz = std::min(req_z, lz / 2);
    std::vector<double> s, c;
    trig_of(lx * ly * lz, theta, s, c);
    correlations_from_trig(lx, ly, lz, s.data(), c.data(), rxy, rz, corr_x, corr_y, corr_xy,
                           corr_xy_by_z, corr_z);
    eff[0] = rxy;
    eff[1] = rz;
}

/* ---- the model ---- */
int or_model_new(size_t lx, size_t ly, size_t lz, const double* jxy, size_t n_jxy,
                 const double* jz, size_t n_jz, double temperature, double width,
                 size_t wolff_steps, uint64_t seed, or_model** out) {
    /* ThetaLattice::new (src/types.rs:120-138), ThetaModel::new (src/model.rs:314-371). */
    if (lx == 0) return fail("L_x must be positive");
    if (ly == 0) return fail("L_y must be positive");
    if (lz == 0) return fail("L_z must be positive");
    if (n_jxy != lz) return fail("J_xy_array length must match Lz");
    if (n_jz != lz) return fail("J_z_array length must match Lz");
    for (size_t i = 0; i < lz; ++i)
        if (jxy[i] < 0.0 || jz[i] < 0.0) return fail("theta simulation requires nonnegative layer couplings");
    or_model* m = new or_model;
    m->lx = lx;
    m->ly = ly;
    m->lz = lz;
    const size_t v = lx * ly * lz;
    m->theta.assign(v, 0.0);
    m->jxy.assign(jxy, jxy + lz);
    m->jz.assign(jz, jz + lz);
    m->sin_t.assign(v, 0.0);
    m->cos_t.assign(v, 1.0);
    m->in_cluster.assign(v, 0);
    or_rng_seed(&m->rng, seed);
    m->temperature = temperature;
    m->width = width;
    m->wolff_steps = wolff_steps;
    m->refresh();
    *out = m;
    return 0;
}

void or_model_free(or_model* m) { delete m; }

void or_model_init(or_model* m, int cold) {
    or_init_angles(m->theta.data(), m->theta.size(), cold, &m->rng);
    m->refresh();
}

void or_model_set_theta(or_model* m, const double* theta) {
    std::memcpy(m->theta.data(), theta, m->theta.size() * sizeof(double));
    m->refresh();
}

void or_model_get_theta(const or_model* m, double* theta) {
    std::memcpy(theta, m->theta.data(), m->theta.size() * sizeof(double));
}

uint64_t or_model_rng_position(const or_model* m) { return m->rng.draws; }

int or_model_metropolis_sweep(or_model* m, int use_batch8, double* acceptance) {
    return metropolis_sweep(*m, use_batch8, acceptance);
}

/* local_metropolis_step (src/updates.rs:273-298, :410-427). */
int or_model_local_metropolis_step(or_model* m, double width, int* accepted) {
    if (!temperature_ok(m->temperature)) return fail(kErrTemperature);
    if (!width_ok(width)) return fail(kErrWidth);
    m->refresh();
    const size_t v = m->volume();
    const size_t idx = rng_range(&m->rng, v);
    const size_t plane = m->lx * m->ly;
    const size_t z = idx / plane, xy = idx - z * plane, y = xy / m->lx, x = xy - y * m->lx;
    *accepted = step_at(*m, width, 1.0 / m->temperature, idx, x, y, z) ? 1 : 0;
    return 0;
}

int or_model_wolff_step(or_model* m, size_t* cluster_size) { return wolff_step(*m, cluster_size); }

/* ThetaModel::sweep (src/model.rs:379-400). */
int or_model_sweep(or_model* m, int use_batch8) {
    double acc;
    if (metropolis_sweep(*m, use_batch8, &acc)) return 1;
    for (size_t k = 0; k < m->wolff_steps; ++k)
        if (wolff_step(*m, nullptr)) return 1;
    return 0;
}

void or_model_measure(const or_model* m, or_obs* out) {
    observables_from_trig(m->lx, m->ly, m->lz, m->sin_t.data(), m->cos_t.data(), m->jxy.data(),
                          m->jz.data(), out);
}

int or_model_run_series(or_model* m, size_t thermalization, size_t sweeps, int use_batch8,
                        double* series, double* acceptance) {
    double acc_sum = 0;
    size_t acc_n = 0;
    for (size_t s = 0; s < thermalization + sweeps; ++s) {
        double acc;
        if (metropolis_sweep(*m, use_batch8, &acc)) return 1;
        acc_sum += acc;
        ++acc_n;
        for (size_t k = 0; k < m->wolff_steps; ++k)
            if (wolff_step(*m, nullptr)) return 1;
        if (s >= thermalization) {
            or_obs o;
            or_model_measure(m, &o);
            double* row = series + (s - thermalization) * OR_SERIES_COLS;
            row[0] = o.energy;
            row[1] = o.energy * o.energy;
            row[2] = o.magnetization_squared;
            row[3] = o.cos_x;
            row[4] = o.cos_y;
            row[5] = o.cos_z;
            row[6] = o.sin_x;
            row[7] = o.sin_y;
            row[8] = o.sin_z;
            row[9] = o.sin_x * o.sin_x;
            row[10] = o.sin_y * o.sin_y;
            row[11] = o.sin_z * o.sin_z;
        }
    }
    if (acceptance) *acceptance = acc_n ? acc_sum / (double)acc_n : 0.0;
    return 0;
}

/* ---- the standalone driver ---- */
double or_blocking_stderr(const double* x, size_t n) {
    /* blocking_stderr (src/simulation.rs:210-226). */
    if (n <= 1) return 0.0;
    std::vector<double> data(x, x + n);
    double err = sample_std(data) / std::sqrt((double)data.size());
    while (data.size() >= 16) {
        const size_t even = data.size() - (data.size() % 2);
        std::vector<double> next;
        next.reserve(even / 2);
        for (size_t i = 0; i < even; i += 2) next.push_back((data[i] + data[i + 1]) / 2.0);
        data.swap(next);
        err = std::max(err, sample_std(data) / std::sqrt((double)data.size()));
    }
    return err;
}

int or_run_theta_simulation(size_t lx, size_t ly, size_t lz, double* theta, double* jxy,
                            double* jz, double j_xy, double j_z_mean, double delta_j_z,
                            double temperature, const or_sim_options* o, or_rng* rng,
                            or_sim_result* res, double* corr_x, double* corr_y, double* corr_xy,
                            double* corr_xy_by_z, double* corr_z) {
    /* run_theta_simulation (src/simulation.rs:13-195). */
    if (o->measure_interval == 0) return fail("measure_interval must be positive");
    if (o->correlation_interval == 0) return fail("correlation_interval must be positive");
    const size_t num_meas = o->measure_sweeps / o->measure_interval;
    if (num_meas == 0)
        return fail("measure_sweeps must include at least one measurement; require measure_sweeps >= measure_interval");
    if (!temperature_ok(temperature)) return fail(kErrTemperature);
    if (!width_ok(o->proposal_width)) return fail(kErrWidth);
    const size_t req_xy = o->correlation_rmax_xy >= 0 ? (size_t)o->correlation_rmax_xy
                          : o->correlation_rmax >= 0  ? (size_t)o->correlation_rmax
                                                      : std::min(lx / 2, ly / 2);
    const size_t req_z = o->correlation_rmax_z >= 0 ? (size_t)o->correlation_rmax_z
                         : o->correlation_rmax >= 0 ? (size_t)o->correlation_rmax
                                                    : lz / 2;
    const size_t rxy = std::min(std::min(req_xy, lx / 2), ly / 2);
    const size_t rz = std::min(req_z, lz / 2);

    /* initialize_disorder (src/initialization.rs:33-46). */
    for (size_t i = 0; i < lz; ++i) jxy[i] = j_xy;
    if (or_two_point_disorder(jz, lz, j_z_mean, delta_j_z, rng, "J_z")) return 1;
    for (size_t i = 0; i < lz; ++i)
        if (jxy[i] < 0.0 || jz[i] < 0.0) return fail("theta simulation requires nonnegative layer couplings");
    const size_t v = lx * ly * lz;
    or_init_angles(theta, v, o->init_cold, rng);

    or_model m;
    m.lx = lx;
    m.ly = ly;
    m.lz = lz;
    m.theta.assign(theta, theta + v);
    m.jxy.assign(jxy, jxy + lz);
    m.jz.assign(jz, jz + lz);
    m.sin_t.assign(v, 0.0);
    m.cos_t.assign(v, 0.0);
    m.in_cluster.assign(v, 0);
    m.rng = *rng;
    m.temperature = temperature;
    m.width = o->proposal_width;
    m.wolff_steps = o->wolff_steps;
    m.refresh();

    double acc_sum = 0;
    size_t acc_n = 0;
    for (size_t s = 0; s < o->thermal_sweeps; ++s) {
        double acc;
        if (metropolis_sweep(m, host_batch8(), &acc)) return 1;
        acc_sum += acc;
        ++acc_n;
        for (size_t k = 0; k < o->wolff_steps; ++k)
            if (wolff_step(m, nullptr)) return 1;
    }
    std::vector<double> energy, cx, cy, cz, sx, sy, sz, m2;
    std::vector<double> cxs(rxy, 0.0), cys(rxy, 0.0), cxys(rxy, 0.0), cbz(lz * rxy, 0.0), czs(rz, 0.0);
    std::vector<double> tx(rxy), ty(rxy), txy(rxy), tbz(lz * rxy), tz(rz);
    size_t corr_meas = 0;
    for (size_t step = 1; step <= o->measure_sweeps; ++step) {
        double acc;
        if (metropolis_sweep(m, host_batch8(), &acc)) return 1;
        acc_sum += acc;
        ++acc_n;
        for (size_t k = 0; k < o->wolff_steps; ++k)
            if (wolff_step(m, nullptr)) return 1;
        if (step % o->measure_interval == 0) {
            or_obs ob;
            or_model_measure(&m, &ob);
            energy.push_back(ob.energy);
            cx.push_back(ob.cos_x);
            cy.push_back(ob.cos_y);
            cz.push_back(ob.cos_z);
            sx.push_back(ob.sin_x);
            sy.push_back(ob.sin_y);
            sz.push_back(ob.sin_z);
            m2.push_back(ob.magnetization_squared);
            const size_t idx = energy.size();
            if ((rxy > 0 || rz > 0) && (idx - 1) % o->correlation_interval == 0) {
                correlations_from_trig(lx, ly, lz, m.sin_t.data(), m.cos_t.data(), rxy, rz,
                                       tx.data(), ty.data(), txy.data(), tbz.data(), tz.data());
                for (size_t i = 0; i < rxy; ++i) {
                    cxs[i] += tx[i];
                    cys[i] += ty[i];
                    cxys[i] += txy[i];
                }
                for (size_t i = 0; i < lz * rxy; ++i) cbz[i] += tbz[i];
                for (size_t i = 0; i < rz; ++i) czs[i] += tz[i];
                ++corr_meas;
            }
        }
    }
    const double vol = (double)v, beta = 1.0 / temperature;
    const double msx = mean_of(sx), msy = mean_of(sy), msz = mean_of(sz);
    res->energy = mean_of(energy);
    res->rho_sx = mean_of(cx) / vol - beta * (mean_square_of(sx) - msx * msx) / vol;
    res->rho_sy = mean_of(cy) / vol - beta * (mean_square_of(sy) - msy * msy) / vol;
    res->rho_sz = mean_of(cz) / vol - beta * (mean_square_of(sz) - msz * msz) / vol;
    auto eff = [&](const std::vector<double>& c, const std::vector<double>& s, double ms) {
        std::vector<double> out(c.size());
        for (size_t i = 0; i < c.size(); ++i) out[i] = c[i] / vol - beta * (s[i] * s[i] - ms * s[i]) / vol;
        return out;
    };
    const auto ex = eff(cx, sx, msx), ey = eff(cy, sy, msy), ez = eff(cz, sz, msz);
    res->std_rho_sx = or_blocking_stderr(ex.data(), ex.size());
    res->std_rho_sy = or_blocking_stderr(ey.data(), ey.size());
    res->std_rho_sz = or_blocking_stderr(ez.data(), ez.size());
    res->magnetization_squared = mean_of(m2);
    res->chi = beta * vol * res->magnetization_squared;
    res->acceptance = acc_n ? acc_sum / (double)acc_n : 0.0;
    res->num_measurements = num_meas;
    res->num_correlation_measurements = corr_meas;
    res->n_corr_xy = rxy;
    res->n_corr_z = rz;
    const double norm = corr_meas > 0 ? (double)corr_meas : 1.0;
    for (size_t i = 0; i < rxy; ++i) {
        if (corr_x) corr_x[i] = cxs[i] / norm;
        if (corr_y) corr_y[i] = cys[i] / norm;
        if (corr_xy) corr_xy[i] = cxys[i] / norm;
    }
    for (size_t i = 0; i < lz * rxy; ++i)
        if (corr_xy_by_z) corr_xy_by_z[i] = cbz[i] / norm;
    for (size_t i = 0; i < rz; ++i)
        if (corr_z) corr_z[i] = czs[i] / norm;
    std::memcpy(theta, m.theta.data(), v * sizeof(double));
    *rng = m.rng;
    return 0;
}

/* ---- binning and derived observables ---- */
int or_binned_estimate(const double* samples, size_t n, size_t binsize, double* mean,
                       double* stderr_out, double* bins, size_t* n_bins) {
    /* BinnedEstimate::from_samples, pinned by src/tests.rs:436-446: bins are
     * the means of complete chunks of `binsize` samples; mean over bins; the
     * standard error is the sample standard deviation of the bins over
     * sqrt(#bins). */
    if (binsize == 0 || binsize > n) return fail("binsize is larger than the sample series");
    const size_t nb = n / binsize;
    std::vector<double> b(nb);
    for (size_t k = 0; k < nb; ++k) {
        double s = 0;
        for (size_t i = 0; i < binsize; ++i) s += samples[k * binsize + i];
        b[k] = s / (double)binsize;
    }
    if (bins)
        for (size_t k = 0; k < nb; ++k) bins[k] = b[k];
    if (n_bins) *n_bins = nb;
    *mean = mean_of(b);
    *stderr_out = sample_std(b) / std::sqrt((double)nb);
    return 0;
}

int or_evaluate_derived(const double* bm, size_t nb, double volume, double beta, double out[5][2]) {
    /* register_theta_evaluables (src/model.rs:857-888) with a delete-one
     * jackknife over bins for the errors. bm is [nb][OR_SERIES_COLS]. */
    if (nb == 0) return fail("no bins");
    auto eval = [&](const double* c, double r[5]) {
        r[0] = std::sqrt(c[2]);
        r[1] = beta * volume * c[2];
        r[2] = beta * beta * volume * (c[1] - c[0] * c[0]);
        const double rx = c[3] / volume - beta * (c[9] - c[6] * c[6]) / volume;
        const double ry = c[4] / volume - beta * (c[10] - c[7] * c[7]) / volume;
        r[3] = (rx + ry) / 2.0;
        r[4] = c[5] / volume - beta * (c[11] - c[8] * c[8]) / volume;
    };
    double total[OR_SERIES_COLS] = {0};
    for (size_t k = 0; k < nb; ++k)
        for (int c = 0; c < OR_SERIES_COLS; ++c) total[c] += bm[k * OR_SERIES_COLS + c];
    double full[OR_SERIES_COLS];
    for (int c = 0; c < OR_SERIES_COLS; ++c) full[c] = total[c] / (double)nb;
    double f[5];
    eval(full, f);
    if (nb == 1) {
        for (int q = 0; q < 5; ++q) {
            out[q][0] = f[q];
            out[q][1] = 0.0;
        }
        return 0;
    }
    std::vector<double> jk(nb * 5);
    double jk_mean[5] = {0};
    for (size_t k = 0; k < nb; ++k) {
        double loo[OR_SERIES_COLS];
        for (int c = 0; c < OR_SERIES_COLS; ++c)
            loo[c] = (total[c] - bm[k * OR_SERIES_COLS + c]) / (double)(nb - 1);
        eval(loo, &jk[k * 5]);
        for (int q = 0; q < 5; ++q) jk_mean[q] += jk[k * 5 + q] / (double)nb;
    }
    for (int q = 0; q < 5; ++q) {
        double v = 0;
        for (size_t k = 0; k < nb; ++k) v += (jk[k * 5 + q] - jk_mean[q]) * (jk[k * 5 + q] - jk_mean[q]);
        out[q][0] = f[q];
        out[q][1] = std::sqrt(v * (double)(nb - 1) / (double)nb);
    }
    return 0;
}

/* ---- counter-based forms ---- */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    slsf_u32x4 c;
    c.x = ctr[0];
    c.y = ctr[1];
    c.z = ctr[2];
    c.w = ctr[3];
    const slsf_u32x4 r = slsf_philox4x32_10(c, key[0], key[1]);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
}

void or_keyed_init_angles(size_t n, uint64_t seed, float* theta) {
    for (size_t i = 0; i < n; ++i) {
        const slsf_u32x4 b = slsf_stream(seed, 0, SLSF_PURPOSE_INIT, 0, (uint32_t)(i >> 2));
        const uint32_t words[4] = {b.x, b.y, b.z, b.w};
        theta[i] = slsf_angle_from_word(words[i & 3]);
    }
}

size_t or_keyed_metro_half(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                           const float* jz, float beta, float width, uint64_t seed,
                           uint64_t sweep, int color, double eps_tie, float* theta_out,
                           int8_t* decision, uint8_t* tie, double* accept_prob) {
    const size_t v = lx * ly * lz, plane = lx * ly;
    std::vector<double> s(v), c(v);
    for (size_t i = 0; i < v; ++i) {
        s[i] = std::sin((double)theta[i]);
        c[i] = std::cos((double)theta[i]);
    }
    if (theta_out != theta) std::memcpy(theta_out, theta, v * sizeof(float));
    size_t accepted = 0;
    for (size_t z = 0; z < lz; ++z)
        for (size_t y = 0; y < ly; ++y)
            for (size_t x = 0; x < lx; ++x) {
                const size_t i = x + lx * (y + ly * z);
                if (((x + y + z) & 1) != (size_t)color) {
                    if (decision) decision[i] = -1;
                    if (tie) tie[i] = 0;
                    if (accept_prob) accept_prob[i] = 0.0;
                    continue;
                }
                const size_t h = i >> 1;
                const slsf_u32x4 b = slsf_stream(seed, sweep, SLSF_PURPOSE_METRO, (uint32_t)color, (uint32_t)(h >> 1));
                float u_prop, u_acc;
                slsf_metro_uniforms(b, (uint32_t)(h & 1), &u_prop, &u_acc);
                const float nw = slsf_propose(theta[i], width, u_prop);
                const size_t zm = minus(z, lz);
                const size_t nb[6] = {plus(x, lx) + lx * (y + ly * z), minus(x, lx) + lx * (y + ly * z),
                                      x + lx * (plus(y, ly) + ly * z), x + lx * (minus(y, ly) + ly * z),
                                      x + lx * (y + ly * plus(z, lz)), x + lx * (y + ly * zm)};
                const double jw[6] = {jxy[z], jxy[z], jxy[z], jxy[z], jz[z], jz[zm]};
                double hx = 0, hy = 0;
                for (int k = 0; k < 6; ++k) {
                    hx += jw[k] * c[nb[k]];
                    hy += jw[k] * s[nb[k]];
                }
                (void)plane;
                const double de = -(std::cos((double)nw) * hx + std::sin((double)nw) * hy) + (c[i] * hx + s[i] * hy);
                const double p = de <= 0.0 ? 1.0 : std::exp(-(double)beta * de);
                const bool acc = de <= 0.0 || (double)u_acc < p;
                if (decision) decision[i] = acc ? 1 : 0;
                if (tie) tie[i] = std::fabs((double)u_acc - p) < eps_tie ? 1 : 0;
                if (accept_prob) accept_prob[i] = p;
                if (acc) {
                    theta_out[i] = nw;
                    ++accepted;
                }
            }
    return accepted;
}

void or_keyed_wolff_pick(size_t lx, size_t ly, size_t lz, uint64_t seed, uint64_t sweep,
                         uint32_t step, float* phi, uint32_t site[3]) {
    const slsf_u32x4 b = slsf_stream(seed, sweep, SLSF_PURPOSE_WOLFF_PICK, step, 0);
    *phi = slsf_angle_from_word(b.x);
    site[0] = slsf_range(b.y, (uint32_t)lx);
    site[1] = slsf_range(b.z, (uint32_t)ly);
    site[2] = slsf_range(b.w, (uint32_t)lz);
}

size_t or_cluster_from_bonds(size_t lx, size_t ly, size_t lz, const uint8_t* bonds,
                             size_t seed_idx, uint8_t* cluster) {
    const size_t v = lx * ly * lz;
    std::memset(cluster, 0, v);
    std::vector<size_t> stack{seed_idx};
    cluster[seed_idx] = 1;
    size_t size = 1;
    while (!stack.empty()) {
        const size_t i = stack.back();
        stack.pop_back();
        const size_t x = i % lx, y = (i / lx) % ly, z = i / (lx * ly);
        const size_t nb[6] = {plus(x, lx) + lx * (y + ly * z), minus(x, lx) + lx * (y + ly * z),
                              x + lx * (plus(y, ly) + ly * z), x + lx * (minus(y, ly) + ly * z),
                              x + lx * (y + ly * plus(z, lz)), x + lx * (y + ly * minus(z, lz))};
        /* bond k of site i is bit k of bonds[i] for + directions, and bit k of
         * bonds[neighbour] for - directions. */
        const bool active[6] = {(bonds[i] & 1) != 0, (bonds[nb[1]] & 1) != 0,
                                (bonds[i] & 2) != 0, (bonds[nb[3]] & 2) != 0,
                                (bonds[i] & 4) != 0, (bonds[nb[5]] & 4) != 0};
        for (int k = 0; k < 6; ++k) {
            if (!active[k] || cluster[nb[k]]) continue;
            cluster[nb[k]] = 1;
            ++size;
            stack.push_back(nb[k]);
        }
    }
    return size;
}

size_t or_keyed_wolff(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                      const float* jz, float beta, uint64_t seed, uint64_t sweep, uint32_t step,
                      double eps_tie, uint8_t* bonds, uint8_t* cluster, float* theta_out) {
    const size_t v = lx * ly * lz;
    float phi;
    uint32_t site[3];
    or_keyed_wolff_pick(lx, ly, lz, seed, sweep, step, &phi, site);
    std::vector<double> r(v);
    for (size_t i = 0; i < v; ++i) r[i] = std::cos((double)theta[i] - (double)phi);
    for (size_t z = 0; z < lz; ++z)
        for (size_t y = 0; y < ly; ++y)
            for (size_t x = 0; x < lx; ++x) {
                const size_t i = x + lx * (y + ly * z);
                const slsf_u32x4 b = slsf_stream(seed, sweep, SLSF_PURPOSE_WOLFF_BOND, step, (uint32_t)i);
                const uint32_t w[3] = {b.x, b.y, b.z};
                const size_t nb[3] = {plus(x, lx) + lx * (y + ly * z), x + lx * (plus(y, ly) + ly * z),
                                      x + lx * (y + ly * plus(z, lz))};
                const double jw[3] = {jxy[z], jxy[z], jz[z]};
                uint8_t bits = 0;
                for (int k = 0; k < 3; ++k) {
                    const double prod = jw[k] * r[i] * r[nb[k]];
                    /* try_add_wolff_neighbor (src/updates.rs:537-548): no
                     * activation when J r_i r_j <= 0. */
                    const double p = prod <= 0.0 ? 0.0 : 1.0 - std::exp(-2.0 * (double)beta * prod);
                    const double u = slsf_u24d(w[k]);
                    if (prod > 0.0 && u < p) bits |= (uint8_t)(1u << k);
                    if (std::fabs(u - p) < eps_tie) bits |= (uint8_t)(8u << k);
                }
                bonds[i] = bits;
            }
    const size_t seed_idx = site[0] + lx * (site[1] + ly * site[2]);
    const size_t size = or_cluster_from_bonds(lx, ly, lz, bonds, seed_idx, cluster);
    if (theta_out) {
        for (size_t i = 0; i < v; ++i) theta_out[i] = cluster[i] ? slsf_reflect(theta[i], phi) : theta[i];
    }
    return size;
}

void or_measure_f32(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                    const float* jz, or_obs* out) {
    const size_t v = lx * ly * lz;
    std::vector<double> s(v), c(v), jx(jxy, jxy + lz), jzz(jz, jz + lz);
    for (size_t i = 0; i < v; ++i) {
        s[i] = std::sin((double)theta[i]);
        c[i] = std::cos((double)theta[i]);
    }
    observables_from_trig(lx, ly, lz, s.data(), c.data(), jx.data(), jzz.data(), out);
}

void or_correlations_f32(size_t lx, size_t ly, size_t lz, const float* theta, size_t rmax_xy,
                         size_t rmax_z, double* corr_x, double* corr_y, double* corr_xy_by_z,
                         double* corr_z) {
    const size_t v = lx * ly * lz;
    std::vector<double> s(v), c(v);
    for (size_t i = 0; i < v; ++i) {
        s[i] = std::sin((double)theta[i]);
        c[i] = std::cos((double)theta[i]);
    }
    correlations_from_trig(lx, ly, lz, s.data(), c.data(), rmax_xy, rmax_z, corr_x, corr_y,
                           nullptr, corr_xy_by_z, corr_z);
}

/* ---- CPU baseline ---- */
int or_bench_tasks(size_t n_tasks, size_t lx, size_t ly, size_t lz, const double* jxy,
                   const double* jz, const double* temperature, double width, size_t wolff_steps,
                   const uint64_t* seeds, size_t sweeps, int threads, double* seconds,
                   double* checksum) {
    if (threads < 1) threads = 1;
    std::atomic<size_t> next{0};
    std::atomic<int> status{0};
    std::vector<double> energies(n_tasks, 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        for (;;) {
            const size_t t = next.fetch_add(1);
            if (t >= n_tasks) return;
            or_model* m = nullptr;
            if (or_model_new(lx, ly, lz, jxy + t * lz, lz, jz + t * lz, lz, temperature[t], width,
                             wolff_steps, seeds[t], &m)) {
                status = 1;
                return;
            }
            or_model_init(m, 0);
            or_obs o{};
            const int batch8 = host_batch8();
            for (size_t s = 0; s < sweeps; ++s) {
                if (or_model_sweep(m, batch8)) {
                    status = 1;
                    break;
                }
                or_model_measure(m, &o);
            }
            energies[t] = o.energy;
            or_model_free(m);
        }
    };
    std::vector<std::thread> pool;
    for (int k = 0; k < threads; ++k) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    const auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    double sum = 0;
    for (double e : energies) sum += e;
    *checksum = sum;
    return status.load();
}

/* ---- independent reference-order tasks with binned series (2-sigma checks) ---- */
int or_series_tasks(size_t n_tasks, size_t lx, size_t ly, size_t lz, const double* jxy,
                    const double* jz, const double* temperature, double width, size_t wolff_steps,
                    const uint64_t* seeds, size_t thermalization, size_t sweeps, size_t n_bins,
                    int threads, double* bin_means) {
    /* Each task is ThetaModel::new + init + the Runner's loop of sweep and
     * measure (src/model.rs:314-442), its measurement stream cut into n_bins
     * bins of equal length (carlo's bins, pinned by src/tests.rs:436-446). */
    if (n_bins == 0 || sweeps % n_bins != 0) return fail("sweeps must be a positive multiple of n_bins");
    if (threads < 1) threads = 1;
    const size_t binsize = sweeps / n_bins;
    std::atomic<size_t> next{0};
    std::atomic<int> status{0};
    auto worker = [&]() {
        std::vector<double> series(sweeps * OR_SERIES_COLS);
        for (;;) {
            const size_t t = next.fetch_add(1);
            if (t >= n_tasks || status.load()) return;
            or_model* m = nullptr;
            if (or_model_new(lx, ly, lz, jxy + t * lz, lz, jz + t * lz, lz, temperature[t], width,
                             wolff_steps, seeds[t], &m)) {
                status = 1;
                return;
            }
            or_model_init(m, 0);
            if (or_model_run_series(m, thermalization, sweeps, host_batch8(), series.data(), nullptr)) {
                status = 1;
                or_model_free(m);
                return;
            }
            or_model_free(m);
            double* out = bin_means + t * n_bins * OR_SERIES_COLS;
            for (size_t b = 0; b < n_bins; ++b)
                for (int c = 0; c < OR_SERIES_COLS; ++c) {
                    double acc = 0;
                    for (size_t i = 0; i < binsize; ++i) acc += series[(b * binsize + i) * OR_SERIES_COLS + c];
                    out[b * OR_SERIES_COLS + c] = acc / (double)binsize;
                }
        }
    };
    std::vector<std::thread> pool;
    for (int k = 0; k < threads; ++k) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
    return status.load();
}

}  // extern "C"
