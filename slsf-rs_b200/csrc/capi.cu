/*
 * C ABI of the library (include/slsf_gpu.h): contexts, tasks, validation with
 * the reference's error strings, and the host side of every launch.
 *
 * Device memory of one task (V = Lx Ly Lz sites):
 *   theta    FP32 [V]          the state, x fastest (src/types.rs:146-149)
 *   jxy, jz  FP32 [Lz]         layer couplings
 *   bonds    u8   [V]          Wolff active-bond bits (+x, +y, +z)
 *   parent   u32  [V]          Wolff union-find forest
 *   partials FP64 [blocks][8]  measurement block sums
 *   result   FP64 [8]          measurement sums
 *   stats    u64  [4]          accepted, cluster sites, clusters, error bits
 *   bins     FP64 [n_bins][12] batched-engine measurement bins
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/slsf_gpu.h"
#include "engine.h"
#include "xy_fp32.h"

using slsf::TaskView;

namespace {

thread_local std::string g_error;

int set_error(int code, const std::string& message) {
    g_error = message;
    return code;
}

int cuda_error(cudaError_t e, const char* what) {
    return set_error(SLSF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SLSF_CUDA(call)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_error(e_, #call); \
    } while (0)

const char* kErrTemperature = "temperature T must be positive and finite";
const char* kErrWidth = "proposal_width must be nonnegative and finite";
const char* kErrEven = "red-black Metropolis sweep requires even lattice dimensions";

bool temperature_ok(double t) { return t > 0.0 && std::isfinite(t); }
bool width_ok(double w) { return w >= 0.0 && std::isfinite(w); }

}  // namespace

struct slsf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    uint64_t used = 0;
    uint64_t live_tasks = 0;
    int sm_count = 0;
    /* batched engine scratch */
    TaskView* d_views = nullptr;
    uint32_t views_cap = 0;
    unsigned int* d_queue = nullptr;
};

struct slsf_task {
    slsf_ctx* ctx = nullptr;
    uint32_t lx = 0, ly = 0, lz = 0;
    uint32_t volume = 0;
    double temperature = 0, width = 0;
    uint32_t wolff_steps = 0;
    uint64_t seed = 0;
    uint32_t thermalization = 0, binsize = 1, n_bins = 0;
    uint64_t metro_sweeps = 0, wolff_done = 0;
    uint64_t measurements = 0;
    uint64_t bytes = 0;
    bool counted = false; /* registered in ctx->used / live_tasks */
    float* theta = nullptr;
    float* jxy = nullptr;
    float* jz = nullptr;
    uint8_t* bonds = nullptr;
    uint32_t* parent = nullptr;
    double* partials = nullptr;
    double* result = nullptr;
    unsigned int* done = nullptr;
    unsigned long long* stats = nullptr;
    double* bins = nullptr;

    TaskView view() const {
        TaskView v;
        v.theta = theta;
        v.jxy = jxy;
        v.jz = jz;
        v.lx = lx;
        v.ly = ly;
        v.lz = lz;
        v.beta = (float)(1.0 / temperature);
        v.width = (float)width;
        v.wolff_steps = wolff_steps;
        v.seed = seed;
        v.metro_sweeps = metro_sweeps;
        v.wolff_done = wolff_done;
        v.bins = bins;
        v.thermalization = thermalization;
        v.binsize = binsize;
        v.n_bins = n_bins;
        v.stats = stats;
        return v;
    }
};

namespace {

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

uint64_t task_bytes(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t n_bins) {
    const uint64_t v = (uint64_t)lx * ly * lz;
    return align256(4 * v) + 2 * align256(4ull * lz) + align256(v) + align256(4 * v) +
           align256(8ull * 8 * slsf::measure_partial_blocks((uint32_t)v)) + align256(8 * 8) + align256(4) +
           align256(8 * slsf::kStatSlots) + align256(8ull * slsf::kBinCols * n_bins);
}

/* Checks the state a sweep needs, with the reference's messages
 * (src/updates.rs:447-450). */
int check_sweepable(const slsf_task* t) {
    if (!temperature_ok(t->temperature)) return set_error(SLSF_ERR_INVALID, kErrTemperature);
    if (!width_ok(t->width)) return set_error(SLSF_ERR_INVALID, kErrWidth);
    if (t->lx % 2 || t->ly % 2 || t->lz % 2) return set_error(SLSF_ERR_INVALID, kErrEven);
    return SLSF_OK;
}

int read_stats(slsf_task* t, unsigned long long out[slsf::kStatSlots]) {
    SLSF_CUDA(cudaMemcpyAsync(out, t->stats, sizeof(unsigned long long) * slsf::kStatSlots,
                              cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    if (out[slsf::kStatError])
        return set_error(SLSF_ERR_TIMEOUT, "a bounded device loop hit its iteration limit");
    return SLSF_OK;
}

int zero_stats(slsf_task* t) {
    SLSF_CUDA(cudaMemsetAsync(t->stats, 0, sizeof(unsigned long long) * slsf::kStatSlots, t->ctx->stream));
    return SLSF_OK;
}

int bind_device(const slsf_ctx* ctx) {
    SLSF_CUDA(cudaSetDevice(ctx->device));
    return SLSF_OK;
}

}  // namespace

extern "C" {

size_t slsf_last_error(char* buf, size_t len) {
    if (buf && len) {
        const size_t n = std::min(len - 1, g_error.size());
        std::memcpy(buf, g_error.data(), n);
        buf[n] = '\0';
    }
    return g_error.size();
}

const char* slsf_version(void) { return "slsf-b200 0.1.0 (sm_100a)"; }

uint64_t slsf_task_bytes(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t n_bins) {
    return task_bytes(lx, ly, lz, n_bins);
}

int slsf_ctx_create(int device, uint64_t budget_bytes, uint32_t flags, slsf_ctx** out) {
    (void)flags;
    if (!out) return set_error(SLSF_ERR_INVALID, "output handle pointer is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return set_error(SLSF_ERR_CUDA, "no CUDA device is available (this library has no CPU path)");
    if (device < 0 || device >= count) return set_error(SLSF_ERR_INVALID, "device index out of range");
    SLSF_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    SLSF_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return set_error(SLSF_ERR_CUDA, "this library is built for sm_100a (B200)");
    slsf_ctx* ctx = new slsf_ctx;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_error(e, "cudaMemGetInfo");
    }
    ctx->budget = budget_bytes ? budget_bytes : (uint64_t)(0.9 * (double)free_b);
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_queue, sizeof(unsigned int));
    if (e != cudaSuccess) {
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return cuda_error(e, "context set-up");
    }
    *out = ctx;
    return SLSF_OK;
}

int slsf_ctx_destroy(slsf_ctx* ctx) {
    if (!ctx) return SLSF_OK;
    if (ctx->live_tasks)
        return set_error(SLSF_ERR_STATE, "context still owns tasks; destroy them first");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->d_views) cudaFree(ctx->d_views);
    if (ctx->d_queue) cudaFree(ctx->d_queue);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SLSF_OK;
}

int slsf_ctx_memory(const slsf_ctx* ctx, uint64_t* used, uint64_t* budget) {
    if (!ctx) return set_error(SLSF_ERR_INVALID, "context is NULL");
    if (used) *used = ctx->used;
    if (budget) *budget = ctx->budget;
    return SLSF_OK;
}

int slsf_task_create(slsf_ctx* ctx, const slsf_task_desc* d, slsf_task** out) {
    if (!ctx || !d || !out) return set_error(SLSF_ERR_INVALID, "NULL argument");
    *out = nullptr;
    /* ThetaLattice::new (src/types.rs:120-129). */
    if (d->lx == 0) return set_error(SLSF_ERR_INVALID, "L_x must be positive");
    if (d->ly == 0) return set_error(SLSF_ERR_INVALID, "L_y must be positive");
    if (d->lz == 0) return set_error(SLSF_ERR_INVALID, "L_z must be positive");
    const uint64_t volume = (uint64_t)d->lx * d->ly * d->lz;
    if (volume > (1ull << 31)) return set_error(SLSF_ERR_INVALID, "lattice volume exceeds 2^31 sites");
    /* ThetaModel::new (src/model.rs:318-348). */
    if (!d->j_xy || d->n_j_xy != d->lz) return set_error(SLSF_ERR_INVALID, "J_xy_array length must match Lz");
    if (!d->j_z || d->n_j_z != d->lz) return set_error(SLSF_ERR_INVALID, "J_z_array length must match Lz");
    for (uint32_t i = 0; i < d->lz; ++i)
        if (d->j_xy[i] < 0.0 || d->j_z[i] < 0.0)
            return set_error(SLSF_ERR_INVALID, "theta simulation requires nonnegative layer couplings");
    if (d->n_bins > 0 && d->binsize == 0) return set_error(SLSF_ERR_INVALID, "binsize must be positive");
    const uint64_t bytes = task_bytes(d->lx, d->ly, d->lz, d->n_bins);
    if (ctx->used + bytes > ctx->budget)
        return set_error(SLSF_ERR_BUDGET, "task does not fit in the context's device memory budget");
    if (int rc = bind_device(ctx)) return rc;

    slsf_task* t = new slsf_task;
    t->ctx = ctx;
    t->lx = d->lx;
    t->ly = d->ly;
    t->lz = d->lz;
    t->volume = (uint32_t)volume;
    t->temperature = d->temperature;
    t->width = d->proposal_width;
    t->wolff_steps = d->wolff_steps;
    t->seed = d->seed;
    t->thermalization = d->thermalization;
    t->binsize = d->binsize ? d->binsize : 1;
    t->n_bins = d->n_bins;
    t->bytes = bytes;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** p, size_t n) {
        if (e == cudaSuccess) e = cudaMalloc(p, std::max<size_t>(n, 1));
    };
    alloc((void**)&t->theta, 4ull * volume);
    alloc((void**)&t->jxy, 4ull * d->lz);
    alloc((void**)&t->jz, 4ull * d->lz);
    alloc((void**)&t->bonds, volume);
    alloc((void**)&t->parent, 4ull * volume);
    alloc((void**)&t->partials, 8ull * 8 * slsf::measure_partial_blocks(t->volume));
    alloc((void**)&t->result, 8 * 8);
    alloc((void**)&t->done, 4);
    alloc((void**)&t->stats, 8 * slsf::kStatSlots);
    alloc((void**)&t->bins, 8ull * slsf::kBinCols * d->n_bins);
    std::vector<float> jx(d->lz), jzv(d->lz);
    for (uint32_t i = 0; i < d->lz; ++i) {
        jx[i] = (float)d->j_xy[i];
        jzv[i] = (float)d->j_z[i];
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->jxy, jx.data(), 4ull * d->lz, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(t->jz, jzv.data(), 4ull * d->lz, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->theta, 0, 4ull * volume, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->done, 0, 4, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(t->stats, 0, 8 * slsf::kStatSlots, ctx->stream);
    if (e == cudaSuccess && d->n_bins)
        e = cudaMemsetAsync(t->bins, 0, 8ull * slsf::kBinCols * d->n_bins, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        slsf_task_destroy(t);
        return cuda_error(e, "task allocation");
    }
    ctx->used += bytes;
    ctx->live_tasks += 1;
    t->counted = true;
    *out = t;
    return SLSF_OK;
}

int slsf_task_destroy(slsf_task* t) {
    if (!t) return SLSF_OK;
    if (t->ctx) {
        cudaSetDevice(t->ctx->device);
        cudaStreamSynchronize(t->ctx->stream);
    }
    void* ptrs[] = {t->theta, t->jxy, t->jz, t->bonds, t->parent, t->partials, t->result, t->done, t->stats, t->bins};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (t->ctx && t->counted) {
        t->ctx->used -= t->bytes;
        t->ctx->live_tasks -= 1;
    }
    delete t;
    return SLSF_OK;
}

int slsf_task_init_random(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = bind_device(t->ctx)) return rc;
    slsf::launch_init_random(t->theta, t->volume, t->seed, t->ctx->stream);
    SLSF_CUDA(cudaGetLastError());
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_init_cold(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = bind_device(t->ctx)) return rc;
    SLSF_CUDA(cudaMemsetAsync(t->theta, 0, 4ull * t->volume, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_set_angles(slsf_task* t, const float* theta, size_t n) {
    if (!t || !theta) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (n != t->volume) return set_error(SLSF_ERR_INVALID, "angle array length must equal the lattice volume");
    if (int rc = bind_device(t->ctx)) return rc;
    SLSF_CUDA(cudaMemcpyAsync(t->theta, theta, 4ull * n, cudaMemcpyHostToDevice, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_get_angles(slsf_task* t, float* theta, size_t n) {
    if (!t || !theta) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (n != t->volume) return set_error(SLSF_ERR_INVALID, "angle array length must equal the lattice volume");
    if (int rc = bind_device(t->ctx)) return rc;
    SLSF_CUDA(cudaMemcpyAsync(theta, t->theta, 4ull * n, cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_get_counters(const slsf_task* t, uint64_t* metro_sweeps, uint64_t* wolff_steps) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (metro_sweeps) *metro_sweeps = t->metro_sweeps;
    if (wolff_steps) *wolff_steps = t->wolff_done;
    return SLSF_OK;
}

int slsf_task_set_counters(slsf_task* t, uint64_t metro_sweeps, uint64_t wolff_steps) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    t->metro_sweeps = metro_sweeps;
    t->wolff_done = wolff_steps;
    return SLSF_OK;
}

int slsf_task_metropolis_color(slsf_task* t, uint32_t colour, uint8_t* accept_mask, uint64_t* accepted) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (colour > 1) return set_error(SLSF_ERR_INVALID, "colour must be 0 or 1");
    if (int rc = check_sweepable(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    uint8_t* d_mask = nullptr;
    if (accept_mask) {
        SLSF_CUDA(cudaMallocAsync((void**)&d_mask, t->volume, t->ctx->stream));
        SLSF_CUDA(cudaMemsetAsync(d_mask, 0, t->volume, t->ctx->stream));
    }
    if (int rc = zero_stats(t)) return rc;
    slsf::launch_metro_colour(t->view(), t->metro_sweeps, colour, d_mask, t->ctx->stream);
    SLSF_CUDA(cudaGetLastError());
    if (accept_mask) {
        SLSF_CUDA(cudaMemcpyAsync(accept_mask, d_mask, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream));
        SLSF_CUDA(cudaFreeAsync(d_mask, t->ctx->stream));
    }
    unsigned long long st[slsf::kStatSlots];
    if (int rc = read_stats(t, st)) return rc;
    if (accepted) *accepted = st[slsf::kStatAccepted];
    return SLSF_OK;
}

int slsf_task_metropolis_sweep(slsf_task* t, double* acceptance) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_sweepable(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    if (int rc = zero_stats(t)) return rc;
    const TaskView v = t->view();
    slsf::launch_metro_colour(v, t->metro_sweeps, 0, nullptr, t->ctx->stream);
    slsf::launch_metro_colour(v, t->metro_sweeps, 1, nullptr, t->ctx->stream);
    SLSF_CUDA(cudaGetLastError());
    unsigned long long st[slsf::kStatSlots];
    if (int rc = read_stats(t, st)) return rc;
    t->metro_sweeps += 1;
    if (acceptance) *acceptance = (double)st[slsf::kStatAccepted] / (double)t->volume;
    return SLSF_OK;
}

int slsf_task_wolff_step_debug(slsf_task* t, uint8_t* bonds, uint8_t* cluster, float* phi,
                               uint32_t seed_site[3], uint64_t* cluster_size) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    /* wolff_cluster_step_with_theta_scratch validates T (src/updates.rs:558). */
    if (!temperature_ok(t->temperature)) return set_error(SLSF_ERR_INVALID, kErrTemperature);
    if (int rc = bind_device(t->ctx)) return rc;
    if (int rc = zero_stats(t)) return rc;
    uint8_t* d_cluster = nullptr;
    if (cluster) SLSF_CUDA(cudaMallocAsync((void**)&d_cluster, t->volume, t->ctx->stream));
    float phi_h = 0;
    uint32_t site[3] = {0, 0, 0};
    slsf::launch_wolff(t->view(), t->wolff_done, t->bonds, t->parent, d_cluster, t->ctx->stream, &phi_h, site);
    SLSF_CUDA(cudaGetLastError());
    if (bonds) SLSF_CUDA(cudaMemcpyAsync(bonds, t->bonds, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream));
    if (cluster) {
        SLSF_CUDA(cudaMemcpyAsync(cluster, d_cluster, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream));
        SLSF_CUDA(cudaFreeAsync(d_cluster, t->ctx->stream));
    }
    unsigned long long st[slsf::kStatSlots];
    if (int rc = read_stats(t, st)) return rc;
    t->wolff_done += 1;
    if (phi) *phi = phi_h;
    if (seed_site) std::memcpy(seed_site, site, sizeof(site));
    if (cluster_size) *cluster_size = st[slsf::kStatClusterSites];
    return SLSF_OK;
}

int slsf_task_wolff_step(slsf_task* t, uint64_t* cluster_size) {
    return slsf_task_wolff_step_debug(t, nullptr, nullptr, nullptr, nullptr, cluster_size);
}

int slsf_task_sweep(slsf_task* t, uint32_t n_sweeps, slsf_sweep_stats* stats) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_sweepable(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    if (int rc = zero_stats(t)) return rc;
    for (uint32_t s = 0; s < n_sweeps; ++s) {
        TaskView v = t->view();
        slsf::launch_metro_colour(v, t->metro_sweeps, 0, nullptr, t->ctx->stream);
        slsf::launch_metro_colour(v, t->metro_sweeps, 1, nullptr, t->ctx->stream);
        t->metro_sweeps += 1;
        for (uint32_t k = 0; k < t->wolff_steps; ++k) {
            slsf::launch_wolff(v, t->wolff_done, t->bonds, t->parent, nullptr, t->ctx->stream, nullptr, nullptr);
            t->wolff_done += 1;
        }
    }
    SLSF_CUDA(cudaGetLastError());
    unsigned long long st[slsf::kStatSlots];
    if (int rc = read_stats(t, st)) return rc;
    if (stats) {
        stats->sweeps = n_sweeps;
        stats->accepted = st[slsf::kStatAccepted];
        stats->wolff_clusters = (uint64_t)n_sweeps * t->wolff_steps;
        stats->wolff_cluster_sites = st[slsf::kStatClusterSites];
    }
    return SLSF_OK;
}

int slsf_task_measure(slsf_task* t, slsf_observables* out) {
    if (!t || !out) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (int rc = bind_device(t->ctx)) return rc;
    slsf::launch_measure(t->view(), t->partials, t->done, t->result, t->ctx->stream);
    SLSF_CUDA(cudaGetLastError());
    double r[8];
    SLSF_CUDA(cudaMemcpyAsync(r, t->result, sizeof(r), cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    const double v = (double)t->volume;
    /* energy_sum = -(sum of the J cos terms) (src/observables.rs:129-138). */
    out->energy = -(r[2] + r[3] + r[4]) / v;
    out->magnetization_squared = (r[0] * r[0] + r[1] * r[1]) / (v * v);
    out->cos_x = r[2];
    out->cos_y = r[3];
    out->cos_z = r[4];
    out->sin_x = r[5];
    out->sin_y = r[6];
    out->sin_z = r[7];
    return SLSF_OK;
}

int slsf_task_correlations(slsf_task* t, uint32_t rmax_xy, uint32_t rmax_z, double* corr_x,
                           double* corr_y, double* corr_xy, double* corr_xy_by_z, double* corr_z) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    /* Clamp as measure_theta_correlations_with_scratch does (src/observables.rs:180-181). */
    rmax_xy = std::min(std::min(rmax_xy, t->lx / 2), t->ly / 2);
    rmax_z = std::min(rmax_z, t->lz / 2);
    if (rmax_xy == 0 && rmax_z == 0) return SLSF_OK;
    if ((size_t)2 * std::max(t->ly, t->lz) * 32 * sizeof(float) > 200 * 1024)
        return set_error(SLSF_ERR_INVALID, "correlation lines longer than 800 sites are not supported");
    if (int rc = bind_device(t->ctx)) return rc;
    const size_t work_n = slsf::correlation_work_doubles(t->lx, t->ly, t->lz, rmax_xy, rmax_z);
    const size_t nsx = (size_t)t->lz * rmax_xy, nsz = rmax_z;
    double* d = nullptr;
    SLSF_CUDA(cudaMallocAsync((void**)&d, 8 * (work_n + 2 * nsx + nsz + 1), t->ctx->stream));
    double* sx = d + work_n;
    double* sy = sx + nsx;
    double* sz = sy + nsx;
    slsf::launch_correlations(t->view(), rmax_xy, rmax_z, d, work_n, sx, sy, sz, t->ctx->stream);
    cudaError_t e = cudaGetLastError();
    std::vector<double> h(2 * nsx + nsz);
    if (e == cudaSuccess && !h.empty())
        e = cudaMemcpyAsync(h.data(), sx, 8 * h.size(), cudaMemcpyDeviceToHost, t->ctx->stream);
    cudaFreeAsync(d, t->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->ctx->stream);
    if (e != cudaSuccess) return cuda_error(e, "correlations");
    const double volume = (double)t->volume, area = (double)t->lx * t->ly;
    for (uint32_t r = 0; r < rmax_xy; ++r) {
        double sxr = 0, syr = 0;
        for (uint32_t z = 0; z < t->lz; ++z) {
            const double lsx = h[z * rmax_xy + r], lsy = h[nsx + z * rmax_xy + r];
            sxr += lsx;
            syr += lsy;
            if (corr_xy_by_z) corr_xy_by_z[z * rmax_xy + r] = (lsx + lsy) / (2.0 * area);
        }
        if (corr_x) corr_x[r] = sxr / volume;
        if (corr_y) corr_y[r] = syr / volume;
        if (corr_xy) corr_xy[r] = (sxr / volume + syr / volume) / 2.0;
    }
    for (uint32_t r = 0; r < rmax_z; ++r)
        if (corr_z) corr_z[r] = h[2 * nsx + r] / volume;
    return SLSF_OK;
}

int slsf_task_get_bins(const slsf_task* t, double* bins, size_t n_rows, uint64_t* measurements) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (measurements) *measurements = t->measurements;
    if (!bins || n_rows == 0) return SLSF_OK;
    if (n_rows > t->n_bins) return set_error(SLSF_ERR_INVALID, "more bin rows requested than the task keeps");
    if (int rc = bind_device(t->ctx)) return rc;
    SLSF_CUDA(cudaMemcpyAsync(bins, t->bins, 8ull * slsf::kBinCols * n_rows, cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    /* Sums -> means: full bins hold binsize measurements, the last one fewer. */
    for (size_t b = 0; b < n_rows; ++b) {
        const uint64_t first = (uint64_t)b * t->binsize;
        const uint64_t count = t->measurements > first ? std::min<uint64_t>(t->binsize, t->measurements - first) : 0;
        for (int c = 0; c < slsf::kBinCols; ++c)
            bins[b * slsf::kBinCols + c] = count ? bins[b * slsf::kBinCols + c] / (double)count : 0.0;
    }
    return SLSF_OK;
}

int slsf_task_reset_bins(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = bind_device(t->ctx)) return rc;
    if (t->n_bins)
        SLSF_CUDA(cudaMemsetAsync(t->bins, 0, 8ull * slsf::kBinCols * t->n_bins, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    t->measurements = 0;
    return SLSF_OK;
}

int slsf_batch_run(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, uint32_t n_sweeps,
                   slsf_sweep_stats* stats) {
    if (!ctx || (!tasks && n)) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (n == 0 || n_sweeps == 0) return SLSF_OK;
    if (int rc = bind_device(ctx)) return rc;
    std::vector<TaskView> views(n);
    uint32_t max_volume = 0, max_rows = 0, max_lz = 0;
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = tasks[i];
        if (!t || t->ctx != ctx) return set_error(SLSF_ERR_INVALID, "task does not belong to this context");
        if (int rc = check_sweepable(t)) return rc;
        if (!slsf::batched_supports(t->lx, t->ly, t->lz, ctx->device))
            return set_error(SLSF_ERR_INVALID,
                             "lattice not supported by the shared-memory batched kernel (needs L_x <= 32, "
                             "L_x % 4 == 0 and the replica in shared memory)");
        views[i] = t->view();
        max_volume = std::max(max_volume, t->volume);
        max_rows = std::max(max_rows, t->ly * t->lz);
        max_lz = std::max(max_lz, t->lz);
        SLSF_CUDA(cudaMemsetAsync(t->stats, 0, 8 * slsf::kStatSlots, ctx->stream));
    }
    /* Largest replicas first, so the persistent grid ends evenly. */
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t a, size_t b) { return tasks[a]->volume > tasks[b]->volume; });
    std::vector<TaskView> sorted(n);
    for (size_t i = 0; i < n; ++i) sorted[i] = views[order[i]];
    views.swap(sorted);
    if (ctx->views_cap < n) {
        if (ctx->d_views) SLSF_CUDA(cudaFree(ctx->d_views));
        ctx->d_views = nullptr;
        SLSF_CUDA(cudaMalloc(&ctx->d_views, sizeof(TaskView) * n));
        ctx->views_cap = (uint32_t)n;
    }
    SLSF_CUDA(cudaMemcpyAsync(ctx->d_views, views.data(), sizeof(TaskView) * n, cudaMemcpyHostToDevice, ctx->stream));
    SLSF_CUDA(cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned int), ctx->stream));
    SLSF_CUDA(slsf::launch_batched(ctx->d_views, (uint32_t)n, n_sweeps, ctx->d_queue, ctx->device, ctx->stream,
                                   max_volume, max_rows, max_lz));
    std::vector<unsigned long long> st(n * slsf::kStatSlots);
    for (size_t i = 0; i < n; ++i)
        SLSF_CUDA(cudaMemcpyAsync(&st[i * slsf::kStatSlots], tasks[i]->stats, 8 * slsf::kStatSlots,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    int rc = SLSF_OK;
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = tasks[i];
        const uint64_t before = t->metro_sweeps;
        t->metro_sweeps += n_sweeps;
        t->wolff_done += (uint64_t)n_sweeps * t->wolff_steps;
        /* Measurements happen after sweeps past the thermalization count. */
        const uint64_t lo = std::max<uint64_t>(before, t->thermalization);
        if (t->metro_sweeps > lo) t->measurements += t->metro_sweeps - lo;
        const unsigned long long* s = &st[i * slsf::kStatSlots];
        if (s[slsf::kStatError]) rc = set_error(SLSF_ERR_TIMEOUT, "a bounded device loop hit its iteration limit");
        if (stats) {
            stats[i].sweeps = n_sweeps;
            stats[i].accepted = s[slsf::kStatAccepted];
            stats[i].wolff_clusters = s[slsf::kStatClusters];
            stats[i].wolff_cluster_sites = s[slsf::kStatClusterSites];
        }
    }
    return rc;
}

}  // extern "C"
