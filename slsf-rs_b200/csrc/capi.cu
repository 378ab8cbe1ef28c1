/*
 * C ABI of the library (include/slsf_gpu.h): contexts, tasks, validation with
 * the reference's error strings, and the host side of every launch.
 *
 * Device memory of one task (V = Lx Ly Lz sites) is one block from the
 * context's pool (pool.h), carved into 256-byte aligned arrays:
 *   theta    FP32 [V]          the state, x fastest (src/types.rs:146-149)
 *   jxy, jz  FP32 [Lz]         layer couplings
 *   bonds    u8   [V]          Wolff active-bond bits (+x, +y, +z)
 *   parent   u32  [V]          Wolff union-find forest
 *   partials FP64 [blocks][8]  measurement block sums
 *   result   FP64 [8]          measurement sums
 *   done     u32               last-block counter of the measurement
 *   stats    u64  [4]          accepted, cluster sites, clusters, error bits
 *   bins     FP64 [n_bins][12] batched-engine measurement bin sums
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/slsf_gpu.h"
#include "engine.h"
#include "pool.h"
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

#define SLSF_CUDA(call)                                      \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_error(e_, #call); \
    } while (0)

}  // namespace

int slsf::report_error(int code, const std::string& message) { return set_error(code, message); }

namespace {

const char* kErrTemperature = "temperature T must be positive and finite";
const char* kErrWidth = "proposal_width must be nonnegative and finite";
const char* kErrEven = "red-black Metropolis sweep requires even lattice dimensions";
const char* kErrCorrLong = "correlation lines plus lags longer than 775 sites are not supported";
const char* kErrFuse =
    "correlations inside the sweeps need the one-CTA kernel (even L_x <= 32, replica in shared memory) or the grid-wide kernels";
const char* kErrFused = "task measures its correlations inside the batched sweeps (slsf_task_corr_fuse)";

bool temperature_ok(double t) { return t > 0.0 && std::isfinite(t); }
bool width_ok(double w) { return w >= 0.0 && std::isfinite(w); }

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

/* Kernels of one correlation measurement (launch_corr): the line items, the
 * spectral z items when there are z items, and the finalize. */
uint32_t corr_launch_count(uint32_t items, uint32_t z_items) { return items ? (z_items ? 3u : 2u) : 1u; }

/* Side streams for the kernel groups of a batch after the first (group g
 * runs on side[(g - 1) % kSideStreams]); each group has its own work-queue
 * counter. */
constexpr int kSideStreams = 7;

/* Offsets of the arrays inside a task's block. */
struct TaskLayout {
    uint64_t theta, jxy, jz, bonds, parent, partials, result, done, stats, bins, total;
};

TaskLayout layout_of(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t n_bins) {
    const uint64_t v = (uint64_t)lx * ly * lz;
    TaskLayout L;
    uint64_t o = 0;
    L.theta = o;
    o += align256(4 * v);
    L.jxy = o;
    o += align256(4ull * lz);
    L.jz = o;
    o += align256(4ull * lz);
    L.bonds = o;
    o += align256(v);
    L.parent = o;
    o += align256(4 * v);
    L.partials = o;
    o += align256(8ull * 8 * slsf::measure_partial_blocks((uint32_t)v));
    L.result = o;
    o += align256(8 * 8);
    L.done = o;
    o += align256(4);
    L.stats = o;
    o += align256(8 * slsf::kStatSlots);
    L.bins = o;
    o += align256(8ull * slsf::kBinCols * n_bins);
    L.total = o;
    return L;
}

}  // namespace

constexpr size_t kSmallReadBack = 256; /* bytes */

struct slsf_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr; /* own_stream or the caller's */
    uint64_t budget = 0;
    uint64_t used = 0;
    uint64_t live_tasks = 0;
    uint64_t launches = 0;
    uint32_t loop_limit = 0; /* slsf_ctx_set_loop_limit */
    int sm_count = 0;
    slsf::DevicePool pool;
    /* batched engine scratch */
    TaskView* d_views = nullptr;
    TaskView* h_views = nullptr; /* pinned */
    slsf::ResidentCorr* d_rcorr = nullptr; /* fused correlations, parallel to d_views */
    slsf::ResidentCorr* h_rcorr = nullptr; /* pinned */
    unsigned long long* d_batch_stats = nullptr;
    unsigned long long* h_batch_stats = nullptr; /* pinned */
    /* pinned landing area of the single-task calls' small read-backs (stats,
     * observables): a pageable destination would be staged by the driver */
    double* h_small = nullptr;
    uint32_t views_cap = 0;
    unsigned int* d_queue = nullptr; /* one counter per kernel group */
    uint32_t queue_cap = 0;
    /* side streams for the kernel groups of a batch, forked from and joined
     * back into `stream` with events, so that groups that do not fill the
     * GPU alone overlap */
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kSideStreams] = {};
    /* kernel choice per lattice shape (slsf_tune_set / slsf_autotune) */
    std::unordered_map<uint64_t, slsf::KernelChoice> tune;
    std::unordered_map<uint64_t, double> tune_rate; /* site-updates/s measured by slsf_autotune */
    /* bins gather scratch */
    const double** d_bin_src = nullptr;
    const double** h_bin_src = nullptr; /* pinned */
    double* d_bin_out = nullptr;
    double* h_bin_out = nullptr; /* pinned */
    size_t gather_tasks_cap = 0, gather_doubles_cap = 0;
    /* task table of slsf_batch_correlations; the pinned copy is rewritten
     * only after the event says its last upload has been read */
    slsf::CorrTask* d_corr = nullptr;
    slsf::CorrTask* h_corr = nullptr; /* pinned */
    size_t corr_cap = 0;
    cudaEvent_t corr_uploaded = nullptr;
    /* the task list (and set-up generations) the device table holds, so a
     * repeated batch reuses it without an upload */
    std::vector<const slsf_task*> corr_last;
    std::vector<uint64_t> corr_last_gen;
    uint32_t corr_last_items = 0, corr_last_zunits = 0, corr_last_len = 0, corr_last_r = 0, corr_last_nz = 0;
    uint64_t corr_gen = 0; /* slsf_task_corr_setup calls so far */
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
    void* block = nullptr;
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
    slsf_batch* session = nullptr; /* open batch session holding the task's device view */
    /* correlation bins (slsf_task_corr_setup): one pool block holding the
     * launch scratch, the bin sums and the device measurement count */
    void* corr_block = nullptr;
    uint64_t corr_bytes = 0;
    uint32_t corr_rxy = 0, corr_rz = 0, corr_binsize = 1, corr_n_bins = 0;
    uint64_t corr_count = 0; /* host mirror of *corr_count_dev */
    uint64_t corr_gen = 0;   /* the context's set-up count when this set-up was made */
    uint32_t corr_interval = 0; /* slsf_task_corr_fuse: measured inside the batched sweeps every this many */
    double* corr_partial = nullptr;
    double* corr_bins = nullptr;
    unsigned long long* corr_count_dev = nullptr;

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
        v.sweeps = 0;
        v.loop_limit = ctx->loop_limit;
        v.stats = stats;
        return v;
    }
};

namespace {

/* Checks the state a sweep needs, with the reference's messages
 * (src/updates.rs:447-450). */
int check_free(const slsf_task* t);

int check_sweepable(const slsf_task* t) {
    if (int rc = check_free(t)) return rc;
    if (!temperature_ok(t->temperature)) return set_error(SLSF_ERR_INVALID, kErrTemperature);
    if (!width_ok(t->width)) return set_error(SLSF_ERR_INVALID, kErrWidth);
    if (t->lx % 2 || t->ly % 2 || t->lz % 2) return set_error(SLSF_ERR_INVALID, kErrEven);
    return SLSF_OK;
}

/* Calls that change a task's state or counters are refused while an open
 * batch session owns its device view. */
int check_free(const slsf_task* t) {
    if (t->session) return set_error(SLSF_ERR_STATE, "task belongs to an open batch session; close it first");
    return SLSF_OK;
}

int read_stats(slsf_task* t, unsigned long long out[slsf::kStatSlots]) {
    static_assert(sizeof(unsigned long long) * slsf::kStatSlots <= kSmallReadBack, "stats fit the landing area");
    SLSF_CUDA(cudaMemcpyAsync(t->ctx->h_small, t->stats, sizeof(unsigned long long) * slsf::kStatSlots,
                              cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    std::memcpy(out, t->ctx->h_small, sizeof(unsigned long long) * slsf::kStatSlots);
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

/* Grows the batched-engine scratch to hold n views. */
int ensure_batch_capacity(slsf_ctx* ctx, size_t n) {
    if (ctx->views_cap >= n) return SLSF_OK;
    if (ctx->d_views) {
        /* queued launches may still read them, on the main stream or on a
         * side stream that an earlier failed call left unjoined */
        SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < kSideStreams; ++k)
            if (ctx->side[k]) SLSF_CUDA(cudaStreamSynchronize(ctx->side[k]));
    }
    if (ctx->d_views) cudaFree(ctx->d_views);
    if (ctx->h_views) cudaFreeHost(ctx->h_views);
    if (ctx->d_rcorr) cudaFree(ctx->d_rcorr);
    if (ctx->h_rcorr) cudaFreeHost(ctx->h_rcorr);
    if (ctx->d_batch_stats) cudaFree(ctx->d_batch_stats);
    if (ctx->h_batch_stats) cudaFreeHost(ctx->h_batch_stats);
    ctx->d_views = nullptr;
    ctx->h_views = nullptr;
    ctx->d_rcorr = nullptr;
    ctx->h_rcorr = nullptr;
    ctx->d_batch_stats = nullptr;
    ctx->h_batch_stats = nullptr;
    ctx->views_cap = 0;
    const size_t cap = std::max<size_t>(n, 64);
    SLSF_CUDA(cudaMalloc(&ctx->d_views, sizeof(TaskView) * cap));
    SLSF_CUDA(cudaHostAlloc(&ctx->h_views, sizeof(TaskView) * cap, cudaHostAllocDefault));
    SLSF_CUDA(cudaMalloc(&ctx->d_rcorr, sizeof(slsf::ResidentCorr) * cap));
    SLSF_CUDA(cudaHostAlloc(&ctx->h_rcorr, sizeof(slsf::ResidentCorr) * cap, cudaHostAllocDefault));
    SLSF_CUDA(cudaMalloc(&ctx->d_batch_stats, 8 * slsf::kStatSlots * cap));
    SLSF_CUDA(cudaHostAlloc(&ctx->h_batch_stats, 8 * slsf::kStatSlots * cap, cudaHostAllocDefault));
    ctx->views_cap = (uint32_t)cap;
    return SLSF_OK;
}

int ensure_gather_capacity(slsf_ctx* ctx, size_t n, size_t doubles) {
    if (ctx->gather_tasks_cap < n) {
        if (ctx->d_bin_src) cudaFree(ctx->d_bin_src);
        if (ctx->h_bin_src) cudaFreeHost(ctx->h_bin_src);
        ctx->d_bin_src = nullptr;
        ctx->h_bin_src = nullptr;
        ctx->gather_tasks_cap = 0;
        SLSF_CUDA(cudaMalloc(&ctx->d_bin_src, sizeof(double*) * n));
        SLSF_CUDA(cudaHostAlloc(&ctx->h_bin_src, sizeof(double*) * n, cudaHostAllocDefault));
        ctx->gather_tasks_cap = n;
    }
    if (ctx->gather_doubles_cap < doubles) {
        if (ctx->d_bin_out) cudaFree(ctx->d_bin_out);
        if (ctx->h_bin_out) cudaFreeHost(ctx->h_bin_out);
        ctx->d_bin_out = nullptr;
        ctx->h_bin_out = nullptr;
        ctx->gather_doubles_cap = 0;
        SLSF_CUDA(cudaMalloc(&ctx->d_bin_out, 8 * doubles));
        SLSF_CUDA(cudaHostAlloc(&ctx->h_bin_out, 8 * doubles, cudaHostAllocDefault));
        ctx->gather_doubles_cap = doubles;
    }
    return SLSF_OK;
}

/* Bin sums -> means: full bins hold binsize measurements, the last fewer. */
void bin_means(const slsf_task* t, const double* sums, double* out, size_t n_rows) {
    for (size_t b = 0; b < n_rows; ++b) {
        const uint64_t first = (uint64_t)b * t->binsize;
        const uint64_t count =
            t->measurements > first ? std::min<uint64_t>(t->binsize, t->measurements - first) : 0;
        for (int c = 0; c < slsf::kBinCols; ++c)
            out[b * slsf::kBinCols + c] = count ? sums[b * slsf::kBinCols + c] / (double)count : 0.0;
    }
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
    return layout_of(lx, ly, lz, n_bins).total;
}

static void destroy_streams(slsf_ctx* ctx) {
    for (int q = 0; q < kSideStreams; ++q) {
        if (ctx->side[q]) cudaStreamSynchronize(ctx->side[q]);
        if (ctx->side[q]) cudaStreamDestroy(ctx->side[q]);
        if (ctx->join[q]) cudaEventDestroy(ctx->join[q]);
    }
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
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
    size_t free_b = 0, total_b = 0;
    SLSF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    slsf_ctx* ctx = new slsf_ctx;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->budget = budget_bytes ? budget_bytes : (uint64_t)(0.9 * (double)free_b);
    e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaHostAlloc(&ctx->h_small, kSmallReadBack, cudaHostAllocDefault);
    for (int q = 0; q < kSideStreams && e == cudaSuccess; ++q) {
        e = cudaStreamCreateWithFlags(&ctx->side[q], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->join[q], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        destroy_streams(ctx);
        if (ctx->d_queue) cudaFree(ctx->d_queue);
        if (ctx->h_small) cudaFreeHost(ctx->h_small);
        delete ctx;
        return cuda_error(e, "context set-up");
    }
    ctx->stream = ctx->own_stream;
    *out = ctx;
    return SLSF_OK;
}

int slsf_ctx_destroy(slsf_ctx* ctx) {
    if (!ctx) return SLSF_OK;
    if (ctx->live_tasks) return set_error(SLSF_ERR_STATE, "context still owns tasks; destroy them first");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->own_stream);
    void* dev[] = {ctx->d_views, ctx->d_batch_stats, ctx->d_queue, (void*)ctx->d_bin_src, ctx->d_bin_out,
                   ctx->d_rcorr};
    for (void* p : dev)
        if (p) cudaFree(p);
    if (ctx->d_corr) cudaFree(ctx->d_corr);
    void* host[] = {ctx->h_views, ctx->h_batch_stats, (void*)ctx->h_bin_src, ctx->h_bin_out, ctx->h_corr,
                    ctx->h_rcorr, ctx->h_small};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    if (ctx->corr_uploaded) cudaEventDestroy(ctx->corr_uploaded);
    ctx->pool.release();
    destroy_streams(ctx);
    delete ctx;
    return SLSF_OK;
}

int slsf_ctx_memory(const slsf_ctx* ctx, uint64_t* used, uint64_t* budget) {
    if (!ctx) return set_error(SLSF_ERR_INVALID, "context is NULL");
    if (used) *used = ctx->used;
    if (budget) *budget = ctx->budget;
    return SLSF_OK;
}

int slsf_ctx_set_stream(slsf_ctx* ctx, void* stream) {
    if (!ctx) return set_error(SLSF_ERR_INVALID, "context is NULL");
    if (int rc = bind_device(ctx)) return rc;
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return SLSF_OK;
}

int slsf_ctx_set_loop_limit(slsf_ctx* ctx, uint32_t limit) {
    if (!ctx) return set_error(SLSF_ERR_INVALID, "context is NULL");
    ctx->loop_limit = limit;
    return SLSF_OK;
}

int slsf_ctx_launch_count(const slsf_ctx* ctx, uint64_t* launches) {
    if (!ctx || !launches) return set_error(SLSF_ERR_INVALID, "NULL argument");
    *launches = ctx->launches;
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
    const TaskLayout L = layout_of(d->lx, d->ly, d->lz, d->n_bins);
    if (ctx->used + L.total > ctx->budget)
        return set_error(SLSF_ERR_BUDGET, "task does not fit in the context's device memory budget");
    if (int rc = bind_device(ctx)) return rc;

    void* block = nullptr;
    cudaError_t e = ctx->pool.allocate(L.total, &block);
    if (e != cudaSuccess) return cuda_error(e, "device pool allocation");
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
    t->bytes = L.total;
    t->block = block;
    char* b = static_cast<char*>(block);
    t->theta = reinterpret_cast<float*>(b + L.theta);
    t->jxy = reinterpret_cast<float*>(b + L.jxy);
    t->jz = reinterpret_cast<float*>(b + L.jz);
    t->bonds = reinterpret_cast<uint8_t*>(b + L.bonds);
    t->parent = reinterpret_cast<uint32_t*>(b + L.parent);
    t->partials = reinterpret_cast<double*>(b + L.partials);
    t->result = reinterpret_cast<double*>(b + L.result);
    t->done = reinterpret_cast<unsigned int*>(b + L.done);
    t->stats = reinterpret_cast<unsigned long long*>(b + L.stats);
    t->bins = reinterpret_cast<double*>(b + L.bins);
    std::vector<float> jv(2 * (size_t)d->lz);
    for (uint32_t i = 0; i < d->lz; ++i) {
        jv[i] = (float)d->j_xy[i];
        jv[d->lz + i] = (float)d->j_z[i];
    }
    /* theta, jxy and jz are separate 256-byte aligned arrays; zero the whole
     * block, then copy J.  The copy is synchronous: jv is pageable. */
    e = cudaMemsetAsync(block, 0, L.total, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpy(t->jxy, jv.data(), 4ull * d->lz, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->jz, jv.data() + d->lz, 4ull * d->lz, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ctx->pool.free(block, L.total);
        delete t;
        return cuda_error(e, "task set-up");
    }
    ctx->used += L.total;
    ctx->live_tasks += 1;
    *out = t;
    return SLSF_OK;
}

int slsf_task_destroy(slsf_task* t) {
    if (!t) return SLSF_OK;
    if (int rc = check_free(t)) return rc;
    slsf_ctx* ctx = t->ctx;
    cudaSetDevice(ctx->device);
    /* Work queued on the stream may still use the block. */
    cudaStreamSynchronize(ctx->stream);
    if (t->corr_block) {
        ctx->pool.free(t->corr_block, t->corr_bytes);
        ctx->used -= t->corr_bytes;
    }
    ctx->pool.free(t->block, t->bytes);
    ctx->used -= t->bytes;
    ctx->live_tasks -= 1;
    delete t;
    return SLSF_OK;
}

int slsf_task_init_random(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_free(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    slsf::launch_init_random(t->theta, t->volume, t->seed, t->ctx->stream);
    t->ctx->launches += 1;
    SLSF_CUDA(cudaGetLastError());
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_init_cold(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_free(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    SLSF_CUDA(cudaMemsetAsync(t->theta, 0, 4ull * t->volume, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    return SLSF_OK;
}

int slsf_task_set_angles(slsf_task* t, const float* theta, size_t n) {
    if (!t || !theta) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (int rc = check_free(t)) return rc;
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
    if (int rc = check_free(t)) return rc;
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
        /* the bonds array doubles as the mask buffer: one byte per site */
        d_mask = t->bonds;
        SLSF_CUDA(cudaMemsetAsync(d_mask, 0, t->volume, t->ctx->stream));
    }
    if (int rc = zero_stats(t)) return rc;
    slsf::launch_metro_colour(t->view(), t->metro_sweeps, colour, d_mask, t->ctx->stream);
    t->ctx->launches += 1;
    SLSF_CUDA(cudaGetLastError());
    if (accept_mask)
        SLSF_CUDA(cudaMemcpyAsync(accept_mask, d_mask, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream));
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
    t->ctx->launches += 2;
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
    if (int rc = check_free(t)) return rc;
    /* wolff_cluster_step_with_theta_scratch validates T (src/updates.rs:558). */
    if (!temperature_ok(t->temperature)) return set_error(SLSF_ERR_INVALID, kErrTemperature);
    if (int rc = bind_device(t->ctx)) return rc;
    if (int rc = zero_stats(t)) return rc;
    /* The exported cluster mask needs a byte per site of its own; it comes
     * from the pool and goes back after the copy. */
    void* d_cluster = nullptr;
    if (cluster) {
        cudaError_t e = t->ctx->pool.allocate(align256(t->volume), &d_cluster);
        if (e != cudaSuccess) return cuda_error(e, "debug buffer");
    }
    float phi_h = 0;
    uint32_t site[3] = {0, 0, 0};
    t->ctx->launches += slsf::launch_wolff(t->view(), t->wolff_done, t->bonds, t->parent, (uint8_t*)d_cluster,
                                           t->ctx->stream, &phi_h, site, bonds != nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && bonds)
        e = cudaMemcpyAsync(bonds, t->bonds, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream);
    if (e == cudaSuccess && cluster)
        e = cudaMemcpyAsync(cluster, d_cluster, t->volume, cudaMemcpyDeviceToHost, t->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(t->ctx->stream);
    if (d_cluster) t->ctx->pool.free(d_cluster, align256(t->volume));
    if (e != cudaSuccess) return cuda_error(e, "wolff step");
    if (bonds) /* the bond bits only (the kernels mark tile roots in bit 3) */
        for (uint32_t i = 0; i < t->volume; ++i) bonds[i] &= 7u;
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
        t->ctx->launches += 2;
        for (uint32_t k = 0; k < t->wolff_steps; ++k) {
            t->ctx->launches +=
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
    t->ctx->launches += 1;
    SLSF_CUDA(cudaGetLastError());
    double r[8];
    SLSF_CUDA(cudaMemcpyAsync(t->ctx->h_small, t->result, sizeof(r), cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    std::memcpy(r, t->ctx->h_small, sizeof(r));
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
    if (!slsf::corr_supports(t->lx, t->ly, t->lz, rmax_xy, rmax_z)) return set_error(SLSF_ERR_INVALID, kErrCorrLong);
    if (int rc = bind_device(t->ctx)) return rc;
    slsf_ctx* ctx = t->ctx;
    const uint32_t nv = slsf::corr_values(t->lz, rmax_xy, rmax_z);
    const size_t np = slsf::corr_partial_doubles(t->lx, t->ly, t->lz, rmax_xy, rmax_z);
    const size_t off_values = align256(8 * np);
    const size_t bytes = off_values + align256(8ull * nv);
    void* dv = nullptr;
    cudaError_t e = ctx->pool.allocate(bytes, &dv);
    if (e != cudaSuccess) return cuda_error(e, "correlation scratch");
    char* d = static_cast<char*>(dv);
    slsf::CorrTask ct = {t->theta, t->lx, t->ly, t->lz, rmax_xy, rmax_z, 0, 1, 0,
                         reinterpret_cast<double*>(d), reinterpret_cast<double*>(d + off_values), nullptr, nullptr};
    std::vector<double> h(nv);
    const uint32_t items = slsf::corr_items(t->lx, t->ly, t->lz, rmax_xy, rmax_z);
    e = slsf::launch_corr(nullptr, &ct, 1, items, slsf::corr_z_units(t->lx, t->ly, t->lz, rmax_xy, rmax_z),
                          slsf::corr_len(t->lx, t->ly, t->lz, rmax_xy, rmax_z), std::max(rmax_xy, rmax_z),
                          slsf::corr_z_items(t->lx, t->ly, t->lz, rmax_xy, rmax_z), ctx->sm_count, ctx->stream);
    ctx->launches += corr_launch_count(items, slsf::corr_z_items(t->lx, t->ly, t->lz, rmax_xy, rmax_z));
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), ct.values, 8ull * nv, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    ctx->pool.free(dv, bytes);
    if (e != cudaSuccess) return cuda_error(e, "correlations");
    const uint32_t R = rmax_xy;
    for (uint32_t r = 0; r < R; ++r) {
        if (corr_x) corr_x[r] = h[r];
        if (corr_y) corr_y[r] = h[R + r];
        if (corr_xy) corr_xy[r] = h[2 * R + r];
    }
    if (corr_xy_by_z)
        for (size_t j = 0; j < (size_t)t->lz * R; ++j) corr_xy_by_z[j] = h[3 * R + j];
    if (corr_z)
        for (uint32_t r = 0; r < rmax_z; ++r) corr_z[r] = h[3 * R + (size_t)t->lz * R + r];
    return SLSF_OK;
}

int slsf_task_corr_setup(slsf_task* t, uint32_t rmax_xy, uint32_t rmax_z, uint32_t binsize, uint32_t n_bins,
                         size_t* n_values) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_free(t)) return rc;
    if (n_bins > 0 && binsize == 0) return set_error(SLSF_ERR_INVALID, "binsize must be positive");
    const uint32_t rxy = std::min(std::min(rmax_xy, t->lx / 2), t->ly / 2), rz = std::min(rmax_z, t->lz / 2);
    const bool on = rxy || rz;
    if (on && !slsf::corr_supports(t->lx, t->ly, t->lz, rxy, rz)) return set_error(SLSF_ERR_INVALID, kErrCorrLong);
    slsf_ctx* ctx = t->ctx;
    const uint32_t nv = on ? slsf::corr_values(t->lz, rxy, rz) : 0;
    const size_t off_bins = align256(8 * slsf::corr_partial_doubles(t->lx, t->ly, t->lz, rxy, rz));
    const size_t off_count = off_bins + align256(8ull * nv * n_bins);
    const uint64_t bytes = on ? off_count + 256 : 0;
    if (int rc = bind_device(ctx)) return rc;
    if (t->corr_block) {
        SLSF_CUDA(cudaStreamSynchronize(ctx->stream)); /* queued launches may still use the block */
        ctx->pool.free(t->corr_block, t->corr_bytes);
        ctx->used -= t->corr_bytes;
        t->corr_block = nullptr;
        t->corr_bytes = 0;
        t->corr_partial = t->corr_bins = nullptr;
        t->corr_count_dev = nullptr;
    }
    t->corr_rxy = t->corr_rz = t->corr_n_bins = 0;
    t->corr_binsize = 1;
    t->corr_count = 0;
    t->corr_interval = 0;
    t->corr_gen = ++ctx->corr_gen;
    if (n_values) *n_values = nv;
    if (!on) return SLSF_OK;
    if (ctx->used + bytes > ctx->budget)
        return set_error(SLSF_ERR_BUDGET, "correlation bins do not fit in the context's device memory budget");
    void* block = nullptr;
    SLSF_CUDA(ctx->pool.allocate(bytes, &block));
    char* b = static_cast<char*>(block);
    const cudaError_t e = cudaMemsetAsync(block, 0, bytes, ctx->stream);
    if (e != cudaSuccess) {
        ctx->pool.free(block, bytes);
        return cuda_error(e, "correlation bins");
    }
    ctx->used += bytes;
    t->corr_block = block;
    t->corr_bytes = bytes;
    t->corr_partial = reinterpret_cast<double*>(b);
    t->corr_bins = reinterpret_cast<double*>(b + off_bins);
    t->corr_count_dev = reinterpret_cast<unsigned long long*>(b + off_count);
    t->corr_rxy = rxy;
    t->corr_rz = rz;
    t->corr_binsize = binsize ? binsize : 1;
    t->corr_n_bins = n_bins;
    return SLSF_OK;
}

int slsf_task_corr_fuse(slsf_task* t, uint32_t interval) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_free(t)) return rc;
    if (interval && !t->corr_block)
        return set_error(SLSF_ERR_STATE, "task has no correlation bins; call slsf_task_corr_setup first");
    /* the context's kernel choice for this shape (default or tuned) must be the
     * one-CTA kernel (correlations from the replica in shared memory) or the
     * grid-wide kernels (the correlation launches queued after the sweep) */
    slsf_kernel_choice kc = {};
    if (interval && (slsf_tune_get(t->ctx, t->lx, t->ly, t->lz, &kc) != SLSF_OK ||
                     (kc.kind != SLSF_KERNEL_RESIDENT && kc.kind != SLSF_KERNEL_GRID)))
        return set_error(SLSF_ERR_INVALID, kErrFuse);
    t->corr_interval = interval;
    return SLSF_OK;
}

int slsf_task_corr_bins(const slsf_task* t, double* bin_means, size_t n_rows, uint64_t* count) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (count) *count = t->corr_count;
    if (!bin_means || n_rows == 0) return SLSF_OK;
    if (n_rows > t->corr_n_bins) return set_error(SLSF_ERR_INVALID, "more bin rows requested than the task keeps");
    if (int rc = bind_device(t->ctx)) return rc;
    const size_t nv = slsf::corr_values(t->lz, t->corr_rxy, t->corr_rz);
    SLSF_CUDA(cudaMemcpyAsync(bin_means, t->corr_bins, 8 * nv * n_rows, cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    /* sums -> means: a full row holds binsize measurements, the last fewer */
    for (size_t row = 0; row < n_rows; ++row) {
        const uint64_t first = (uint64_t)row * t->corr_binsize;
        const uint64_t filled = t->corr_count > first ? std::min<uint64_t>(t->corr_binsize, t->corr_count - first) : 0;
        for (size_t j = 0; j < nv; ++j) bin_means[row * nv + j] = filled ? bin_means[row * nv + j] / (double)filled : 0.0;
    }
    return SLSF_OK;
}

int slsf_batch_correlations(slsf_ctx* ctx, slsf_task* const* tasks, size_t n) {
    if (!ctx || (!tasks && n)) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (n == 0) return SLSF_OK;
    /* Correlations read the angles and write only the correlation bins, so
     * tasks held by an open batch session are accepted (their steps and this
     * launch are ordered on the context's stream). */
    bool same = ctx->corr_last.size() == n;
    for (size_t i = 0; i < n; ++i) {
        const slsf_task* t = tasks[i];
        if (!t || t->ctx != ctx) return set_error(SLSF_ERR_INVALID, "task does not belong to this context");
        if (!t->corr_block)
            return set_error(SLSF_ERR_STATE, "task has no correlation bins; call slsf_task_corr_setup first");
        if (t->corr_interval) return set_error(SLSF_ERR_STATE, kErrFused);
        if (same && (ctx->corr_last[i] != t || ctx->corr_last_gen[i] != t->corr_gen)) same = false;
    }
    if (int rc = bind_device(ctx)) return rc;
    if (!same) {
        std::unordered_set<const slsf_task*> seen;
        for (size_t i = 0; i < n; ++i)
            if (!seen.insert(tasks[i]).second) return set_error(SLSF_ERR_INVALID, "a task appears twice in the batch");
        if (!ctx->corr_uploaded) SLSF_CUDA(cudaEventCreateWithFlags(&ctx->corr_uploaded, cudaEventDisableTiming));
        /* the pinned table may still be the source of the last queued upload */
        SLSF_CUDA(cudaEventSynchronize(ctx->corr_uploaded));
        ctx->corr_last.clear();
        ctx->corr_last_gen.clear();
        if (ctx->corr_cap < n) {
            SLSF_CUDA(cudaStreamSynchronize(ctx->stream)); /* queued launches may still read the device table */
            if (ctx->d_corr) cudaFree(ctx->d_corr);
            if (ctx->h_corr) cudaFreeHost(ctx->h_corr);
            ctx->d_corr = nullptr;
            ctx->h_corr = nullptr;
            ctx->corr_cap = 0;
            SLSF_CUDA(cudaMalloc(&ctx->d_corr, sizeof(slsf::CorrTask) * n));
            SLSF_CUDA(cudaHostAlloc(&ctx->h_corr, sizeof(slsf::CorrTask) * n, cudaHostAllocDefault));
            ctx->corr_cap = n;
        }
        uint32_t items = 0, zunits = 0, max_len = 0, max_r = 0, max_nz = 0;
        for (size_t i = 0; i < n; ++i) {
            slsf_task* t = tasks[i];
            ctx->h_corr[i] = slsf::CorrTask{t->theta, t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz, items,
                                            t->corr_binsize, t->corr_n_bins, t->corr_partial, nullptr, t->corr_bins,
                                            t->corr_count_dev, zunits};
            items += slsf::corr_items(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz);
            zunits += slsf::corr_z_units(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz);
            max_len = std::max(max_len, slsf::corr_len(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz));
            max_r = std::max(max_r, std::max(t->corr_rxy, t->corr_rz));
            max_nz = std::max(max_nz, slsf::corr_z_items(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz));
        }
        SLSF_CUDA(cudaMemcpyAsync(ctx->d_corr, ctx->h_corr, sizeof(slsf::CorrTask) * n, cudaMemcpyHostToDevice,
                                  ctx->stream));
        SLSF_CUDA(cudaEventRecord(ctx->corr_uploaded, ctx->stream));
        ctx->corr_last.assign(tasks, tasks + n);
        for (size_t i = 0; i < n; ++i) ctx->corr_last_gen.push_back(tasks[i]->corr_gen);
        ctx->corr_last_items = items;
        ctx->corr_last_zunits = zunits;
        ctx->corr_last_len = max_len;
        ctx->corr_last_r = max_r;
        ctx->corr_last_nz = max_nz;
    }
    SLSF_CUDA(slsf::launch_corr(ctx->d_corr, nullptr, (uint32_t)n, ctx->corr_last_items, ctx->corr_last_zunits,
                                ctx->corr_last_len,
                                ctx->corr_last_r, ctx->corr_last_nz, ctx->sm_count, ctx->stream));
    ctx->launches += corr_launch_count(ctx->corr_last_items, ctx->corr_last_nz);
    for (size_t i = 0; i < n; ++i) tasks[i]->corr_count += 1;
    return SLSF_OK;
}

int slsf_task_get_bins(const slsf_task* t, double* bins, size_t n_rows, uint64_t* measurements) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (measurements) *measurements = t->measurements;
    if (!bins || n_rows == 0) return SLSF_OK;
    if (n_rows > t->n_bins) return set_error(SLSF_ERR_INVALID, "more bin rows requested than the task keeps");
    if (int rc = bind_device(t->ctx)) return rc;
    std::vector<double> sums(n_rows * slsf::kBinCols);
    SLSF_CUDA(cudaMemcpyAsync(sums.data(), t->bins, 8 * sums.size(), cudaMemcpyDeviceToHost, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    bin_means(t, sums.data(), bins, n_rows);
    return SLSF_OK;
}

/* ---- device state blob (checkpoints) ----
 * Layout, little-endian: StateHeader, then J_xy and J_z as stored on the
 * device (FP32, L_z each), theta (FP32, x fastest), the bin sums
 * ([n_bins][12] FP64) and the correlation bin sums ([corr_n_bins][values]
 * FP64), each section padded to 8 bytes. */
namespace {

struct StateHeader {
    char magic[8]; /* "SLSFST01" */
    uint32_t lx, ly, lz, wolff_steps;
    uint64_t seed;
    double temperature, width;
    uint32_t thermalization, binsize, n_bins, corr_rxy;
    uint32_t corr_rz, corr_binsize, corr_n_bins, corr_values;
    uint64_t metro_sweeps, wolff_done, measurements, corr_count;
    uint64_t user[4];
    uint64_t bytes; /* the whole blob */
};
static_assert(sizeof(StateHeader) % 8 == 0, "state header is 8-byte aligned");
constexpr char kStateMagic[8] = {'S', 'L', 'S', 'F', 'S', 'T', '0', '1'};

uint64_t pad8(uint64_t b) { return (b + 7) & ~7ull; }

struct StateLayout {
    uint64_t j, theta, bins, corr, total;
    uint32_t nv;
};

StateLayout state_layout(const slsf_task* t) {
    StateLayout L;
    L.nv = t->corr_block ? slsf::corr_values(t->lz, t->corr_rxy, t->corr_rz) : 0;
    L.j = sizeof(StateHeader);
    L.theta = L.j + pad8(8ull * t->lz);
    L.bins = L.theta + pad8(4ull * t->volume);
    L.corr = L.bins + 8ull * slsf::kBinCols * t->n_bins;
    L.total = L.corr + 8ull * L.nv * (t->corr_block ? t->corr_n_bins : 0);
    return L;
}

}  // namespace

int slsf_task_state_size(const slsf_task* t, size_t* bytes) {
    if (!t || !bytes) return set_error(SLSF_ERR_INVALID, "NULL argument");
    *bytes = state_layout(t).total;
    return SLSF_OK;
}

int slsf_task_state_save(const slsf_task* t, const uint64_t user[4], void* buf, size_t bytes) {
    if (!t || !buf) return set_error(SLSF_ERR_INVALID, "NULL argument");
    const StateLayout L = state_layout(t);
    if (bytes < L.total) return set_error(SLSF_ERR_INVALID, "state buffer is smaller than slsf_task_state_size");
    if (int rc = bind_device(t->ctx)) return rc;
    char* b = static_cast<char*>(buf);
    std::memset(b, 0, L.total);
    StateHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kStateMagic, 8);
    h.lx = t->lx, h.ly = t->ly, h.lz = t->lz, h.wolff_steps = t->wolff_steps;
    h.seed = t->seed;
    h.temperature = t->temperature, h.width = t->width;
    h.thermalization = t->thermalization, h.binsize = t->binsize, h.n_bins = t->n_bins;
    h.corr_rxy = t->corr_rxy, h.corr_rz = t->corr_rz, h.corr_binsize = t->corr_binsize;
    h.corr_n_bins = t->corr_block ? t->corr_n_bins : 0, h.corr_values = L.nv;
    h.metro_sweeps = t->metro_sweeps, h.wolff_done = t->wolff_done, h.measurements = t->measurements;
    h.corr_count = t->corr_count;
    if (user) std::memcpy(h.user, user, sizeof(h.user));
    h.bytes = L.total;
    std::memcpy(b, &h, sizeof(h));
    cudaStream_t st = t->ctx->stream;
    SLSF_CUDA(cudaMemcpyAsync(b + L.j, t->jxy, 4ull * t->lz, cudaMemcpyDeviceToHost, st));
    SLSF_CUDA(cudaMemcpyAsync(b + L.j + 4ull * t->lz, t->jz, 4ull * t->lz, cudaMemcpyDeviceToHost, st));
    SLSF_CUDA(cudaMemcpyAsync(b + L.theta, t->theta, 4ull * t->volume, cudaMemcpyDeviceToHost, st));
    if (t->n_bins)
        SLSF_CUDA(cudaMemcpyAsync(b + L.bins, t->bins, L.corr - L.bins, cudaMemcpyDeviceToHost, st));
    if (L.total > L.corr)
        SLSF_CUDA(cudaMemcpyAsync(b + L.corr, t->corr_bins, L.total - L.corr, cudaMemcpyDeviceToHost, st));
    SLSF_CUDA(cudaStreamSynchronize(st));
    return SLSF_OK;
}

int slsf_task_state_load(slsf_task* t, const void* buf, size_t bytes, uint64_t user[4]) {
    if (!t || !buf) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (int rc = check_free(t)) return rc;
    const StateLayout L = state_layout(t);
    const char* b = static_cast<const char*>(buf);
    StateHeader h;
    if (bytes < sizeof(h)) return set_error(SLSF_ERR_INVALID, "not a task state (too short)");
    std::memcpy(&h, b, sizeof(h));
    if (std::memcmp(h.magic, kStateMagic, 8) != 0) return set_error(SLSF_ERR_INVALID, "not a task state (bad magic)");
    auto mismatch = [](const char* what) {
        return set_error(SLSF_ERR_INVALID, std::string("state does not match the task: ") + what);
    };
    if (h.bytes != bytes || bytes != L.total) return mismatch("size");
    if (h.lx != t->lx || h.ly != t->ly || h.lz != t->lz) return mismatch("lattice dimensions");
    if (h.seed != t->seed) return mismatch("seed");
    if (std::memcmp(&h.temperature, &t->temperature, 8) || std::memcmp(&h.width, &t->width, 8))
        return mismatch("temperature or proposal width");
    if (h.wolff_steps != t->wolff_steps) return mismatch("wolff_steps");
    if (h.thermalization != t->thermalization || h.binsize != t->binsize || h.n_bins != t->n_bins)
        return mismatch("thermalization or bins");
    const uint32_t corr_n_bins = t->corr_block ? t->corr_n_bins : 0;
    if (h.corr_rxy != t->corr_rxy || h.corr_rz != t->corr_rz || h.corr_binsize != t->corr_binsize ||
        h.corr_n_bins != corr_n_bins || h.corr_values != L.nv)
        return mismatch("correlation set-up");
    if (int rc = bind_device(t->ctx)) return rc;
    cudaStream_t st = t->ctx->stream;
    std::vector<float> j(2ull * t->lz);
    SLSF_CUDA(cudaMemcpyAsync(j.data(), t->jxy, 4ull * t->lz, cudaMemcpyDeviceToHost, st));
    SLSF_CUDA(cudaMemcpyAsync(j.data() + t->lz, t->jz, 4ull * t->lz, cudaMemcpyDeviceToHost, st));
    SLSF_CUDA(cudaStreamSynchronize(st));
    if (std::memcmp(j.data(), b + L.j, 8ull * t->lz) != 0) return mismatch("layer couplings");
    SLSF_CUDA(cudaMemcpyAsync(t->theta, b + L.theta, 4ull * t->volume, cudaMemcpyHostToDevice, st));
    if (t->n_bins)
        SLSF_CUDA(cudaMemcpyAsync(t->bins, b + L.bins, L.corr - L.bins, cudaMemcpyHostToDevice, st));
    const unsigned long long corr_count = h.corr_count;
    if (t->corr_block) {
        if (L.total > L.corr)
            SLSF_CUDA(cudaMemcpyAsync(t->corr_bins, b + L.corr, L.total - L.corr, cudaMemcpyHostToDevice, st));
        SLSF_CUDA(cudaMemcpyAsync(t->corr_count_dev, &corr_count, 8, cudaMemcpyHostToDevice, st));
    }
    SLSF_CUDA(cudaStreamSynchronize(st));
    t->metro_sweeps = h.metro_sweeps;
    t->wolff_done = h.wolff_done;
    t->measurements = h.measurements;
    t->corr_count = t->corr_block ? h.corr_count : 0;
    if (user) std::memcpy(user, h.user, sizeof(h.user));
    return SLSF_OK;
}

int slsf_task_reset_bins(slsf_task* t) {
    if (!t) return set_error(SLSF_ERR_INVALID, "task is NULL");
    if (int rc = check_free(t)) return rc;
    if (int rc = bind_device(t->ctx)) return rc;
    if (t->n_bins)
        SLSF_CUDA(cudaMemsetAsync(t->bins, 0, 8ull * slsf::kBinCols * t->n_bins, t->ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(t->ctx->stream));
    t->measurements = 0;
    return SLSF_OK;
}

/* `v.sweeps` sweeps of one task through the grid-wide kernels, measuring
 * after every sweep past thermalization into the task's bin sums as the
 * persistent kernels do: the state after a sweep is measured by the next
 * sweep's colour-0 kernel, the launch's last state by the measurement
 * kernel; counters accumulate into v.stats. */
static void run_grid_task(slsf_ctx* ctx, const slsf_task* t, const TaskView& v, cudaStream_t st) {
    double* pending = nullptr; /* bin row of the state after the previous sweep, not yet measured */
    for (uint32_t sw = 0; sw < v.sweeps; ++sw) {
        const uint64_t sweep = t->metro_sweeps + sw;
        if (pending)
            slsf::launch_metro_colour0_measure(v, sweep, t->partials, t->done, t->result, pending, st);
        else
            slsf::launch_metro_colour(v, sweep, 0, nullptr, st);
        pending = nullptr;
        slsf::launch_metro_colour(v, sweep, 1, nullptr, st);
        ctx->launches += 2;
        for (uint32_t k = 0; k < t->wolff_steps; ++k) {
            ctx->launches += slsf::launch_wolff(v, t->wolff_done + (uint64_t)sw * t->wolff_steps + k, t->bonds,
                                                t->parent, nullptr, st, nullptr, nullptr);
        }
        const uint64_t done = sweep + 1;
        if (done > t->thermalization && t->n_bins) {
            const uint64_t b = (done - t->thermalization - 1) / t->binsize;
            if (b < t->n_bins) pending = t->bins + b * slsf::kBinCols;
        }
        /* ThetaModel::measure's correlations of the state after this sweep
         * (slsf_task_corr_fuse), as the one-CTA kernel takes them: measurement
         * m = sweep - thermalization, every corr_interval-th, into the bins */
        if (t->corr_interval && t->corr_block && sweep >= t->thermalization &&
            (sweep - t->thermalization) % t->corr_interval == 0) {
            const slsf::CorrTask ct = {t->theta,         t->lx,         t->ly,          t->lz,
                                       t->corr_rxy,      t->corr_rz,    0,              t->corr_binsize,
                                       t->corr_n_bins,   t->corr_partial, nullptr,      t->corr_bins,
                                       t->corr_count_dev};
            const uint32_t items = slsf::corr_items(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz);
            slsf::launch_corr(nullptr, &ct, 1, items, slsf::corr_z_units(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz),
                              slsf::corr_len(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz),
                              std::max(t->corr_rxy, t->corr_rz),
                              slsf::corr_z_items(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz), ctx->sm_count, st);
            ctx->launches +=
                corr_launch_count(items, slsf::corr_z_items(t->lx, t->ly, t->lz, t->corr_rxy, t->corr_rz));
        }
    }
    if (pending) {
        slsf::launch_measure_into_bin(v, t->partials, t->done, t->result, pending, st);
        ctx->launches += 1;
    }
}

namespace {

uint64_t shape_key(uint32_t lx, uint32_t ly, uint32_t lz) {
    return (uint64_t)lx | ((uint64_t)ly << 21) | ((uint64_t)lz << 42);
}

bool choice_feasible(const slsf::KernelChoice& c, uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    switch (c.kind) {
        case slsf::kKernelResident:
            return c.cluster == 1 && c.threads >= 64 && c.threads <= 1024 && c.threads % 32 == 0 &&
                   slsf::resident_supports(lx, ly, lz, device);
        case slsf::kKernelCluster:
            return c.threads >= 64 && c.threads <= 1024 && c.threads % 32 == 0 &&
                   slsf::cluster_feasible(lx, ly, lz, c.cluster, device);
        case slsf::kKernelGrid:
            return true;
        default:
            return false;
    }
}

/* Without a tuned entry: the one-CTA kernel when the replica fits, with a CTA
 * of about one thread per 32 sites (128 .. 1024; measured on B200: L = 8 and
 * 16 run 1.4-2x faster on 128 threads than on 1024, L = 24 best on 512, L = 32
 * on 1024); else the smallest cluster that holds it, 1024 threads; else the
 * grid-wide kernels. */
slsf::KernelChoice default_choice(uint32_t lx, uint32_t ly, uint32_t lz, int device) {
    if (slsf::resident_supports(lx, ly, lz, device)) {
        const uint64_t v = (uint64_t)lx * ly * lz;
        uint32_t t = 128;
        while (t < 1024 && 32ull * t < v) t <<= 1;
        return {slsf::kKernelResident, 1, t};
    }
    if (const uint32_t c = slsf::batched_cluster_size(lx, ly, lz, device)) return {slsf::kKernelCluster, c, 1024};
    return {slsf::kKernelGrid, 1, 256};
}

slsf::KernelChoice choice_for(const slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz) {
    const auto it = ctx->tune.find(shape_key(lx, ly, lz));
    if (it != ctx->tune.end()) return it->second;
    return default_choice(lx, ly, lz, ctx->device);
}

int ensure_queue_capacity(slsf_ctx* ctx, uint32_t n) {
    if (n <= ctx->queue_cap) return SLSF_OK;
    if (ctx->d_queue) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_queue);
        ctx->d_queue = nullptr;
        ctx->queue_cap = 0;
    }
    const uint32_t cap = std::max<uint32_t>(16, n);
    SLSF_CUDA(cudaMalloc(&ctx->d_queue, sizeof(unsigned int) * cap));
    ctx->queue_cap = cap;
    return SLSF_OK;
}

}  // namespace

/* Shared body of slsf_batch_run (every task n_sweeps), slsf_batch_run_v
 * (task i per_task[i] sweeps; tasks with 0 sweeps are left out of the
 * launch) and the autotuner (`force`: one kernel choice for every task). */
/* The fused-correlation entry of a task's view (bins NULL without). */
static slsf::ResidentCorr rcorr_of(const slsf_task* t) {
    if (!t->corr_interval || !t->corr_block) return slsf::ResidentCorr{nullptr, nullptr, 0, 0, 1, 0, 1};
    return slsf::ResidentCorr{t->corr_bins, t->corr_count_dev, t->corr_rxy, t->corr_rz,
                              t->corr_binsize, t->corr_n_bins, t->corr_interval};
}

static uint32_t rcorr_doubles(const slsf_task* t) {
    return t->corr_interval ? slsf::resident_corr_doubles(t->ly, t->lz, t->corr_rxy, t->corr_rz) : 0;
}

/* Host mirrors of a task's counters after `sweeps` batched sweeps: sweep and
 * Wolff counters, measurements (every sweep past thermalization) and fused
 * correlation measurements (measurement m = sweep - thermalization when m is
 * a multiple of the interval). */
static void advance_counters(slsf_task* t, uint64_t sweeps) {
    const uint64_t before = t->metro_sweeps;
    t->metro_sweeps += sweeps;
    t->wolff_done += sweeps * t->wolff_steps;
    const uint64_t lo = std::max<uint64_t>(before, t->thermalization);
    if (t->metro_sweeps > lo && t->n_bins) t->measurements += t->metro_sweeps - lo;
    if (t->corr_interval && t->metro_sweeps > lo) {
        const uint64_t q = t->corr_interval, a = lo - t->thermalization, b = t->metro_sweeps - t->thermalization;
        t->corr_count += (b + q - 1) / q - (a + q - 1) / q; /* multiples of q in [a, b) */
    }
}

static int batch_run_impl(slsf_ctx* ctx, slsf_task* const* all_tasks, size_t n_all, uint32_t n_sweeps,
                          const uint32_t* per_task, slsf_sweep_stats* all_stats,
                          const slsf::KernelChoice* force = nullptr) {
    if (!ctx || (!all_tasks && n_all)) return set_error(SLSF_ERR_INVALID, "NULL argument");
    std::vector<slsf_task*> task_list;
    std::vector<size_t> slot_of;
    std::vector<uint32_t> sweeps_of;
    for (size_t i = 0; i < n_all; ++i) {
        const uint32_t sw = per_task ? per_task[i] : n_sweeps;
        if (all_stats) all_stats[i] = slsf_sweep_stats{0, 0, 0, 0};
        if (sw == 0) continue;
        task_list.push_back(all_tasks[i]);
        slot_of.push_back(i);
        sweeps_of.push_back(sw);
    }
    const size_t n = task_list.size();
    slsf_task* const* tasks = task_list.data();
    if (n == 0) return SLSF_OK;
    if (int rc = bind_device(ctx)) return rc;
    /* Kernel of each task (kernel_resident.cu, kernel_cluster.cu, or the
     * grid-wide single-task kernels of kernels_plain.cu for lattices too
     * large for one cluster's shared memory, which fill the GPU on their
     * own), from the context's tuning table or the default. */
    std::vector<slsf::KernelChoice> ch(n);
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = tasks[i];
        if (!t || t->ctx != ctx) return set_error(SLSF_ERR_INVALID, "task does not belong to this context");
        if (int rc = check_sweepable(t)) return rc;
        ch[i] = force ? *force : choice_for(ctx, t->lx, t->ly, t->lz);
        if (!choice_feasible(ch[i], t->lx, t->ly, t->lz, ctx->device))
            return set_error(SLSF_ERR_INVALID, "the kernel choice does not hold this lattice");
        if (t->corr_interval && ch[i].kind == slsf::kKernelCluster) return set_error(SLSF_ERR_INVALID, kErrFuse);
    }
    if (int rc = ensure_batch_capacity(ctx, n)) return rc;
    /* Grouped by kernel choice (one persistent launch each; cluster groups
     * first, grid-wide tasks last), largest replicas first within a group so
     * the grid ends evenly; each view accumulates its counters into its own
     * slot of the batch stats array. */
    auto rank = [&](size_t i) {
        const slsf::KernelChoice& c = ch[i];
        const uint32_t k = c.kind == slsf::kKernelCluster ? 2u : (c.kind == slsf::kKernelResident ? 1u : 0u);
        const uint64_t fused = tasks[i]->corr_interval ? 1u : 0u;
        return ((uint64_t)k << 48) | (fused << 40) | ((uint64_t)c.cluster << 16) | c.threads;
    };
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        const uint64_t ra = rank(a), rb = rank(b);
        if (ra != rb) return ra > rb;
        return tasks[a]->volume > tasks[b]->volume;
    });
    uint32_t n_groups = 0;
    for (size_t k = 0; k < n; ++k)
        if (k == 0 || rank(order[k]) != rank(order[k - 1])) ++n_groups;
    if (int rc = ensure_queue_capacity(ctx, n_groups)) return rc;
    bool any_fused = false;
    for (size_t k = 0; k < n; ++k) {
        TaskView v = tasks[order[k]]->view();
        v.stats = ctx->d_batch_stats + slsf::kStatSlots * order[k];
        v.sweeps = sweeps_of[order[k]];
        ctx->h_views[k] = v;
        ctx->h_rcorr[k] = rcorr_of(tasks[order[k]]);
        any_fused |= tasks[order[k]]->corr_interval != 0;
    }
    SLSF_CUDA(cudaMemcpyAsync(ctx->d_views, ctx->h_views, sizeof(TaskView) * n, cudaMemcpyHostToDevice, ctx->stream));
    if (any_fused)
        SLSF_CUDA(cudaMemcpyAsync(ctx->d_rcorr, ctx->h_rcorr, sizeof(slsf::ResidentCorr) * n, cudaMemcpyHostToDevice,
                                  ctx->stream));
    SLSF_CUDA(cudaMemsetAsync(ctx->d_batch_stats, 0, 8 * slsf::kStatSlots * n, ctx->stream));
    SLSF_CUDA(cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned int) * n_groups, ctx->stream));
    /* Group g runs on ctx->stream (g == 0) or on a side stream, forked after
     * the uploads above and joined before the stats read-back below. */
    if (n_groups > 1) SLSF_CUDA(cudaEventRecord(ctx->fork, ctx->stream));
    for (size_t lo = 0, q = 0; lo < n; ++q) {
        const slsf::KernelChoice c = ch[order[lo]];
        const uint64_t key = rank(order[lo]);
        cudaStream_t st = ctx->stream;
        const int side = q > 0 ? (int)((q - 1) % kSideStreams) : -1;
        if (side >= 0) {
            st = ctx->side[side];
            SLSF_CUDA(cudaStreamWaitEvent(st, ctx->fork, 0));
        }
        size_t hi = lo;
        const uint32_t parts = c.kind == slsf::kKernelCluster ? c.cluster : 1;
        uint32_t max_vs = 0, max_rows = 0, max_lz = 0, max_plane = 0, max_lx = 0, max_cd = 0;
        bool cube32 = false;
        while (hi < n && rank(order[hi]) == key) {
            const slsf_task* t = tasks[order[hi]];
            cube32 |= t->lx == 32 && t->ly == 32 && t->lz == 32;
            max_cd = std::max(max_cd, rcorr_doubles(t));
            max_vs = std::max(max_vs, t->volume / parts);
            max_rows = std::max(max_rows, t->ly * (t->lz / parts));
            max_lz = std::max(max_lz, t->lz);
            max_plane = std::max(max_plane, t->lx * t->ly);
            max_lx = std::max(max_lx, t->lx);
            ++hi;
        }
        if (c.kind == slsf::kKernelGrid) {
            for (size_t k = lo; k < hi; ++k) run_grid_task(ctx, tasks[order[k]], ctx->h_views[k], st);
        } else if (c.kind == slsf::kKernelResident) {
            SLSF_CUDA(slsf::launch_resident(ctx->d_views + lo, (uint32_t)(hi - lo), n_sweeps, ctx->d_queue + q,
                                            ctx->device, st, max_vs, max_rows, max_lz, c.threads, nullptr,
                                            max_cd ? ctx->d_rcorr + lo : nullptr, max_cd, cube32));
            ctx->launches += 1;
        } else {
            SLSF_CUDA(slsf::launch_batched(ctx->d_views + lo, (uint32_t)(hi - lo), n_sweeps, ctx->d_queue + q,
                                           ctx->device, st, c.cluster, c.threads, max_vs, max_rows, max_lz,
                                           max_plane, max_lx, nullptr));
            ctx->launches += 1;
        }
        if (side >= 0) {
            SLSF_CUDA(cudaEventRecord(ctx->join[side], st));
            SLSF_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join[side], 0));
        }
        lo = hi;
    }
    SLSF_CUDA(cudaMemcpyAsync(ctx->h_batch_stats, ctx->d_batch_stats, 8 * slsf::kStatSlots * n,
                              cudaMemcpyDeviceToHost, ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    int rc = SLSF_OK;
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = tasks[i];
        const uint32_t sw = sweeps_of[i];
        advance_counters(t, sw);
        const unsigned long long* s = &ctx->h_batch_stats[i * slsf::kStatSlots];
        if (s[slsf::kStatError]) rc = set_error(SLSF_ERR_TIMEOUT, "a bounded device loop hit its iteration limit");
        if (all_stats) {
            slsf_sweep_stats& o = all_stats[slot_of[i]];
            o.sweeps = sw;
            o.accepted = s[slsf::kStatAccepted];
            o.wolff_clusters =
                ch[i].kind == slsf::kKernelGrid ? (uint64_t)sw * t->wolff_steps : s[slsf::kStatClusters];
            o.wolff_cluster_sites = s[slsf::kStatClusterSites];
        }
    }
    return rc;
}

/* ---- batch sessions: one captured step replayed as a CUDA graph ---- */

struct slsf_batch {
    slsf_ctx* ctx = nullptr;
    std::vector<slsf_task*> tasks; /* in the caller's order */
    uint32_t n_sweeps = 0;
    TaskView* d_views = nullptr;
    unsigned long long* d_stats = nullptr;
    unsigned long long* h_stats = nullptr; /* pinned */
    unsigned int* d_queue = nullptr;
    unsigned long long* d_counters = nullptr; /* [view][Metropolis, Wolff], advanced by the kernels */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    slsf::ResidentCorr* d_rcorr = nullptr; /* fused correlations, parallel to d_views */
    unsigned long long* d_acc = nullptr; /* stats summed over the cycles of slsf_batch_step_correlations */
    unsigned long long* h_acc = nullptr; /* pinned */
};

static void batch_free(slsf_batch* b) {
    if (b->d_acc) cudaFree(b->d_acc);
    if (b->d_rcorr) cudaFree(b->d_rcorr);
    if (b->h_acc) cudaFreeHost(b->h_acc);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_views) cudaFree(b->d_views);
    if (b->d_stats) cudaFree(b->d_stats);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_counters) cudaFree(b->d_counters);
    if (b->h_stats) cudaFreeHost(b->h_stats);
    for (slsf_task* t : b->tasks)
        if (t && t->session == b) t->session = nullptr;
    delete b;
}

int slsf_batch_open(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, uint32_t n_sweeps, slsf_batch** out) {
    if (!ctx || !out || (!tasks && n)) return set_error(SLSF_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (n == 0 || n_sweeps == 0) return set_error(SLSF_ERR_INVALID, "a session needs tasks and sweeps");
    if (int rc = bind_device(ctx)) return rc;
    std::vector<slsf::KernelChoice> ch(n);
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = tasks[i];
        if (!t || t->ctx != ctx) return set_error(SLSF_ERR_INVALID, "task does not belong to this context");
        if (int rc = check_sweepable(t)) return rc;
        for (size_t j = 0; j < i; ++j)
            if (tasks[j] == t) return set_error(SLSF_ERR_INVALID, "a task appears twice in the session");
        ch[i] = choice_for(ctx, t->lx, t->ly, t->lz);
        if (ch[i].kind == slsf::kKernelGrid || !choice_feasible(ch[i], t->lx, t->ly, t->lz, ctx->device))
            return set_error(SLSF_ERR_INVALID,
                             "batch sessions hold lattices that fit one thread-block cluster's shared memory");
        if (t->corr_interval && ch[i].kind == slsf::kKernelCluster) return set_error(SLSF_ERR_INVALID, kErrFuse);
    }
    auto rank = [&](size_t i) {
        const slsf::KernelChoice& c = ch[i];
        const uint64_t fused = tasks[i]->corr_interval ? 1u : 0u;
        return ((uint64_t)(c.kind == slsf::kKernelCluster ? 2u : 1u) << 48) | (fused << 40) |
               ((uint64_t)c.cluster << 16) | c.threads;
    };
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        const uint64_t ra = rank(a), rb = rank(b);
        if (ra != rb) return ra > rb;
        return tasks[a]->volume > tasks[b]->volume;
    });
    uint32_t n_groups = 0;
    for (size_t k = 0; k < n; ++k)
        if (k == 0 || rank(order[k]) != rank(order[k - 1])) ++n_groups;
    slsf_batch* b = new slsf_batch;
    b->ctx = ctx;
    b->tasks.assign(tasks, tasks + n);
    b->n_sweeps = n_sweeps;
    cudaError_t e = cudaMalloc(&b->d_views, sizeof(TaskView) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_stats, 8 * slsf::kStatSlots * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, sizeof(unsigned int) * n_groups);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_stats, 8 * slsf::kStatSlots * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, 16 * n);
    std::vector<unsigned long long> counters(2 * n);
    for (size_t k = 0; k < n; ++k) {
        counters[2 * k] = tasks[order[k]]->metro_sweeps;
        counters[2 * k + 1] = tasks[order[k]]->wolff_done;
    }
    if (e == cudaSuccess) e = cudaMemcpy(b->d_counters, counters.data(), 16 * n, cudaMemcpyHostToDevice);
    std::vector<TaskView> views(n);
    for (size_t k = 0; k < n && e == cudaSuccess; ++k) {
        TaskView v = tasks[order[k]]->view();
        v.stats = b->d_stats + slsf::kStatSlots * order[k];
        v.sweeps = n_sweeps;
        views[k] = v;
    }
    if (e == cudaSuccess) e = cudaMemcpy(b->d_views, views.data(), sizeof(TaskView) * n, cudaMemcpyHostToDevice);
    {
        std::vector<slsf::ResidentCorr> rc(n);
        bool any = false;
        for (size_t k = 0; k < n; ++k) {
            rc[k] = rcorr_of(tasks[order[k]]);
            any |= tasks[order[k]]->corr_interval != 0;
        }
        if (any && e == cudaSuccess) e = cudaMalloc(&b->d_rcorr, sizeof(slsf::ResidentCorr) * n);
        if (any && e == cudaSuccess)
            e = cudaMemcpy(b->d_rcorr, rc.data(), sizeof(slsf::ResidentCorr) * n, cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_error(e, "batch session set-up");
    }
    /* capture one step */
    cudaStream_t main = ctx->stream;
    e = cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_stats, 0, 8 * slsf::kStatSlots * n, main);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int) * n_groups, main);
    if (e == cudaSuccess && n_groups > 1) e = cudaEventRecord(ctx->fork, main);
    uint64_t launches = 0;
    for (size_t lo = 0, q = 0; lo < n && e == cudaSuccess; ++q) {
        const slsf::KernelChoice c = ch[order[lo]];
        const uint64_t key = rank(order[lo]);
        cudaStream_t st = main;
        const int side = q > 0 ? (int)((q - 1) % kSideStreams) : -1;
        if (side >= 0) {
            st = ctx->side[side];
            e = cudaStreamWaitEvent(st, ctx->fork, 0);
        }
        size_t hi = lo;
        const uint32_t parts = c.kind == slsf::kKernelCluster ? c.cluster : 1;
        uint32_t max_vs = 0, max_rows = 0, max_lz = 0, max_plane = 0, max_lx = 0, max_cd = 0;
        bool cube32 = false;
        while (hi < n && rank(order[hi]) == key) {
            const slsf_task* t = tasks[order[hi]];
            cube32 |= t->lx == 32 && t->ly == 32 && t->lz == 32;
            max_cd = std::max(max_cd, rcorr_doubles(t));
            max_vs = std::max(max_vs, t->volume / parts);
            max_rows = std::max(max_rows, t->ly * (t->lz / parts));
            max_lz = std::max(max_lz, t->lz);
            max_plane = std::max(max_plane, t->lx * t->ly);
            max_lx = std::max(max_lx, t->lx);
            ++hi;
        }
        if (e == cudaSuccess) {
            if (c.kind == slsf::kKernelResident)
                e = slsf::launch_resident(b->d_views + lo, (uint32_t)(hi - lo), n_sweeps, b->d_queue + q, ctx->device,
                                          st, max_vs, max_rows, max_lz, c.threads, b->d_counters + 2 * lo,
                                          max_cd ? b->d_rcorr + lo : nullptr, max_cd, cube32);
            else
                e = slsf::launch_batched(b->d_views + lo, (uint32_t)(hi - lo), n_sweeps, b->d_queue + q, ctx->device,
                                         st, c.cluster, c.threads, max_vs, max_rows, max_lz, max_plane, max_lx,
                                         b->d_counters + 2 * lo);
            ++launches;
        }
        if (e == cudaSuccess && side >= 0) {
            e = cudaEventRecord(ctx->join[side], st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(main, ctx->join[side], 0);
        }
        lo = hi;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_stats, b->d_stats, 8 * slsf::kStatSlots * n, cudaMemcpyDeviceToHost, main);
    const cudaError_t e_end = cudaStreamEndCapture(main, &b->graph);
    if (e == cudaSuccess) e = e_end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        batch_free(b);
        return cuda_error(e, "batch session capture");
    }
    (void)launches;
    for (slsf_task* t : b->tasks) t->session = b;
    *out = b;
    return SLSF_OK;
}

int slsf_batch_step(slsf_batch* b, slsf_sweep_stats* stats) {
    if (!b) return set_error(SLSF_ERR_INVALID, "session is NULL");
    slsf_ctx* ctx = b->ctx;
    if (int rc = bind_device(ctx)) return rc;
    SLSF_CUDA(cudaGraphLaunch(b->exec, ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->launches += 1;
    int rc = SLSF_OK;
    for (size_t i = 0; i < b->tasks.size(); ++i) {
        slsf_task* t = b->tasks[i];
        advance_counters(t, b->n_sweeps);
        const unsigned long long* s = &b->h_stats[i * slsf::kStatSlots];
        if (s[slsf::kStatError]) rc = set_error(SLSF_ERR_TIMEOUT, "a bounded device loop hit its iteration limit");
        if (stats) stats[i] = slsf_sweep_stats{b->n_sweeps, s[slsf::kStatAccepted], s[slsf::kStatClusters],
                                               s[slsf::kStatClusterSites]};
    }
    return rc;
}

namespace {

/* acc[i] += add[i], one thread per counter. */
__global__ void k_stats_add(const unsigned long long* __restrict__ add, unsigned long long* __restrict__ acc,
                            uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) acc[i] += add[i];
}

}  // namespace

int slsf_batch_step_correlations(slsf_batch* b, uint32_t n_cycles, slsf_sweep_stats* stats) {
    if (!b) return set_error(SLSF_ERR_INVALID, "session is NULL");
    slsf_ctx* ctx = b->ctx;
    const size_t n = b->tasks.size();
    for (slsf_task* t : b->tasks) {
        if (!t->corr_block)
            return set_error(SLSF_ERR_STATE, "task has no correlation bins; call slsf_task_corr_setup first");
        if (t->corr_interval) return set_error(SLSF_ERR_STATE, kErrFused);
    }
    if (n_cycles == 0) {
        if (stats)
            for (size_t i = 0; i < n; ++i) stats[i] = slsf_sweep_stats{0, 0, 0, 0};
        return SLSF_OK;
    }
    if (int rc = bind_device(ctx)) return rc;
    const size_t slots = slsf::kStatSlots * n;
    if (!b->d_acc) {
        SLSF_CUDA(cudaMalloc(&b->d_acc, 8 * slots));
        SLSF_CUDA(cudaHostAlloc(&b->h_acc, 8 * slots, cudaHostAllocDefault));
    }
    SLSF_CUDA(cudaMemsetAsync(b->d_acc, 0, 8 * slots, ctx->stream));
    for (uint32_t c = 0; c < n_cycles; ++c) {
        /* the step's stats are reset inside its graph; they are summed here
         * on the device, so the cycles need no host round trip */
        SLSF_CUDA(cudaGraphLaunch(b->exec, ctx->stream));
        k_stats_add<<<(uint32_t)((slots + 255) / 256), 256, 0, ctx->stream>>>(b->d_stats, b->d_acc, (uint32_t)slots);
        SLSF_CUDA(cudaGetLastError());
        if (int rc = slsf_batch_correlations(ctx, b->tasks.data(), n)) return rc;
        ctx->launches += 2;
    }
    SLSF_CUDA(cudaMemcpyAsync(b->h_acc, b->d_acc, 8 * slots, cudaMemcpyDeviceToHost, ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    const uint64_t sweeps = (uint64_t)n_cycles * b->n_sweeps;
    int rc = SLSF_OK;
    for (size_t i = 0; i < n; ++i) {
        slsf_task* t = b->tasks[i];
        advance_counters(t, sweeps);
        const unsigned long long* a = &b->h_acc[i * slsf::kStatSlots];
        if (a[slsf::kStatError]) rc = set_error(SLSF_ERR_TIMEOUT, "a bounded device loop hit its iteration limit");
        if (stats) stats[i] = slsf_sweep_stats{sweeps, a[slsf::kStatAccepted], a[slsf::kStatClusters],
                                               a[slsf::kStatClusterSites]};
    }
    return rc;
}

int slsf_batch_close(slsf_batch* b) {
    if (!b) return SLSF_OK;
    bind_device(b->ctx);
    cudaStreamSynchronize(b->ctx->stream);
    batch_free(b);
    return SLSF_OK;
}

static slsf::KernelChoice to_choice(const slsf_kernel_choice& c) { return {c.kind, c.cluster, c.threads}; }
static slsf_kernel_choice from_choice(const slsf::KernelChoice& c) { return {c.kind, c.cluster, c.threads}; }

int slsf_tune_get(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, slsf_kernel_choice* out) {
    if (!ctx || !out) return set_error(SLSF_ERR_INVALID, "NULL argument");
    *out = from_choice(choice_for(ctx, lx, ly, lz));
    return SLSF_OK;
}

int slsf_tune_set(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, const slsf_kernel_choice* c) {
    if (!ctx || !c) return set_error(SLSF_ERR_INVALID, "NULL argument");
    const slsf::KernelChoice k = to_choice(*c);
    if (!choice_feasible(k, lx, ly, lz, ctx->device))
        return set_error(SLSF_ERR_INVALID, "the kernel choice does not hold this lattice");
    ctx->tune[shape_key(lx, ly, lz)] = k;
    ctx->tune_rate.erase(shape_key(lx, ly, lz));
    return SLSF_OK;
}

int slsf_autotune(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, uint32_t sweeps, slsf_kernel_choice* best,
                  double* rate) {
    if (!ctx) return set_error(SLSF_ERR_INVALID, "context is NULL");
    if (lx == 0 || ly == 0 || lz == 0 || lx % 2 || ly % 2 || lz % 2)
        return set_error(SLSF_ERR_INVALID, kErrEven);
    if (int rc = bind_device(ctx)) return rc;
    /* candidates */
    std::vector<slsf::KernelChoice> cand;
    for (uint32_t t : {128u, 256u, 512u, 1024u}) {
        const slsf::KernelChoice c = {slsf::kKernelResident, 1, t};
        if (choice_feasible(c, lx, ly, lz, ctx->device)) cand.push_back(c);
    }
    for (uint32_t cl = 1; cl <= 16; cl <<= 1)
        for (uint32_t t : {512u, 1024u}) {
            const slsf::KernelChoice c = {slsf::kKernelCluster, cl, t};
            if (choice_feasible(c, lx, ly, lz, ctx->device)) cand.push_back(c);
        }
    if (cand.empty()) cand.push_back({slsf::kKernelGrid, 1, 256});
    /* scratch replicas: about 2^25 sites, at most 4096, within the budget */
    const uint64_t v = (uint64_t)lx * ly * lz;
    uint64_t n = std::max<uint64_t>(1, std::min<uint64_t>(4096, (1ull << 25) / v));
    const uint64_t per = slsf_task_bytes(lx, ly, lz, 1);
    if (ctx->budget > ctx->used) n = std::min<uint64_t>(n, (ctx->budget - ctx->used) / per);
    if (n == 0) return set_error(SLSF_ERR_BUDGET, "task does not fit in the context's device memory budget");
    std::vector<double> jx(lz, 1.2), jz(lz, 1.0);
    std::vector<slsf_task*> tasks;
    int rc = SLSF_OK;
    for (uint64_t i = 0; i < n && rc == SLSF_OK; ++i) {
        slsf_task_desc d = {};
        d.lx = lx;
        d.ly = ly;
        d.lz = lz;
        d.temperature = 1.1 + 0.4 * (double)(i % 16) / 15.0;
        d.proposal_width = 3.141592653589793;
        d.wolff_steps = 1;
        d.seed = 0x5eed0000ull + i;
        d.j_xy = jx.data();
        d.n_j_xy = lz;
        d.j_z = jz.data();
        d.n_j_z = lz;
        d.binsize = 1;
        d.n_bins = 1;
        slsf_task* t = nullptr;
        rc = slsf_task_create(ctx, &d, &t);
        if (rc == SLSF_OK) {
            tasks.push_back(t);
            rc = slsf_task_init_random(t);
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == SLSF_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = set_error(SLSF_ERR_CUDA, "event creation failed");
    double best_rate = -1.0;
    slsf::KernelChoice best_c = cand[0];
    for (const slsf::KernelChoice& c : cand) {
        if (rc != SLSF_OK) break;
        /* warm-up, then a run sized to ~20 ms unless `sweeps` is given */
        rc = batch_run_impl(ctx, tasks.data(), tasks.size(), 1, nullptr, nullptr, &c);
        uint32_t s_run = sweeps ? sweeps : 2;
        for (int pass = 0; pass < 2 && rc == SLSF_OK; ++pass) {
            cudaEventRecord(e0, ctx->stream);
            rc = batch_run_impl(ctx, tasks.data(), tasks.size(), s_run, nullptr, nullptr, &c);
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rc != SLSF_OK) break;
            const double r = (double)tasks.size() * (double)v * s_run / (ms * 1e-3);
            if (sweeps || pass == 1) {
                if (r > best_rate) {
                    best_rate = r;
                    best_c = c;
                }
                break;
            }
            s_run = (uint32_t)std::min<double>(200.0, std::max<double>(2.0, s_run * 20.0 / std::max(ms, 1e-3f)));
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    for (slsf_task* t : tasks) slsf_task_destroy(t);
    if (rc != SLSF_OK) return rc;
    ctx->tune[shape_key(lx, ly, lz)] = best_c;
    ctx->tune_rate[shape_key(lx, ly, lz)] = best_rate;
    if (best) *best = from_choice(best_c);
    if (rate) *rate = best_rate;
    return SLSF_OK;
}

int slsf_tune_save(const slsf_ctx* ctx, const char* path) {
    if (!ctx || !path) return set_error(SLSF_ERR_INVALID, "NULL argument");
    FILE* f = std::fopen(path, "w");
    if (!f) return set_error(SLSF_ERR_INVALID, std::string("cannot write ") + path);
    std::fprintf(f, "# slsf-b200 kernel choices: lx ly lz kind cluster threads site_updates_per_s\n");
    for (const auto& kv : ctx->tune) {
        const uint64_t k = kv.first;
        const auto r = ctx->tune_rate.find(k);
        std::fprintf(f, "%u %u %u %u %u %u %.6e\n", (unsigned)(k & 0x1fffff), (unsigned)((k >> 21) & 0x1fffff),
                     (unsigned)(k >> 42), kv.second.kind, kv.second.cluster, kv.second.threads,
                     r == ctx->tune_rate.end() ? 0.0 : r->second);
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? SLSF_OK : set_error(SLSF_ERR_INVALID, std::string("cannot write ") + path);
}

int slsf_tune_load(slsf_ctx* ctx, const char* path) {
    if (!ctx || !path) return set_error(SLSF_ERR_INVALID, "NULL argument");
    FILE* f = std::fopen(path, "r");
    if (!f) return set_error(SLSF_ERR_INVALID, std::string("cannot read ") + path);
    char line[256];
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        unsigned lx, ly, lz, kind, cl, th;
        double r = 0.0;
        if (std::sscanf(line, "%u %u %u %u %u %u %lf", &lx, &ly, &lz, &kind, &cl, &th, &r) < 6) continue;
        const slsf::KernelChoice c = {kind, cl, th};
        if (!choice_feasible(c, lx, ly, lz, ctx->device)) continue;
        ctx->tune[shape_key(lx, ly, lz)] = c;
        if (r > 0.0) ctx->tune_rate[shape_key(lx, ly, lz)] = r;
    }
    std::fclose(f);
    return SLSF_OK;
}

int slsf_batch_run(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, uint32_t n_sweeps, slsf_sweep_stats* stats) {
    if (n_sweeps == 0) return SLSF_OK;
    return batch_run_impl(ctx, tasks, n, n_sweeps, nullptr, stats);
}

int slsf_batch_run_v(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, const uint32_t* sweeps,
                     slsf_sweep_stats* stats) {
    if (!sweeps && n) return set_error(SLSF_ERR_INVALID, "NULL argument");
    return batch_run_impl(ctx, tasks, n, 0, sweeps, stats);
}

int slsf_batch_get_bins(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, size_t n_rows, double* out,
                        uint64_t* measurements) {
    if (!ctx || (!tasks && n)) return set_error(SLSF_ERR_INVALID, "NULL argument");
    if (n == 0) return SLSF_OK;
    for (size_t i = 0; i < n; ++i) {
        if (!tasks[i] || tasks[i]->ctx != ctx) return set_error(SLSF_ERR_INVALID, "task does not belong to this context");
        if (n_rows > tasks[i]->n_bins) return set_error(SLSF_ERR_INVALID, "more bin rows requested than the task keeps");
        if (measurements) measurements[i] = tasks[i]->measurements;
    }
    if (!out || n_rows == 0) return SLSF_OK;
    if (int rc = bind_device(ctx)) return rc;
    const size_t per = n_rows * slsf::kBinCols;
    if (int rc = ensure_gather_capacity(ctx, n, n * per)) return rc;
    for (size_t i = 0; i < n; ++i) ctx->h_bin_src[i] = tasks[i]->bins;
    SLSF_CUDA(cudaMemcpyAsync(ctx->d_bin_src, ctx->h_bin_src, sizeof(double*) * n, cudaMemcpyHostToDevice, ctx->stream));
    slsf::launch_gather(ctx->d_bin_src, (uint32_t)n, (uint32_t)per, ctx->d_bin_out, ctx->stream);
    ctx->launches += 1;
    SLSF_CUDA(cudaGetLastError());
    SLSF_CUDA(cudaMemcpyAsync(ctx->h_bin_out, ctx->d_bin_out, 8 * n * per, cudaMemcpyDeviceToHost, ctx->stream));
    SLSF_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < n; ++i) bin_means(tasks[i], ctx->h_bin_out + i * per, out + i * per, n_rows);
    return SLSF_OK;
}

}  // extern "C"
