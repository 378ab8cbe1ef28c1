/*
 * Internal interface between the C ABI (capi.cu) and the kernel files.
 * Nothing here is exported from the shared library.
 */
#ifndef SLSF_ENGINE_H
#define SLSF_ENGINE_H

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace slsf {

/* Device-side counters of one task. */
enum StatSlot : int {
    kStatAccepted = 0,     /* Metropolis acceptances */
    kStatClusterSites = 1, /* sum of Wolff cluster sizes */
    kStatClusters = 2,     /* Wolff steps */
    kStatError = 3,        /* nonzero: a bounded device loop gave up */
    kStatSlots = 4
};

/* Error bits written to stats[kStatError]. */
constexpr unsigned long long kErrUnionFindLimit = 1ull;
constexpr unsigned long long kErrQueueLimit = 2ull;
constexpr unsigned long long kErrGrowthLimit = 4ull; /* a Wolff growth did not converge */

constexpr int kBinCols = 12;

/* Everything a kernel needs to know about one task. */
struct TaskView {
    float* theta;
    const float* jxy;
    const float* jz;
    uint32_t lx, ly, lz;
    float beta;
    float width;
    uint32_t wolff_steps;
    uint64_t seed;
    uint64_t metro_sweeps; /* Metropolis sweeps done before this launch */
    uint64_t wolff_done;   /* Wolff steps done before this launch */
    double* bins;          /* [n_bins][kBinCols] sums */
    uint32_t thermalization, binsize, n_bins;
    uint32_t sweeps;       /* sweeps of this task in a batched launch; 0: the launch's count */
    uint32_t loop_limit;   /* 0, or a lower bound on device loops (slsf_ctx_set_loop_limit) */
    unsigned long long* stats;
};

/* Correlations measured inside the sweeps of the one-CTA kernel
 * (slsf_task_corr_fuse), one entry per task view of a launch; bins NULL for
 * a task without them. */
struct ResidentCorr {
    double* bins;               /* [n_bins][values] sums */
    unsigned long long* count;  /* correlation measurements so far */
    uint32_t rxy, rz, binsize, n_bins, interval;
};

/* How a batched launch runs one lattice shape: which kernel, how many CTAs
 * hold a replica (cluster kernel) and how many threads a CTA has.  The
 * choice changes neither a task's trajectory nor its bins beyond FP32
 * partial-sum rounding. */
struct KernelChoice {
    uint32_t kind;    /* kKernelResident, kKernelCluster or kKernelGrid */
    uint32_t cluster; /* CTAs per replica (cluster kernel), else 1 */
    uint32_t threads; /* threads per CTA (batched kernels) */
};
constexpr uint32_t kKernelResident = 0, kKernelCluster = 1, kKernelGrid = 2;

/* Records `message` as the calling thread's slsf_last_error text and returns
 * `code` (capi.cu). */
int report_error(int code, const std::string& message);

/* ---- single-task kernels (kernels_plain.cu) ---- */
void launch_init_random(float* theta, uint32_t volume, uint64_t seed, cudaStream_t s);
void launch_metro_colour(const TaskView& t, uint64_t sweep, uint32_t colour, uint8_t* record,
                         cudaStream_t s);
/* Colour 0 of a sweep fused with the measurement of the state it starts from
 * (the observables' sums into `result`, added into `bin_row` if given). */
void launch_metro_colour0_measure(const TaskView& t, uint64_t sweep, double* partials, unsigned int* done,
                                  double* result, double* bin_row, cudaStream_t s);
/* One Wolff update; returns the number of kernels launched.  bonds [V] and
 * parent [V] are the task's scratch; with record_bonds the per-site bond
 * bits (+x, +y, +z in bits 0-2) are left in `bonds`. */
int launch_wolff(const TaskView& t, uint64_t wolff_counter, uint8_t* bonds, uint32_t* parent,
                 uint8_t* cluster_out, cudaStream_t s, float* phi_out, uint32_t seed_site[3],
                 bool record_bonds = false);
/* ---- Wolff on bit-packed bonds, the seed's cluster only (kernel_wolff_bits.cu) ---- */
/* Sides that are multiples of 32 (regions of 32^3 sites). */
bool wolff_bits_supports(uint32_t lx, uint32_t ly, uint32_t lz);
uint64_t wolff_bits_scratch_bytes(uint32_t lx, uint32_t ly, uint32_t lz);
/* `scratch` holds wolff_bits_scratch_bytes(); bond_bytes (or NULL) receives
 * the per-site bond bits, cluster_out (or NULL) the cluster mask. */
int launch_wolff_bits(const TaskView& t, uint64_t counter, void* scratch, uint8_t* bond_bytes, uint8_t* cluster_out,
                      cudaStream_t s, float* phi_out, uint32_t seed_site[3]);
/* Fused observables: writes 8 FP64 sums (mx, my, cos xyz, sin xyz) to result. */
void launch_measure(const TaskView& t, double* partials, unsigned int* done, double* result,
                    cudaStream_t s);
/* launch_measure that also adds the measurement's kBinCols stream values to
 * bin_row (a task's bin sums row). */
void launch_measure_into_bin(const TaskView& t, double* partials, unsigned int* done, double* result,
                             double* bin_row, cudaStream_t s);
/* Blocks of a measurement launch: one per 256 sites, at most kMeasureMaxBlocks
 * (148 SMs x 8), so its per-block partial sums fit kMeasureMaxBlocks rows. */
constexpr int kMeasureMaxBlocks = 148 * 8;
int measure_partial_blocks(uint32_t volume);
/* dst[i * per + k] = src[i][k] for i < n, k < per. */
void launch_gather(const double* const* src, uint32_t n, uint32_t per, double* dst, cudaStream_t s);

/* ---- correlation functions, batched over tasks (kernel_corr.cu) ---- */
/* One task of a correlation launch.  `partial` holds corr_partial_doubles()
 * of scratch; the measurement's corr_values() values (C_x(r), C_y(r),
 * C_xy(r), C_xy(z, r) z-major, C_z(r)) go to `values` and/or are added into
 * row *count / binsize of `bins` (rows past n_bins are dropped), after which
 * *count grows by one. */
struct CorrTask {
    const float* theta;
    uint32_t lx, ly, lz;
    uint32_t rxy, rz;   /* radii, already clamped to Lx/2, Ly/2 and Lz/2 */
    uint32_t item0;     /* the task's first work item in the launch */
    uint32_t binsize, n_bins;
    double* partial;
    double* values;     /* or NULL */
    double* bins;       /* [n_bins][values] sums, or NULL */
    unsigned long long* count; /* or NULL */
    uint32_t zunit0;    /* the task's first spectral z unit in the launch */
};
uint32_t corr_items(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
size_t corr_partial_doubles(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
uint32_t corr_values(uint32_t lz, uint32_t rxy, uint32_t rz);
/* Longest measured line of a task (the correlation tile's rows); its
 * longest line plus lags (corr_supports bounds it to 775 sites). */
uint32_t corr_len(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
uint32_t corr_ext(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
bool corr_supports(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
/* tasks_dev: n_tasks entries in item order (item0 and zunit0 ascending,
 * n_items and n_zunits in all) in device memory; or, for one task, `one` on
 * the host (passed to the kernels by value, no copy).  max_len, max_r,
 * max_nz: the largest corr_len, radius and corr_z_items of them (they size
 * the launches). */
cudaError_t launch_corr(const CorrTask* tasks_dev, const CorrTask* one, uint32_t n_tasks, uint32_t n_items,
                        uint32_t n_zunits, uint32_t max_len, uint32_t max_r, uint32_t max_nz, int sm_count,
                        cudaStream_t s);
/* z-line work items of a task (0 without C_z). */
uint32_t corr_z_items(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);
/* Spectral z units of a task: groups of consecutive z items whose power
 * spectra one block sums (0 off the spectral route). */
uint32_t corr_z_units(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);

/* ---- batched persistent engine, one CTA per replica (kernel_resident.cu) ---- */
bool resident_supports(uint32_t lx, uint32_t ly, uint32_t lz, int device);
/* Runs n_sweeps sweeps of every view in `views_dev` (device array of n);
 * `queue` is a zeroed device counter.  With `counters` (2 per view, may be
 * NULL) the Metropolis and Wolff counters come from there instead of the
 * views and are advanced in place, so a replayed launch continues.  max_* are the largest volume, row
 * count (Ly Lz) and Lz over the views; cube32: some view is a 32^3 lattice (its Wolff growth then runs
 * the warp-scan closure of bitgrow.cuh in 17 KB of extra shared memory). */
cudaError_t launch_resident(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                            int device, cudaStream_t s, uint32_t max_volume, uint32_t max_rows, uint32_t max_lz,
                            uint32_t threads, unsigned long long* counters, const ResidentCorr* corr_dev = nullptr,
                            uint32_t corr_doubles = 0, bool cube32 = false);
/* Shared doubles the fused correlation measurement of one task needs (0 without). */
uint32_t resident_corr_doubles(uint32_t ly, uint32_t lz, uint32_t rxy, uint32_t rz);

/* ---- batched persistent engine, one cluster per replica (kernel_cluster.cu) ---- */
/* Whether a cluster of c CTAs (a power of two up to 16) holds one replica of
 * these dimensions in shared memory. */
bool cluster_feasible(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t c, int device);
/* Smallest portable cluster size (1, 2, 4 or 8) that holds the replica, or 0. */
uint32_t batched_cluster_size(uint32_t lx, uint32_t ly, uint32_t lz, int device);
bool batched_supports(uint32_t lx, uint32_t ly, uint32_t lz, int device);
/* Runs n_sweeps sweeps of every task view in `views_dev` (device array of
 * n, all needing the same cluster size) with a persistent grid of clusters;
 * `queue` is a zeroed device counter the kernel consumes.  max_* are the
 * largest per-CTA slab volume, slab row count, Lz, Lx Ly and Lx over the views. */
cudaError_t launch_batched(const TaskView* views_dev, uint32_t n, uint32_t n_sweeps, unsigned int* queue,
                           int device, cudaStream_t s, uint32_t cluster, uint32_t threads, uint32_t max_vs,
                           uint32_t max_rows, uint32_t max_lz, uint32_t max_plane, uint32_t max_lx,
                           unsigned long long* counters);

}  // namespace slsf

#endif /* SLSF_ENGINE_H */
