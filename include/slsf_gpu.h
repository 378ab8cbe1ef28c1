/*
 * slsf_gpu.h -- C ABI of the B200 (sm_100a) update-and-measure library for
 * the 3D layered-disorder XY model of SLSF-rs.
 *
 * The reference is a Rust crate whose hot path sits behind the carlo-mc
 * `MonteCarlo` trait implemented by `ThetaModel` (src/model.rs:308-477) and
 * behind the re-exported lower-level functions of src/lib.rs:21-29.  It has no
 * FFI of its own; every entry point below is the `extern "C"` function a Rust
 * `GpuThetaModel` would bind in place of one of those calls, and its comment
 * cites the reference item it replaces.
 *
 * Conventions
 *   - Every function returns an int status: SLSF_OK (0) or an SLSF_ERR_*
 *     code.  slsf_last_error() copies the calling thread's last message; for
 *     argument errors that message is the reference's string, character for
 *     character (src/types.rs:120-129, :373-385, src/updates.rs:430-438,
 *     src/model.rs:318-348).
 *   - Handles are single-owner: one host thread issues all calls on a context
 *     and its tasks, as carlo-mc's Runner does (src/results.rs:200-202).
 *   - Angles cross the boundary as FP32 (the device state).  J arrays cross
 *     as FP64, as in ThetaTask (src/model.rs:45-46), and are stored as FP32.
 *   - Randoms are Philox4x32-10 keyed by (seed, sweep counter, purpose,
 *     site); a task's trajectory depends only on its seed, counters and state,
 *     never on what else runs on the device.
 *   - There is no CPU fallback: without a usable CUDA device every compute
 *     entry point fails with SLSF_ERR_CUDA.
 */
#ifndef SLSF_GPU_H
#define SLSF_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLSF_OK 0
#define SLSF_ERR_INVALID 1 /* argument rejected; message is the reference's string */
#define SLSF_ERR_CUDA 2    /* CUDA runtime or device error, or no device */
#define SLSF_ERR_BUDGET 3  /* allocation would exceed the context's HBM budget */
#define SLSF_ERR_TIMEOUT 4 /* a bounded device loop hit its iteration limit */
#define SLSF_ERR_STATE 5   /* call not valid in the handle's current state */

typedef struct slsf_ctx slsf_ctx;
typedef struct slsf_task slsf_task;

/* Task parameters: the fields of ThetaTask (src/model.rs:20-47) that the
 * update-and-measure step reads.  j_xy / j_z are the explicit per-layer
 * arrays (ThetaTask::j_xy_array / j_z_array); the two-point disorder
 * generator stays on the host. */
typedef struct slsf_task_desc {
    uint32_t lx, ly, lz;
    double temperature;
    double proposal_width;
    uint32_t wolff_steps;
    uint64_t seed;
    const double* j_xy;
    size_t n_j_xy;
    const double* j_z;
    size_t n_j_z;
    /* Measurement plan of the batched engine: sweeps before the first
     * measurement, measurements per bin, and the number of bins to keep. */
    uint32_t thermalization;
    uint32_t binsize;
    uint32_t n_bins;
} slsf_task_desc;

/* ThetaObservables (src/types.rs:253-263). */
typedef struct slsf_observables {
    double energy;
    double magnetization_squared;
    double cos_x, cos_y, cos_z;
    double sin_x, sin_y, sin_z;
} slsf_observables;

/* Counters accumulated over the sweeps of one call. */
typedef struct slsf_sweep_stats {
    uint64_t sweeps;
    uint64_t accepted;            /* Metropolis acceptances (sum over sweeps) */
    uint64_t wolff_clusters;      /* Wolff steps performed */
    uint64_t wolff_cluster_sites; /* sum of cluster sizes */
} slsf_sweep_stats;

/* Columns of one measurement in the per-task bin accumulators: the
 * observable stream of ThetaModel::measure (src/model.rs:406-409) and
 * measure_theta_helicity (src/model.rs:890-904). */
#define SLSF_BIN_COLS 12 /* Energy, EnergySquared, MagnetizationSquared,
                            cos_x, cos_y, cos_z, sin_x, sin_y, sin_z,
                            sin2_x, sin2_y, sin2_z */

/* ---------------------------------------------------------------- library */

/* Copies the calling thread's last error message (NUL-terminated, truncated
 * to len) and returns its full length. */
size_t slsf_last_error(char* buf, size_t len);

/* Library version string. */
const char* slsf_version(void);

/* Creates a context on CUDA device `device` that may allocate up to
 * `budget_bytes` of device memory (0 = 90% of the device's free memory).
 * No reference counterpart: carlo-mc owns no device. */
int slsf_ctx_create(int device, uint64_t budget_bytes, uint32_t flags, slsf_ctx** out);
int slsf_ctx_destroy(slsf_ctx* ctx);
/* Device bytes in use by the context's tasks, and its budget. */
int slsf_ctx_memory(const slsf_ctx* ctx, uint64_t* used, uint64_t* budget);
/* Device bytes a task of these dimensions and measurement plan would take. */
uint64_t slsf_task_bytes(uint32_t lx, uint32_t ly, uint32_t lz, uint32_t n_bins);
/* Runs the context's work on `stream` (a cudaStream_t; NULL restores the
 * context's own stream), so a host framework can order and time it with its
 * own events.  No reference counterpart. */
int slsf_ctx_set_stream(slsf_ctx* ctx, void* stream);
/* Number of kernels the library has launched on this context. */
int slsf_ctx_launch_count(const slsf_ctx* ctx, uint64_t* launches);
/* Lowers the bound of every device loop of this context's later launches
 * (union-find path lengths and retries, Wolff growth passes) to `limit`;
 * 0 restores the defaults (paths <= V, 2^22 union retries, growth <= V
 * passes).  A loop that reaches its bound makes the kernel record the
 * failure and return, and the call reports SLSF_ERR_TIMEOUT.  For testing
 * the error path without faulting a GPU; the task's state after such a
 * failure is undefined.  No reference counterpart. */
int slsf_ctx_set_loop_limit(slsf_ctx* ctx, uint32_t limit);

/* ---------------------------------------------------------------- sessions
 * A batch session captures one batched step -- n_sweeps sweeps of every task,
 * with the kernel groups of slsf_batch_run -- in a CUDA graph once, keeps the
 * task table on the device and replays the graph per step; the tasks'
 * counters advance on the device and are mirrored on the host after each
 * step.  While a session is open its tasks refuse the calls that change
 * their state (SLSF_ERR_STATE); measuring and reading angles, counters and
 * bins work between steps.  Lattices too large for one thread-block cluster
 * (run by the grid-wide kernels) are refused.  No reference counterpart. */
typedef struct slsf_batch slsf_batch;

int slsf_batch_open(slsf_ctx* ctx, slsf_task* const* tasks, size_t n, uint32_t n_sweeps, slsf_batch** out);
/* Replays the step and waits for it; stats (may be NULL) receives each
 * task's counters of this step, in the order of the tasks at open. */
int slsf_batch_step(slsf_batch* b, slsf_sweep_stats* stats);
int slsf_batch_close(slsf_batch* b);
/* n_cycles times: the session's step followed by one correlation
 * measurement of every task (slsf_batch_correlations; every task needs
 * slsf_task_corr_setup), all queued back to back with the step counters
 * summed on the device; waits once at the end.  stats (may be NULL) receives
 * each task's counters summed over the cycles.  The loop of
 * ThetaModel::measure with correlation_interval = the session's sweeps. */
int slsf_batch_step_correlations(slsf_batch* b, uint32_t n_cycles, slsf_sweep_stats* stats);

/* ---------------------------------------------------------------- tuning
 * How the batched entry points run each lattice shape: the one-CTA kernel
 * with a CTA of `threads`, the cluster kernel with `cluster` CTAs per replica
 * (a power of two up to 16) of `threads` each, or the grid-wide single-task
 * kernels.  The choice changes neither a task's trajectory nor its bins
 * beyond FP32 partial-sum rounding, only the speed.  A context starts from a
 * default per shape; slsf_autotune times every feasible choice on scratch
 * replicas and keeps the fastest; the table can be saved and loaded.  No
 * reference counterpart (the reference's tasks are single-threaded). */
#define SLSF_KERNEL_RESIDENT 0
#define SLSF_KERNEL_CLUSTER 1
#define SLSF_KERNEL_GRID 2

typedef struct slsf_kernel_choice {
    uint32_t kind;    /* SLSF_KERNEL_* */
    uint32_t cluster; /* CTAs per replica (SLSF_KERNEL_CLUSTER), else 1 */
    uint32_t threads; /* threads per CTA */
} slsf_kernel_choice;

/* The choice the context uses for this shape (its table entry or the default). */
int slsf_tune_get(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, slsf_kernel_choice* out);
/* Sets the shape's choice; SLSF_ERR_INVALID if it cannot hold the lattice. */
int slsf_tune_set(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, const slsf_kernel_choice* c);
/* Times every feasible choice for the shape over `sweeps` sweeps of scratch
 * replicas that fill the GPU (0: a default that runs ~20 ms per choice),
 * stores the fastest in the table and returns it with its rate in
 * site-updates/s.  Uses device memory for the scratch replicas while it runs. */
int slsf_autotune(slsf_ctx* ctx, uint32_t lx, uint32_t ly, uint32_t lz, uint32_t sweeps, slsf_kernel_choice* best,
                  double* site_updates_per_s);
/* The table as text lines "lx ly lz kind cluster threads rate"; loading
 * skips entries that this device cannot run. */
int slsf_tune_save(const slsf_ctx* ctx, const char* path);
int slsf_tune_load(slsf_ctx* ctx, const char* path);

/* ---------------------------------------------------------------- one task */

/* Replaces ThetaModel::new (src/model.rs:314-371): validates the lattice
 * dimensions (src/types.rs:120-129), the J array lengths and signs
 * (src/model.rs:318-348), allocates the device state and uploads J.  Like the
 * reference, T and proposal_width are checked when a sweep runs. */
int slsf_task_create(slsf_ctx* ctx, const slsf_task_desc* desc, slsf_task** out);
int slsf_task_destroy(slsf_task* task);

/* Replaces ThetaModel::init (src/model.rs:373-377): theta_i = 2 pi u_i with
 * u_i from the task's Philox stream (purpose INIT). */
int slsf_task_init_random(slsf_task* task);
/* InitMode::Cold (src/initialization.rs:58): all angles 0. */
int slsf_task_init_cold(slsf_task* task);
/* ThetaLattice::theta as FP32, index x + Lx (y + Ly z) (src/types.rs:146-149). */
int slsf_task_set_angles(slsf_task* task, const float* theta, size_t n);
int slsf_task_get_angles(slsf_task* task, float* theta, size_t n);

/* Checkpoint counters: Metropolis sweeps and Wolff steps done so far.  With
 * the angles they are the whole random state (the serde FastRng position of
 * src/types.rs:9-37 has no other counterpart). */
int slsf_task_get_counters(const slsf_task* task, uint64_t* metro_sweeps, uint64_t* wolff_steps);
int slsf_task_set_counters(slsf_task* task, uint64_t metro_sweeps, uint64_t wolff_steps);

/* Replaces ThetaModel::sweep (src/model.rs:379-400) n_sweeps times: one
 * checkerboard Metropolis sweep then wolff_steps Wolff updates per sweep.
 * stats may be NULL. */
int slsf_task_sweep(slsf_task* task, uint32_t n_sweeps, slsf_sweep_stats* stats);

/* Replaces metropolis_sweep_with_scratch (src/updates.rs:440-486): returns
 * accepted / V. */
int slsf_task_metropolis_sweep(slsf_task* task, double* acceptance);

/* One colour of the checkerboard sweep (the parity loop body of
 * src/updates.rs:455-483) without advancing the sweep counter.  When
 * accept_mask is not NULL it receives one byte per site: 1 if the site was
 * updated and accepted, 0 otherwise.  accepted may be NULL. */
int slsf_task_metropolis_color(slsf_task* task, uint32_t color, uint8_t* accept_mask,
                               uint64_t* accepted);

/* Replaces wolff_cluster_step_with_theta_scratch (src/updates.rs:551-620):
 * bond activation, cluster labelling from the seed site, reflection.
 * cluster_size may be NULL. */
int slsf_task_wolff_step(slsf_task* task, uint64_t* cluster_size);

/* A Wolff step that also exports, per site, the active-bond bits (bit 0/1/2
 * = bond to +x/+y/+z) and the cluster membership, plus the reflection axis
 * and seed site it used.  Any output pointer may be NULL. */
int slsf_task_wolff_step_debug(slsf_task* task, uint8_t* bonds, uint8_t* cluster, float* phi,
                               uint32_t seed_site[3], uint64_t* cluster_size);

/* Replaces measure_theta_observables_with_scratch (src/observables.rs:80-154):
 * one fused pass; per-site terms in FP32, sums in FP64. */
int slsf_task_measure(slsf_task* task, slsf_observables* out);

/* Replaces measure_theta_correlations_with_scratch (src/observables.rs:166-265)
 * for explicit rmax values (clamped to L/2 as at :177-181).  Outputs (any may
 * be NULL): corr_x, corr_y, corr_xy [rmax_xy], corr_xy_by_z [lz][rmax_xy],
 * corr_z [rmax_z].  Blocks until the values are on the host. */
int slsf_task_correlations(slsf_task* task, uint32_t rmax_xy, uint32_t rmax_z, double* corr_x,
                           double* corr_y, double* corr_xy, double* corr_xy_by_z,
                           double* corr_z);

/* Correlation measurements binned on the device, for ThetaModel::measure's
 * correlation observables (src/model.rs:410-438).  slsf_task_corr_setup
 * gives the task radii (clamped as slsf_task_correlations clamps them; both
 * 0 turns the measurements off and frees the bins), a bin size and n_bins
 * rows of bin sums, and resets the measurement count.  One measurement
 * (slsf_batch_correlations) produces *n_values values in the order
 *   CorrX_r (r = 1..R), CorrY_r, CorrXY_r, CorrXY_z{z}_r (z-major), CorrZ_r (r = 1..R_z)
 * with R and R_z the clamped radii, n_values = 3 R + L_z R + R_z, and adds
 * them into row count / binsize (rows past n_bins are not kept). */
int slsf_task_corr_setup(slsf_task* task, uint32_t rmax_xy, uint32_t rmax_z, uint32_t binsize, uint32_t n_bins,
                         size_t* n_values);
/* Correlations measured inside the batched sweeps: with interval > 0,
 * every batched run or session step of the task measures the correlation
 * functions of the state after each sweep whose measurement index
 * m = sweep - thermalization is a multiple of `interval` into the bins of
 * slsf_task_corr_setup (ThetaModel::measure, src/model.rs:410, with
 * correlation_interval = interval): from the replica in shared memory on the
 * one-CTA kernel (even L_x <= 32 and a replica that fits shared memory), or
 * by the correlation kernels queued after those sweeps on the grid-wide
 * kernels (lattices too large for one cluster; not in sessions).  Tasks on
 * the cluster kernel are refused.  0 turns it off.
 * Such a task refuses the separate measurements (slsf_batch_correlations,
 * slsf_batch_step_correlations).  Values agree with the separate kernels to
 * FP32 partial-sum rounding. */
int slsf_task_corr_fuse(slsf_task* task, uint32_t interval);
/* The first n_rows rows of bin means ([n_rows][n_values]) and the number of
 * correlation measurements taken (either output may be NULL).  Blocks. */
int slsf_task_corr_bins(const slsf_task* task, double* bin_means, size_t n_rows, uint64_t* count);
/* One correlation measurement of every task (each set up with
 * slsf_task_corr_setup) in two launches for the whole batch, queued on the
 * context's stream after the work already queued there (a batched run's
 * sweeps or a session step included); does not wait for it.  Tasks may
 * differ in size and may belong to an open batch session (the measurement
 * only reads their angles).  Repeating the same task list reuses the
 * device task table. */
int slsf_batch_correlations(slsf_ctx* ctx, slsf_task* const* tasks, size_t n_tasks);

/* Per-task bin accumulators of the batched engine: n_bins rows of
 * SLSF_BIN_COLS bin means, and the number of measurements taken so far. */
int slsf_task_get_bins(const slsf_task* task, double* bins, size_t n_rows, uint64_t* measurements);
int slsf_task_reset_bins(slsf_task* task);

/* Device state of a task as one byte blob, for checkpoints: the parts of
 * ThetaModel's serialized state (src/model.rs:255-271) that live on the
 * device -- angles, counters (Metropolis sweeps, Wolff steps, measurements,
 * correlation measurements), bin sums and correlation bin sums -- with the
 * task's configuration to check against.  The random streams are keyed by
 * (seed, counters, site), so a task loaded from a state continues exactly as
 * the saved one would have.  `user` carries four caller words through the
 * blob (e.g. host-side acceptance sums; may be NULL).  Loading requires a
 * task created with the same description (dimensions, seed, temperature,
 * proposal width, Wolff steps, couplings, thermalization, bins) and the same
 * correlation set-up; anything else fails with "state does not match the
 * task: ...". */
int slsf_task_state_size(const slsf_task* task, size_t* bytes);
int slsf_task_state_save(const slsf_task* task, const uint64_t user[4], void* buf, size_t bytes);
int slsf_task_state_load(slsf_task* task, const void* buf, size_t bytes, uint64_t user[4]);

/* ---------------------------------------------------------------- batches */

/* Runs n_sweeps sweeps of every task in `tasks` in one persistent launch
 * (the carlo-mc Runner's per-task loop of src/results.rs:200-202, batched):
 * each sweep is ThetaModel::sweep followed, once the task's thermalization
 * is done, by ThetaModel::measure accumulated into the task's bins.  Tasks
 * may have different sizes.  stats (one per task) may be NULL.  Blocks until
 * the work is done. */
int slsf_batch_run(slsf_ctx* ctx, slsf_task* const* tasks, size_t n_tasks, uint32_t n_sweeps,
                   slsf_sweep_stats* stats);

/* slsf_batch_run with its own sweep count per task (sweeps[i]; tasks with 0
 * are left out of the launch): how a scheduler advances tasks with different
 * remaining work in one persistent launch (carlo-mc's dynamic runner,
 * src/results.rs:211-239, batched). */
int slsf_batch_run_v(slsf_ctx* ctx, slsf_task* const* tasks, size_t n_tasks, const uint32_t* sweeps,
                     slsf_sweep_stats* stats);

/* Bin means of many tasks in one device gather and one copy: out is
 * [n_tasks][n_rows][SLSF_BIN_COLS]; measurements (may be NULL) receives each
 * task's measurement count.  The batched form of slsf_task_get_bins, feeding
 * carlo-mc's binned estimates (src/model.rs:906-934). */
int slsf_batch_get_bins(slsf_ctx* ctx, slsf_task* const* tasks, size_t n_tasks, size_t n_rows,
                        double* out, uint64_t* measurements);

/* ---------------------------------------------------- no device allocation */

/* Largest lattice slsf_measure_noalloc accepts (2^31 - 1 sites). */
#define SLSF_NOALLOC_MAX_SITES 2147483647ull

/* The fused measurement of slsf_task_measure for a lattice held in the
 * caller's own device memory (theta [Lx Ly Lz], j_xy [Lz], j_z [Lz], FP32,
 * layout x + Lx (y + Ly z)), for callers that cannot allocate device memory:
 * hosts whose own memory pool owns the device, services under a fixed device
 * memory budget, and loops that must not risk cudaMalloc/cudaFree's
 * device-wide synchronisation.  It calls no allocating routine.  Its scratch
 * (per-block partial sums, about 75 KiB) is a static device array that every
 * GPU loading this library holds until the process exits.
 *   - Lattices beyond SLSF_NOALLOC_MAX_SITES sites are rejected.
 *   - All calls share that array and it keeps the last call's contents;
 *     calls that overlap on the GPU race on it, so serialise them.
 *   - The first call on a device sets the scratch up on the current device
 *     (takes its address, zeroes its counter); make it before any stream
 *     capture.
 * `stream` is a cudaStream_t (NULL: the default stream); the call waits for
 * it.  No counterpart in the reference. */
int slsf_measure_noalloc(const float* theta, const float* j_xy, const float* j_z, uint32_t lx, uint32_t ly,
                         uint32_t lz, void* stream, slsf_observables* out);

#ifdef __cplusplus
}
#endif

#endif /* SLSF_GPU_H */
