/*
 * slsf_host.h -- host layer above the C ABI of slsf_gpu.h (libslsf_host.so).
 *
 * The reference's host side is Rust (ThetaModel's MonteCarlo impl, carlo-mc's
 * Runner, Context and binning, the task expansion).  Its toolchain is not
 * available here, so this C++ layer restates the parts that drive the hot
 * path, calling the GPU library only through slsf_gpu.h:
 *   - the model driver: ThetaModel::new/init/sweep/measure and
 *     finalize_estimates (src/model.rs:308-477, :857-934) with carlo-style
 *     binned estimates (BinnedEstimate::from_samples, src/tests.rs:436-446);
 *   - the task expansion and seed formula (src/model.rs:697-810);
 *   - a continuous-batching server: requests of mixed size are admitted by
 *     device-memory budget as memory frees up, advanced together in
 *     persistent launches (slsf_batch_run_v), and retired with their binned
 *     estimates and latency.
 * Status codes are those of slsf_gpu.h; slsf_host_last_error gives the
 * message of the calling thread's last failed call into this layer (a GPU
 * library failure's text is copied there).
 */
#ifndef SLSF_HOST_H
#define SLSF_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "slsf_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

size_t slsf_host_last_error(char* buf, size_t len);

/* Derived observables (register_theta_evaluables, src/model.rs:857-888). */
#define SLSF_DERIVED 5 /* Magnetization, Chi, SpecificHeat, RhoXY, RhoZ */

/* Binned estimates of one task: bin means of the measurement stream
 * (SLSF_BIN_COLS columns, slsf_gpu.h), their standard errors over bins, and
 * the derived observables with jackknife errors. */
typedef struct slsf_estimates {
    uint64_t measurements;
    uint32_t n_bins;
    double acceptance;
    double mean[SLSF_BIN_COLS];
    double err[SLSF_BIN_COLS];
    double derived[SLSF_DERIVED];
    double derived_err[SLSF_DERIVED];
} slsf_estimates;

/* Binned estimate of a series (BinnedEstimate::from_samples): bins are means
 * of complete chunks of `binsize`; stderr = sample std of bins / sqrt(#bins).
 * Fails with "binsize is larger than the sample series". */
int slsf_binned_estimate(const double* samples, size_t n, size_t binsize, double* mean, double* stderr_out,
                         size_t* n_bins);

/* Estimates from bin means [n_bins][SLSF_BIN_COLS] of a task of `volume`
 * sites at inverse temperature beta (finalize_theta_estimates,
 * src/model.rs:906-934). */
int slsf_estimates_from_bins(const double* bin_means, size_t n_bins, double volume, double beta,
                             slsf_estimates* out);

/* ---------------------------------------------------------------- tasks */

/* ThetaTask (src/model.rs:20-47).  j_xy_array / j_z_array may be NULL: the
 * layer couplings are then drawn two-point from FastRng(disorder_seed),
 * J_xy first (src/model.rs:317-345). */
typedef struct slsf_theta_task {
    uint32_t lx, ly, lz;
    double temperature;
    double j_xy, delta_j_xy, j_z_mean, delta_j_z;
    uint64_t disorder_seed;
    uint64_t seed;
    uint32_t sweeps, thermalization, binsize;
    double proposal_width;
    uint32_t wolff_steps;
    const double* j_xy_array;
    const double* j_z_array;
} slsf_theta_task;

/* The run seed of make_theta_tasks (src/model.rs:742-747). */
uint64_t slsf_task_seed(uint64_t base_seed, uint32_t l_z, uint32_t sample, double temperature, double delta_j_xy,
                        double delta_j_z);

/* Layer couplings of a task: explicit arrays, or two-point disorder
 * (src/initialization.rs:5-31) from FastRng(disorder_seed). */
int slsf_task_couplings(const slsf_theta_task* task, double* j_xy, double* j_z);

/* Runs one task the way carlo-mc drives ThetaModel: new, init,
 * `thermalization` sweeps, then `sweeps` x (sweep + measure), then the
 * binned estimates.  batched != 0 runs it through the persistent kernel
 * (bins on the device), otherwise through the single-task entry points. */
int slsf_model_run(slsf_ctx* ctx, const slsf_theta_task* task, int batched, slsf_estimates* out);

/* ---------------------------------------------------------------- server */

typedef struct slsf_server slsf_server;

typedef struct slsf_server_config {
    uint32_t epoch_sweeps; /* sweeps per launch: the admission granularity (default 100) */
    uint32_t max_active;   /* tasks on the device at once (0: only the budget limits) */
    uint64_t budget_bytes; /* device bytes for task state (0: the context's budget) */
    uint32_t keep_bins;    /* nonzero: keep each completed request's bin means for
                              slsf_server_take_bins */
} slsf_server_config;

/* One request: a task, its sweep count and measurement plan. */
typedef struct slsf_request {
    uint64_t tag; /* echoed in the result */
    uint32_t lx, ly, lz;
    double temperature;
    double proposal_width;
    uint32_t wolff_steps;
    uint64_t seed;
    const double* j_xy; /* [lz], copied at submission */
    const double* j_z;  /* [lz], copied at submission */
    uint32_t sweeps;         /* total sweeps */
    uint32_t thermalization; /* sweeps before the first measurement */
    uint32_t n_bins;         /* bins of the measured sweeps (used when binsize is 0) */
    uint32_t binsize;        /* sweeps per bin; 0: measured sweeps / n_bins.  Only complete
                                bins are kept (carlo drops a partial last bin). */
} slsf_request;

typedef struct slsf_result {
    uint64_t tag;
    int status;            /* SLSF_OK, or why the request failed or was cancelled */
    char message[160];     /* error text when status != SLSF_OK */
    double submit_s;       /* seconds since the server was created */
    double admit_s;
    double finish_s;
    uint64_t sweeps;
    uint64_t accepted;
    uint64_t cluster_sites;
    slsf_estimates est;
} slsf_result;

typedef struct slsf_server_stats {
    uint64_t submitted, completed, failed, cancelled;
    uint64_t epochs, launches;
    uint64_t site_updates;    /* Metropolis proposals of finished and running tasks */
    double busy_s;            /* wall seconds spent in epochs */
    uint64_t peak_active;
    uint64_t peak_bytes;
} slsf_server_stats;

int slsf_server_create(slsf_ctx* ctx, const slsf_server_config* cfg, slsf_server** out);
/* Stops the worker (if started) and destroys every task still held. */
int slsf_server_destroy(slsf_server* s);
/* Queues a request (thread-safe, never blocks on the GPU).  Requests that
 * can never fit the budget, or that fail validation, come back as results
 * with an error status. */
int slsf_server_submit(slsf_server* s, const slsf_request* r);
/* Cancels a queued or running request; its result reports SLSF_ERR_STATE
 * "cancelled".  Returns SLSF_ERR_INVALID if the tag is unknown. */
int slsf_server_cancel(slsf_server* s, uint64_t tag);
/* One epoch on the calling thread: retire finished tasks, admit queued
 * requests that fit, advance every active task by up to epoch_sweeps. */
int slsf_server_step(slsf_server* s, uint32_t* active, uint32_t* pending);
/* Runs epochs on a worker thread until slsf_server_stop. */
int slsf_server_start(slsf_server* s);
int slsf_server_stop(slsf_server* s);
/* Blocks until nothing is queued or running, or timeout_s passes
 * (SLSF_ERR_TIMEOUT). */
int slsf_server_wait_idle(slsf_server* s, double timeout_s);
/* Moves up to `max` finished results to `out` (thread-safe). */
int slsf_server_poll(slsf_server* s, slsf_result* out, size_t max, size_t* n);
int slsf_server_stats_get(slsf_server* s, slsf_server_stats* out);
/* The complete bins of a finished request, kept when the server was created
 * with keep_bins (the measurement_bins of ThetaTaskResult,
 * src/model.rs:81, that src/results.rs:55-105 writes to .meas.h5): bin means
 * [n_rows][SLSF_BIN_COLS], one row per `binsize` measured sweeps.  *n_rows
 * receives the row count; with out != NULL and max_rows >= *n_rows the rows
 * are copied and released.  SLSF_ERR_INVALID when nothing is kept for the
 * tag (not finished, failed, cancelled, already taken, or keep_bins off). */
int slsf_server_take_bins(slsf_server* s, uint64_t tag, double* out, size_t max_rows, size_t* n_rows);
/* Checkpoint of the serving loop (carlo-mc's checkpoint directory and
 * restart, src/results.rs:211-239): with the worker stopped, writes one file
 * per unfinished request to `dir` -- queued ones as submitted, running ones
 * with their progress and the task's device state (slsf_task_state_save) --
 * and keeps running them.  Finished results stay with slsf_server_poll. */
int slsf_server_checkpoint(slsf_server* s, const char* dir, size_t* n_saved);
/* Queues the requests a checkpoint saved in `dir`, in tag order; running
 * ones resume where they stopped and finish with the results they would
 * have had without the interruption. */
int slsf_server_restore(slsf_server* s, const char* dir, size_t* n_restored);

#ifdef __cplusplus
}
#endif

#endif /* SLSF_HOST_H */
