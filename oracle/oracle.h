/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of SLSF-rs's update-and-measure path.  It is the
 * checker for the CUDA library and the timed CPU baseline; nothing in the
 * product library links, loads or calls it.  Only tests/, the smoke check and
 * the benchmark's CPU-baseline leg may use it.
 *
 * Every function names the reference lines it restates.  The reference is a
 * Rust crate that cannot be built here; its arithmetic comes from three crates
 * that are not in the reference tree:
 *   - sleef 0.3.3 (sincos_u10, exp_u10, cos_u10): replaced by glibc sin, cos,
 *     exp; the reference pins sleef only to within 1e-14 of std
 *     (src/tests.rs:11-23);
 *   - rand 0.10.2 (f64, bool and range sampling from FastRng): restated from
 *     rand's published sampling methods (53-bit multiply for f64, sign of the
 *     low 32-bit word for bool, Canon's widening-multiply method for ranges);
 *     no reference test pins a trajectory, so trajectory-level parity with the
 *     Rust binary is unpinned;
 *   - carlo-mc @3547ec9 (binning, estimates): restated from the binning
 *     known-answer test (src/tests.rs:436-446).
 *
 * Error strings are the reference's, character for character.
 */
#ifndef SLSF_ORACLE_H
#define SLSF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FastRng: SplitMix64 stream (src/types.rs:9-82) ---- */
typedef struct or_rng {
    uint64_t seed;
    uint64_t state;
    uint64_t draws;
} or_rng;

void or_rng_seed(or_rng* rng, uint64_t seed);
void or_rng_set_position(or_rng* rng, uint64_t position);
uint64_t or_rng_next_u64(or_rng* rng);
double or_rng_f64(or_rng* rng);
int or_rng_bool(or_rng* rng);
uint64_t or_rng_range(or_rng* rng, uint64_t n);

const char* or_last_error(void);

/* ---- scalar helpers (src/types.rs:334-385, src/updates.rs:498-506) ---- */
double or_wrap_angle(double theta);
double or_wolff_add_probability(double beta, double coupling, double ri, double rj);
double or_wolff_reflect_angle(double theta, double phi);
int or_validate_temperature(double temperature);
int or_validate_proposal_width(double width);

/* ---- initialisation (src/initialization.rs) ---- */
int or_two_point_disorder(double* values, size_t n, double mean, double delta, or_rng* rng,
                          const char* coupling_name);
void or_uniform_disorder(double* values, size_t n, double lo, double hi, uint64_t seed);
void or_init_angles(double* theta, size_t n, int cold, or_rng* rng);

/* ---- observables on an FP64 lattice (src/observables.rs) ---- */
typedef struct or_obs {
    double energy;
    double magnetization_squared;
    double cos_x, cos_y, cos_z;
    double sin_x, sin_y, sin_z;
} or_obs;

double or_measure_energy(size_t lx, size_t ly, size_t lz, const double* theta, const double* jxy,
                         const double* jz);
double or_magnetization_squared(size_t n, const double* theta);
void or_helicity_sums(size_t lx, size_t ly, size_t lz, const double* theta, const double* jxy,
                      const double* jz, double out[6]);
int or_helicity_modulus(size_t lx, size_t ly, size_t lz, const double* theta, const double* jxy,
                        const double* jz, double temperature, double out[3]);
void or_measure_observables(size_t lx, size_t ly, size_t lz, const double* theta,
                            const double* jxy, const double* jz, or_obs* out);
/* corr_xy_by_z is [lz][rmax_xy_eff]; rmax < 0 means "None". Writes the
 * effective rmax values to eff[2]. */
void or_measure_correlations(size_t lx, size_t ly, size_t lz, const double* theta, long rmax,
                             long rmax_xy, long rmax_z, double* corr_x, double* corr_y,
                             double* corr_xy, double* corr_xy_by_z, double* corr_z,
                             size_t eff[2]);

/* ---- the model (ThetaModel, src/model.rs:254-442) ---- */
typedef struct or_model or_model;

int or_model_new(size_t lx, size_t ly, size_t lz, const double* jxy, size_t n_jxy,
                 const double* jz, size_t n_jz, double temperature, double proposal_width,
                 size_t wolff_steps, uint64_t seed, or_model** out);
void or_model_free(or_model* m);
void or_model_init(or_model* m, int cold);
void or_model_set_theta(or_model* m, const double* theta);
void or_model_get_theta(const or_model* m, double* theta);
uint64_t or_model_rng_position(const or_model* m);
int or_model_metropolis_sweep(or_model* m, int use_batch8, double* acceptance);
int or_model_local_metropolis_step(or_model* m, double proposal_width, int* accepted);
int or_model_wolff_step(or_model* m, size_t* cluster_size);
int or_model_sweep(or_model* m, int use_batch8);
void or_model_measure(const or_model* m, or_obs* out);
/* Per-measurement stream of ThetaModel::measure (src/model.rs:402-409,
 * :890-904): columns Energy, EnergySquared, MagnetizationSquared, cos_x,
 * cos_y, cos_z, sin_x, sin_y, sin_z, sin2_x, sin2_y, sin2_z. Runs
 * `thermalization` sweeps, then `sweeps` sweeps each followed by a measure. */
#define OR_SERIES_COLS 12
int or_model_run_series(or_model* m, size_t thermalization, size_t sweeps, int use_batch8,
                        double* series, double* acceptance);

/* ---- the standalone driver (src/simulation.rs:13-230) ---- */
typedef struct or_sim_options {
    size_t thermal_sweeps;
    size_t measure_sweeps;
    size_t measure_interval;
    double proposal_width;
    size_t wolff_steps;
    size_t correlation_interval;
    long correlation_rmax;    /* -1 = None */
    long correlation_rmax_xy; /* -1 = None */
    long correlation_rmax_z;  /* -1 = None */
    int init_cold;
} or_sim_options;

typedef struct or_sim_result {
    double energy;
    double rho_sx, rho_sy, rho_sz;
    double std_rho_sx, std_rho_sy, std_rho_sz;
    double magnetization_squared;
    double chi;
    double acceptance;
    size_t num_measurements;
    size_t num_correlation_measurements;
    size_t n_corr_xy;
    size_t n_corr_z;
} or_sim_result;

/* Correlation outputs are caller-sized: corr_x/corr_y/corr_xy [lx/2],
 * corr_xy_by_z [lz * (lx/2)], corr_z [lz/2]; theta/jxy/jz are the lattice
 * arrays (jxy, jz are overwritten by the disorder initialisation). */
int or_run_theta_simulation(size_t lx, size_t ly, size_t lz, double* theta, double* jxy,
                            double* jz, double j_xy, double j_z_mean, double delta_j_z,
                            double temperature, const or_sim_options* options, or_rng* rng,
                            or_sim_result* result, double* corr_x, double* corr_y,
                            double* corr_xy, double* corr_xy_by_z, double* corr_z);
double or_blocking_stderr(const double* x, size_t n);

/* ---- binning and derived observables (carlo-mc restated; src/model.rs:857-888) ---- */
int or_binned_estimate(const double* samples, size_t n, size_t binsize, double* mean,
                       double* stderr_out, double* bins, size_t* n_bins);
/* Jackknife over bins of the series columns above; out[k] = {mean, err} for
 * Magnetization, Chi, SpecificHeat, RhoXY, RhoZ. */
int or_evaluate_derived(const double* bin_means, size_t n_bins, double volume, double beta,
                        double out[5][2]);

/* ---- counter-based (Philox) forms for device parity ---- */
/* The raw Philox4x32-10 block of the shared device header. */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void or_keyed_init_angles(size_t n, uint64_t seed, float* theta);
/* One colour half-sweep from an FP32 state, randoms from the shared Philox
 * streams, Delta E in FP64.  decision[i]: -1 other colour, 0 reject,
 * 1 accept; tie[i] = 1 when |u_accept - min(1, exp(-beta dE))| < eps_tie.
 * accept_prob may be NULL.  Returns the number of accepted sites. */
size_t or_keyed_metro_half(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                           const float* jz, float beta, float width, uint64_t seed,
                           uint64_t sweep, int color, double eps_tie, float* theta_out,
                           int8_t* decision, uint8_t* tie, double* accept_prob);
void or_keyed_wolff_pick(size_t lx, size_t ly, size_t lz, uint64_t seed, uint64_t sweep,
                         uint32_t step, float* phi, uint32_t site[3]);
/* Bond activation (bits 0..2 = +x,+y,+z) with FP64 probabilities, ties in
 * bits 3..5, DFS labelling from the seed site and the FP32 reflection. */
size_t or_keyed_wolff(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                      const float* jz, float beta, uint64_t seed, uint64_t sweep, uint32_t step,
                      double eps_tie, uint8_t* bonds, uint8_t* cluster, float* theta_out);
/* Connected component of `seed_idx` over the active bonds (bits 0..2). */
size_t or_cluster_from_bonds(size_t lx, size_t ly, size_t lz, const uint8_t* bonds,
                             size_t seed_idx, uint8_t* cluster);
void or_measure_f32(size_t lx, size_t ly, size_t lz, const float* theta, const float* jxy,
                    const float* jz, or_obs* out);
void or_correlations_f32(size_t lx, size_t ly, size_t lz, const float* theta, size_t rmax_xy,
                         size_t rmax_z, double* corr_x, double* corr_y, double* corr_xy_by_z,
                         double* corr_z);

/* ---- CPU baseline: independent tasks, one task per thread at a time ---- */
/* Each task: ThetaModel::new with explicit J arrays, random init, then
 * `sweeps` x (sweep + measure).  jxy/jz are [n_tasks][lz].  Returns wall
 * seconds in *seconds and the summed energy of the final measurements. */
int or_bench_tasks(size_t n_tasks, size_t lx, size_t ly, size_t lz, const double* jxy,
                   const double* jz, const double* temperature, double proposal_width,
                   size_t wolff_steps, const uint64_t* seeds, size_t sweeps, int threads,
                   double* seconds, double* checksum);

/* Independent tasks in the reference's order (FastRng streams), each run
 * for `thermalization` + `sweeps` sweeps with a measurement after every
 * measured sweep; bin_means is [n_tasks][n_bins][OR_SERIES_COLS], n_bins
 * equal bins of the measured series (sweeps must be a multiple of n_bins). */
int or_series_tasks(size_t n_tasks, size_t lx, size_t ly, size_t lz, const double* jxy,
                    const double* jz, const double* temperature, double proposal_width,
                    size_t wolff_steps, const uint64_t* seeds, size_t thermalization, size_t sweeps,
                    size_t n_bins, int threads, double* bin_means);

#ifdef __cplusplus
}
#endif

#endif /* SLSF_ORACLE_H */
