/*
 * fw_oracle.h -- C ABI of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. This is an f64, OpenMP restatement of the CPU engine of
 * WyssCenter/fastwarp (crate fastwarp-reg, `engine="cpu"`), used by tests/ as the parity
 * checker and by bench.py as the timed CPU baseline. The product library
 * (fastwarp_b200/csrc) never links, loads or calls it.
 *
 * Parity pinning: the reference is Rust and cannot be built here (no cargo/rustc), so the
 * restatement is pinned against the known-answer tests the reference's own unit tests hold
 * (MT19937 published outputs, Gaussian operator taps, CC identities and brute-force window
 * statistics, B-spline partition of unity, inversion/compose identities, convergence-monitor
 * closed form). See tests/test_oracle.py.
 *
 * Conventions (as the reference): grids are ITK LPS grids, x-fastest; images are f64 arrays of
 * size[0]*size[1]*size[2]; displacement fields are AoS f64 triples in millimetres.
 */
#ifndef FW_ORACLE_H
#define FW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* crates/fastwarp-reg/src/grid.rs:33-40 (size, spacing, origin, direction[row][axis]). */
typedef struct fwo_grid {
    int64_t size[3];
    double spacing[3];
    double origin[3];
    double direction[9]; /* row-major, columns are the axis directions */
} fwo_grid;

/* y = matrix * p + offset (crates/fastwarp-reg/src/transform/affine.rs:77-86). */
typedef struct fwo_affine {
    double matrix[9];
    double offset[3];
} fwo_affine;

/* crates/fastwarp-reg/src/field_ops.rs:276-296 */
typedef struct fwo_invert_params {
    int32_t max_iterations;
    double mean_error_tolerance;
    double max_error_tolerance;
    int32_t enforce_boundary_condition;
} fwo_invert_params;

/* crates/fastwarp-reg/src/field_ops.rs:300-307 */
typedef struct fwo_invert_stats {
    int32_t iterations;
    double mean_error_norm;
    double max_error_norm;
} fwo_invert_stats;

/* Mattes binning, crates/fastwarp-reg/src/metric/mi.rs:117-137 */
typedef struct fwo_mi_binning {
    int32_t bins;
    double fixed_min, fixed_max, moving_min, moving_max;
    double fixed_bin_size, moving_bin_size;
    double fixed_normalized_min, moving_normalized_min;
} fwo_mi_binning;

/* LinearMovingTransform, crates/fastwarp-reg/src/transform/param.rs: outer(optimised(p)).
 * kind 0 = Euler3D (6 params: angles x,y,z then translation; zyx selects Rz Ry Rx),
 * kind 1 = Affine (12 params: matrix row-major then translation). */
typedef struct fwo_linear_transform {
    double outer_matrix[9];
    double outer_translation[3];
    double outer_center[3];
    int32_t kind;
    int32_t zyx;
    double parameters[12];
    double center[3];
} fwo_linear_transform;

/* SyN recipe, crates/fastwarp-reg/src/recipe.rs:52-100 (masks are passed beside it as
 * fwo_syn_masks). channel_metrics: 0 = CC[radius], 1 = dense Mattes MI[mi_bins] (SynMetric). */
#define FWO_MAX_LEVELS 8
#define FWO_MAX_CHANNELS 4
typedef struct fwo_syn_recipe {
    double gradient_step;
    double update_field_variance;
    double total_field_variance;
    int32_t cc_radius;
    int32_t levels;
    uint32_t iterations[FWO_MAX_LEVELS];
    uint32_t shrink_factors[FWO_MAX_LEVELS];
    double smoothing_sigmas[FWO_MAX_LEVELS];
    int32_t sigma_units_mm; /* 0 = voxels, 1 = millimetres */
    double convergence_threshold;
    int32_t convergence_window;
    int32_t channels;
    double channel_weights[FWO_MAX_CHANNELS];
    int32_t channel_metrics[FWO_MAX_CHANNELS];
    int32_t mi_bins;
} fwo_syn_recipe;

/* One SyN iteration record, crates/fastwarp-reg/src/syn.rs:96-113. */
typedef struct fwo_syn_iteration {
    int32_t level;
    double energy;
    double energy_weighted;
    double convergence_value;
    double fixed_update_scale;
    double moving_update_scale;
    fwo_invert_stats inversions[4];
} fwo_syn_iteration;

const char* fwo_last_error(void);
int fwo_num_threads(void);
void fwo_set_num_threads(int n);

/* grid helpers */
int fwo_shrink_factors(uint32_t factor, const double spacing[3], uint32_t out[3]);
int fwo_shrink_grid(const fwo_grid* grid, const uint32_t factors[3], fwo_grid* out);
int fwo_point_to_index(const fwo_grid* grid, const double p[3], double out[3]);
int fwo_index_to_point(const fwo_grid* grid, const double c[3], double out[3]);

/* Backend ops, crates/fastwarp-reg/src/cpu/mod.rs */
int fwo_warp(const fwo_grid* src_grid, const double* src, const fwo_grid* grid, const double* field,
             const fwo_grid* pre_grid, const double* pre, const fwo_affine* affine, double* out);
int fwo_warp_mask(const fwo_grid* mask_grid, const double* mask, const fwo_grid* grid,
                  const double* field, const fwo_grid* pre_grid, const double* pre,
                  const fwo_affine* affine, const double* product, double* out);
int fwo_cc(const fwo_grid* grid, const double* fixed, const double* moving, const double* valid,
           int32_t radius, double* value, double* derivative, double* local_cc,
           double* coefficient, int64_t* num_valid);
int fwo_cc_pair(const fwo_grid* grid, const double* fixed, const double* moving,
                const double* valid, int32_t radius, double values[2], double* d_fwd,
                double* d_bwd);
int64_t fwo_gaussian_taps(double variance, double max_error, int64_t max_width, double* out,
                          int64_t cap);
int fwo_smooth_field(const fwo_grid* grid, const double* field, double variance, double* out);
double fwo_max_scaled_norm(const fwo_grid* grid, const double* field);
double fwo_l2_norm(const fwo_grid* grid, const double* field);
int fwo_scale(const fwo_grid* grid, double* field, double s);
int fwo_axpy(const fwo_grid* grid, double* acc, double a, const double* x);
int fwo_compose(const fwo_grid* grid, const double* displacement, const double* warping,
                double* out);
int fwo_invert(const fwo_grid* grid, const double* field, double* inverse,
               const fwo_invert_params* params, fwo_invert_stats* stats);
int fwo_resample_field(const fwo_grid* src_grid, const double* field, const fwo_grid* grid,
                       double* out);

/* pyramid, crates/fastwarp-reg/src/pyramid.rs */
int fwo_smooth_recursive(const fwo_grid* grid, const double* img, const double sigma_mm[3],
                         double* out);

/* sampling, crates/fastwarp-reg/src/sampling.rs */
int fwo_mt19937(uint32_t seed, int64_t n, uint32_t* out);
int64_t fwo_sample_points_regular(const fwo_grid* grid, float percentage, uint32_t seed,
                                  double* out, int64_t cap);

/* Mattes MI, crates/fastwarp-reg/src/metric/mi.rs */
double fwo_bspline3(double u);
double fwo_bspline3_derivative(double u);
int fwo_mi_binning_from_ranges(int32_t bins, double fmin, double fmax, double mmin, double mmax,
                               fwo_mi_binning* out);
int fwo_prepare_samples(const fwo_grid* fgrid, const double* fixed, const fwo_grid* mgrid,
                        const double* moving, const double* points, int64_t n, int32_t bins,
                        double* kept_points, uint32_t* fixed_bin, int64_t* kept,
                        fwo_mi_binning* binning);
int fwo_linear_map(const fwo_linear_transform* t, fwo_affine* out);
int fwo_linear_jacobian(const fwo_linear_transform* t, const double p[3], double* cols);
int fwo_mi_evaluate(const fwo_mi_binning* binning, const fwo_grid* mgrid, const double* moving,
                    const double* points, const uint32_t* fixed_bin, int64_t n,
                    const fwo_linear_transform* t, int32_t want_derivative, double* value,
                    double* derivative, int64_t* num_valid, double* joint_pdf);

/* dense Mattes MI (SyN-stage metric), metric/mi.rs:553-680: the moving point of virtual voxel l
 * is p + field[l] (AoS mm); masks may be NULL. Pinned against the reference's ITK fixtures. */
int fwo_mi_dense(const fwo_grid* fgrid, const double* fixed, const fwo_grid* mgrid,
                 const double* moving, const double* field, const fwo_grid* fmask_grid,
                 const double* fmask, const fwo_grid* mmask_grid, const double* mmask,
                 int32_t bins, double* value, int64_t* num_valid, double* derivative);

/* the linear-stage optimiser, crates/fastwarp-reg/src/optimizer.rs:60-435 */
typedef struct fwo_cg_settings {
    double max_step_mm, lower_limit, upper_limit, epsilon;
    int32_t max_line_search_iterations;
    int32_t iterations;
    double convergence_threshold;
    int32_t convergence_window;
    double small_parameter_variation;
} fwo_cg_settings;
typedef struct fwo_cg_trace {
    int32_t iterations;
    int32_t converged;
    double converged_value;
    double best_value;
    double initial_learning_rate;
    double final_learning_rate;
    uint64_t line_search_evaluations;
    double scales[12];
    int64_t nvalues;
} fwo_cg_trace;
typedef int (*fwo_metric_value_fn)(void* user, const fwo_linear_transform* t, double* value);
typedef int (*fwo_metric_value_derivative_fn)(void* user, const fwo_linear_transform* t,
                                              double* value, double* derivative);
int fwo_estimate_scales(const double* corners, const fwo_linear_transform* t, double small,
                        double* scales);
double fwo_estimate_step_scale(const double* corners, const fwo_linear_transform* t,
                               const double* step, double small);
int fwo_cg_optimize_level(const fwo_cg_settings* st, const double* corners,
                          fwo_linear_transform* t, fwo_metric_value_fn value,
                          fwo_metric_value_derivative_fn value_derivative, void* user,
                          fwo_cg_trace* trace, double* values, int64_t cap);

/* convergence, crates/fastwarp-reg/src/convergence.rs */
double fwo_convergence_value(const double* values, int64_t n, int32_t window,
                             double total_energy);

/* SyN, crates/fastwarp-reg/src/syn.rs:337-445, 776-986 */
int fwo_syn_level_grid(const fwo_syn_recipe* r, const fwo_grid* fixed_grid, int32_t level,
                       fwo_grid* out);
int fwo_syn_step(const fwo_syn_recipe* r, const fwo_grid* level_grid,
                 const fwo_grid* fixed_grid, const double* const* fixed_smooth,
                 const fwo_grid* moving_grid, const double* const* moving_smooth,
                 const fwo_affine* initial, double* f2m, double* f2m_inv, double* m2m,
                 double* m2m_inv, double* fixed_update, double* moving_update,
                 fwo_syn_iteration* record);
int fwo_syn_run(const fwo_syn_recipe* r, const fwo_grid* fixed_grid, const double* const* fixed,
                const fwo_grid* moving_grid, const double* const* moving,
                const fwo_affine* initial, double* warp, double* inverse_warp,
                fwo_syn_iteration* records, int64_t cap, int64_t* count);

/* The recipe's fixed and moving masks (recipe.rs fixed_mask / moving_mask), each on its own grid
 * (NULL data = not given); syn.rs:496-580 resolves them on the level grid every iteration. */
typedef struct fwo_syn_masks {
    const fwo_grid* fixed_grid;
    const double* fixed;
    const fwo_grid* moving_grid;
    const double* moving;
} fwo_syn_masks;
int fwo_syn_step_masked(const fwo_syn_recipe* r, const fwo_grid* level_grid,
                        const fwo_grid* fixed_grid, const double* const* fixed_smooth,
                        const fwo_grid* moving_grid, const double* const* moving_smooth,
                        const fwo_affine* initial, const fwo_syn_masks* masks, double* f2m,
                        double* f2m_inv, double* m2m, double* m2m_inv, double* fixed_update,
                        double* moving_update, fwo_syn_iteration* record);
int fwo_syn_run_masked(const fwo_syn_recipe* r, const fwo_grid* fixed_grid,
                       const double* const* fixed, const fwo_grid* moving_grid,
                       const double* const* moving, const fwo_affine* initial,
                       const fwo_syn_masks* masks, double* warp, double* inverse_warp,
                       fwo_syn_iteration* records, int64_t cap, int64_t* count);

/* run_syn_from, syn.rs:620-660, 761-774, 803-820, 971-977: a later SyN stage whose moving side
 * goes through the earlier stages' collapsed field (prior, AoS on prior_grid = the grid of this
 * stage's last level; NULL for a first stage), collapsed with it at the end. masks may be NULL. */
int fwo_syn_run_from(const fwo_syn_recipe* r, const fwo_grid* fixed_grid,
                     const double* const* fixed, const fwo_grid* moving_grid,
                     const double* const* moving, const fwo_affine* initial,
                     const fwo_syn_masks* masks, const fwo_grid* prior_grid, const double* prior,
                     const double* prior_inverse, double* warp, double* inverse_warp,
                     fwo_syn_iteration* records, int64_t cap, int64_t* count);

/* Image preparation (crates/fastwarp-reg/src/preprocess.rs, register.rs). */
/* quantile_window (preprocess.rs:168-173): the window of a 256-bin histogram of the finite
 * values, each bound rounded to float32. Fails for an image without finite values. */
int fwo_quantile_window(const double* values, int64_t n, float lower, float upper,
                        double out[2]);
/* preprocess_values (preprocess.rs:180-209): the window mapped onto [out_min, out_max], values
 * outside clamped, NaN passed through; fails for a degenerate window (hi <= lo). */
int fwo_preprocess(const double* values, int64_t n, float lower, float upper, double out_min,
                   double out_max, double* out);
/* resample_isotropic's grid rule (register.rs:112-129): same origin and direction, mm spacing,
 * floor((n - 1) * spacing / mm + 1e-9) + 1 voxels; the grid itself when every axis has mm. */
int fwo_isotropic_grid(const fwo_grid* grid, double mm, fwo_grid* out);
/* resample_isotropic (register.rs:112-146): trilinear at index min(i * mm / spacing, n - 1),
 * rounded to float32; `out` holds fwo_isotropic_grid's voxel count. */
int fwo_resample_isotropic(const fwo_grid* grid, const double* img, double mm, double* out);

#ifdef __cplusplus
}
#endif
#endif
