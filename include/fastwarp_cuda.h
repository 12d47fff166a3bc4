/*
 * fastwarp_cuda.h -- C ABI of the B200 (sm_100a) registration engine.
 *
 * This is the drop-in boundary for the hot path of WyssCenter/fastwarp: every entry point
 * replaces one operation of the engine interface that the registration loops drive,
 *   - trait `Backend`      crates/fastwarp-reg/src/backend.rs:39-305 (SyN loop),
 *   - trait `LinearEngine` crates/fastwarp-reg/src/linear.rs:288-320 and
 *     trait `LinearMetric` crates/fastwarp-reg/src/optimizer.rs:60-65 (Rigid/Affine Mattes MI),
 * and the SyN stage driver `syn_fields` crates/fastwarp-reg/src/syn.rs:776-986.
 * The reference declaration each function replaces is cited beside it.
 *
 * Conventions
 *  - Grids are ITK LPS grids (crates/fastwarp-reg/src/grid.rs:33-40): size, spacing (mm),
 *    origin (mm) and the 3x3 direction matrix row-major with the axis directions as columns.
 *    Voxels are x-fastest.
 *  - Images live on the device as float32 (one value per voxel). Fields live on the device as
 *    float32 SoA planes x | y | z of LPS millimetre displacements. Host-side fields are AoS
 *    (x, y, z per voxel), float64 (`VectorField`, field_ops.rs:58-64) or float32
 *    (`DisplacementField`).
 *  - Every call returns 0 on success and a negative status on failure; fw_last_error() gives
 *    the message of the last failure on the calling thread (RegError::Invalid's text where the
 *    reference has one).
 *  - One CUDA stream per context. Every call is synchronous from the caller's view (its results
 *    are ready when it returns), as the reference's native futures are ready on first poll
 *    (crates/fastwarp-reg/src/exec.rs:14-30). Contexts are independent and may be used from
 *    different threads at the same time; one context must not be used by two threads at once.
 *  - Nothing falls back to the CPU: a call on a machine without a usable sm_100 GPU fails.
 */
#ifndef FASTWARP_CUDA_H
#define FASTWARP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FW_OK 0
#define FW_ERR_INVALID -1   /* RegError::Invalid: bad argument, mismatched grids, no overlap */
#define FW_ERR_CUDA -2      /* a CUDA runtime error */
#define FW_ERR_MEMORY -3    /* device allocation failed or the HBM budget is exhausted */
#define FW_ERR_NOT_FINITE -4 /* "the metric gradient is not finite" / "the displacement field is not finite" */
#define FW_ERR_TIMEOUT -5   /* a bounded device-side wait ran out */
#define FW_ERR_CANCELLED -6 /* RegError::Cancelled (syn.rs:826, 891) */

typedef struct fw_ctx fw_ctx;
typedef struct fw_image fw_image;
typedef struct fw_field fw_field;
typedef struct fw_mi_level fw_mi_level;

/* crates/fastwarp-reg/src/grid.rs:33-40 */
typedef struct fw_grid {
    int64_t size[3];
    double spacing[3];
    double origin[3];
    double direction[9];
} fw_grid;

/* AffineTransform as one map y = matrix * p + offset (transform/affine.rs:77-86). */
typedef struct fw_affine {
    double matrix[9];
    double offset[3];
} fw_affine;

/* InvertParams, field_ops.rs:276-296 (SyN: 20, 0.001, 0.1, true). */
typedef struct fw_invert_params {
    int32_t max_iterations;
    double mean_error_tolerance;
    double max_error_tolerance;
    int32_t enforce_boundary_condition;
} fw_invert_params;

/* InvertStats, field_ops.rs:300-307. */
typedef struct fw_invert_stats {
    int32_t iterations;
    double mean_error_norm;
    double max_error_norm;
} fw_invert_stats;

/* MiBinning, metric/mi.rs:117-137. */
typedef struct fw_mi_binning {
    int32_t bins;
    double fixed_min, fixed_max, moving_min, moving_max;
    double fixed_bin_size, moving_bin_size;
    double fixed_normalized_min, moving_normalized_min;
} fw_mi_binning;

/* LinearMovingTransform, transform/param.rs:392-420: outer(optimised(p)).
 * kind 0 = Euler3DTransform (parameters: angles x, y, z in radians, then translation; zyx
 * selects the Rz Ry Rx composition), kind 1 = AffineTransform (matrix row-major, then
 * translation). `center` is the optimised transform's centre. */
typedef struct fw_linear_transform {
    double outer_matrix[9];
    double outer_translation[3];
    double outer_center[3];
    int32_t kind;
    int32_t zyx;
    double parameters[12];
    double center[3];
} fw_linear_transform;

/* SynRecipe, recipe.rs:52-100 (masks are passed beside it as images). channel_metrics (SynMetric):
 * FW_METRIC_CC (neighbourhood CC of cc_radius) or FW_METRIC_MATTES (dense Mattes MI of mi_bins). */
#define FW_METRIC_CC 0
#define FW_METRIC_MATTES 1
#define FW_MAX_LEVELS 8
#define FW_MAX_CHANNELS 4
typedef struct fw_syn_recipe {
    double gradient_step;
    double update_field_variance;
    double total_field_variance;
    int32_t cc_radius;
    int32_t levels;
    uint32_t iterations[FW_MAX_LEVELS];
    uint32_t shrink_factors[FW_MAX_LEVELS];
    double smoothing_sigmas[FW_MAX_LEVELS];
    int32_t sigma_units_mm;
    double convergence_threshold;
    int32_t convergence_window;
    int32_t channels;
    double channel_weights[FW_MAX_CHANNELS];
    int32_t channel_metrics[FW_MAX_CHANNELS];
    int32_t mi_bins;
} fw_syn_recipe;

/* SynIteration, syn.rs:96-113. */
typedef struct fw_syn_iteration {
    int32_t level;
    double energy;
    double energy_weighted;
    double convergence_value;
    double fixed_update_scale;
    double moving_update_scale;
    fw_invert_stats inversions[4];
} fw_syn_iteration;

/* Counters of BackendStats (crates/fastwarp-gpu/src/wgpu_backend.rs:209-220) plus device
 * launches. */
typedef struct fw_stats {
    uint64_t kernel_launches;
    uint64_t graph_launches;
    uint64_t host_syncs;
    uint64_t bytes_uploaded;
    uint64_t bytes_downloaded;
    uint64_t peak_device_bytes;
    uint64_t live_device_bytes;
} fw_stats;

/* ---- errors, context ------------------------------------------------------------------- */

/* The message of the last failure on this thread (RegError's Display text). */
const char* fw_last_error(void);

/* Opens a context on `device` with its own stream. Fails on a GPU that is not sm_100.
 * Replaces the device open of the wgpu engine (crates/fastwarp-gpu/src/device.rs). */
int fw_ctx_create(int device, fw_ctx** out);
/* Destroys the context and its stream. Free every image, field and MI level made on it first:
 * their free functions use the context's stream. */
void fw_ctx_destroy(fw_ctx* ctx);
/* Backend::release_idle_buffers (backend.rs:48-50): a context keeps the device buffers it frees
 * for the next allocation of the same size (so repeated registrations of one shape allocate
 * nothing after the first); this returns them and the pool's unused memory to the device. */
int fw_ctx_release_idle_buffers(fw_ctx* ctx);
/* Bytes held by that cache. */
int fw_ctx_cached_bytes(const fw_ctx* ctx, uint64_t* out);
/* The context's cudaStream_t, for callers that interleave their own device work. */
void* fw_ctx_stream(fw_ctx* ctx);
int fw_ctx_synchronize(fw_ctx* ctx);
int fw_ctx_stats(const fw_ctx* ctx, fw_stats* out);
void fw_ctx_reset_stats(fw_ctx* ctx);
/* Free and total device memory (cudaMemGetInfo): the capacity budget that engine.rs:843-861
 * builds from its device caps. */
int fw_device_memory(int device, uint64_t* free_bytes, uint64_t* total_bytes);
/* Backend::name (backend.rs:46). */
const char* fw_backend_name(void);

/* ---- images and fields (backend.rs:52-87) ----------------------------------------------- */

/* Backend::upload_image (backend.rs:53): a float64 volume, stored as float32. */
int fw_image_upload(fw_ctx* ctx, const fw_grid* grid, const double* host, fw_image** out);
/* The same from float32 host data (no conversion). */
int fw_image_upload_f32(fw_ctx* ctx, const fw_grid* grid, const float* host, fw_image** out);
int fw_image_download(fw_ctx* ctx, const fw_image* img, float* host);
int fw_image_grid(const fw_image* img, fw_grid* out);
/* Device address of the float32 voxels (for zero-copy interop). */
void* fw_image_device_ptr(fw_image* img);
void fw_image_free(fw_image* img);

/* Backend::zero_field (backend.rs:61). */
int fw_field_zero(fw_ctx* ctx, const fw_grid* grid, fw_field** out);
/* Backend::upload_field (backend.rs:64): AoS float64 (VectorField). */
int fw_field_upload(fw_ctx* ctx, const fw_grid* grid, const double* aos, fw_field** out);
/* Backend::download_field (backend.rs:67): AoS float64 (VectorField). */
int fw_field_download(fw_ctx* ctx, const fw_field* field, double* aos);
/* The same as AoS float32 (DisplacementField, what run_syn returns). */
int fw_field_download_f32(fw_ctx* ctx, const fw_field* field, float* aos);
/* Backend::field_grid (backend.rs:70). */
int fw_field_grid(const fw_field* field, fw_grid* out);
/* Backend::copy_field (backend.rs:73). */
int fw_field_copy(fw_ctx* ctx, const fw_field* field, fw_field** out);
/* Device address of plane 0 and the plane stride in floats (planes x | y | z). */
void* fw_field_device_ptr(fw_field* field, int64_t* plane_stride);
void fw_field_free(fw_field* field);

/* ---- SyN operations (backend.rs:75-304) ------------------------------------------------- */

/* Backend::warp_through_field (backend.rs:82-88): out(x) = source(affine(q + pre(q))),
 * q = x + field(x), trilinear with ITK's buffer rule, zero outside. pre and affine may be NULL.
 * The result lives on the grid of `field`. */
int fw_warp_through_field(fw_ctx* ctx, const fw_image* source, const fw_field* field,
                          const fw_field* pre, const fw_affine* affine, fw_image** out);

/* Backend::warp_mask_through_field (backend.rs:98-105): nearest neighbour (half up), 1 where the
 * mask is not zero; with `product` the result is multiplied into it and returned in it
 * (*out == product). */
int fw_warp_mask_through_field(fw_ctx* ctx, const fw_image* mask, const fw_field* field,
                               const fw_field* pre, const fw_affine* affine, fw_image* product,
                               fw_image** out);

/* Backend::cc_value_derivative (backend.rs:110-115). */
int fw_cc_value_derivative(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                           int32_t radius, double* value, fw_field** derivative);

/* Backend::cc_value_derivative_pair (backend.rs:120-130): both directions from one set of
 * window sums; values[0] = (fixed, moving), values[1] = (moving, fixed). */
int fw_cc_value_derivative_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                int32_t radius, double values[2], fw_field** d_fixed,
                                fw_field** d_moving);

/* Backend::cc_value_derivative_pair_with_norms (backend.rs:164-177): plus both L2 norms. */
int fw_cc_value_derivative_pair_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                           const fw_image* moving, int32_t radius,
                                           double values[2], fw_field** d_fixed,
                                           fw_field** d_moving, double norms[2]);

/* Backend::cc_value_derivative_pair_masked (backend.rs:128-140; cpu/mod.rs:134-163 ->
 * metric/cc.rs:170-321 with Some(valid)): only voxels where `valid` (on the images' grid) is not
 * zero enter the window sums and their count; other voxels get a zero derivative; each value is
 * the mean over the valid voxels. No valid voxel: FW_ERR_INVALID with FW_NO_VOXEL_IN_MASKS in
 * the message (metric/cc.rs:49-50). */
#define FW_NO_VOXEL_IN_MASKS \
    "no voxel of the registration level lies inside both the fixed and the moving mask"
int fw_cc_value_derivative_pair_masked(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                       const fw_image* valid, int32_t radius, double values[2],
                                       fw_field** d_fixed, fw_field** d_moving);

/* Backend::cc_value_derivative_pair_masked_with_norms (backend.rs:142-152). */
int fw_cc_value_derivative_pair_masked_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                                  const fw_image* moving, const fw_image* valid,
                                                  int32_t radius, double values[2],
                                                  fw_field** d_fixed, fw_field** d_moving,
                                                  double norms[2]);

/* Backend::mi_value_derivative_pair (backend.rs:179-190; cpu/mod.rs:352-381 ->
 * MattesMi::evaluate_dense, metric/mi.rs:601-680): dense Mattes MI of two images on one grid in
 * both directions, (fixed, moving) then (moving, fixed). Each value is -MI; each derivative is
 * sum_k B3'(k - term) ratio[fixed bin, k] * grad(moving image of the direction) per voxel. The
 * intensity ranges of the bins are measured anew from the images on every call. bins 5..=32. */
int fw_mi_value_derivative_pair(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                int32_t bins, double values[2], fw_field** d_fixed,
                                fw_field** d_moving);

/* Backend::mi_value_derivative_pair_masked (backend.rs:192-205): masks on the images' grid
 * (NULL: not given); a voxel counts where both masks are not zero, each image's range is
 * measured inside its own mask; no voxel inside both: FW_NO_VOXEL_IN_MASKS. */
int fw_mi_value_derivative_pair_masked(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving,
                                       const fw_image* fixed_mask, const fw_image* moving_mask,
                                       int32_t bins, double values[2], fw_field** d_fixed,
                                       fw_field** d_moving);

/* ..._with_norms (backend.rs:207-240): plus the L2 norms of both derivatives. */
int fw_mi_value_derivative_pair_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                           const fw_image* moving, int32_t bins, double values[2],
                                           fw_field** d_fixed, fw_field** d_moving,
                                           double norms[2]);
int fw_mi_value_derivative_pair_masked_with_norms(fw_ctx* ctx, const fw_image* fixed,
                                                  const fw_image* moving,
                                                  const fw_image* fixed_mask,
                                                  const fw_image* moving_mask, int32_t bins,
                                                  double values[2], fw_field** d_fixed,
                                                  fw_field** d_moving, double norms[2]);

/* No counterpart in the reference (its CPU engine sums in float64, its GPU engine in plain
 * float32 after subtracting each image's intensity mode). The arithmetic of the CC window sums
 * (sum f, sum m, sum f^2, sum m^2, sum fm over each voxel's box) of the unmasked CC pair, for the
 * whole process: FW_CC_SUMS_F64 (the default: float64, in which products of float32 voxels are
 * exact) or FW_CC_SUMS_C32 (compensated float32: a float hi/lo pair per sum, TwoSum additions and
 * exact products by fma). The per-voxel CC and its derivative are float64 either way; the
 * masked pair, the batched kernels and the allocation-free entry point always use float64. */
#define FW_CC_SUMS_F64 0
#define FW_CC_SUMS_C32 1
int fw_set_cc_window_sums(int32_t kind);

/* No counterpart in the reference. The CC pair above for callers that cannot allocate device
 * memory: hosts whose own pool allocator owns the GPU's memory (a framework's caching allocator
 * that must see every byte, a server under a fixed HBM budget), plug-ins that run inside such a
 * host and get only the buffers it hands them, and real-time pipelines that plan all memory up
 * front and may not allocate once running. This call
 * allocates nothing and needs no context: `fixed` and `moving` are float32 device images on
 * `grid`, `d_fixed` / `d_moving` receive the two derivative fields as three float32 planes of
 * `plane_stride` (>= voxel count) floats, and `result` (device, 3 doubles) receives the value,
 * sum |d_fixed|^2 and sum |d_moving|^2. It runs asynchronously on `stream` (a cudaStream_t;
 * NULL = the default stream) of the current device and does not wait for it.
 * Its scratch is a static device array compiled into the library (block partials for at most
 * FW_NOALLOC_MAX_BLOCKS thread blocks, about 196 KB, held on every GPU that loads the library
 * until the process exits); a grid that needs more blocks is rejected with FW_ERR_INVALID. The
 * first call on a device looks the array's address up, so make it before any stream capture;
 * the address is kept for the life of the process, so do not use this call on a device after
 * cudaDeviceReset (or after the device's primary context was destroyed and the library's module
 * reloaded): the kept address would then name freed memory.
 * All calls share the array: calls whose kernels overlap on the GPU race and must be ordered
 * on one stream (or otherwise serialised) by the caller. */
#define FW_NOALLOC_MAX_BLOCKS 8192
int fw_cc_value_derivative_pair_noalloc(const fw_grid* grid, const float* fixed,
                                        const float* moving, int32_t radius, float* d_fixed,
                                        float* d_moving, int64_t plane_stride, double* result,
                                        void* stream);

/* Backend::smooth_field (backend.rs:249): in place; variance <= 0 leaves the field unchanged. */
int fw_smooth_field(fw_ctx* ctx, fw_field* field, double variance);

/* Backend::max_scaled_norm / max_scaled_norm_pair (backend.rs:252-262). */
int fw_max_scaled_norm(fw_ctx* ctx, const fw_field* field, double* out);
int fw_max_scaled_norm_pair(fw_ctx* ctx, const fw_field* a, const fw_field* b, double out[2]);

/* Backend::l2_norm (backend.rs:265). */
int fw_l2_norm(fw_ctx* ctx, const fw_field* field, double* out);

/* Backend::scale (backend.rs:268) and Backend::axpy (backend.rs:271). */
int fw_scale(fw_ctx* ctx, fw_field* field, double s);
int fw_axpy(fw_ctx* ctx, fw_field* acc, double a, const fw_field* x);

/* Backend::compose (backend.rs:275-279): out(x) = warping(x) + displacement(x + warping(x)). */
int fw_compose(fw_ctx* ctx, const fw_field* displacement, const fw_field* warping,
               fw_field** out);

/* Backend::invert (backend.rs:283-288): `initial` is updated in place and is the inverse. */
int fw_invert(fw_ctx* ctx, const fw_field* field, fw_field* initial,
              const fw_invert_params* params, fw_invert_stats* stats);

/* Backend::invert_pair (backend.rs:293-302): inverse = invert(field, init = inverse), then
 * field = invert(inverse, init = field), both in place; stats in call order. */
int fw_invert_pair(fw_ctx* ctx, fw_field* field, fw_field* inverse,
                   const fw_invert_params* params, fw_invert_stats stats[2]);

/* Backend::resample_field (backend.rs:305). */
int fw_resample_field(fw_ctx* ctx, const fw_field* field, const fw_grid* grid, fw_field** out);

/* ---- level pyramid (pyramid.rs:58-129, 418-460) ---------------------------------------- */

/* shrink_factors_per_dimension (pyramid.rs:58-93). */
int fw_shrink_factors(uint32_t factor, const double spacing[3], uint32_t out[3]);
/* level_virtual_grid / shrink_grid (pyramid.rs:99-158). */
int fw_shrink_grid(const fw_grid* grid, const uint32_t factors[3], fw_grid* out);
/* smooth_recursive_gaussian (pyramid.rs:418-427) on the device: a new image. */
int fw_smooth_recursive(fw_ctx* ctx, const fw_image* img, const double sigma_mm[3],
                        fw_image** out);

/* ---- image preparation (register.rs:82-249, preprocess.rs:45-215) ----------------------- */

/* resample_isotropic (register.rs:112-146): a new image on the isotropic `mm` grid (same origin
 * and direction, floor((n - 1) * spacing / mm + 1e-9) + 1 voxels per axis); output voxel i
 * samples source index min(i * mm / spacing, n - 1) trilinearly. A copy when every axis already
 * has `mm` spacing (within 1e-6 mm). */
int fw_resample_isotropic(fw_ctx* ctx, const fw_image* img, double mm, fw_image** out);
/* quantile_window (preprocess.rs:168-173): the (lower, upper) quantiles of a 256-bin histogram
 * of the finite voxels, each rounded to float32. Fails for an image without finite voxels. */
int fw_quantile_window(fw_ctx* ctx, const fw_image* img, float lower, float upper,
                       double window[2]);
/* preprocess_volume (preprocess.rs:180-223): a new image, the quantile window mapped linearly
 * onto [out_min, out_max], values outside it clamped, NaN passed through. `window` (nullable)
 * receives the window. Fails for no finite voxels and for a degenerate window (hi <= lo). */
int fw_preprocess(fw_ctx* ctx, const fw_image* img, float lower, float upper, double out_min,
                  double out_max, fw_image** out, double window[2]);
/* prepare_channels_with (register.rs:201-249): rejects images with non-finite voxels, resamples
 * every channel onto the isotropic grid (`iso_mm` NULL: copies as they are), and preprocesses
 * each onto [0, 1] with the quantile window `winsorize` = {lower, upper} (NULL: (0, 1), the plain
 * rescale). fixed_out / moving_out receive `channels` new images each; fixed_raw / moving_raw
 * (nullable) the resampled images before preprocessing. */
int fw_prepare_channels(fw_ctx* ctx, int32_t channels, const fw_image* const* fixed,
                        const fw_image* const* moving, const double* iso_mm,
                        const float* winsorize, fw_image** fixed_out, fw_image** moving_out,
                        fw_image** fixed_raw, fw_image** moving_raw);

/* ---- Mattes MI of the linear stages (linear.rs:288-320, optimizer.rs:60-65) ------------- */

/* LinearEngine::prepare_level (linear.rs:303-308): the moving level image and the prepared
 * samples (points in LPS mm, n x 3; fixed bins; binning) become device-resident. */
int fw_mi_level_prepare(fw_ctx* ctx, const fw_grid* moving_grid, const double* moving,
                        const double* points, const uint32_t* fixed_bin, int64_t n,
                        const fw_mi_binning* binning, fw_mi_level** out);
/* The same with the moving image already on the device (no upload): the level reads it in
 * place, so it must outlive the level. */
int fw_mi_level_prepare_image(fw_ctx* ctx, const fw_image* moving, const double* points,
                              const uint32_t* fixed_bin, int64_t n,
                              const fw_mi_binning* binning, fw_mi_level** out);
/* The level a linear stage prepares (linear.rs:474-492, 251-280, 940-945; sampling.rs:196-238)
 * from device images already at the level's smoothing: the regular sample set of `level_grid`
 * from `seed` (only the points inside `fixed_mask`, which may be NULL), the binning (fixed range at
 * the samples' nearest voxels, moving range over the whole moving image) and the kept points with
 * their trilinear fixed bins, all on the device (the host draws only the generator's integers);
 * `moving` must outlive the level. Fails with the reference's reason when Mattes MI is undefined
 * on the samples. */
int fw_mi_level_prepare_regular(fw_ctx* ctx, const fw_grid* level_grid, const fw_image* fixed,
                                const fw_image* moving, const fw_image* fixed_mask,
                                float percentage, uint32_t seed, int32_t bins,
                                fw_mi_level** out);
/* A level's samples, for inspection: the count in *n and, when cap >= *n, each sample's point
 * (3 per sample, physical mm: the cloud centre plus the record's float32 offset) and fixed bin;
 * `points`, `fixed_bins` and `binning` may be NULL. */
int fw_mi_level_samples(const fw_mi_level* level, double* points, uint32_t* fixed_bins,
                        int64_t cap, int64_t* n, fw_mi_binning* binning);
/* LinearMetric::value (optimizer.rs:61): -MI. */
int fw_mi_level_value(fw_mi_level* level, const fw_linear_transform* t, double* value);
/* LinearMetric::value_and_derivative (optimizer.rs:62-64): -MI and +dMI/dtheta (6 or 12). */
int fw_mi_level_value_and_derivative(fw_mi_level* level, const fw_linear_transform* t,
                                     double* value, double* derivative);
/* Several value() evaluations in one pass over the samples (a line search's bracket). */
int fw_mi_level_values(fw_mi_level* level, const fw_linear_transform* ts, int32_t count,
                       double* values);
/* Samples that contributed to the last evaluation. */
int fw_mi_level_num_valid(const fw_mi_level* level, int64_t* out);
/* Profiling (crates/fastwarp-gpu/src/profiler.rs:8-60, per-op device timestamps): after one
 * evaluation at `t`, times `reps` back-to-back launches of each pass of the level with CUDA events
 * on the context's stream and writes the mean milliseconds per launch and the algorithmic bytes
 * per launch of [0] the joint histogram (clear + k_mi_hist), [1] ComputeResults (k_mi_finish),
 * [2] the gradient moments (k_mi_deriv). A pass's bytes are the 16-byte sample records and the
 * moving image's gathers, min(4 Nm, 32 S) for S samples on Nm moving voxels. */
int fw_mi_level_time(fw_mi_level* level, const fw_linear_transform* t, int32_t reps,
                     double ms[3], double bytes[3]);
void fw_mi_level_free(fw_mi_level* level);

/* ---- SyN stage (syn.rs:776-986) --------------------------------------------------------- */

/* The virtual grid of one level of `recipe` on the fixed grid. */
int fw_syn_level_grid(const fw_syn_recipe* recipe, const fw_grid* fixed_grid, int32_t level,
                      fw_grid* out);

/* One SyN iteration (syn.rs:890-958) on device-resident state: f2m, f2m_inv, m2m, m2m_inv are
 * replaced in place; fixed/moving are the level-smoothed full-resolution images (one per
 * channel). Optional outputs: the two scaled update fields (host AoS float64, may be NULL). */
int fw_syn_step(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                const fw_image* const* moving, const fw_affine* initial, fw_field* f2m,
                fw_field* f2m_inv, fw_field* m2m, fw_field* m2m_inv, double* fixed_update,
                double* moving_update, fw_syn_iteration* record);

/* run_syn (syn.rs:555-564) from device-resident full-resolution images (one per channel):
 * the forward and inverse SyN fields on the grid of the last level (new fields) and the
 * per-iteration records (up to cap; *count = all iterations). */
int fw_syn_run_device(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                      const fw_image* const* moving, const fw_affine* initial,
                      fw_field** warp, fw_field** inverse_warp, fw_syn_iteration* records,
                      int64_t cap, int64_t* count);

/* The same two with the recipe's masks (recipe.rs fixed_mask / moving_mask, each on its own
 * grid, either may be NULL): every iteration resolves them on the level grid (syn.rs:555-580:
 * the fixed mask through F^-1, times the moving mask through affine(M^-1), nearest voxel) and
 * the CC pairs take only those voxels. A given mask without a non-zero voxel is refused
 * (recipe.rs:239-246); a level grid without a valid voxel fails with FW_NO_VOXEL_IN_MASKS. */
int fw_syn_step_masked(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                       const fw_image* const* moving, const fw_image* fixed_mask,
                       const fw_image* moving_mask, const fw_affine* initial, fw_field* f2m,
                       fw_field* f2m_inv, fw_field* m2m, fw_field* m2m_inv, double* fixed_update,
                       double* moving_update, fw_syn_iteration* record);
int fw_syn_run_device_masked(fw_ctx* ctx, const fw_syn_recipe* recipe,
                             const fw_image* const* fixed, const fw_image* const* moving,
                             const fw_image* fixed_mask, const fw_image* moving_mask,
                             const fw_affine* initial, fw_field** warp, fw_field** inverse_warp,
                             fw_syn_iteration* records, int64_t cap, int64_t* count);

/* run_syn_from (syn.rs:620-660, 803-820, 971-977): a later SyN stage. `prior` / `prior_inverse`
 * are the earlier SyN stages' collapsed fields (PriorWarp), on the grid of this stage's last
 * level; the moving images and mask are sampled at affine(prior(M^-1(x))) every iteration, and
 * the result is collapsed with the prior: warp = W + P(x + W), inverse = Pinv + Winv(x + Pinv).
 * Masks may be NULL; both prior fields NULL is a first stage (fw_syn_run_device_masked). */
int fw_syn_run_device_from(fw_ctx* ctx, const fw_syn_recipe* recipe,
                           const fw_image* const* fixed, const fw_image* const* moving,
                           const fw_image* fixed_mask, const fw_image* moving_mask,
                           const fw_affine* initial, const fw_field* prior,
                           const fw_field* prior_inverse, fw_field** warp,
                           fw_field** inverse_warp, fw_syn_iteration* records, int64_t cap,
                           int64_t* count);

/* run_syn from host float32 images: uploads, runs, and writes the two fields as AoS float32
 * (DisplacementField) on the grid of the last level (fw_syn_level_grid). */
int fw_syn_run(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_grid* fixed_grid,
               const float* const* fixed, const fw_grid* moving_grid, const float* const* moving,
               const fw_affine* initial, float* warp, float* inverse_warp,
               fw_syn_iteration* records, int64_t cap, int64_t* count);

/* ---- linear-stage optimiser (optimizer.rs:60-435) ---------------------------------------- */

/* CgSettings, optimizer.rs:67-106 (fw_cg_settings_ants: the antsRegistration settings). */
typedef struct fw_cg_settings {
    double max_step_mm;            /* MaximumStepSizeInPhysicalUnits, the first learning rate */
    double lower_limit, upper_limit;  /* the line search's bracket, times the learning rate */
    double epsilon;                /* relative width at which the line search stops */
    int32_t max_line_search_iterations;
    int32_t iterations;            /* iterations of the level */
    double convergence_threshold;
    int32_t convergence_window;
    double small_parameter_variation;  /* of the scale estimator */
} fw_cg_settings;

/* CgTrace, optimizer.rs:108-140. */
typedef struct fw_cg_trace {
    int32_t iterations;            /* steps taken */
    int32_t converged;             /* the monitor ended the level before its limit */
    double converged_value;        /* the value the monitor stopped on (NaN if none) */
    double best_value;
    double initial_learning_rate;
    double final_learning_rate;
    uint64_t line_search_evaluations;
    double scales[12];             /* parameter scales of the level */
    int64_t nvalues;               /* values written (all of them, even past `cap`) */
} fw_cg_trace;

/* The metric the optimiser drives (trait LinearMetric, optimizer.rs:56-65): return 0, or a
 * non-zero status with the message in fw_last_error(). `derivative` has 6 (Euler) or 12
 * (affine) entries in ITK's sign: the direction that decreases the value. */
typedef int (*fw_metric_value_fn)(void* user, const fw_linear_transform* t, double* value);
typedef int (*fw_metric_value_derivative_fn)(void* user, const fw_linear_transform* t,
                                             double* value, double* derivative);

void fw_cg_settings_ants(double max_step_mm, int32_t iterations, double threshold,
                         int32_t window, fw_cg_settings* out);
/* corner_points (optimizer.rs:142-166): the 8 corner points (x, y, z mm) of a grid. */
int fw_grid_corners(const fw_grid* grid, double corners[24]);
/* estimate_scales / estimate_step_scale (optimizer.rs:185-231). */
int fw_linear_estimate_scales(const double corners[24], const fw_linear_transform* t,
                              double small_variation, double* scales);
int fw_linear_estimate_step_scale(const double corners[24], const fw_linear_transform* t,
                                  const double* step, double small_variation, double* out);
/* optimise_level (optimizer.rs:311-435): ITK's conjugate-gradient optimiser with a golden-
 * section line search over `transform`'s parameters from its current values; on return it holds
 * the best transform. `values` (may be NULL) receives the value of every iteration that stepped,
 * up to `cap`. `cancel` (may be NULL) is polled before every iteration. */
int fw_cg_optimize_level(const fw_cg_settings* settings, const double corners[24],
                         fw_linear_transform* transform, fw_metric_value_fn value,
                         fw_metric_value_derivative_fn value_derivative, void* user,
                         fw_cg_trace* trace, double* values, int64_t cap,
                         const volatile int32_t* cancel);
/* The same on a device MI level (fw_mi_level_value / _value_and_derivative). */
int fw_mi_level_optimize(fw_mi_level* level, const fw_cg_settings* settings,
                         const double corners[24], fw_linear_transform* transform,
                         fw_cg_trace* trace, double* values, int64_t cap);

/* ---- one linear stage (linear.rs:512-597, 873-1068) -------------------------------------- */

/* LinearRecipe (linear.rs:75-128); its fixed mask is an argument of the _masked entry points.
 * The transform kind is the start transform's (Euler3D: rigid, affine: affine). */
typedef struct fw_linear_recipe {
    int32_t levels;
    uint32_t iterations[FW_MAX_LEVELS];
    uint32_t shrink_factors[FW_MAX_LEVELS];
    double smoothing_sigmas[FW_MAX_LEVELS];
    int32_t sigma_units_mm;          /* 0: sigmas in voxels (the cohort recipe), 1: in mm */
    double gradient_step;            /* Rigid[step] / Affine[step]: maximum step in mm */
    double convergence_threshold;
    int32_t convergence_window;
    int32_t bins;                    /* MI[...] histogram bins */
    float sampling_percentage;       /* MI[...] regular sampling percentage, (0, 1] */
    uint32_t seed;                   /* --random-seed: the first level's generator seed */
} fw_linear_recipe;

/* LinearLevelTrace (linear.rs:420-470). */
typedef struct fw_linear_level_trace {
    int32_t level;
    uint32_t shrink_factors[3];
    int64_t grid_size[3];
    int64_t samples;                 /* prepared samples (0 when skipped) */
    int32_t skipped;                 /* 1: Mattes MI undefined on the level's samples */
    fw_cg_trace cg;
    double parameters[12];           /* the optimised parameters after the level */
    double prepare_ms;               /* wall time: smoothing, sampling, sample preparation */
    double optimize_ms;              /* wall time: the optimiser's metric evaluations */
    int32_t samples_cached;          /* 1: the samples came from the chain's earlier stage */
} fw_linear_level_trace;

/* run_linear_stage (linear.rs:512-597): per level, the fixed grid shrunk by the level's factors,
 * both images smoothed at full resolution on the device, one regular sample set from the next
 * seed, the samples prepared (nearest-voxel fixed range, whole-image moving range, trilinear
 * fixed bins), and the conjugate-gradient optimiser over the device MI level. A level whose
 * samples leave MI undefined is skipped; every level skipped is an error. `transform` holds the
 * start (with the earlier transforms as its outer part) and receives the result; `traces`
 * (nullable) receives recipe->levels entries. */
int fw_linear_stage_run(fw_ctx* ctx, const fw_linear_recipe* recipe, const fw_image* fixed,
                        const fw_image* moving, fw_linear_transform* transform,
                        fw_linear_level_trace* traces);
/* The same with a fixed-image mask (LinearRecipe::mask, linear.rs:98-100, 130-134: `--masks
 * [fixed,NULL]`): `fixed_mask` is an image on its own grid whose non-zero voxels are inside
 * (MaskVolume::is_inside, mask.rs:76-78: the nearest voxel, rounding half up, inside the buffer
 * and not zero); only the jittered sample points inside it are kept (linear.rs:940-945,
 * sampling.rs:225-228), and a level left without a point is skipped with the reference's "no
 * sample point lands on the fixed image inside the fixed mask" reason (linear.rs:474-482). A mask
 * with no voxel inside is refused. NULL runs the unmasked stage. */
int fw_linear_stage_run_masked(fw_ctx* ctx, const fw_linear_recipe* recipe, const fw_image* fixed,
                               const fw_image* moving, const fw_image* fixed_mask,
                               fw_linear_transform* transform, fw_linear_level_trace* traces);

/* LinearChainResult (linear.rs:1078-1101): the centre-of-mass initial transform, both stages
 * (each optimised transform with its outer part, and its level traces) and the collapsed
 * initial(rigid(affine(x))) with the affine stage's centre (what 0GenericAffine.mat holds). An
 * affine transform here is y = matrix (x - center) + center + translation. */
typedef struct fw_linear_chain_result {
    double initial_matrix[9], initial_translation[3], initial_center[3];
    fw_linear_transform rigid;
    fw_linear_transform affine;
    fw_linear_level_trace rigid_levels[FW_MAX_LEVELS];
    fw_linear_level_trace affine_levels[FW_MAX_LEVELS];
    double total_matrix[9], total_translation[3], total_center[3];
    double initial_ms;               /* wall time of the centre-of-mass initialiser */
} fw_linear_chain_result;

/* run_linear_chain (linear.rs:1105-1212): the initial transform from the centres of mass of the
 * raw (resampled, un-preprocessed) images, then the rigid stage and the affine stage on the
 * preprocessed images (`rigid` and `affine` recipes, fw_linear_stage_run each). The centres of
 * mass are summed in float64 over the images' float32 device values (init.rs:50-74 sums the f64
 * volume): a caller holding float64 raw data that float32 cannot represent exactly gets the
 * centre of its float32 rounding. */
int fw_linear_chain_run(fw_ctx* ctx, const fw_linear_recipe* rigid, const fw_linear_recipe* affine,
                        const fw_image* fixed_raw, const fw_image* moving_raw,
                        const fw_image* fixed, const fw_image* moving,
                        fw_linear_chain_result* out);
/* The chain with a fixed-image mask restricting both stages' samples (as
 * fw_linear_stage_run_masked). */
int fw_linear_chain_run_masked(fw_ctx* ctx, const fw_linear_recipe* rigid,
                               const fw_linear_recipe* affine, const fw_image* fixed_raw,
                               const fw_image* moving_raw, const fw_image* fixed,
                               const fw_image* moving, const fw_image* fixed_mask,
                               fw_linear_chain_result* out);

/* ---- the batching form: many subjects to one template in one run ------------------------- */

/* One subject of a batch: its moving channels (device images on the subject's own grid, one grid
 * for all its channels) and its initial affine (the linear stages' result). */
typedef struct fw_batch_subject {
    const fw_image* moving[FW_MAX_CHANNELS];
    fw_affine initial;
    int32_t has_initial;
} fw_batch_subject;

/* The autotuner's choice for one level: z slices per tile of each tiled kernel family and the
 * persistent grid of each (blocks per SM), the time spent tuning, and whether it came from the
 * process-wide cache of earlier batches of the same shape. The inversion body's fields:
 * measure_zchunk = step tiles (4 slices each) per work item, as the single inversion plans them;
 * measure_blocks_per_sm = the step kernel's grid; body_blocks_per_sm = the fix kernel's grid. */
typedef struct fw_batch_tuning {
    int32_t level;
    int64_t grid_size[3];
    int32_t warp_zchunk, warp_blocks_per_sm;
    int32_t compose_zchunk, compose_blocks_per_sm;
    int32_t cc_zchunk, cc_blocks_per_sm;
    int32_t measure_zchunk, measure_blocks_per_sm;
    int32_t body_blocks_per_sm;
    int32_t smooth_blocks_per_sm;
    int32_t from_cache;
    double tune_ms;
    /* the tuned time of one launch over all subjects (ms; 0 when the shapes were not timed):
     * moving-side warp, CC pair, smoothing pair, compose, inversion step (after its bound),
     * inversion body (bound, step and fix) */
    double kernel_ms[6];
} fw_batch_tuning;

typedef struct fw_batch_report {
    int32_t subjects;
    int32_t levels;
    fw_batch_tuning tuning[FW_MAX_LEVELS];
    double level_ms[FW_MAX_LEVELS]; /* device time of each level's graph (CUDA events) */
    uint64_t device_bytes;          /* device memory the batch held at its largest level */
    double prepare_ms[FW_MAX_LEVELS]; /* wall time of each level's buffers and smoothed sources */
    double finish_ms;               /* wall time of the statuses, records and output fields */
} fw_batch_report;

/* No counterpart in the reference, whose nearest path registers several moving images to one
 * fixed image as independent runs (register_atlases, crates/fastwarp-cli/src/engine.rs:1016-1072).
 * The SyN stage (as fw_syn_run_device, syn.rs:776-986) of `subjects` subjects against ONE
 * template (`fixed`, recipe->channels device images), in lockstep: every sub-step of an
 * iteration is one persistent launch over a device-side work list of (subject, tile) items, each
 * level one CUDA graph, the list shrinking as subjects converge; tile shapes and persistent grids
 * come from an autotuner (`report->tuning`). Each subject's result equals its own
 * fw_syn_run_device result up to last-bit rounding of the tiled reductions. CC channels only, the
 * update field smoothed (variance > 0), no total-field smoothing, no masks; 1..=256 subjects.
 * Outputs per subject b: warps[b] / inverse_warps[b] (NULL when the subject failed),
 * records[b * cap ...] and counts[b] (nullable), statuses[b] (nullable: FW_OK or the subject's
 * FW_ERR_*). The call fails only for invalid arguments or a device error. */
int fw_batch_syn_run(fw_ctx* ctx, const fw_syn_recipe* recipe, const fw_image* const* fixed,
                     int32_t subjects, const fw_batch_subject* subject, fw_field** warps,
                     fw_field** inverse_warps, fw_syn_iteration* records, int64_t cap,
                     int64_t* counts, int32_t* statuses, fw_batch_report* report);

/* ---- profiling (crates/fastwarp-gpu/src/profiler.rs:8-60: per-op device timestamps) ----- */

/* Times `reps` launches of each kernel of one SyN iteration on the grid of `fixed` with CUDA
 * events on the context's stream: mean ms per launch and algorithmic bytes per launch of
 * [0] warp, [1] CC pair, [2] Gaussian smoothing + max norm, [3] compose + scale,
 * [4] one inversion body (its bound, step and fix kernels: measurement and update of every
 * voxel), [5] the body's bound kernel alone (the error on one voxel in 64), [6] its fix kernel
 * alone (the update of the tiles the step left for the clamp; bytes counts their voxels). */
int fw_time_kernels(fw_ctx* ctx, const fw_image* fixed, const fw_image* moving, int32_t radius,
                    double variance, int32_t reps, double ms[7], double bytes[7]);

/* Sets a flag polled before every level and iteration (SynOptions::cancel, syn.rs:80-85);
 * a run that sees it set fails with FW_ERR_CANCELLED. The flag is caller memory the device
 * cannot read, so inside a SyN level graph it is seen only at the next level; pass NULL to
 * clear. */
int fw_ctx_set_cancel_flag(fw_ctx* ctx, const volatile int32_t* flag);

/* Sets (on != 0) or clears the context's own cancel flag, which lives in mapped pinned host
 * memory: the host polls it before every level and linear-optimiser iteration, and the SyN level
 * graph's record kernel reads it once per iteration, so a run stops after the iteration in
 * flight and fails with FW_ERR_CANCELLED (SynOptions::cancel, syn.rs:80-85). It stays set until
 * cleared: a later run on the context fails at once. Safe to call from any thread. */
int fw_ctx_request_cancel(fw_ctx* ctx, int32_t on);

#ifdef __cplusplus
}
#endif
#endif
