// fw_linear.cu -- one linear (rigid or affine) registration stage: run_linear_stage
// (crates/fastwarp-reg/src/linear.rs:512-597, 873-1068) over the device Mattes MI level, and the
// rigid + affine chain (linear.rs:1105-1212).
//
// Per level: the fixed grid shrunk by the level's factors is the virtual domain, both images are
// smoothed at full resolution on the device (Deriche, pyramid.rs:418-460), one regular sample set
// is drawn with the stage's next seed and prepared on the device (fw_samples.cu: the fixed mask,
// the fixed range from the nearest voxels, the moving range from the whole image, the fixed bins
// from trilinear values), a level whose samples leave Mattes MI undefined is skipped
// (linear.rs:474-492), and the conjugate-gradient optimiser runs on the device level
// (fw_mi_level_optimize). In a chain the rigid and the affine stage share a level's smoothed
// moving image and prepared samples when their recipes give the same level grid, smoothing,
// seed, sampling percentage and bins (the reference's SmoothCache, linear.rs:573-667).
#include "fw_internal.cuh"

#include <algorithm>
#include <chrono>
#include <deque>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace fw {
namespace {

// The optimised part of a stage's transform alone (ParametricTransform::to_affine) as a matrix
// and an offset.
void stage_map(const fw_linear_transform* t, double M[9], double off[3]) {
    fw_linear_transform inner = *t;
    const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(inner.outer_matrix, eye, sizeof(eye));
    for (int a = 0; a < 3; ++a) inner.outer_translation[a] = inner.outer_center[a] = 0.0;
    linear_transform_map(&inner, M, off);
}

}  // namespace
}  // namespace fw

namespace fw {
namespace {

// What a level's prepared samples depend on (SampleKey, linear.rs:582-594): the level grid, the
// smoothing, the seed, the sampling percentage and the bins (the images and the fixed mask are
// the chain's own).
struct LevelKey {
    fw_grid grid;
    double sigma;
    int32_t sigma_mm;
    uint32_t seed;
    float percentage;
    int32_t bins;
    bool operator==(const LevelKey& o) const {
        return std::memcmp(&grid, &o.grid, sizeof(grid)) == 0 && sigma == o.sigma &&
               sigma_mm == o.sigma_mm && seed == o.seed && percentage == o.percentage &&
               bins == o.bins;
    }
};

// The chain's cache of prepared levels: the level's smoothed moving image (null when the level
// is not smoothed) and its samples, kept from the rigid stage for the affine stage.
struct SampleCache {
    struct Entry {
        LevelKey key;
        fw_image* moving_s = nullptr;
        LevelSamples samples;
    };
    fw_ctx* ctx;
    std::deque<Entry> entries;
    explicit SampleCache(fw_ctx* c) : ctx(c) {}
    ~SampleCache() {
        for (auto& e : entries) {
            free_level_samples(ctx, e.samples);
            if (e.moving_s) fw_image_free(e.moving_s);
        }
    }
    Entry* find(const LevelKey& k) {
        for (auto& e : entries)
            if (e.key == k) return &e;
        return nullptr;
    }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int linear_stage_run(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                     const fw_image* moving, const fw_image* mask, SampleCache* cache,
                     fw_linear_transform* transform, fw_linear_level_trace* traces) {
    FW_CHECK(r->levels >= 1 && r->levels <= FW_MAX_LEVELS, "linear recipe: 1 to 8 levels");
    FW_CHECK(r->bins > 4, "at least five histogram bins are required");
    FW_CHECK(r->sampling_percentage > 0.0f && r->sampling_percentage <= 1.0f,
             "linear recipe: the sampling percentage must lie in (0, 1]");
    FW_CHECK(transform->kind == 0 || transform->kind == 1, "unknown linear transform kind");
    const HostGrid& fg = fixed->grid;
    const fw_grid fgc = to_c(fg);
    auto level_grid = [&](int level, uint32_t f[3], fw_grid& lgc, HostGrid& lg) {
        FW_TRY(fw_shrink_factors(r->shrink_factors[level], fg.sp, f));
        FW_TRY(fw_shrink_grid(&fgc, f, &lgc));
        return make_grid(&lgc, lg);
    };
    // the generator integers of every level to prepare, drawn ahead on host threads
    DrawPlan plan;
    for (int level = 0; level < r->levels; ++level) {
        uint32_t f[3];
        fw_grid lgc;
        HostGrid lg;
        FW_TRY(level_grid(level, f, lgc, lg));
        const LevelKey key{lgc, r->smoothing_sigmas[level], r->sigma_units_mm,
                           r->seed + (uint32_t)level, r->sampling_percentage, r->bins};
        if (!(cache && cache->find(key))) plan_draws(ctx, plan, lg, r->sampling_percentage, key.seed);
    }
    uint32_t seed = r->seed;  // SeedSequence: one generator per level, never reset
    int skipped = 0;
    std::string why;
    for (int level = 0; level < r->levels; ++level) {
        if (cancel_requested(ctx)) return fail(FW_ERR_CANCELLED, "registration cancelled");
        const auto t0 = std::chrono::steady_clock::now();
        uint32_t f[3];
        fw_grid lgc;
        HostGrid lg;
        FW_TRY(level_grid(level, f, lgc, lg));
        fw_linear_level_trace tr{};
        tr.level = level;
        for (int a = 0; a < 3; ++a) {
            tr.shrink_factors[a] = f[a];
            tr.grid_size[a] = lg.n[a];
        }
        const double sigma = r->smoothing_sigmas[level];
        const LevelKey key{lgc, sigma, r->sigma_units_mm, seed++, r->sampling_percentage, r->bins};
        SampleCache::Entry* hit = cache ? cache->find(key) : nullptr;
        LevelSamples local;
        fw_image* ms_local = nullptr;
        const LevelSamples* S = nullptr;
        const fw_image* ml = moving;
        int rc = 0;
        if (hit) {
            S = &hit->samples;
            if (hit->moving_s) ml = hit->moving_s;
            tr.samples_cached = 1;
        } else {
            // the level's smoothed images (full resolution)
            fw_image* fs = nullptr;
            if (sigma > 0.0) {
                double sf[3], sm[3];
                for (int a = 0; a < 3; ++a) {
                    sf[a] = r->sigma_units_mm ? sigma : sigma * fg.sp[a];
                    sm[a] = r->sigma_units_mm ? sigma : sigma * moving->grid.sp[a];
                }
                rc = fw_smooth_recursive(ctx, fixed, sf, &fs);
                if (!rc) rc = fw_smooth_recursive(ctx, moving, sm, &ms_local);
            }
            if (!rc)
                rc = prepare_level_samples(ctx, lg, fs ? fs : fixed, ms_local ? ms_local : moving,
                                           mask, r->sampling_percentage, key.seed, r->bins, local,
                                           &plan);
            if (fs) fw_image_free(fs);
            if (rc) {
                if (ms_local) fw_image_free(ms_local);
                return rc;
            }
            if (cache) {
                cache->entries.push_back(SampleCache::Entry{key, ms_local, std::move(local)});
                ms_local = nullptr;
                local = LevelSamples{};
                S = &cache->entries.back().samples;
                if (cache->entries.back().moving_s) ml = cache->entries.back().moving_s;
            } else {
                S = &local;
                if (ms_local) ml = ms_local;
            }
        }
        tr.prepare_ms = ms_since(t0);
        const auto t1 = std::chrono::steady_clock::now();
        if (S->skip) {
            why += std::string(why.empty() ? "" : "; ") + "level " + std::to_string(level + 1) +
                   ": " + S->why;
        } else {
            fw_mi_level* lvl = nullptr;
            rc = mi_level_create(ctx, const_cast<fw_image*>(ml), false, S->d_rec, false, S->n,
                                 S->center, &S->binning, &lvl);
            if (!rc) {
                double corners[24];
                fw_cg_settings st;
                fw_cg_settings_ants(r->gradient_step, (int32_t)r->iterations[level],
                                    r->convergence_threshold, r->convergence_window, &st);
                rc = fw_grid_corners(&lgc, corners);
                if (!rc) rc = fw_mi_level_optimize(lvl, &st, corners, transform, &tr.cg, nullptr, 0);
                fw_mi_level_free(lvl);
            }
            tr.samples = S->n;
        }
        tr.optimize_ms = ms_since(t1);
        const bool skip = S->skip;
        free_level_samples(ctx, local);
        if (ms_local) fw_image_free(ms_local);
        if (rc) return rc;
        if (skip) {
            ++skipped;
            tr.skipped = 1;
            tr.cg.best_value = NAN;
            tr.cg.converged_value = NAN;
        }
        std::memcpy(tr.parameters, transform->parameters, sizeof(tr.parameters));
        if (traces) traces[level] = tr;
    }
    if (skipped == r->levels)
        return fail(FW_ERR_INVALID,
                    std::string("linear stage: every level of the ") +
                        (transform->kind == 0 ? "rigid" : "affine") +
                        " stage has too few usable samples for Mattes mutual information (" + why +
                        "); use smaller shrink factors, a larger sampling percentage, a larger "
                        "fixed mask, or a finer registration grid (iso_mm)");
    return 0;
}

int check_mask(fw_ctx* ctx, const fw_image* mask) {
    bool any = false;
    FW_TRY(mask_has_inside(ctx, mask, &any));
    if (!any)
        return fail(FW_ERR_INVALID, "linear recipe: the fixed mask has no voxel inside (every voxel is zero)");
    return 0;
}

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

int fw_linear_stage_run(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                        const fw_image* moving, fw_linear_transform* transform,
                        fw_linear_level_trace* traces) {
    FW_CHECK(ctx && r && fixed && moving && transform, "null argument");
    return linear_stage_run(ctx, r, fixed, moving, nullptr, nullptr, transform, traces);
}

int fw_mi_level_prepare_regular(fw_ctx* ctx, const fw_grid* level_grid, const fw_image* fixed,
                                const fw_image* moving, const fw_image* fixed_mask,
                                float percentage, uint32_t seed, int32_t bins,
                                fw_mi_level** out) {
    FW_CHECK(ctx && level_grid && fixed && moving && out, "null argument");
    FW_CHECK(bins > 4 && bins <= 32, "mattes: bins must be in 5..=32");
    FW_CHECK(percentage > 0.0f && percentage <= 1.0f,
             "linear recipe: the sampling percentage must lie in (0, 1]");
    HostGrid lg;
    FW_TRY(make_grid(level_grid, lg));
    if (fixed_mask) FW_TRY(check_mask(ctx, fixed_mask));
    LevelSamples S;
    FW_TRY(prepare_level_samples(ctx, lg, fixed, moving, fixed_mask, percentage, seed, bins, S));
    if (S.skip) return fail(FW_ERR_INVALID, "mattes: " + S.why);
    // the level takes the records
    return mi_level_create(ctx, const_cast<fw_image*>(moving), false, S.d_rec, true, S.n, S.center,
                           &S.binning, out);
}

int fw_linear_stage_run_masked(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                               const fw_image* moving, const fw_image* fixed_mask,
                               fw_linear_transform* transform, fw_linear_level_trace* traces) {
    FW_CHECK(ctx && r && fixed && moving && transform, "null argument");
    if (fixed_mask) FW_TRY(check_mask(ctx, fixed_mask));
    return linear_stage_run(ctx, r, fixed, moving, fixed_mask, nullptr, transform, traces);
}

// run_linear_chain_cached_async (linear.rs:1148-1212): the centre-of-mass initial transform
// of the raw images (init.rs:76-86), the rigid stage from it, the affine stage from the rigid
// result, and their collapse recentred on the affine stage's centre (with_center, :1071-1076).
// The fixed mask (nullable) restricts both stages' samples (LinearRecipe::mask of each stage).
// The affine stage takes a level's smoothed moving image and samples from the rigid stage when
// its recipe gives the same level (plan_samples, linear.rs:631-667).
static int linear_chain_run(fw_ctx* ctx, const fw_linear_recipe* rigid,
                            const fw_linear_recipe* affine, const fw_image* fixed_raw,
                            const fw_image* moving_raw, const fw_image* fixed,
                            const fw_image* moving, const fw_image* fixed_mask,
                            fw_linear_chain_result* out) {
    FW_CHECK(ctx && rigid && affine && fixed_raw && moving_raw && fixed && moving && out,
             "null argument");
    std::memset(out, 0, sizeof(*out));
    if (fixed_mask) FW_TRY(check_mask(ctx, fixed_mask));
    const auto t0 = std::chrono::steady_clock::now();
    double fc[3], mc[3];
    FW_TRY(centre_of_mass(ctx, fixed_raw, fc));
    FW_TRY(centre_of_mass(ctx, moving_raw, mc));
    out->initial_ms = ms_since(t0);
    SampleCache cache(ctx);
    const double eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(out->initial_matrix, eye, sizeof(eye));
    for (int a = 0; a < 3; ++a) {
        out->initial_translation[a] = mc[a] - fc[a];
        out->initial_center[a] = fc[a];
    }
    // the rigid stage: Euler3D at zero about the initial centre, the initial transform outside
    fw_linear_transform& tr = out->rigid;
    std::memcpy(tr.outer_matrix, eye, sizeof(eye));
    for (int a = 0; a < 3; ++a) {
        tr.outer_translation[a] = out->initial_translation[a];
        tr.outer_center[a] = fc[a];
        tr.center[a] = fc[a];
    }
    tr.kind = 0;
    FW_TRY(linear_stage_run(ctx, rigid, fixed, moving, fixed_mask, &cache, &tr, out->rigid_levels));
    // after_rigid = initial o rigid as a matrix and an offset (the initial transform's matrix is
    // the identity, so its offset is its translation)
    double Mr[9], offr[3];
    stage_map(&tr, Mr, offr);
    double off_after[3];
    for (int a = 0; a < 3; ++a) off_after[a] = offr[a] + out->initial_translation[a];
    // the affine stage: identity about the rigid centre, after_rigid outside (centre zero)
    fw_linear_transform& ta = out->affine;
    std::memcpy(ta.outer_matrix, Mr, sizeof(Mr));
    for (int a = 0; a < 3; ++a) {
        ta.outer_translation[a] = off_after[a];
        ta.outer_center[a] = 0.0;
        ta.center[a] = tr.center[a];
    }
    ta.kind = 1;
    for (int k = 0; k < 12; ++k) ta.parameters[k] = k < 9 ? eye[k] : 0.0;
    FW_TRY(linear_stage_run(ctx, affine, fixed, moving, fixed_mask, &cache, &ta,
                            out->affine_levels));
    // collapsed = after_rigid o affine, recentred on the affine centre
    double Ma[9], offa[3], M[9], off[3], mo[3];
    stage_map(&ta, Ma, offa);
    mat3_mul(Mr, Ma, M);
    mat3_vec(Mr, offa, mo);
    for (int a = 0; a < 3; ++a) off[a] = mo[a] + off_after[a];
    double mcen[3];
    mat3_vec(M, ta.center, mcen);
    std::memcpy(out->total_matrix, M, sizeof(M));
    for (int a = 0; a < 3; ++a) {
        out->total_center[a] = ta.center[a];
        out->total_translation[a] = off[a] - ta.center[a] + mcen[a];
    }
    return 0;
}

int fw_linear_chain_run(fw_ctx* ctx, const fw_linear_recipe* rigid, const fw_linear_recipe* affine,
                        const fw_image* fixed_raw, const fw_image* moving_raw,
                        const fw_image* fixed, const fw_image* moving,
                        fw_linear_chain_result* out) {
    return linear_chain_run(ctx, rigid, affine, fixed_raw, moving_raw, fixed, moving, nullptr, out);
}

int fw_linear_chain_run_masked(fw_ctx* ctx, const fw_linear_recipe* rigid,
                               const fw_linear_recipe* affine, const fw_image* fixed_raw,
                               const fw_image* moving_raw, const fw_image* fixed,
                               const fw_image* moving, const fw_image* fixed_mask,
                               fw_linear_chain_result* out) {
    return linear_chain_run(ctx, rigid, affine, fixed_raw, moving_raw, fixed, moving, fixed_mask,
                            out);
}

}  // extern "C"
