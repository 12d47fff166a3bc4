// fw_linear.cu -- one linear (rigid or affine) registration stage: run_linear_stage
// (crates/fastwarp-reg/src/linear.rs:512-597, 873-1068) over the device Mattes MI level.
//
// Per level: the fixed grid shrunk by the level's factors is the virtual domain, both images are
// smoothed at full resolution on the device (Deriche, pyramid.rs:418-460), one regular sample set
// is drawn with the stage's next seed (sampling.rs:181-238), a level whose samples leave Mattes
// MI undefined is skipped (linear.rs:474-492), the samples are prepared (fixed range from the
// nearest voxels, moving range from the whole image, fixed bins from trilinear values;
// linear.rs:251-280, metric/mi.rs:121-317) and the conjugate-gradient optimiser runs on the
// device level (fw_mi_level_optimize). With a fixed mask only the sample points inside it are
// kept (linear.rs:940-945). Sampling and sample preparation are host work, as in the
// reference (they run once per level over the level's samples); every metric evaluation is on
// the device.
#include "fw_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace fw {
namespace {

// MT19937 (Matsumoto & Nishimura 1998) with the reference's seeding (sampling.rs:40-120).
struct Mt19937 {
    uint32_t s[624];
    int next = 0, left = 0;
    static uint32_t twist(uint32_t m, uint32_t s0, uint32_t s1) {
        return m ^ (((s0 & 0x80000000u) | (s1 & 0x7fffffffu)) >> 1) ^ ((s1 & 1u) ? 0x9908b0dfu : 0u);
    }
    explicit Mt19937(uint32_t seed) {
        s[0] = seed;
        for (uint32_t i = 1; i < 624; ++i) s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + i;
        reload();
    }
    void reload() {
        for (int p = 0; p < 624; ++p) s[p] = twist(s[(p + 397) % 624], s[p], s[(p + 1) % 624]);
        left = 624;
        next = 0;
    }
    uint32_t integer() {
        if (left == 0) reload();
        --left;
        uint32_t y = s[next++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        return y ^ (y >> 18);
    }
};

// sampling.rs:163-171: ITK's Box-Muller variate (cosine branch) from two integer draws.
double normal_from(uint32_t open, uint32_t open_upper) {
    const double o = ((double)open + 0.5) * (1.0 / 4294967296.0);
    const double ou = (double)open_upper * (1.0 / 4294967296.0);
    const double r = std::sqrt(-2.0 * std::log(1.0 - o) * 1.0);
    return r * std::cos(2.0 * M_PI * ou);
}

void index_to_point(const HostGrid& g, const double c[3], double p[3]) {
    const double s[3] = {c[0] * g.sp[0], c[1] * g.sp[1], c[2] * g.sp[2]};
    for (int r = 0; r < 3; ++r)
        p[r] = g.org[r] + (g.dir[r * 3] * s[0] + g.dir[r * 3 + 1] * s[1] + g.dir[r * 3 + 2] * s[2]);
}

void point_to_index(const HostGrid& g, const double p[3], double c[3]) {
    const double d[3] = {p[0] - g.org[0], p[1] - g.org[1], p[2] - g.org[2]};
    for (int r = 0; r < 3; ++r) c[r] = g.inv[r * 3] * d[0] + g.inv[r * 3 + 1] * d[1] + g.inv[r * 3 + 2] * d[2];
}

// sampling.rs:196-238: voxel 0 and every ceil(1 / percentage)-th voxel in raster order, each
// jittered by N(0, 1) * spacing / 3 per axis (two draws per variate, x first).
std::vector<double> regular_samples(const HostGrid& g, float percentage, uint32_t seed) {
    Mt19937 mt(seed);
    const int64_t stride = (int64_t)std::max(std::ceil(1.0 / (double)percentage), 1.0);
    const int64_t picks = (g.count() + stride - 1) / stride;
    std::vector<double> out((size_t)(3 * picks));
    for (int64_t q = 0; q < picks; ++q) {
        uint32_t d[6];
        for (auto& v : d) v = mt.integer();
        const int64_t flat = q * stride;
        const double c[3] = {(double)(flat % g.n[0]), (double)((flat / g.n[0]) % g.n[1]),
                             (double)(flat / (g.n[0] * g.n[1]))};
        double* p = &out[(size_t)(3 * q)];
        index_to_point(g, c, p);
        for (int a = 0; a < 3; ++a) p[a] += normal_from(d[2 * a], d[2 * a + 1]) * (g.sp[a] / 3.0);
    }
    return out;
}

// interp.rs:43-85 on the host: ITK's linear interpolation at a continuous index inside the
// buffer ([-0.5, n - 0.5) per axis), neighbours clamped, float64.
bool linear_at_point(const HostGrid& g, const std::vector<double>& img, const double p[3],
                     double& out) {
    double c[3];
    point_to_index(g, p, c);
    for (int a = 0; a < 3; ++a)
        if (!(c[a] >= -0.5 && c[a] < (double)g.n[a] - 0.5)) return false;
    int64_t b[3];
    double w[3];
    for (int a = 0; a < 3; ++a) {
        const double fl = std::floor(c[a]);
        double d;
        if (fl < 0.0) {
            b[a] = 0;
            d = c[a];
        } else if (!(fl <= (double)(g.n[a] - 1))) {
            b[a] = g.n[a] - 1;
            d = c[a] - (double)(g.n[a] - 1);
        } else {
            b[a] = (int64_t)fl;
            d = c[a] - fl;
        }
        w[a] = (d <= 0.0 || b[a] + 1 > g.n[a] - 1) ? 0.0 : d;
    }
    const int64_t sy = g.n[0], sz = g.n[0] * g.n[1];
    const int64_t base = b[0] + sy * b[1] + sz * b[2];
    const int64_t ox = w[0] > 0.0 ? 1 : 0, oy = w[1] > 0.0 ? sy : 0, oz = w[2] > 0.0 ? sz : 0;
    auto plane = [&](int64_t o) {
        const double x0 = img[base + o] + (img[base + o + ox] - img[base + o]) * w[0];
        const double x1 = img[base + o + oy] + (img[base + o + oy + ox] - img[base + o + oy]) * w[0];
        return x0 + (x1 - x0) * w[1];
    };
    const double y0 = plane(0);
    out = w[2] > 0.0 ? y0 + (plane(oz) - y0) * w[2] : y0;
    return true;
}

// linear.rs:474-492 / metric/mi.rs:156-200 (fixed_sample_range): the finite fixed values at the
// nearest voxel of each sample point inside the buffer.
bool fixed_sample_range(const HostGrid& g, const std::vector<double>& img,
                        const std::vector<double>& pts, double& lo, double& hi, int64_t& seen) {
    bool have = false;
    seen = 0;
    for (size_t i = 0; i < pts.size() / 3; ++i) {
        double c[3];
        point_to_index(g, &pts[3 * i], c);
        int64_t q[3];
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            const double r = std::floor(c[a] + 0.5);
            if (r < 0.0 || r >= (double)g.n[a]) ok = false;
            else q[a] = (int64_t)r;
        }
        if (!ok) continue;
        const double v = img[q[0] + g.n[0] * (q[1] + g.n[1] * q[2])];
        if (!std::isfinite(v)) continue;
        ++seen;
        if (!have) {
            lo = hi = v;
            have = true;
        } else {
            lo = std::min(lo, v);
            hi = std::max(hi, v);
        }
    }
    return have;
}

int download(fw_ctx* ctx, const fw_image* img, std::vector<double>& out) {
    std::vector<float> f((size_t)img->grid.count());
    FW_TRY(fw_image_download(ctx, img, f.data()));
    out.assign(f.begin(), f.end());
    return 0;
}

// init.rs:50-74 (centre_of_gravity): the intensity-weighted mean of the voxel centres, summed in
// raster order.
int centre_of_gravity(fw_ctx* ctx, const fw_image* img, double out[3]) {
    std::vector<double> h;
    FW_TRY(download(ctx, img, h));
    const HostGrid& g = img->grid;
    double mass = 0.0, cg[3] = {0.0, 0.0, 0.0};
    size_t lin = 0;
    for (int64_t k = 0; k < g.n[2]; ++k)
        for (int64_t j = 0; j < g.n[1]; ++j)
            for (int64_t i = 0; i < g.n[0]; ++i, ++lin) {
                const double v = h[lin];
                const double c[3] = {(double)i, (double)j, (double)k};
                double p[3];
                index_to_point(g, c, p);
                mass += v;
                for (int a = 0; a < 3; ++a) cg[a] += p[a] * v;
            }
    if (mass == 0.0) return fail(FW_ERR_INVALID, "total mass of the image is zero");
    for (int a = 0; a < 3; ++a) out[a] = cg[a] / mass;
    return 0;
}

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

// mask.rs:76-110 (MaskVolume::is_inside): the nearest voxel of the mask (rounding half up) must be
// inside its buffer and not zero; the mask is evaluated in physical space on its own grid.
struct HostMask {
    HostGrid grid;
    std::vector<float> data;
    bool inside(const double p[3]) const {
        double c[3];
        point_to_index(grid, p, c);
        int64_t q[3];
        for (int a = 0; a < 3; ++a) {
            const double r = std::floor(c[a] + 0.5);
            if (!(r >= 0.0 && r < (double)grid.n[a])) return false;
            q[a] = (int64_t)r;
        }
        return data[(size_t)(q[0] + grid.n[0] * (q[1] + grid.n[1] * q[2]))] != 0.0f;
    }
};

int load_mask(fw_ctx* ctx, const fw_image* mask, HostMask& out) {
    out.grid = mask->grid;
    out.data.resize((size_t)mask->grid.count());
    FW_TRY(fw_image_download(ctx, mask, out.data.data()));
    for (float v : out.data)
        if (v != 0.0f) return 0;
    return fail(FW_ERR_INVALID, "linear recipe: the fixed mask has no voxel inside (every voxel is zero)");
}

// One level's Mattes MI samples (linear.rs:474-492, 251-280, 940-945): the regular sample set
// of the level grid `lg` from `seed` (only the points inside the fixed mask, when one is given);
// `skip` with the reference's reason when MI is undefined on them; otherwise the binning (fixed
// range at the samples' nearest voxels, moving range over the whole image, MiBinning::new,
// metric/mi.rs:229-262) and the kept points with their trilinear fixed bins.
int level_samples(const HostGrid& lg, const HostGrid& fg, const std::vector<double>& fh,
                  const std::vector<double>& mh, const HostMask* mask, float percentage,
                  uint32_t seed, int bins, std::vector<double>& kept, std::vector<uint32_t>& fbin,
                  fw_mi_binning& b, bool& skip, std::string& why) {
    skip = false;
    kept.clear();
    fbin.clear();
    std::vector<double> raw = regular_samples(lg, percentage, seed);
    if (mask) {
        // linear.rs:940-945 / sampling.rs:225-228: with a fixed mask only the jittered points
        // inside it are kept (every point still takes its six draws)
        size_t w = 0;
        for (size_t i = 0; i < raw.size() / 3; ++i) {
            if (!mask->inside(&raw[3 * i])) continue;
            for (int a = 0; a < 3; ++a) raw[3 * w + a] = raw[3 * i + a];
            ++w;
        }
        raw.resize(3 * w);
    }
    const int64_t candidates = (int64_t)(raw.size() / 3);
    double lo = 0, hi = 0;
    int64_t seen = 0;
    char msg[256];
    if (!fixed_sample_range(fg, fh, raw, lo, hi, seen)) {
        std::snprintf(msg, sizeof(msg), "no sample point lands on the fixed image inside the fixed "
                      "mask, if one is given (%lld candidate points on the level grid)",
                      (long long)candidates);
        skip = true;
    } else if (hi - lo <= DBL_EPSILON) {
        std::snprintf(msg, sizeof(msg), "the fixed image takes a single value at its %lld sample "
                      "point(s) (%lld candidate points)", (long long)seen, (long long)candidates);
        skip = true;
    }
    if (skip) {
        why = msg;
        return 0;
    }
    bool mhave = false;
    double mlo = 0, mhi = 0;
    for (double v : mh) {
        if (!std::isfinite(v)) continue;
        if (!mhave) {
            mlo = mhi = v;
            mhave = true;
        } else {
            mlo = std::min(mlo, v);
            mhi = std::max(mhi, v);
        }
    }
    if (!mhave) return fail(FW_ERR_INVALID, "the moving image has no finite voxel");
    if (mhi - mlo <= DBL_EPSILON) return fail(FW_ERR_INVALID, "the moving image is constant");
    const double span = (double)(bins - 4);
    b.bins = bins;
    b.fixed_min = lo;
    b.fixed_max = hi;
    b.moving_min = mlo;
    b.moving_max = mhi;
    b.fixed_bin_size = (hi - lo) / span;
    b.moving_bin_size = (mhi - mlo) / span;
    b.fixed_normalized_min = lo / b.fixed_bin_size - 2.0;
    b.moving_normalized_min = mlo / b.moving_bin_size - 2.0;
    // prepare_samples (linear.rs:251-280): points whose trilinear fixed value exists, with its
    // box-window bin
    for (int64_t i = 0; i < candidates; ++i) {
        double v;
        if (!linear_at_point(fg, fh, &raw[(size_t)(3 * i)], v) || !std::isfinite(v)) continue;
        kept.insert(kept.end(), &raw[(size_t)(3 * i)], &raw[(size_t)(3 * i)] + 3);
        const double term = v / b.fixed_bin_size - b.fixed_normalized_min;
        const int64_t idx = std::isnan(term) ? 0 : (int64_t)term;
        fbin.push_back((uint32_t)std::min<int64_t>(std::max<int64_t>(idx, 2), bins - 3));
    }
    if (kept.empty()) {
        std::snprintf(msg, sizeof(msg), "no sample point lies inside the fixed image (%lld "
                      "candidate points)", (long long)candidates);
        why = msg;
        skip = true;
    }
    return 0;
}

int linear_stage_run(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                     const fw_image* moving, const HostMask* mask, fw_linear_transform* transform,
                     fw_linear_level_trace* traces) {
    FW_CHECK(r->levels >= 1 && r->levels <= FW_MAX_LEVELS, "linear recipe: 1 to 8 levels");
    FW_CHECK(r->bins > 4, "at least five histogram bins are required");
    FW_CHECK(r->sampling_percentage > 0.0f && r->sampling_percentage <= 1.0f,
             "linear recipe: the sampling percentage must lie in (0, 1]");
    FW_CHECK(transform->kind == 0 || transform->kind == 1, "unknown linear transform kind");
    const HostGrid& fg = fixed->grid;
    uint32_t seed = r->seed;  // SeedSequence: one generator per level, never reset
    int skipped = 0;
    std::string why;
    for (int level = 0; level < r->levels; ++level) {
        if (cancel_requested(ctx)) return fail(FW_ERR_CANCELLED, "registration cancelled");
        uint32_t f[3];
        FW_TRY(fw_shrink_factors(r->shrink_factors[level], fg.sp, f));
        const fw_grid fgc = to_c(fg);
        fw_grid lgc;
        FW_TRY(fw_shrink_grid(&fgc, f, &lgc));
        HostGrid lg;
        FW_TRY(make_grid(&lgc, lg));
        fw_linear_level_trace tr{};
        tr.level = level;
        for (int a = 0; a < 3; ++a) {
            tr.shrink_factors[a] = f[a];
            tr.grid_size[a] = lg.n[a];
        }
        // the level's smoothed images (full resolution), on the device and as host float64
        const double sigma = r->smoothing_sigmas[level];
        fw_image *fs = nullptr, *ms = nullptr;
        int rc = 0;
        if (sigma > 0.0) {
            double sf[3], sm[3];
            for (int a = 0; a < 3; ++a) {
                sf[a] = r->sigma_units_mm ? sigma : sigma * fg.sp[a];
                sm[a] = r->sigma_units_mm ? sigma : sigma * moving->grid.sp[a];
            }
            rc = fw_smooth_recursive(ctx, fixed, sf, &fs);
            if (!rc) rc = fw_smooth_recursive(ctx, moving, sm, &ms);
        }
        const fw_image* fl = fs ? fs : fixed;
        const fw_image* ml = ms ? ms : moving;
        std::vector<double> fh, mh;
        if (!rc) rc = download(ctx, fl, fh);
        if (!rc) rc = download(ctx, ml, mh);
        // sampling and the level's usable samples
        std::vector<double> kept;
        std::vector<uint32_t> fbin;
        fw_mi_binning b{};
        bool skip = false;
        std::string msg;
        if (!rc)
            rc = level_samples(lg, fg, fh, mh, mask, r->sampling_percentage, seed++, r->bins, kept,
                               fbin, b, skip, msg);
        if (!rc && skip)
            why += std::string(why.empty() ? "" : "; ") + "level " + std::to_string(level + 1) +
                   ": " + msg;
        if (!rc && !skip) {
            fw_mi_level* lvl = nullptr;
            rc = fw_mi_level_prepare_image(ctx, ml, kept.data(), fbin.data(),
                                           (int64_t)fbin.size(), &b, &lvl);
            if (!rc) {
                double corners[24];
                fw_cg_settings s;
                fw_cg_settings_ants(r->gradient_step, (int32_t)r->iterations[level],
                                    r->convergence_threshold, r->convergence_window, &s);
                rc = fw_grid_corners(&lgc, corners);
                if (!rc) rc = fw_mi_level_optimize(lvl, &s, corners, transform, &tr.cg, nullptr, 0);
                fw_mi_level_free(lvl);
            }
            tr.samples = (int64_t)fbin.size();
        }
        if (fs) fw_image_free(fs);
        if (ms) fw_image_free(ms);
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

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

int fw_linear_stage_run(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                        const fw_image* moving, fw_linear_transform* transform,
                        fw_linear_level_trace* traces) {
    FW_CHECK(ctx && r && fixed && moving && transform, "null argument");
    return linear_stage_run(ctx, r, fixed, moving, nullptr, transform, traces);
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
    HostMask m;
    if (fixed_mask) FW_TRY(load_mask(ctx, fixed_mask, m));
    std::vector<double> fh, mh, kept;
    FW_TRY(download(ctx, fixed, fh));
    FW_TRY(download(ctx, moving, mh));
    std::vector<uint32_t> fbin;
    fw_mi_binning b{};
    bool skip = false;
    std::string why;
    FW_TRY(level_samples(lg, fixed->grid, fh, mh, fixed_mask ? &m : nullptr, percentage, seed,
                         bins, kept, fbin, b, skip, why));
    if (skip) return fail(FW_ERR_INVALID, "mattes: " + why);
    return fw_mi_level_prepare_image(ctx, moving, kept.data(), fbin.data(), (int64_t)fbin.size(),
                                     &b, out);
}

int fw_linear_stage_run_masked(fw_ctx* ctx, const fw_linear_recipe* r, const fw_image* fixed,
                               const fw_image* moving, const fw_image* fixed_mask,
                               fw_linear_transform* transform, fw_linear_level_trace* traces) {
    FW_CHECK(ctx && r && fixed && moving && transform, "null argument");
    if (!fixed_mask) return linear_stage_run(ctx, r, fixed, moving, nullptr, transform, traces);
    HostMask m;
    FW_TRY(load_mask(ctx, fixed_mask, m));
    return linear_stage_run(ctx, r, fixed, moving, &m, transform, traces);
}

// run_linear_chain_cached_async (linear.rs:1148-1212): the centre-of-mass initial transform
// of the raw images (init.rs:76-86), the rigid stage from it, the affine stage from the rigid
// result, and their collapse recentred on the affine stage's centre (with_center, :1071-1076).
// The fixed mask (nullable) restricts both stages' samples (LinearRecipe::mask of each stage).
static int linear_chain_run(fw_ctx* ctx, const fw_linear_recipe* rigid,
                            const fw_linear_recipe* affine, const fw_image* fixed_raw,
                            const fw_image* moving_raw, const fw_image* fixed,
                            const fw_image* moving, const fw_image* fixed_mask,
                            fw_linear_chain_result* out) {
    FW_CHECK(ctx && rigid && affine && fixed_raw && moving_raw && fixed && moving && out,
             "null argument");
    std::memset(out, 0, sizeof(*out));
    HostMask mask;
    if (fixed_mask) FW_TRY(load_mask(ctx, fixed_mask, mask));
    const HostMask* mp = fixed_mask ? &mask : nullptr;
    double fc[3], mc[3];
    FW_TRY(centre_of_gravity(ctx, fixed_raw, fc));
    FW_TRY(centre_of_gravity(ctx, moving_raw, mc));
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
    FW_TRY(linear_stage_run(ctx, rigid, fixed, moving, mp, &tr, out->rigid_levels));
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
    FW_TRY(linear_stage_run(ctx, affine, fixed, moving, mp, &ta, out->affine_levels));
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
