// fw_optimize.cu -- the optimiser of the linear (Rigid / Affine) stages: parameter scales from
// physical shifts and ITK's conjugate-gradient optimiser with a golden-section line search, as
// crates/fastwarp-reg/src/optimizer.rs:142-435 runs it (ITK ConjugateGradientLineSearch-
// Optimizerv4, GradientDescentLineSearchOptimizerv4::GoldenSectionSearch,
// RegistrationParameterScalesFromPhysicalShift; ANTs' linear-stage settings).
//
// The optimiser is host code over a metric: C callbacks (`fw_metric_value_fn`,
// `fw_metric_value_derivative_fn`) stand for the reference's `LinearMetric` trait, so a host can
// drive it with any metric; `fw_mi_level_optimize` runs it on the device-resident sampled Mattes
// MI of a level (one device evaluation and one read-back per metric call, the line search's
// evaluations one after another as the search needs them).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "fw_internal.cuh"

namespace fw {

namespace {

constexpr double RESPHI = 2.0 - 1.618034;

int num_params(const fw_linear_transform& t) { return t.kind == 0 ? 6 : 12; }

void apply(const fw_linear_transform& t, const double p[3], double out[3]) {
    double M[9], o[3];
    linear_transform_map(&t, M, o);
    for (int r = 0; r < 3; ++r) out[r] = M[r * 3] * p[0] + M[r * 3 + 1] * p[1] + M[r * 3 + 2] * p[2] + o[r];
}

// optimizer.rs:168-183
double max_voxel_shift(const double* corners, const fw_linear_transform& t, const double* delta) {
    fw_linear_transform moved = t;
    for (int i = 0; i < num_params(t); ++i) moved.parameters[i] += delta[i];
    double mx = 0.0;
    for (int c = 0; c < 8; ++c) {
        double a[3], b[3];
        apply(moved, corners + 3 * c, a);
        apply(t, corners + 3 * c, b);
        double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
        mx = std::max(mx, std::sqrt(d0 * d0 + d1 * d1 + d2 * d2));
    }
    return mx;
}

// optimizer.rs:185-216
void estimate_scales(const double* corners, const fw_linear_transform& t, double small,
                     double* scales) {
    const int n = num_params(t);
    double min_non_zero = DBL_MAX;
    for (int i = 0; i < n; ++i) {
        double delta[12] = {0};
        delta[i] = small;
        const double shift = max_voxel_shift(corners, t, delta);
        scales[i] = shift;
        if (shift > DBL_EPSILON && shift < min_non_zero) min_non_zero = shift;
    }
    if (min_non_zero == DBL_MAX) {
        for (int i = 0; i < n; ++i) scales[i] = 1.0;
        return;
    }
    for (int i = 0; i < n; ++i) {
        if (scales[i] <= DBL_EPSILON) scales[i] = min_non_zero * min_non_zero;
        else scales[i] *= scales[i];
        scales[i] *= 1.0 / (small * small);
    }
}

// optimizer.rs:218-231
double estimate_step_scale(const double* corners, const fw_linear_transform& t, const double* step,
                           double small) {
    const int n = num_params(t);
    double max_step = 0.0;
    for (int i = 0; i < n; ++i) max_step = std::max(max_step, std::fabs(step[i]));
    if (max_step <= DBL_EPSILON) return 0.0;
    const double factor = small / max_step;
    double s[12];
    for (int i = 0; i < n; ++i) s[i] = step[i] * factor;
    return max_voxel_shift(corners, t, s) / factor;
}

// convergence.rs:47-126: the window convergence monitor (the two-control-point fit's closed form)
struct Monitor {
    int window;
    std::vector<double> values;  // the last `window` energies
    double total = 0.0;
    explicit Monitor(int w) : window(w) {}
    void add(double e) {
        values.push_back(e);
        if ((int)values.size() > window) values.erase(values.begin());
        total += std::fabs(e);
    }
    double value() const {
        if ((int)values.size() < window) return DBL_MAX;
        if (window < 2) return 0.0;
        const double spline_eps = 1e-3, domain_spacing = 0.1, domain_size = 11.0;
        const double r = 1.0 / ((domain_size - 1.0) * domain_spacing);
        const double epsilon = r * domain_spacing * spline_eps;
        double delta[2] = {0, 0}, omega[2] = {0, 0};
        for (size_t k = 0; k < values.size(); ++k) {
            double p = ((double)k / (double)(window - 1)) * r;
            if (std::fabs(p - 1.0) <= epsilon) p = 1.0 - epsilon;
            if (p < 0.0 && std::fabs(p) <= epsilon) p = 0.0;
            const double t = p - std::floor(p);
            const double w[2] = {1.0 - t, t};
            const double w2 = w[0] * w[0] + w[1] * w[1];
            const double v = values[k] / total;
            for (int j = 0; j < 2; ++j) {
                omega[j] += w[j] * w[j];
                delta[j] += v * (w[j] * w[j] * w[j] / w2);
            }
        }
        double phi[2] = {0, 0};
        for (int j = 0; j < 2; ++j) {
            if (std::fabs(omega[j]) > DBL_EPSILON) {
                const double q = delta[j] / omega[j];
                phi[j] = std::isfinite(q) ? q : 0.0;
            }
        }
        return phi[0] - phi[1];
    }
};

struct Metric {
    fw_metric_value_fn value;
    fw_metric_value_derivative_fn value_derivative;
    void* user;
};

// optimizer.rs:236-309
struct LineSearch {
    const Metric& metric;
    const fw_linear_transform& start;
    const double* direction;
    const fw_cg_settings& s;
    int iterations = 0;
    uint64_t evaluations = 0;

    int value_at(double step, double* out) {
        ++evaluations;
        fw_linear_transform t = start;
        for (int i = 0; i < num_params(start); ++i) t.parameters[i] = start.parameters[i] + step * direction[i];
        if (metric.value(metric.user, &t, out) != 0)
            return fail(FW_ERR_INVALID, std::string("linear metric: ") + fw_last_error());
        return 0;
    }

    int golden(double a, double b, double c, double* out) {
        double metric_b = DBL_MAX;
        for (;;) {
            if (iterations > s.max_line_search_iterations) {
                *out = (c + a) / 2.0;
                return 0;
            }
            ++iterations;
            const double x = c - b > b - a ? b + RESPHI * (c - b) : b - RESPHI * (b - a);
            if (std::fabs(c - a) < s.epsilon * (std::fabs(b) + std::fabs(x))) {
                *out = (c + a) / 2.0;
                return 0;
            }
            double metric_x;
            FW_TRY(value_at(x, &metric_x));
            if (metric_b == DBL_MAX) FW_TRY(value_at(b, &metric_b));
            if (metric_x < metric_b) {
                if (c - b > b - a) {
                    a = b;
                    b = x;
                } else {
                    c = b;
                    b = x;
                }
                metric_b = metric_x;
            } else if (c - b > b - a) {
                c = x;
            } else if (metric_x == DBL_MAX) {
                c = b;
                b = x;
                metric_b = metric_x;
            } else {
                a = x;
            }
        }
    }
};

double inner(const double* a, const double* b, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// optimizer.rs:311-435
int optimise_level(const Metric& metric, const double* corners, fw_linear_transform* t,
                   const fw_cg_settings& s, fw_cg_trace* trace, double* values, int64_t cap,
                   const volatile int32_t* cancel, const fw_ctx* ctx = nullptr) {
    const int n = num_params(*t);
    double scales[12];
    estimate_scales(corners, *t, s.small_parameter_variation, scales);
    fw_linear_transform current = *t, best = *t;
    double conjugate[12] = {0}, last_gradient[12] = {0}, gradient[12];
    double learning_rate = s.max_step_mm;
    Monitor monitor(s.convergence_window);
    double best_value = DBL_MAX;
    std::memset(trace, 0, sizeof(*trace));
    trace->converged_value = NAN;
    for (int i = 0; i < n; ++i) trace->scales[i] = scales[i];
    trace->initial_learning_rate = learning_rate;
    int iteration = 0;
    while (iteration < s.iterations) {
        if ((cancel && *cancel) || (ctx && cancel_requested(ctx)))
            return fail(FW_ERR_CANCELLED, "registration cancelled");
        double value;
        if (metric.value_derivative(metric.user, &current, &value, gradient) != 0)
            return fail(FW_ERR_INVALID, std::string("linear metric: ") + fw_last_error());
        monitor.add(value);
        if (monitor.value() <= s.convergence_threshold) {
            trace->converged = 1;
            trace->converged_value = value;
            break;
        }
        if (values && trace->nvalues < cap) values[trace->nvalues] = value;
        trace->nvalues++;
        for (int i = 0; i < n; ++i) gradient[i] *= 1.0 / scales[i];
        if (iteration == 0) {
            const double step_scale =
                estimate_step_scale(corners, current, gradient, s.small_parameter_variation);
            learning_rate = step_scale <= DBL_EPSILON ? 1.0 : s.max_step_mm / step_scale;
            trace->initial_learning_rate = learning_rate;
        }
        double gamma = 0.0;
        const double denom = inner(last_gradient, last_gradient, n);
        if (denom > DBL_EPSILON) {
            double diff[12];
            for (int i = 0; i < n; ++i) diff[i] = gradient[i] - last_gradient[i];
            gamma = inner(diff, gradient, n) / denom;
        }
        if (!(gamma >= 0.0 && gamma <= 5.0)) gamma = 0.0;
        for (int i = 0; i < n; ++i) {
            last_gradient[i] = gradient[i];
            conjugate[i] = gradient[i] + conjugate[i] * gamma;
        }
        LineSearch search{metric, current, conjugate, s};
        FW_TRY(search.golden(learning_rate * s.lower_limit, learning_rate,
                             learning_rate * s.upper_limit, &learning_rate));
        trace->line_search_evaluations += search.evaluations;
        for (int i = 0; i < n; ++i) current.parameters[i] += learning_rate * conjugate[i];
        if (value < best_value) {
            best_value = value;
            best = current;
        }
        ++iteration;
    }
    trace->iterations = iteration;
    trace->best_value = best_value;
    trace->final_learning_rate = learning_rate;
    *t = best;
    return 0;
}

int mi_value(void* user, const fw_linear_transform* t, double* value) {
    return fw_mi_level_value(static_cast<fw_mi_level*>(user), t, value);
}

int mi_value_derivative(void* user, const fw_linear_transform* t, double* value, double* d) {
    return fw_mi_level_value_and_derivative(static_cast<fw_mi_level*>(user), t, value, d);
}

}  // namespace
}  // namespace fw

using namespace fw;

extern "C" {

void fw_cg_settings_ants(double max_step_mm, int32_t iterations, double threshold,
                         int32_t window, fw_cg_settings* out) {
    if (!out) return;
    out->max_step_mm = max_step_mm;
    out->lower_limit = 0.0;
    out->upper_limit = 2.0;
    out->epsilon = 0.2;
    out->max_line_search_iterations = 20;
    out->iterations = iterations;
    out->convergence_threshold = threshold;
    out->convergence_window = window;
    out->small_parameter_variation = 0.01;
}

int fw_grid_corners(const fw_grid* grid, double corners[24]) {
    FW_CHECK(grid && corners, "null argument");
    HostGrid g;
    FW_TRY(make_grid(grid, g));
    for (int i = 0; i < 8; ++i) {
        const double idx[3] = {(i & 1) ? (double)(g.n[0] - 1) : 0.0,
                               (i & 2) ? (double)(g.n[1] - 1) : 0.0,
                               (i & 4) ? (double)(g.n[2] - 1) : 0.0};
        for (int r = 0; r < 3; ++r)
            corners[3 * i + r] = g.org[r] + (g.ds[r * 3] * idx[0] + g.ds[r * 3 + 1] * idx[1] +
                                             g.ds[r * 3 + 2] * idx[2]);
    }
    return 0;
}

int fw_linear_estimate_scales(const double corners[24], const fw_linear_transform* t,
                              double small_variation, double* scales) {
    FW_CHECK(corners && t && scales, "null argument");
    FW_CHECK(t->kind == 0 || t->kind == 1, "linear transform: unknown kind");
    estimate_scales(corners, *t, small_variation, scales);
    return 0;
}

int fw_linear_estimate_step_scale(const double corners[24], const fw_linear_transform* t,
                                  const double* step, double small_variation, double* out) {
    FW_CHECK(corners && t && step && out, "null argument");
    FW_CHECK(t->kind == 0 || t->kind == 1, "linear transform: unknown kind");
    *out = estimate_step_scale(corners, *t, step, small_variation);
    return 0;
}

int fw_cg_optimize_level(const fw_cg_settings* settings, const double corners[24],
                         fw_linear_transform* transform, fw_metric_value_fn value,
                         fw_metric_value_derivative_fn value_derivative, void* user,
                         fw_cg_trace* trace, double* values, int64_t cap,
                         const volatile int32_t* cancel) {
    FW_CHECK(settings && corners && transform && value && value_derivative && trace,
             "null argument");
    FW_CHECK(transform->kind == 0 || transform->kind == 1, "linear transform: unknown kind");
    const Metric m{value, value_derivative, user};
    return optimise_level(m, corners, transform, *settings, trace, values, cap, cancel);
}

int fw_mi_level_optimize(fw_mi_level* level, const fw_cg_settings* settings,
                         const double corners[24], fw_linear_transform* transform,
                         fw_cg_trace* trace, double* values, int64_t cap) {
    FW_CHECK(level && settings && corners && transform && trace, "null argument");
    FW_CHECK(transform->kind == 0 || transform->kind == 1, "linear transform: unknown kind");
    const Metric m{mi_value, mi_value_derivative, level};
    // the level's context: its cancel flags are polled before every iteration
    return optimise_level(m, corners, transform, *settings, trace, values, cap, nullptr,
                          mi_level_context(level));
}

}  // extern "C"
