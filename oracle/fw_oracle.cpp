// fw_oracle.cpp -- f64 CPU oracle of the fastwarp registration hot path.
//
// TEST INFRASTRUCTURE ONLY: the parity checker of tests/ and the CPU baseline of bench.py.
// Nothing in the product library links or calls this file.
//
// Every function restates the reference's CPU engine (WyssCenter/fastwarp, crate fastwarp-reg,
// paths below relative to crates/fastwarp-reg/src) in plain C++ with OpenMP; the file:line it
// follows is cited beside each one. Reductions use the reference's fixed chunk order
// (field_ops.rs:47-56) so results do not depend on the thread count.

#include "fw_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_error;

int fail(const std::string& what) {
    g_error = what;
    return -1;
}

typedef double V3[3];

struct Grid {
    int64_t n[3];
    double sp[3], org[3], dir[9];  // dir[row*3+axis]
    double inv[9];                 // (dir * diag(sp))^-1, row-major

    int64_t count() const { return n[0] * n[1] * n[2]; }
    int64_t lin(int64_t i, int64_t j, int64_t k) const { return i + n[0] * (j + n[1] * k); }
    void ijk(int64_t l, int64_t out[3]) const {
        out[0] = l % n[0];
        out[1] = (l / n[0]) % n[1];
        out[2] = l / (n[0] * n[1]);
    }
    // grid.rs:131-143
    void index_to_point(const double c[3], double p[3]) const {
        double s[3] = {c[0] * sp[0], c[1] * sp[1], c[2] * sp[2]};
        for (int r = 0; r < 3; ++r)
            p[r] = org[r] + (dir[r * 3 + 0] * s[0] + dir[r * 3 + 1] * s[1] + dir[r * 3 + 2] * s[2]);
    }
    // grid.rs:145-156
    void point_to_index(const double p[3], double c[3]) const {
        double d[3] = {p[0] - org[0], p[1] - org[1], p[2] - org[2]};
        for (int r = 0; r < 3; ++r)
            c[r] = inv[r * 3 + 0] * d[0] + inv[r * 3 + 1] * d[1] + inv[r * 3 + 2] * d[2];
    }
    // grid.rs:159-161, ITK IsInsideBuffer
    bool inside(const double c[3]) const {
        for (int a = 0; a < 3; ++a)
            if (!(c[a] >= -0.5 && c[a] < (double)n[a] - 0.5)) return false;
        return true;
    }
    void voxel_point(int64_t l, double p[3]) const {
        int64_t q[3];
        ijk(l, q);
        double c[3] = {(double)q[0], (double)q[1], (double)q[2]};
        index_to_point(c, p);
    }
    bool boundary(int64_t l) const {
        int64_t q[3];
        ijk(l, q);
        return q[0] == 0 || q[1] == 0 || q[2] == 0 || q[0] == n[0] - 1 || q[1] == n[1] - 1 ||
               q[2] == n[2] - 1;
    }
    bool same(const Grid& o) const {
        for (int a = 0; a < 3; ++a)
            if (n[a] != o.n[a] || sp[a] != o.sp[a] || org[a] != o.org[a]) return false;
        for (int a = 0; a < 9; ++a)
            if (dir[a] != o.dir[a]) return false;
        return true;
    }
};

// linalg.rs:53-70
bool mat3_inverse(const double m[9], double out[9]) {
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (det == 0.0 || !std::isfinite(det)) return false;
    double id = 1.0 / det;
    out[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    out[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    out[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
    return true;
}

void mat3_mul(const double a[9], const double b[9], double out[9]) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            out[r * 3 + c] = a[r * 3] * b[c] + a[r * 3 + 1] * b[3 + c] + a[r * 3 + 2] * b[6 + c];
}

void mat3_vec(const double m[9], const double v[3], double out[3]) {
    for (int r = 0; r < 3; ++r) out[r] = m[r * 3] * v[0] + m[r * 3 + 1] * v[1] + m[r * 3 + 2] * v[2];
}

// grid.rs:45-88 (validation and index_from_offset)
bool make_grid(const fwo_grid* g, Grid& out) {
    if (!g) return fail("null grid") == 0;
    for (int a = 0; a < 3; ++a) {
        if (g->size[a] <= 0) return fail("zero size") == 0;
        if (!std::isfinite(g->spacing[a]) || g->spacing[a] <= 0) return fail("bad spacing") == 0;
        out.n[a] = g->size[a];
        out.sp[a] = g->spacing[a];
        out.org[a] = g->origin[a];
    }
    std::memcpy(out.dir, g->direction, sizeof(out.dir));
    double scaled[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) scaled[r * 3 + c] = out.dir[r * 3 + c] * out.sp[c];
    if (!mat3_inverse(scaled, out.inv)) return fail("singular direction matrix") == 0;
    return true;
}

fwo_grid to_c(const Grid& g) {
    fwo_grid o;
    for (int a = 0; a < 3; ++a) {
        o.size[a] = g.n[a];
        o.spacing[a] = g.sp[a];
        o.origin[a] = g.org[a];
    }
    std::memcpy(o.direction, g.dir, sizeof(o.direction));
    return o;
}

// field_ops.rs:47-56: sums in chunks of 4096 in a fixed order.
const int64_t REDUCE_CHUNK = 4096;
double ordered_sum(const std::vector<double>& v) {
    int64_t n = (int64_t)v.size();
    int64_t chunks = (n + REDUCE_CHUNK - 1) / REDUCE_CHUNK;
    std::vector<double> part(chunks, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < chunks; ++c) {
        double s = 0.0;
        int64_t hi = std::min(n, (c + 1) * REDUCE_CHUNK);
        for (int64_t i = c * REDUCE_CHUNK; i < hi; ++i) s += v[i];
        part[c] = s;
    }
    double s = 0.0;
    for (double x : part) s += x;
    return s;
}

// interp.rs:43-85 -- ITK LinearInterpolateImageFunction::EvaluateAtContinuousIndex.
double linear_at_index(const Grid& g, const double* data, const double c[3]) {
    int64_t base[3];
    double w[3];
    for (int a = 0; a < 3; ++a) {
        double fl = std::floor(c[a]);
        int64_t b = fl < 0.0 ? 0 : (int64_t)fl;
        if (fl >= 9.2e18) b = g.n[a] - 1;
        b = std::min(b, g.n[a] - 1);
        double d = c[a] - (double)b;
        base[a] = b;
        w[a] = (d <= 0.0 || b + 1 > g.n[a] - 1) ? 0.0 : d;
    }
    auto at = [&](int dx, int dy, int dz) {
        return data[g.lin(base[0] + dx, base[1] + dy, base[2] + dz)];
    };
    auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
    auto xr = [&](int dy, int dz) {
        double v0 = at(0, dy, dz);
        return w[0] > 0.0 ? lerp(v0, at(1, dy, dz), w[0]) : v0;
    };
    auto yr = [&](int dz) {
        double v0 = xr(0, dz);
        return w[1] > 0.0 ? lerp(v0, xr(1, dz), w[1]) : v0;
    };
    double v0 = yr(0);
    return w[2] > 0.0 ? lerp(v0, yr(1), w[2]) : v0;
}

// interp.rs:87-94
bool linear_at_point(const Grid& g, const double* data, const double p[3], double& out) {
    double c[3];
    g.point_to_index(p, c);
    if (!g.inside(c)) return false;
    out = linear_at_index(g, data, c);
    return true;
}

// interp.rs:96-120 -- half-spacing central difference along the physical axes.
void central_difference(const Grid& g, const double* data, const double p[3], double out[3]) {
    for (int d = 0; d < 3; ++d) {
        out[d] = 0.0;
        double off = 0.5 * g.sp[d];
        double p1[3] = {p[0], p[1], p[2]}, p2[3] = {p[0], p[1], p[2]};
        p1[d] = p[d] - off;
        p2[d] = p[d] + off;
        double v1, v2;
        if (!linear_at_point(g, data, p1, v1) || !linear_at_point(g, data, p2, v2)) continue;
        double delta = p2[d] - p1[d];
        if (delta > 10.0 * DBL_EPSILON) out[d] = (v2 - v1) / delta;
    }
}

// field_ops.rs:143-172 -- ITK VectorLinearInterpolateImageFunction (neighbours clamped).
void vector_interpolate_index(const Grid& g, const double* f, const double c[3], double out[3]) {
    int64_t idx[3][2];
    double w[3][2];
    for (int a = 0; a < 3; ++a) {
        double fl = std::floor(c[a]);
        double d = c[a] - fl;
        int64_t base = (int64_t)fl;
        int64_t last = g.n[a] - 1;
        idx[a][0] = std::min(std::max(base, (int64_t)0), last);
        idx[a][1] = std::min(std::max(base + 1, (int64_t)0), last);
        w[a][0] = 1.0 - d;
        w[a][1] = d;
    }
    out[0] = out[1] = out[2] = 0.0;
    for (int counter = 0; counter < 8; ++counter) {
        int bx = counter & 1, by = (counter >> 1) & 1, bz = (counter >> 2) & 1;
        double overlap = w[0][bx] * w[1][by] * w[2][bz];
        if (overlap != 0.0) {
            const double* v = f + 3 * g.lin(idx[0][bx], idx[1][by], idx[2][bz]);
            out[0] += overlap * v[0];
            out[1] += overlap * v[1];
            out[2] += overlap * v[2];
        }
    }
}

// field_ops.rs:176-181
bool vector_interpolate(const Grid& g, const double* f, const double p[3], double out[3]) {
    double c[3];
    g.point_to_index(p, c);
    if (!g.inside(c)) return false;
    vector_interpolate_index(g, f, c, out);
    return true;
}

// mask.rs:99-111 -- nearest voxel, rounding half up.
bool nearest_voxel(const Grid& g, const double p[3], int64_t& out) {
    double c[3];
    g.point_to_index(p, c);
    int64_t q[3];
    for (int a = 0; a < 3; ++a) {
        double r = std::floor(c[a] + 0.5);
        if (!(r >= 0.0 && r < (double)g.n[a])) return false;
        q[a] = (int64_t)r;
    }
    out = g.lin(q[0], q[1], q[2]);
    return true;
}

void apply_affine(const fwo_affine* a, const double p[3], double out[3]) {
    double q[3];
    mat3_vec(a->matrix, p, q);
    for (int r = 0; r < 3; ++r) out[r] = q[r] + a->offset[r];
}

// cpu/mod.rs:60-86 / 88-132: the point sampled for output voxel l.
void warp_point(const Grid& g, const double* field, int64_t l, const Grid* pg, const double* pre,
                const fwo_affine* affine, double p[3]) {
    double x[3];
    g.voxel_point(l, x);
    const double* u = field + 3 * l;
    p[0] = x[0] + u[0];
    p[1] = x[1] + u[1];
    p[2] = x[2] + u[2];
    if (pg) {
        double d[3];
        if (vector_interpolate(*pg, pre, p, d)) {
            p[0] += d[0];
            p[1] += d[1];
            p[2] += d[2];
        }
    }
    if (affine) {
        double q[3];
        apply_affine(affine, p, q);
        p[0] = q[0];
        p[1] = q[1];
        p[2] = q[2];
    }
}

double scaled_norm(const double* v, const double sp[3]) {
    double a = v[0] / sp[0], b = v[1] / sp[1], c = v[2] / sp[2];
    return std::sqrt(a * a + b * b + c * c);
}

// field_ops.rs:251-272 -- ITK ComposeDisplacementFieldsImageFilter.
void compose(const Grid& g, const double* disp, const double* warping, double* out) {
    int64_t n = g.count();
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        double p1[3];
        g.voxel_point(l, p1);
        const double* w = warping + 3 * l;
        double p2[3] = {p1[0] + w[0], p1[1] + w[1], p1[2] + w[2]};
        double d[3] = {0, 0, 0};
        if (!vector_interpolate(g, disp, p2, d)) d[0] = d[1] = d[2] = 0.0;
        out[3 * l] = w[0] + d[0];
        out[3 * l + 1] = w[1] + d[1];
        out[3 * l + 2] = w[2] + d[2];
    }
}

// field_ops.rs:394-416 -- ITK GaussianOperator::ModifiedBesselI0 (Abramowitz & Stegun 9.8.1-2
// polynomial fits; the published coefficient tables).
double bessel_i0(double y) {
    double d = std::fabs(y);
    if (d < 3.75) {
        double m = y / 3.75;
        m *= m;
        return 1.0 + m * (3.5156229 + m * (3.0899424 + m * (1.2067492 +
                      m * (0.2659732 + m * (0.360768e-1 + m * 0.45813e-2)))));
    }
    double m = 3.75 / d;
    return (std::exp(d) / std::sqrt(d)) *
           (0.39894228 + m * (0.1328592e-1 + m * (0.225319e-2 + m * (-0.157565e-2 +
            m * (0.916281e-2 + m * (-0.2057706e-1 + m * (0.2635537e-1 +
            m * (-0.1647633e-1 + m * 0.392377e-2))))))));
}

// field_ops.rs:418-441 -- A&S 9.8.3-4.
double bessel_i1(double y) {
    double d = std::fabs(y), acc;
    if (d < 3.75) {
        double m = y / 3.75;
        m *= m;
        acc = d * (0.5 + m * (0.87890594 + m * (0.51498869 + m * (0.15084934 +
              m * (0.2658733e-1 + m * (0.301532e-2 + m * 0.32411e-3))))));
    } else {
        double m = 3.75 / d;
        double a = 0.2282967e-1 + m * (-0.2895312e-1 + m * (0.1787654e-1 - m * 0.420059e-2));
        a = 0.39894228 + m * (-0.3988024e-1 + m * (-0.362018e-2 + m * (0.163801e-2 +
            m * (-0.1031555e-1 + m * a))));
        acc = a * (std::exp(d) / std::sqrt(d));
    }
    return y < 0.0 ? -acc : acc;
}

// field_ops.rs:443-476 -- Miller's downward recurrence normalised by I0.
double bessel_in(int n, double y) {
    const double accuracy = 40.0;
    if (y == 0.0) return 0.0;
    double toy = 2.0 / std::fabs(y);
    double qip = 0.0, acc = 0.0, qi = 1.0;
    int start = 2 * (n + (int)std::sqrt(accuracy * (double)n));
    for (int j = start; j > 0; --j) {
        double qim = qip + (double)j * toy * qi;
        qip = qi;
        qi = qim;
        if (std::fabs(qi) > 1.0e10) {
            acc *= 1.0e-10;
            qi *= 1.0e-10;
            qip *= 1.0e-10;
        }
        if (j == n) acc = qip;
    }
    acc *= bessel_i0(y) / qi;
    return (y < 0.0 && (n & 1)) ? -acc : acc;
}

// field_ops.rs:478-506 -- the taps of ITK's GaussianOperator.
std::vector<double> gaussian_taps(double variance, double max_error, int64_t max_width) {
    double et = std::exp(-variance);
    double cap = 1.0 - max_error;
    std::vector<double> half;
    half.push_back(et * bessel_i0(variance));
    double sum = half[0];
    half.push_back(et * bessel_i1(variance));
    sum += half[1] * 2.0;
    int i = 2;
    while (sum < cap) {
        half.push_back(et * bessel_in(i, variance));
        sum += half[i] * 2.0;
        if (half[i] <= 0.0) break;
        if ((int64_t)half.size() > max_width) break;
        ++i;
    }
    for (double& c : half) c /= sum;
    std::vector<double> full;
    for (size_t k = half.size() - 1; k >= 1; --k) full.push_back(half[k]);
    for (double c : half) full.push_back(c);
    return full;
}

// field_ops.rs:508-528 -- one axis, edge replication.
void convolve_axis(const double* in, double* out, const int64_t n[3], int axis,
                   const std::vector<double>& k) {
    int64_t radius = (int64_t)k.size() / 2;
    int64_t stride = axis == 0 ? 1 : (axis == 1 ? n[0] : n[0] * n[1]);
    int64_t len = n[axis];
    int64_t total = n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < total; ++idx) {
        int64_t pos = (idx / stride) % len;
        int64_t base = idx - pos * stride;
        double acc[3] = {0, 0, 0};
        for (size_t t = 0; t < k.size(); ++t) {
            int64_t q = std::min(std::max(pos + (int64_t)t - radius, (int64_t)0), len - 1);
            const double* v = in + 3 * (base + q * stride);
            acc[0] += k[t] * v[0];
            acc[1] += k[t] * v[1];
            acc[2] += k[t] * v[2];
        }
        out[3 * idx] = acc[0];
        out[3 * idx + 1] = acc[1];
        out[3 * idx + 2] = acc[2];
    }
}

// field_ops.rs:530-574 -- SyN's GaussianSmoothDisplacementField.
void smooth_field(const Grid& g, const double* field, double variance, double* out) {
    int64_t n = g.count();
    if (variance <= 0.0) {
        std::memcpy(out, field, sizeof(double) * 3 * n);
        return;
    }
    std::vector<double> a(field, field + 3 * n), b(3 * n);
    for (int axis = 0; axis < 3; ++axis) {
        std::vector<double> k = gaussian_taps(variance, 0.001, g.n[axis]);
        convolve_axis(a.data(), b.data(), g.n, axis, k);
        std::swap(a, b);
    }
    double w1 = variance < 0.5 ? 1.0 - variance / 0.5 : 1.0;
    double w2 = 1.0 - w1;
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        for (int c = 0; c < 3; ++c)
            out[3 * l + c] = g.boundary(l) ? 0.0 : a[3 * l + c] * w1 + field[3 * l + c] * w2;
    }
}

// field_ops.rs:191-203 (NaN propagates)
double max_scaled_norm(const Grid& g, const double* f) {
    int64_t n = g.count();
    double m = 0.0;
    bool nan = false;
    for (int64_t l = 0; l < n; ++l) {
        double v = scaled_norm(f + 3 * l, g.sp);
        if (std::isnan(v)) nan = true;
        m = std::max(m, v);
    }
    return nan ? std::numeric_limits<double>::quiet_NaN() : m;
}

// field_ops.rs:205-213
double l2_norm(const Grid& g, const double* f) {
    int64_t n = g.count();
    std::vector<double> sq(n);
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        const double* v = f + 3 * l;
        sq[l] = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    }
    return std::sqrt(ordered_sum(sq));
}

// field_ops.rs:309-392 -- ITK InvertDisplacementFieldImageFilter.
void invert(const Grid& g, const double* field, double* inverse, const fwo_invert_params& prm,
            fwo_invert_stats& stats) {
    int64_t n = g.count();
    double count = (double)n;
    double max_error = DBL_MAX, mean_error = DBL_MAX;
    uint32_t iteration = 0, executed = 0;
    std::vector<double> composed(3 * n), norms(n);
    for (;;) {
        uint32_t current = iteration++;
        if (!((int64_t)current < prm.max_iterations && max_error > prm.max_error_tolerance &&
              mean_error > prm.mean_error_tolerance))
            break;
        ++executed;
        compose(g, field, inverse, composed.data());
#pragma omp parallel for schedule(static)
        for (int64_t l = 0; l < n; ++l) norms[l] = scaled_norm(&composed[3 * l], g.sp);
        mean_error = ordered_sum(norms) / count;
        double mx = 0.0;
        for (int64_t l = 0; l < n; ++l) mx = std::max(mx, norms[l]);
        max_error = mx;
        double eps = current == 0 ? 0.75 : 0.5;
        double limit = eps * max_error;
#pragma omp parallel for schedule(static)
        for (int64_t l = 0; l < n; ++l) {
            double up[3] = {-composed[3 * l], -composed[3 * l + 1], -composed[3 * l + 2]};
            if (norms[l] > limit) {
                double f = limit / norms[l];
                up[0] *= f;
                up[1] *= f;
                up[2] *= f;
            }
            double* psi = inverse + 3 * l;
            psi[0] = psi[0] + up[0] * eps;
            psi[1] = psi[1] + up[1] * eps;
            psi[2] = psi[2] + up[2] * eps;
            if (prm.enforce_boundary_condition && g.boundary(l)) psi[0] = psi[1] = psi[2] = 0.0;
        }
    }
    stats.iterations = (int32_t)executed;
    stats.mean_error_norm = executed == 0 ? 0.0 : mean_error;
    stats.max_error_norm = executed == 0 ? 0.0 : max_error;
}

// field_ops.rs:580-605 -- DisplacementFieldTransformParametersAdaptor (scalar interpolation).
void resample_field(const Grid& src, const double* f, const Grid& dst, double* out) {
    int64_t n = dst.count(), ns = src.count();
    if (src.same(dst)) {
        std::memcpy(out, f, sizeof(double) * 3 * n);
        return;
    }
    std::vector<double> comp[3];
    for (int c = 0; c < 3; ++c) {
        comp[c].resize(ns);
        for (int64_t l = 0; l < ns; ++l) comp[c][l] = f[3 * l + c];
    }
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        double p[3], c[3];
        dst.voxel_point(l, p);
        src.point_to_index(p, c);
        if (!src.inside(c)) {
            out[3 * l] = out[3 * l + 1] = out[3 * l + 2] = 0.0;
            continue;
        }
        for (int k = 0; k < 3; ++k) out[3 * l + k] = linear_at_index(src, comp[k].data(), c);
    }
}

// metric/cc.rs:137-157 -- clamped box sum along one axis of the six window planes.
void box_sum_axis(const std::vector<double>& in, std::vector<double>& out, const int64_t n[3],
                  int axis, int64_t radius) {
    int64_t stride = axis == 0 ? 1 : (axis == 1 ? n[0] : n[0] * n[1]);
    int64_t len = n[axis];
    int64_t total = n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < total; ++idx) {
        int64_t pos = (idx / stride) % len;
        int64_t lo = std::max(pos - radius, (int64_t)0);
        int64_t hi = std::min(pos + radius, len - 1);
        int64_t base = idx - pos * stride;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t t = lo; t <= hi; ++t) {
            const double* v = &in[6 * (base + t * stride)];
            for (int c = 0; c < 6; ++c) acc[c] += v[c];
        }
        for (int c = 0; c < 6; ++c) out[6 * idx + c] = acc[c];
    }
}

// metric/cc.rs:170-321 -- CcMetric::evaluate_masked with identity transforms on one grid
// (what cpu/mod.rs:134-197 passes).
int cc_evaluate(const Grid& g, const double* fixed, const double* moving, const double* valid_img,
                int64_t radius, double& value, double* derivative, double* local_cc_out,
                double* coeff_out, int64_t& num_valid_out) {
    int64_t n = g.count();
    std::vector<unsigned char> valid(n, 0);
    std::vector<double> f(n, 0.0), m(n, 0.0), grad(derivative ? 3 * n : 0, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        if (valid_img && valid_img[l] == 0.0) continue;
        double p[3], fv, mv;
        g.voxel_point(l, p);
        if (!linear_at_point(g, fixed, p, fv)) continue;
        if (!linear_at_point(g, moving, p, mv)) continue;
        if (derivative) central_difference(g, moving, p, &grad[3 * l]);
        valid[l] = 1;
        f[l] = fv;
        m[l] = mv;
    }
    int64_t num_valid = 0;
    for (int64_t l = 0; l < n; ++l) num_valid += valid[l];
    if (num_valid == 0) {
        return fail(valid_img ? "no voxel of the registration level lies inside both the fixed "
                                "and the moving mask"
                              : "no virtual voxel maps inside both image buffers");
    }
    std::vector<double> s(6 * n, 0.0), t(6 * n);
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        if (!valid[l]) continue;
        double* q = &s[6 * l];
        q[0] = f[l] * f[l];
        q[1] = m[l] * m[l];
        q[2] = f[l];
        q[3] = m[l];
        q[4] = f[l] * m[l];
        q[5] = 1.0;
    }
    for (int axis = 0; axis < 3; ++axis) {
        box_sum_axis(s, t, g.n, axis, radius);
        std::swap(s, t);
    }
    const double eps = DBL_EPSILON;
    std::vector<double> cc(n, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        if (coeff_out) coeff_out[l] = 0.0;
        if (derivative) derivative[3 * l] = derivative[3 * l + 1] = derivative[3 * l + 2] = 0.0;
        if (!valid[l]) continue;
        const double* q = &s[6 * l];
        double sum_f2 = q[0], sum_m2 = q[1], sum_f = q[2], sum_m = q[3], sum_fm = q[4], cnt = q[5];
        double fm = sum_f / cnt, mm = sum_m / cnt;
        double s_ff = sum_f2 - fm * sum_f - fm * sum_f + cnt * fm * fm;
        double s_mm = sum_m2 - mm * sum_m - mm * sum_m + cnt * mm * mm;
        double s_fm = sum_fm - mm * sum_f - fm * sum_m + cnt * mm * fm;
        double fi = f[l] - fm, mi = m[l] - mm;
        double product = s_ff * s_mm;
        double c = 1.0;
        if (std::fabs(product) > eps) c = s_fm * s_fm / product;
        cc[l] = c;
        if (derivative && s_ff > eps && s_mm > eps) {
            double coeff = 2.0 * s_fm / product * (fi - s_fm / s_mm * mi);
            if (coeff_out) coeff_out[l] = coeff;
            for (int k = 0; k < 3; ++k) derivative[3 * l + k] = coeff * grad[3 * l + k];
        }
    }
    double total = 0.0;
    for (int64_t l = 0; l < n; ++l) {
        if (!valid[l]) continue;
        total -= cc[l];
        if (local_cc_out) local_cc_out[l] = cc[l];
    }
    if (local_cc_out)
        for (int64_t l = 0; l < n; ++l)
            if (!valid[l]) local_cc_out[l] = 0.0;
    value = total / (double)num_valid;
    num_valid_out = num_valid;
    return 0;
}

// pyramid.rs:58-93 -- ANTs CalculateShrinkFactorsPerDimension.
void shrink_factors(uint32_t factor, const double sp[3], uint32_t out[3]) {
    factor = std::max(factor, 1u);
    int mi = 0;
    double ms = sp[0];
    for (int n = 1; n < 3; ++n)
        if (ms > sp[n]) {
            ms = sp[n];
            mi = n;
        }
    double target = sp[mi] * (double)factor;
    out[0] = out[1] = out[2] = 0;
    out[mi] = factor;
    for (int n = 0; n < 3; ++n) {
        if (out[n] != 0) continue;
        double best_diff = std::fabs(sp[n] * (double)factor - target);
        uint32_t best = factor;
        for (uint32_t f = factor - 1; f >= 1; --f) {
            double diff = std::fabs(sp[n] * (double)f - target);
            if (diff <= best_diff) {
                best_diff = diff;
                best = f;
            }
        }
        out[n] = best;
    }
}

// pyramid.rs:99-129 -- ITK ShrinkImageFilter output grid (centres coincide).
bool shrink_grid(const Grid& g, const uint32_t f[3], Grid& out) {
    fwo_grid o = to_c(g);
    for (int a = 0; a < 3; ++a) {
        uint32_t fa = std::max(f[a], 1u);
        o.spacing[a] = g.sp[a] * (double)fa;
        o.size[a] = std::max((int64_t)std::floor((double)g.n[a] / (double)fa), (int64_t)1);
    }
    double ic[3], oc[3], ip[3], op[3];
    for (int a = 0; a < 3; ++a) {
        ic[a] = ((double)g.n[a] - 1.0) / 2.0;
        oc[a] = ((double)o.size[a] - 1.0) / 2.0;
    }
    g.index_to_point(ic, ip);
    Grid prov;
    if (!make_grid(&o, prov)) return false;
    prov.index_to_point(oc, op);
    for (int a = 0; a < 3; ++a) o.origin[a] = g.org[a] + (ip[a] - op[a]);
    return make_grid(&o, out);
}

// pyramid.rs:186-300 -- Deriche's fourth-order recursive Gaussian (ITK RecursiveGaussian,
// zero order); the constants are Deriche's published fit.
struct Deriche {
    double n[4], d[4], m[4], bn[4], bm[4];
};

bool deriche_zero_order(double sigma, double spacing, Deriche& out) {
    if (spacing < 1e-8) return fail("spacing is too small") == 0;
    double sd_ = sigma / spacing;
    const double a1 = 1.3530, b1 = 1.8151, w1 = 0.6681, l1 = -1.3932;
    const double a2 = -0.3531, b2 = 0.0902, w2 = 2.0787, l2 = -1.3732;
    double sin1 = std::sin(w1 / sd_), sin2 = std::sin(w2 / sd_);
    double cos1 = std::cos(w1 / sd_), cos2 = std::cos(w2 / sd_);
    double exp1 = std::exp(l1 / sd_), exp2 = std::exp(l2 / sd_);
    double d4 = exp1 * exp1 * exp2 * exp2;
    double d3 = -2.0 * cos1 * exp1 * exp2 * exp2;
    d3 += -2.0 * cos2 * exp2 * exp1 * exp1;
    double d2 = 4.0 * cos2 * cos1 * exp1 * exp2;
    d2 += exp1 * exp1 + exp2 * exp2;
    double d1 = -2.0 * (exp2 * cos2 + exp1 * cos1);
    double sd = 1.0 + d1 + d2 + d3 + d4;
    double n0 = a1 + a2;
    double n1 = exp2 * (b2 * sin2 - (a2 + 2.0 * a1) * cos2);
    n1 += exp1 * (b1 * sin1 - (a1 + 2.0 * a2) * cos1);
    double n2 = (a1 + a2) * cos2 * cos1;
    n2 -= b1 * cos2 * sin1 + b2 * cos1 * sin2;
    n2 *= 2.0 * exp1 * exp2;
    n2 += a2 * exp1 * exp1 + a1 * exp2 * exp2;
    double n3 = exp2 * exp1 * exp1 * (b2 * sin2 - a2 * cos2);
    n3 += exp1 * exp2 * exp2 * (b1 * sin1 - a1 * cos1);
    double sn = n0 + n1 + n2 + n3;
    double alpha0 = 2.0 * sn / sd - n0;
    n0 *= 1.0 / alpha0;
    n1 *= 1.0 / alpha0;
    n2 *= 1.0 / alpha0;
    n3 *= 1.0 / alpha0;
    double m1 = n1 - d1 * n0, m2 = n2 - d2 * n0, m3 = n3 - d3 * n0, m4 = -d4 * n0;
    sn = n0 + n1 + n2 + n3;
    double sm = m1 + m2 + m3 + m4;
    sd = 1.0 + d1 + d2 + d3 + d4;
    double nn[4] = {n0, n1, n2, n3}, dd[4] = {d1, d2, d3, d4}, mm[4] = {m1, m2, m3, m4};
    for (int k = 0; k < 4; ++k) {
        out.n[k] = nn[k];
        out.d[k] = dd[k];
        out.m[k] = mm[k];
        out.bn[k] = dd[k] * sn / sd;
        out.bm[k] = dd[k] * sm / sd;
    }
    return true;
}

void deriche_line(const Deriche& c, const double* x, double* ca, double* an, double* out, int64_t ln) {
    const double *n = c.n, *d = c.d, *m = c.m, *bn = c.bn, *bm = c.bm;
    double v1 = x[0];
    ca[0] = v1 * n[0] + v1 * n[1] + v1 * n[2] + v1 * n[3];
    ca[1] = x[1] * n[0] + v1 * n[1] + v1 * n[2] + v1 * n[3];
    ca[2] = x[2] * n[0] + x[1] * n[1] + v1 * n[2] + v1 * n[3];
    ca[3] = x[3] * n[0] + x[2] * n[1] + x[1] * n[2] + v1 * n[3];
    ca[0] -= v1 * bn[0] + v1 * bn[1] + v1 * bn[2] + v1 * bn[3];
    ca[1] -= ca[0] * d[0] + v1 * bn[1] + v1 * bn[2] + v1 * bn[3];
    ca[2] -= ca[1] * d[0] + ca[0] * d[1] + v1 * bn[2] + v1 * bn[3];
    ca[3] -= ca[2] * d[0] + ca[1] * d[1] + ca[0] * d[2] + v1 * bn[3];
    for (int64_t i = 4; i < ln; ++i) {
        ca[i] = x[i] * n[0] + x[i - 1] * n[1] + x[i - 2] * n[2] + x[i - 3] * n[3];
        ca[i] -= ca[i - 1] * d[0] + ca[i - 2] * d[1] + ca[i - 3] * d[2] + ca[i - 4] * d[3];
    }
    double v2 = x[ln - 1];
    an[ln - 1] = v2 * m[0] + v2 * m[1] + v2 * m[2] + v2 * m[3];
    an[ln - 2] = x[ln - 1] * m[0] + v2 * m[1] + v2 * m[2] + v2 * m[3];
    an[ln - 3] = x[ln - 2] * m[0] + x[ln - 1] * m[1] + v2 * m[2] + v2 * m[3];
    an[ln - 4] = x[ln - 3] * m[0] + x[ln - 2] * m[1] + x[ln - 1] * m[2] + v2 * m[3];
    an[ln - 1] -= v2 * bm[0] + v2 * bm[1] + v2 * bm[2] + v2 * bm[3];
    an[ln - 2] -= an[ln - 1] * d[0] + v2 * bm[1] + v2 * bm[2] + v2 * bm[3];
    an[ln - 3] -= an[ln - 2] * d[0] + an[ln - 1] * d[1] + v2 * bm[2] + v2 * bm[3];
    an[ln - 4] -= an[ln - 3] * d[0] + an[ln - 2] * d[1] + an[ln - 1] * d[2] + v2 * bm[3];
    for (int64_t i = ln - 4; i >= 1; --i) {
        an[i - 1] = x[i] * m[0] + x[i + 1] * m[1] + x[i + 2] * m[2] + x[i + 3] * m[3];
        an[i - 1] -= an[i] * d[0] + an[i + 1] * d[1] + an[i + 2] * d[2] + an[i + 3] * d[3];
    }
    for (int64_t i = 0; i < ln; ++i) out[i] = ca[i] + an[i];
}

// pyramid.rs:418-427 -- SmoothingRecursiveGaussianImageFilter: axes z, x, y.
int smooth_recursive(const Grid& g, const double* img, const double sigma_mm[3], double* out) {
    int64_t n = g.count();
    std::memcpy(out, img, sizeof(double) * n);
    const int order[3] = {2, 0, 1};
    for (int oi = 0; oi < 3; ++oi) {
        int axis = order[oi];
        int64_t ln = g.n[axis];
        if (ln < 4) return fail("smoothing axis needs at least 4 voxels");
        if (!(sigma_mm[axis] > 0.0)) return fail("sigma must be greater than zero");
        Deriche c;
        if (!deriche_zero_order(sigma_mm[axis], g.sp[axis], c)) return -1;
        int64_t stride = axis == 0 ? 1 : (axis == 1 ? g.n[0] : g.n[0] * g.n[1]);
        int64_t lines = n / ln;
#pragma omp parallel
        {
            std::vector<double> x(ln), ca(ln), an(ln), r(ln);
#pragma omp for schedule(static)
            for (int64_t li = 0; li < lines; ++li) {
                // line li: enumerate the voxels whose axis coordinate is 0.
                int64_t base;
                if (axis == 0) base = li * g.n[0];
                else if (axis == 1) base = (li % g.n[0]) + (li / g.n[0]) * g.n[0] * g.n[1];
                else base = li;
                for (int64_t t = 0; t < ln; ++t) x[t] = out[base + t * stride];
                deriche_line(c, x.data(), ca.data(), an.data(), r.data(), ln);
                for (int64_t t = 0; t < ln; ++t) out[base + t * stride] = r[t];
            }
        }
    }
    return 0;
}

// sampling.rs:37-118 -- MT19937 as ITK seeds it.
struct Mt {
    uint32_t s[624];
    int next = 0, left = 0;
    static uint32_t twist(uint32_t m, uint32_t s0, uint32_t s1) {
        uint32_t mix = (s0 & 0x80000000u) | (s1 & 0x7fffffffu);
        uint32_t mag = (s1 & 1u) ? 0x9908b0dfu : 0u;
        return m ^ (mix >> 1) ^ mag;
    }
    explicit Mt(uint32_t seed) {
        s[0] = seed;
        for (int i = 1; i < 624; ++i) s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + (uint32_t)i;
        reload();
    }
    void reload() {
        for (int p = 0; p < 624 - 397; ++p) s[p] = twist(s[p + 397], s[p], s[p + 1]);
        for (int p = 624 - 397; p < 623; ++p) s[p] = twist(s[p + 397 - 624], s[p], s[p + 1]);
        s[623] = twist(s[623 + 397 - 624], s[623], s[0]);
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

// sampling.rs:163-171 -- ITK's Box-Muller, cosine branch.
double normal_from(uint32_t open, uint32_t open_upper) {
    double o = ((double)open + 0.5) * (1.0 / 4294967296.0);
    double ou = (double)open_upper * (1.0 / 4294967296.0);
    double r = std::sqrt(-2.0 * std::log(1.0 - o) * 1.0);
    double phi = 2.0 * M_PI * ou;
    return r * std::cos(phi);
}

// metric/mi.rs:61-88 -- ITK BSplineKernelFunction<3> and its derivative.
double bspline3(double u) {
    double a = std::fabs(u);
    if (a < 1.0) {
        double s = a * a;
        return (4.0 - 6.0 * s + 3.0 * s * a) / 6.0;
    }
    if (a < 2.0) {
        double s = a * a;
        return (8.0 - 12.0 * a + 6.0 * s - s * a) / 6.0;
    }
    return 0.0;
}

double bspline3_derivative(double u) {
    if (u >= 0.0 && u < 1.0) return -2.0 * u + 1.5 * u * u;
    if (u > -1.0 && u < 0.0) return -2.0 * u - 1.5 * u * u;
    if (u >= 1.0 && u < 2.0) return -2.0 + 2.0 * u - 0.5 * u * u;
    if (u > -2.0 && u <= -1.0) return 2.0 + 2.0 * u + 0.5 * u * u;
    return 0.0;
}

int clamp_bin(const fwo_mi_binning& b, double term) {
    int64_t idx = (int64_t)term;  // truncation toward zero, as Rust's `as i64`
    if (std::isnan(term)) idx = 0;
    return (int)std::min(std::max(idx, (int64_t)2), (int64_t)b.bins - 3);
}

// transform/affine.rs:152-190 (Euler3D) and :121-150 (affine parameters) as matrix + offset.
void parametric_affine(const fwo_linear_transform* t, double M[9], double off[3]) {
    double tr[3];
    if (t->kind == 0) {
        const double* p = t->parameters;
        double cx = std::cos(p[0]), sx = std::sin(p[0]);
        double cy = std::cos(p[1]), sy = std::sin(p[1]);
        double cz = std::cos(p[2]), sz = std::sin(p[2]);
        double rx[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
        double ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
        double rz[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
        double tmp[9];
        if (t->zyx) {
            mat3_mul(rz, ry, tmp);
            mat3_mul(tmp, rx, M);
        } else {
            mat3_mul(rz, rx, tmp);
            mat3_mul(tmp, ry, M);
        }
        tr[0] = p[3];
        tr[1] = p[4];
        tr[2] = p[5];
    } else {
        for (int k = 0; k < 9; ++k) M[k] = t->parameters[k];
        tr[0] = t->parameters[9];
        tr[1] = t->parameters[10];
        tr[2] = t->parameters[11];
    }
    double mc[3];
    mat3_vec(M, t->center, mc);
    for (int r = 0; r < 3; ++r) off[r] = tr[r] + t->center[r] - mc[r];
}

// transform/param.rs:421-446 -- outer(optimised(p)) as one affine map.
void linear_map(const fwo_linear_transform* t, fwo_affine* out) {
    double M[9], off[3];
    parametric_affine(t, M, off);
    double oc[3], ooff[3];
    mat3_vec(t->outer_matrix, t->outer_center, oc);
    for (int r = 0; r < 3; ++r) ooff[r] = t->outer_translation[r] + t->outer_center[r] - oc[r];
    mat3_mul(t->outer_matrix, M, out->matrix);
    double mo[3];
    mat3_vec(t->outer_matrix, off, mo);
    for (int r = 0; r < 3; ++r) out->offset[r] = mo[r] + ooff[r];
}

// transform/param.rs:188-288 + 448-457 -- Jacobian columns, left-multiplied by the outer matrix.
int linear_jacobian(const fwo_linear_transform* t, const double p[3], double cols[36]) {
    for (int k = 0; k < 36; ++k) cols[k] = 0.0;
    int nparam;
    if (t->kind == 0) {
        const double* q = t->parameters;
        double cx = std::cos(q[0]), sx = std::sin(q[0]);
        double cy = std::cos(q[1]), sy = std::sin(q[1]);
        double cz = std::cos(q[2]), sz = std::sin(q[2]);
        double px = p[0] - t->center[0], py = p[1] - t->center[1], pz = p[2] - t->center[2];
        double* o0 = cols;
        double* o1 = cols + 3;
        double* o2 = cols + 6;
        if (t->zyx) {
            o0[0] = (cz * sy * cx + sz * sx) * py + (-cz * sy * sx + sz * cx) * pz;
            o0[1] = (sz * sy * cx - cz * sx) * py + (-sz * sy * sx - cz * cx) * pz;
            o0[2] = (cy * cx) * py + (-cy * sx) * pz;
            o1[0] = (-cz * sy) * px + (cz * cy * sx) * py + (cz * cy * cx) * pz;
            o1[1] = (-sz * sy) * px + (sz * cy * sx) * py + (sz * cy * cx) * pz;
            o1[2] = (-cy) * px + (-sy * sx) * py + (-sy * cx) * pz;
            o2[0] = (-sz * cy) * px + (-sz * sy * sx - cz * cx) * py + (-sz * sy * cx + cz * sx) * pz;
            o2[1] = (cz * cy) * px + (cz * sy * sx - sz * cx) * py + (cz * sy * cx + sz * sx) * pz;
            o2[2] = 0.0;
        } else {
            o0[0] = (-sz * cx * sy) * px + (sz * sx) * py + (sz * cx * cy) * pz;
            o0[1] = (cz * cx * sy) * px + (-cz * sx) * py + (-cz * cx * cy) * pz;
            o0[2] = (sx * sy) * px + (cx)*py + (-sx * cy) * pz;
            o1[0] = (-cz * sy - sz * sx * cy) * px + (cz * cy - sz * sx * sy) * pz;
            o1[1] = (-sz * sy + cz * sx * cy) * px + (sz * cy + cz * sx * sy) * pz;
            o1[2] = (-cx * cy) * px + (-cx * sy) * pz;
            o2[0] = (-sz * cy - cz * sx * sy) * px + (-cz * cx) * py + (-sz * sy + cz * sx * cy) * pz;
            o2[1] = (cz * cy - sz * sx * sy) * px + (-sz * cx) * py + (cz * sy + sz * sx * cy) * pz;
            o2[2] = 0.0;
        }
        for (int d = 0; d < 3; ++d) cols[3 * (3 + d) + d] = 1.0;
        nparam = 6;
    } else {
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) cols[3 * (r * 3 + c) + r] = p[c] - t->center[c];
            cols[3 * (9 + r) + r] = 1.0;
        }
        nparam = 12;
    }
    for (int k = 0; k < nparam; ++k) {
        double v[3] = {cols[3 * k], cols[3 * k + 1], cols[3 * k + 2]}, o[3];
        mat3_vec(t->outer_matrix, v, o);
        cols[3 * k] = o[0];
        cols[3 * k + 1] = o[1];
        cols[3 * k + 2] = o[2];
    }
    return nparam;
}

struct Kahan {
    double sum = 0.0, comp = 0.0;
    void add(double x) {
        double y = x - comp;
        double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
};

// convergence.rs:47-126
struct Monitor {
    int window;
    std::deque<double> values;
    double total = 0.0;
    explicit Monitor(int w) : window(w) {}
    void add(double v) {
        values.push_back(v);
        if ((int)values.size() > window) values.pop_front();
        total += std::fabs(v);
    }
    double value() const {
        std::vector<double> v(values.begin(), values.end());
        return fwo_convergence_value(v.data(), (int64_t)v.size(), window, total);
    }
};

struct Recipe {
    const fwo_syn_recipe* r;
};

}  // namespace

extern "C" {

const char* fwo_last_error(void) { return g_error.c_str(); }

int fwo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void fwo_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int fwo_shrink_factors(uint32_t factor, const double spacing[3], uint32_t out[3]) {
    shrink_factors(factor, spacing, out);
    return 0;
}

int fwo_shrink_grid(const fwo_grid* grid, const uint32_t factors[3], fwo_grid* out) {
    Grid g, o;
    if (!make_grid(grid, g)) return -1;
    if (!shrink_grid(g, factors, o)) return -1;
    *out = to_c(o);
    return 0;
}

int fwo_point_to_index(const fwo_grid* grid, const double p[3], double out[3]) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    g.point_to_index(p, out);
    return 0;
}

int fwo_index_to_point(const fwo_grid* grid, const double c[3], double out[3]) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    g.index_to_point(c, out);
    return 0;
}

int fwo_warp(const fwo_grid* src_grid, const double* src, const fwo_grid* grid, const double* field,
             const fwo_grid* pre_grid, const double* pre, const fwo_affine* affine, double* out) {
    Grid sg, g, pg;
    if (!make_grid(src_grid, sg) || !make_grid(grid, g)) return -1;
    if (pre_grid && !make_grid(pre_grid, pg)) return -1;
    int64_t n = g.count();
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        double p[3], v;
        warp_point(g, field, l, pre_grid ? &pg : nullptr, pre, affine, p);
        out[l] = linear_at_point(sg, src, p, v) ? v : 0.0;
    }
    return 0;
}

int fwo_warp_mask(const fwo_grid* mask_grid, const double* mask, const fwo_grid* grid,
                  const double* field, const fwo_grid* pre_grid, const double* pre,
                  const fwo_affine* affine, const double* product, double* out) {
    Grid mg, g, pg;
    if (!make_grid(mask_grid, mg) || !make_grid(grid, g)) return -1;
    if (pre_grid && !make_grid(pre_grid, pg)) return -1;
    int64_t n = g.count();
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        double p[3];
        int64_t v;
        warp_point(g, field, l, pre_grid ? &pg : nullptr, pre, affine, p);
        double r = (nearest_voxel(mg, p, v) && mask[v] != 0.0) ? 1.0 : 0.0;
        out[l] = product ? r * product[l] : r;
    }
    return 0;
}

int fwo_cc(const fwo_grid* grid, const double* fixed, const double* moving, const double* valid,
           int32_t radius, double* value, double* derivative, double* local_cc,
           double* coefficient, int64_t* num_valid) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    double v = 0.0;
    int64_t nv = 0;
    if (cc_evaluate(g, fixed, moving, valid, radius, v, derivative, local_cc, coefficient, nv))
        return -1;
    if (value) *value = v;
    if (num_valid) *num_valid = nv;
    return 0;
}

// cpu/mod.rs:134-163 (masked pair) and :299-309 (plain pair: two evaluations).
int fwo_cc_pair(const fwo_grid* grid, const double* fixed, const double* moving,
                const double* valid, int32_t radius, double values[2], double* d_fwd,
                double* d_bwd) {
    if (fwo_cc(grid, fixed, moving, valid, radius, &values[0], d_fwd, nullptr, nullptr, nullptr))
        return -1;
    return fwo_cc(grid, moving, fixed, valid, radius, &values[1], d_bwd, nullptr, nullptr, nullptr);
}

int64_t fwo_gaussian_taps(double variance, double max_error, int64_t max_width, double* out,
                          int64_t cap) {
    std::vector<double> k = gaussian_taps(variance, max_error, max_width);
    for (int64_t i = 0; i < (int64_t)k.size() && i < cap; ++i) out[i] = k[i];
    return (int64_t)k.size();
}

int fwo_smooth_field(const fwo_grid* grid, const double* field, double variance, double* out) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    smooth_field(g, field, variance, out);
    return 0;
}

double fwo_max_scaled_norm(const fwo_grid* grid, const double* field) {
    Grid g;
    if (!make_grid(grid, g)) return std::numeric_limits<double>::quiet_NaN();
    return max_scaled_norm(g, field);
}

double fwo_l2_norm(const fwo_grid* grid, const double* field) {
    Grid g;
    if (!make_grid(grid, g)) return std::numeric_limits<double>::quiet_NaN();
    return l2_norm(g, field);
}

// field_ops.rs:231-238
int fwo_scale(const fwo_grid* grid, double* field, double s) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    int64_t n = 3 * g.count();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) field[i] *= s;
    return 0;
}

// field_ops.rs:215-229
int fwo_axpy(const fwo_grid* grid, double* acc, double a, const double* x) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    int64_t n = 3 * g.count();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) acc[i] += a * x[i];
    return 0;
}

int fwo_compose(const fwo_grid* grid, const double* displacement, const double* warping,
                double* out) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    compose(g, displacement, warping, out);
    return 0;
}

int fwo_invert(const fwo_grid* grid, const double* field, double* inverse,
               const fwo_invert_params* params, fwo_invert_stats* stats) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    invert(g, field, inverse, *params, *stats);
    return 0;
}

int fwo_resample_field(const fwo_grid* src_grid, const double* field, const fwo_grid* grid,
                       double* out) {
    Grid s, d;
    if (!make_grid(src_grid, s) || !make_grid(grid, d)) return -1;
    resample_field(s, field, d, out);
    return 0;
}

int fwo_smooth_recursive(const fwo_grid* grid, const double* img, const double sigma_mm[3],
                         double* out) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    return smooth_recursive(g, img, sigma_mm, out);
}

int fwo_mt19937(uint32_t seed, int64_t n, uint32_t* out) {
    Mt mt(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = mt.integer();
    return 0;
}

// sampling.rs:181-238 -- REGULAR sampling: every ceil(1/percentage)-th voxel, jittered by
// N(0,1) * spacing / 3 per axis (two integer draws per normal variate, x first).
int64_t fwo_sample_points_regular(const fwo_grid* grid, float percentage, uint32_t seed,
                                  double* out, int64_t cap) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    Mt mt(seed);
    int64_t stride = (int64_t)std::max(std::ceil(1.0 / (double)percentage), 1.0);
    int64_t total = g.count();
    int64_t picks = (total + stride - 1) / stride;
    if (!out) return picks;
    for (int64_t q = 0; q < picks && q < cap; ++q) {
        uint32_t d[6];
        for (int k = 0; k < 6; ++k) d[k] = mt.integer();
        int64_t flat = q * stride;
        double c[3] = {(double)(flat % g.n[0]), (double)((flat / g.n[0]) % g.n[1]),
                       (double)(flat / (g.n[0] * g.n[1]))};
        double p[3];
        g.index_to_point(c, p);
        for (int a = 0; a < 3; ++a) p[a] += normal_from(d[2 * a], d[2 * a + 1]) * (g.sp[a] / 3.0);
        out[3 * q] = p[0];
        out[3 * q + 1] = p[1];
        out[3 * q + 2] = p[2];
    }
    return picks;
}

double fwo_bspline3(double u) { return bspline3(u); }
double fwo_bspline3_derivative(double u) { return bspline3_derivative(u); }

// metric/mi.rs:229-262
int fwo_mi_binning_from_ranges(int32_t bins, double fmin, double fmax, double mmin, double mmax,
                               fwo_mi_binning* out) {
    if (bins <= 4) return fail("at least five histogram bins are required");
    if (fmax - fmin <= DBL_EPSILON) return fail("the fixed image is constant");
    if (mmax - mmin <= DBL_EPSILON) return fail("the moving image is constant");
    double span = (double)(bins - 4);
    out->bins = bins;
    out->fixed_min = fmin;
    out->fixed_max = fmax;
    out->moving_min = mmin;
    out->moving_max = mmax;
    out->fixed_bin_size = (fmax - fmin) / span;
    out->moving_bin_size = (mmax - mmin) / span;
    out->fixed_normalized_min = fmin / out->fixed_bin_size - 2.0;
    out->moving_normalized_min = mmin / out->moving_bin_size - 2.0;
    return 0;
}

// linear.rs:251-279 with MiBinning::new (metric/mi.rs:199-227): fixed range over the samples'
// nearest voxels, moving range over the whole moving image, fixed bin of each kept sample.
int fwo_prepare_samples(const fwo_grid* fgrid, const double* fixed, const fwo_grid* mgrid,
                        const double* moving, const double* points, int64_t n, int32_t bins,
                        double* kept_points, uint32_t* fixed_bin, int64_t* kept,
                        fwo_mi_binning* binning) {
    Grid fg, mg;
    if (!make_grid(fgrid, fg) || !make_grid(mgrid, mg)) return -1;
    if (bins <= 4) return fail("at least five histogram bins are required");
    bool have = false;
    double fmin = 0, fmax = 0;
    for (int64_t i = 0; i < n; ++i) {
        double c[3];
        fg.point_to_index(points + 3 * i, c);
        int64_t q[3] = {0, 0, 0};
        bool ok = true;
        for (int a = 0; a < 3; ++a) {
            double r = std::floor(c[a] + 0.5);
            if (r < 0.0 || r >= (double)fg.n[a]) ok = false;
            else q[a] = (int64_t)r;
        }
        if (!ok) continue;
        double v = fixed[fg.lin(q[0], q[1], q[2])];
        if (!std::isfinite(v)) continue;
        if (!have) {
            fmin = fmax = v;
            have = true;
        } else {
            fmin = std::min(fmin, v);
            fmax = std::max(fmax, v);
        }
    }
    if (!have) return fail("no fixed-image samples were observed");
    if (fmax - fmin <= DBL_EPSILON) return fail("the fixed image is constant over the samples");
    bool mh = false;
    double mmin = 0, mmax = 0;
    for (int64_t i = 0; i < mg.count(); ++i) {
        double v = moving[i];
        if (!std::isfinite(v)) continue;
        if (!mh) {
            mmin = mmax = v;
            mh = true;
        } else {
            mmin = std::min(mmin, v);
            mmax = std::max(mmax, v);
        }
    }
    if (!mh) return fail("the moving image has no finite voxel");
    if (fwo_mi_binning_from_ranges(bins, fmin, fmax, mmin, mmax, binning)) return -1;
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
        double v;
        if (!linear_at_point(fg, fixed, points + 3 * i, v) || !std::isfinite(v)) continue;
        kept_points[3 * k] = points[3 * i];
        kept_points[3 * k + 1] = points[3 * i + 1];
        kept_points[3 * k + 2] = points[3 * i + 2];
        fixed_bin[k] = (uint32_t)clamp_bin(*binning, v / binning->fixed_bin_size -
                                                         binning->fixed_normalized_min);
        ++k;
    }
    *kept = k;
    return 0;
}

int fwo_linear_map(const fwo_linear_transform* t, fwo_affine* out) {
    linear_map(t, out);
    return 0;
}

int fwo_linear_jacobian(const fwo_linear_transform* t, const double p[3], double* cols) {
    return linear_jacobian(t, p, cols);
}

// metric/mi.rs:364-511 (accumulate + evaluate) and :702-768 (finish_histogram).
int fwo_mi_evaluate(const fwo_mi_binning* binning, const fwo_grid* mgrid, const double* moving,
                    const double* points, const uint32_t* fixed_bin, int64_t n,
                    const fwo_linear_transform* t, int32_t want_derivative, double* value,
                    double* derivative, int64_t* num_valid_out, double* joint_pdf) {
    Grid mg;
    if (!make_grid(mgrid, mg)) return -1;
    const fwo_mi_binning& b = *binning;
    const int bins = b.bins;
    int params = t->kind == 0 ? 6 : 12;
    fwo_affine map;
    linear_map(t, &map);
    const int64_t SAMPLE_CHUNK = 8192;
    int64_t chunks = (n + SAMPLE_CHUNK - 1) / SAMPLE_CHUNK;
    std::vector<std::vector<double>> pj(chunks), pf(chunks), pd(chunks);
    std::vector<int64_t> pv(chunks, 0);
#pragma omp parallel for schedule(dynamic)
    for (int64_t c = 0; c < chunks; ++c) {
        std::vector<double> joint(bins * bins, 0.0), fm(bins, 0.0);
        std::vector<double> dpdf(want_derivative ? bins * bins * params : 0, 0.0);
        int64_t valid = 0;
        double cols[36];
        int64_t hi = std::min(n, (c + 1) * SAMPLE_CHUNK);
        for (int64_t i = c * SAMPLE_CHUNK; i < hi; ++i) {
            int f_index = (int)fixed_bin[i];
            const double* s = points + 3 * i;
            double mp[3];
            apply_affine(&map, s, mp);
            double mv;
            if (!linear_at_point(mg, moving, mp, mv)) continue;
            if (!std::isfinite(mv) || mv < b.moving_min || mv > b.moving_max) continue;
            double term = mv / b.moving_bin_size - b.moving_normalized_min;
            int m_index = clamp_bin(b, term);
            fm[f_index] += 1.0;
            double grad[3] = {0, 0, 0};
            int ncols = 0;
            if (want_derivative) {
                central_difference(mg, moving, mp, grad);
                ncols = linear_jacobian(t, s, cols);
                if (!(std::isfinite(grad[0]) && std::isfinite(grad[1]) && std::isfinite(grad[2])))
                    grad[0] = grad[1] = grad[2] = 0.0;
            }
            for (int pm = m_index - 1; pm <= m_index + 2; ++pm) {
                double arg = (double)pm - term;
                int cell = f_index * bins + pm;
                joint[cell] += bspline3(arg);
                if (want_derivative) {
                    double db = bspline3_derivative(arg);
                    for (int mu = 0; mu < ncols; ++mu) {
                        double inner = cols[3 * mu] * grad[0] + cols[3 * mu + 1] * grad[1] +
                                       cols[3 * mu + 2] * grad[2];
                        dpdf[cell * params + mu] += inner * db;
                    }
                }
            }
            ++valid;
        }
        pj[c] = std::move(joint);
        pf[c] = std::move(fm);
        pd[c] = std::move(dpdf);
        pv[c] = valid;
    }
    std::vector<double> joint(bins * bins, 0.0), fmarg(bins, 0.0);
    std::vector<double> dpdf(want_derivative ? bins * bins * params : 0, 0.0);
    int64_t num_valid = 0;
    for (int64_t c = 0; c < chunks; ++c) {
        for (int i = 0; i < bins * bins; ++i) joint[i] += pj[c][i];
        for (int i = 0; i < bins; ++i) fmarg[i] += pf[c][i];
        for (size_t i = 0; i < dpdf.size(); ++i) dpdf[i] += pd[c][i];
        num_valid += pv[c];
    }
    if (num_valid == 0) return fail("all samples map outside the moving image buffer");
    Kahan ks;
    for (double v : joint) ks.add(v);
    if (ks.sum < DBL_EPSILON) return fail("joint PDF summed to zero");
    double norm = 1.0 / ks.sum;
    for (double& v : joint) v *= norm;
    for (double& v : fmarg) v *= norm;
    std::vector<double> mmarg(bins, 0.0);
    for (int col = 0; col < bins; ++col)
        for (int row = 0; row < bins; ++row) mmarg[col] += joint[row * bins + col];
    double n_factor = -1.0 / (b.moving_bin_size * (double)num_valid);
    std::vector<double> ratio(bins * bins, 0.0);
    double sum = 0.0;
    for (int f = 0; f < bins; ++f) {
        double fmv = fmarg[f];
        if (fmv <= DBL_EPSILON) continue;
        double log_fm = std::log(fmv);
        for (int m = 0; m < bins; ++m) {
            double mm = mmarg[m], jv = joint[f * bins + m];
            if (mm > DBL_EPSILON && jv > DBL_EPSILON) {
                double pr = std::log(jv / mm);
                sum += jv * (pr - log_fm);
                ratio[f * bins + m] = n_factor * pr;
            }
        }
    }
    *value = -sum;
    if (want_derivative && derivative) {
        for (int mu = 0; mu < params; ++mu) derivative[mu] = 0.0;
        for (int cell = 0; cell < bins * bins; ++cell) {
            if (ratio[cell] == 0.0) continue;
            for (int mu = 0; mu < params; ++mu) derivative[mu] += dpdf[cell * params + mu] * ratio[cell];
        }
    }
    if (num_valid_out) *num_valid_out = num_valid;
    if (joint_pdf) std::memcpy(joint_pdf, joint.data(), sizeof(double) * bins * bins);
    return 0;
}

// metric/mi.rs:553-680 -- MattesMi::evaluate_dense on the fixed grid as the virtual domain, the
// moving point p + u(p) of a displacement field given per virtual voxel (the fixtures' field on
// the fixed grid), masks looked up at the nearest voxel (metric/mi.rs:149-151). Binning:
// MiBinning::dense (metric/mi.rs:270-290), ranges over the voxels inside each image's mask.
int fwo_mi_dense(const fwo_grid* fgrid, const double* fixed, const fwo_grid* mgrid,
                 const double* moving, const double* field, const fwo_grid* fmask_grid,
                 const double* fmask, const fwo_grid* mmask_grid, const double* mmask,
                 int32_t bins, double* value, int64_t* num_valid_out, double* derivative) {
    Grid fg, mg, fmg, mmg;
    if (!make_grid(fgrid, fg) || !make_grid(mgrid, mg)) return -1;
    if (fmask && !make_grid(fmask_grid, fmg)) return -1;
    if (mmask && !make_grid(mmask_grid, mmg)) return -1;
    auto inside_mask = [](const Grid& g, const double* m, const double p[3]) {
        int64_t v;
        return nearest_voxel(g, p, v) && m[v] != 0.0;
    };
    auto range = [&](const Grid& g, const double* img, const Grid* mgp, const double* m,
                     double& lo, double& hi) {
        bool have = false;
        for (int64_t l = 0; l < g.count(); ++l) {
            if (m) {
                double p[3];
                g.voxel_point(l, p);
                if (!inside_mask(*mgp, m, p)) continue;
            }
            double v = img[l];
            if (!std::isfinite(v)) continue;
            if (!have) {
                lo = hi = v;
                have = true;
            } else {
                lo = std::min(lo, v);
                hi = std::max(hi, v);
            }
        }
        return have;
    };
    double fmin = 0, fmax = 0, mmin = 0, mmax = 0;
    if (!range(fg, fixed, &fmg, fmask, fmin, fmax))
        return fail(fmask ? "no finite fixed-image voxel lies inside the fixed mask"
                          : "the fixed image has no finite voxel");
    if (!range(mg, moving, &mmg, mmask, mmin, mmax))
        return fail(mmask ? "no finite moving-image voxel lies inside the moving mask"
                          : "the moving image has no finite voxel");
    fwo_mi_binning b;
    if (fwo_mi_binning_from_ranges(bins, fmin, fmax, mmin, mmax, &b)) return -1;
    const int64_t n = fg.count();
    struct Pt {
        bool ok;
        int fbin, mbin;
        double term;
        double grad[3];
    };
    std::vector<Pt> pts(n);
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < n; ++l) {
        Pt& q = pts[l];
        q.ok = false;
        double p[3];
        fg.voxel_point(l, p);
        if (fmask && !inside_mask(fmg, fmask, p)) continue;
        double fv, mv;
        if (!linear_at_point(fg, fixed, p, fv)) continue;
        double mp[3] = {p[0] + field[3 * l], p[1] + field[3 * l + 1], p[2] + field[3 * l + 2]};
        if (mmask && !inside_mask(mmg, mmask, mp)) continue;
        if (!linear_at_point(mg, moving, mp, mv)) continue;
        if (!std::isfinite(fv) || !std::isfinite(mv) || mv < b.moving_min || mv > b.moving_max)
            continue;
        q.term = mv / b.moving_bin_size - b.moving_normalized_min;
        central_difference(mg, moving, mp, q.grad);
        if (!(std::isfinite(q.grad[0]) && std::isfinite(q.grad[1]) && std::isfinite(q.grad[2])))
            q.grad[0] = q.grad[1] = q.grad[2] = 0.0;
        q.fbin = clamp_bin(b, fv / b.fixed_bin_size - b.fixed_normalized_min);
        q.mbin = clamp_bin(b, q.term);
        q.ok = true;
    }
    const int64_t CH = 8192;
    std::vector<double> joint(bins * bins, 0.0), fmarg(bins, 0.0);
    int64_t num_valid = 0;
    for (int64_t c0 = 0; c0 < n; c0 += CH) {
        std::vector<double> pj(bins * bins, 0.0), pf(bins, 0.0);
        int64_t pv = 0;
        for (int64_t l = c0; l < std::min(n, c0 + CH); ++l) {
            const Pt& q = pts[l];
            if (!q.ok) continue;
            pf[q.fbin] += 1.0;
            for (int pm = q.mbin - 1; pm <= q.mbin + 2; ++pm)
                pj[q.fbin * bins + pm] += bspline3((double)pm - q.term);
            ++pv;
        }
        for (int i = 0; i < bins * bins; ++i) joint[i] += pj[i];
        for (int i = 0; i < bins; ++i) fmarg[i] += pf[i];
        num_valid += pv;
    }
    if (num_valid == 0 && (fmask || mmask))
        return fail("no voxel of the registration level lies inside both the fixed and the moving mask");
    if (num_valid == 0) return fail("all samples map outside the moving image buffer");
    Kahan ks;
    for (double v : joint) ks.add(v);
    if (ks.sum < DBL_EPSILON) return fail("joint PDF summed to zero");
    double norm = 1.0 / ks.sum;
    for (double& v : joint) v *= norm;
    for (double& v : fmarg) v *= norm;
    std::vector<double> mmarg(bins, 0.0);
    for (int col = 0; col < bins; ++col)
        for (int row = 0; row < bins; ++row) mmarg[col] += joint[row * bins + col];
    double n_factor = -1.0 / (b.moving_bin_size * (double)num_valid);
    std::vector<double> ratio(bins * bins, 0.0);
    double sum = 0.0;
    for (int f = 0; f < bins; ++f) {
        double fmv = fmarg[f];
        if (fmv <= DBL_EPSILON) continue;
        double log_fm = std::log(fmv);
        for (int m = 0; m < bins; ++m) {
            double mm = mmarg[m], jv = joint[f * bins + m];
            if (mm > DBL_EPSILON && jv > DBL_EPSILON) {
                double pr = std::log(jv / mm);
                sum += jv * (pr - log_fm);
                ratio[f * bins + m] = n_factor * pr;
            }
        }
    }
    *value = -sum;
    if (num_valid_out) *num_valid_out = num_valid;
    if (derivative) {
#pragma omp parallel for schedule(static)
        for (int64_t l = 0; l < n; ++l) {
            const Pt& q = pts[l];
            double s = 0.0;
            if (q.ok)
                for (int pm = q.mbin - 1; pm <= q.mbin + 2; ++pm)
                    s += bspline3_derivative((double)pm - q.term) * ratio[q.fbin * bins + pm];
            for (int k = 0; k < 3; ++k) derivative[3 * l + k] = q.ok ? s * q.grad[k] : 0.0;
        }
    }
    return 0;
}

// convergence.rs:91-126 -- the closed-form two-control-point B-spline fit.
double fwo_convergence_value(const double* values, int64_t n, int32_t window, double total) {
    if (n < window) return DBL_MAX;
    if (window < 2) return 0.0;
    const double spline_eps = 1e-3, domain_spacing = 0.1, domain_size = 11.0;
    double r = 1.0 / ((domain_size - 1.0) * domain_spacing);
    double epsilon = r * domain_spacing * spline_eps;
    double delta[2] = {0, 0}, omega[2] = {0, 0};
    for (int64_t k = 0; k < n; ++k) {
        double p = ((double)k / (double)(window - 1)) * r;
        if (std::fabs(p - 1.0) <= epsilon) p = 1.0 - epsilon;
        if (p < 0.0 && std::fabs(p) <= epsilon) p = 0.0;
        double t = p - std::floor(p);
        double w[2] = {1.0 - t, t};
        double w2 = w[0] * w[0] + w[1] * w[1];
        double v = values[k] / total;
        for (int j = 0; j < 2; ++j) {
            omega[j] += w[j] * w[j];
            delta[j] += v * (w[j] * w[j] * w[j] / w2);
        }
    }
    double phi[2] = {0, 0};
    for (int j = 0; j < 2; ++j) {
        if (std::fabs(omega[j]) > DBL_EPSILON) {
            double q = delta[j] / omega[j];
            phi[j] = std::isfinite(q) ? q : 0.0;
        }
    }
    return phi[0] - phi[1];
}

int fwo_syn_level_grid(const fwo_syn_recipe* r, const fwo_grid* fixed_grid, int32_t level,
                       fwo_grid* out) {
    Grid g, o;
    if (!make_grid(fixed_grid, g)) return -1;
    if (level < 0 || level >= r->levels) return fail("bad level");
    uint32_t f[3];
    shrink_factors(r->shrink_factors[level], g.sp, f);
    if (!shrink_grid(g, f, o)) return -1;
    *out = to_c(o);
    return 0;
}

}  // extern "C"

namespace {

// syn.rs:337-420 (side_updates) + 422-445 (update_total_field) + 890-958 (one iteration).
// With masks, syn.rs:555-580 (StageMasks::validity): the fixed mask resampled (nearest voxel)
// through F^-1, times the moving mask through affine(M^-1); the CC pair takes only those voxels.
int syn_iteration(const fwo_syn_recipe* r, const Grid& lg, const Grid& fg,
                  const double* const* fixed_s, const Grid& mg, const double* const* moving_s,
                  const fwo_affine* initial, const fwo_syn_masks* masks, double* f2m,
                  double* f2m_inv, double* m2m, double* m2m_inv, double* fixed_update_out,
                  double* moving_update_out, fwo_syn_iteration* rec,
                  const fwo_grid* prior_grid = nullptr, const double* prior = nullptr) {
    int64_t n = lg.count();
    int channels = r->channels;
    double wsum = 0.0;
    for (int c = 0; c < channels; ++c) wsum += r->channel_weights[c];
    std::vector<double> fmid(n), mmid(n);
    std::vector<double> dF(3 * n), dM(3 * n);
    std::vector<double> gF, gM;  // multichannel accumulators
    double totF = 0.0, totM = 0.0;
    std::vector<double> valsF, valsM;
    fwo_grid lgc = to_c(lg), fgc = to_c(fg), mgc = to_c(mg);
    // syn.rs:496-580: each given mask resolved on the level grid (the fixed one through F^-1, the
    // moving one through affine(M^-1)); CC takes the voxels inside both, Mattes each on its own
    std::vector<double> valid, fvalid, mvalid;
    const bool has_fm = masks && masks->fixed, has_mm = masks && masks->moving;
    if (has_fm) {
        fvalid.resize(n);
        if (fwo_warp_mask(masks->fixed_grid, masks->fixed, &lgc, f2m_inv, nullptr, nullptr,
                          nullptr, nullptr, fvalid.data()))
            return -1;
    }
    if (has_mm) {
        mvalid.resize(n);
        if (fwo_warp_mask(masks->moving_grid, masks->moving, &lgc, m2m_inv, prior_grid, prior,
                          initial, nullptr, mvalid.data()))
            return -1;
    }
    if (has_fm || has_mm) {
        valid.resize(n);
        for (int64_t l = 0; l < n; ++l)
            valid[l] = (has_fm ? fvalid[l] : 1.0) * (has_mm ? mvalid[l] : 1.0);
    }
    std::vector<double> zero;
    for (int c = 0; c < channels; ++c) {
        if (fwo_warp(&fgc, fixed_s[c], &lgc, f2m_inv, nullptr, nullptr, nullptr, fmid.data()))
            return -1;
        if (fwo_warp(&mgc, moving_s[c], &lgc, m2m_inv, prior_grid, prior, initial, mmid.data()))
            return -1;
        double vals[2];
        if (r->channel_metrics[c] == 1) {
            // cpu/mod.rs:352-381 (mi_pair): evaluate_dense (fixed, moving) then (moving, fixed)
            if (zero.empty()) zero.assign(3 * n, 0.0);
            const fwo_grid* fmg = has_fm ? &lgc : nullptr;
            const fwo_grid* mmg = has_mm ? &lgc : nullptr;
            const double* fm = has_fm ? fvalid.data() : nullptr;
            const double* mm = has_mm ? mvalid.data() : nullptr;
            int64_t nv = 0;
            if (fwo_mi_dense(&lgc, fmid.data(), &lgc, mmid.data(), zero.data(), fmg, fm, mmg, mm,
                             r->mi_bins, &vals[0], &nv, dF.data()))
                return -1;
            if (fwo_mi_dense(&lgc, mmid.data(), &lgc, fmid.data(), zero.data(), mmg, mm, fmg, fm,
                             r->mi_bins, &vals[1], &nv, dM.data()))
                return -1;
        } else if (fwo_cc_pair(&lgc, fmid.data(), mmid.data(),
                               valid.empty() ? nullptr : valid.data(), r->cc_radius, vals,
                               dF.data(), dM.data())) {
            return -1;
        }
        valsF.push_back(vals[0]);
        valsM.push_back(vals[1]);
        if (channels == 1) {
            gF = dF;
            gM = dM;
        } else {
            double normF = l2_norm(lg, dF.data()), normM = l2_norm(lg, dM.data());
            if (gF.empty()) {
                gF.assign(3 * n, 0.0);
                gM.assign(3 * n, 0.0);
            }
            double wn = r->channel_weights[c] / wsum;
            if (!std::isfinite(normF) || !std::isfinite(normM))
                return fail("the metric gradient is not finite");
            totF += normF;
            totM += normM;
            if (normF > DBL_EPSILON) fwo_axpy(&lgc, gF.data(), wn / normF, dF.data());
            if (normM > DBL_EPSILON) fwo_axpy(&lgc, gM.data(), wn / normM, dM.data());
        }
    }
    double weightedF = valsF[0], weightedM = valsM[0];
    if (channels > 1) {
        fwo_scale(&lgc, gF.data(), totF / channels);
        fwo_scale(&lgc, gM.data(), totM / channels);
        weightedF = weightedM = 0.0;
        for (int c = 0; c < channels; ++c) {
            weightedF += valsF[c] * r->channel_weights[c] / wsum;
            weightedM += valsM[c] * r->channel_weights[c] / wsum;
        }
    }
    std::vector<double> sF(3 * n), sM(3 * n);
    smooth_field(lg, gF.data(), r->update_field_variance, sF.data());
    smooth_field(lg, gM.data(), r->update_field_variance, sM.data());
    double maxF = max_scaled_norm(lg, sF.data()), maxM = max_scaled_norm(lg, sM.data());
    if (!(std::isfinite(maxF) && std::isfinite(maxM))) return fail("the metric gradient is not finite");
    double scaleF = r->gradient_step, scaleM = r->gradient_step;
    if (maxF > 0.0) scaleF /= maxF;
    if (maxM > 0.0) scaleM /= maxM;
    fwo_scale(&lgc, sF.data(), scaleF);
    fwo_scale(&lgc, sM.data(), scaleM);
    if (fixed_update_out) std::memcpy(fixed_update_out, sF.data(), sizeof(double) * 3 * n);
    if (moving_update_out) std::memcpy(moving_update_out, sM.data(), sizeof(double) * 3 * n);
    const fwo_invert_params SYN = {20, 0.001, 0.1, 1};
    fwo_invert_stats st[4];
    double* fields[2][2] = {{f2m, f2m_inv}, {m2m, m2m_inv}};
    std::vector<double>* upd[2] = {&sF, &sM};
    for (int side = 0; side < 2; ++side) {
        double* field = fields[side][0];
        double* inverse = fields[side][1];
        std::vector<double> composed(3 * n), tmp(3 * n);
        compose(lg, upd[side]->data(), field, composed.data());
        smooth_field(lg, composed.data(), r->total_field_variance, tmp.data());
        // invert_pair: inverse = invert(tmp, init = inverse); field = invert(inverse, init = tmp)
        invert(lg, tmp.data(), inverse, SYN, st[2 * side]);
        std::memcpy(field, tmp.data(), sizeof(double) * 3 * n);
        invert(lg, inverse, field, SYN, st[2 * side + 1]);
        for (int k = 0; k < 2; ++k) {
            const fwo_invert_stats& s = st[2 * side + k];
            if (!(std::isfinite(s.mean_error_norm) && std::isfinite(s.max_error_norm)))
                return fail("the displacement field is not finite");
        }
    }
    rec->energy = 0.5 * (valsF[0] + valsM[0]);
    rec->energy_weighted = 0.5 * (weightedF + weightedM);
    rec->fixed_update_scale = scaleF;
    rec->moving_update_scale = scaleM;
    for (int k = 0; k < 4; ++k) rec->inversions[k] = st[k];
    return 0;
}

}  // namespace

extern "C" {

int fwo_syn_step(const fwo_syn_recipe* r, const fwo_grid* level_grid,
                 const fwo_grid* fixed_grid, const double* const* fixed_smooth,
                 const fwo_grid* moving_grid, const double* const* moving_smooth,
                 const fwo_affine* initial, double* f2m, double* f2m_inv, double* m2m,
                 double* m2m_inv, double* fixed_update, double* moving_update,
                 fwo_syn_iteration* record) {
    return fwo_syn_step_masked(r, level_grid, fixed_grid, fixed_smooth, moving_grid,
                               moving_smooth, initial, nullptr, f2m, f2m_inv, m2m, m2m_inv,
                               fixed_update, moving_update, record);
}

int fwo_syn_step_masked(const fwo_syn_recipe* r, const fwo_grid* level_grid,
                        const fwo_grid* fixed_grid, const double* const* fixed_smooth,
                        const fwo_grid* moving_grid, const double* const* moving_smooth,
                        const fwo_affine* initial, const fwo_syn_masks* masks, double* f2m,
                        double* f2m_inv, double* m2m, double* m2m_inv, double* fixed_update,
                        double* moving_update, fwo_syn_iteration* record) {
    Grid lg, fg, mg;
    if (!make_grid(level_grid, lg) || !make_grid(fixed_grid, fg) || !make_grid(moving_grid, mg))
        return -1;
    fwo_syn_iteration rec{};
    int rc = syn_iteration(r, lg, fg, fixed_smooth, mg, moving_smooth, initial, masks, f2m,
                           f2m_inv, m2m, m2m_inv, fixed_update, moving_update, &rec);
    rec.convergence_value = DBL_MAX;
    if (record) *record = rec;
    return rc;
}

// syn.rs:776-986 -- syn_fields for a first SyN stage (no prior field).
int fwo_syn_run(const fwo_syn_recipe* r, const fwo_grid* fixed_grid, const double* const* fixed,
                const fwo_grid* moving_grid, const double* const* moving,
                const fwo_affine* initial, double* warp, double* inverse_warp,
                fwo_syn_iteration* records, int64_t cap, int64_t* count) {
    return fwo_syn_run_masked(r, fixed_grid, fixed, moving_grid, moving, initial, nullptr, warp,
                              inverse_warp, records, cap, count);
}

int fwo_syn_run_masked(const fwo_syn_recipe* r, const fwo_grid* fixed_grid,
                       const double* const* fixed, const fwo_grid* moving_grid,
                       const double* const* moving, const fwo_affine* initial,
                       const fwo_syn_masks* masks, double* warp, double* inverse_warp,
                       fwo_syn_iteration* records, int64_t cap, int64_t* count) {
    return fwo_syn_run_from(r, fixed_grid, fixed, moving_grid, moving, initial, masks, nullptr,
                            nullptr, nullptr, warp, inverse_warp, records, cap, count);
}

// syn.rs:620-660, 776-986 -- syn_fields from a SynStart: after earlier SyN stages their collapsed
// field (on the grid of this stage's last level) enters every moving-side warp, and the result is
// collapsed with it (syn.rs:761-774, 971-977).
int fwo_syn_run_from(const fwo_syn_recipe* r, const fwo_grid* fixed_grid,
                     const double* const* fixed, const fwo_grid* moving_grid,
                     const double* const* moving, const fwo_affine* initial,
                     const fwo_syn_masks* masks, const fwo_grid* prior_grid, const double* prior,
                     const double* prior_inverse, double* warp, double* inverse_warp,
                     fwo_syn_iteration* records, int64_t cap, int64_t* count) {
    Grid fg, mg;
    if (!make_grid(fixed_grid, fg) || !make_grid(moving_grid, mg)) return -1;
    if (r->levels <= 0 || r->levels > FWO_MAX_LEVELS) return fail("bad level count");
    if (r->channels <= 0 || r->channels > FWO_MAX_CHANNELS) return fail("bad channel count");
    if (!prior != !prior_inverse) return fail("syn: the prior needs both the warp and its inverse");
    if (prior) {
        uint32_t factors[3];
        shrink_factors(r->shrink_factors[r->levels - 1], fg.sp, factors);
        Grid last, pg;
        if (!shrink_grid(fg, factors, last) || !make_grid(prior_grid, pg)) return -1;
        bool same = true;
        for (int a = 0; a < 3; ++a)
            same = same && pg.n[a] == last.n[a] && pg.sp[a] == last.sp[a] && pg.org[a] == last.org[a];
        for (int k = 0; k < 9; ++k) same = same && pg.dir[k] == last.dir[k];
        if (!same)
            return fail("syn: the field of the earlier SyN stages is not on the grid of this "
                        "stage's last level: every SyN stage must end with the same shrink factor");
    }
    // recipe.rs:239-246: a given mask must have a voxel inside
    if (masks) {
        const fwo_grid* mgs[2] = {masks->fixed_grid, masks->moving_grid};
        const double* mds[2] = {masks->fixed, masks->moving};
        const char* names[2] = {"fixed", "moving"};
        for (int q = 0; q < 2; ++q) {
            if (!mds[q]) continue;
            Grid m;
            if (!make_grid(mgs[q], m)) return -1;
            bool any = false;
            for (int64_t l = 0; l < m.count() && !any; ++l) any = mds[q][l] != 0.0;
            if (!any)
                return fail(std::string("syn recipe: the ") + names[q] +
                            " mask has no voxel inside (every voxel is zero)");
        }
    }
    int channels = r->channels;
    std::vector<std::vector<double>> fs(channels), ms(channels);
    std::vector<double> f2m, f2m_inv, m2m, m2m_inv;
    Grid prev;
    bool have_prev = false;
    int64_t nrec = 0;
    for (int level = 0; level < r->levels; ++level) {
        uint32_t factors[3];
        shrink_factors(r->shrink_factors[level], fg.sp, factors);
        Grid lg;
        if (!shrink_grid(fg, factors, lg)) return -1;
        double sigma = r->smoothing_sigmas[level];
        std::vector<const double*> fptr(channels), mptr(channels);
        for (int c = 0; c < channels; ++c) {
            if (sigma > 0.0) {
                double sf[3], sm[3];
                for (int a = 0; a < 3; ++a) {
                    sf[a] = r->sigma_units_mm ? sigma : sigma * fg.sp[a];
                    sm[a] = r->sigma_units_mm ? sigma : sigma * mg.sp[a];
                }
                fs[c].resize(fg.count());
                ms[c].resize(mg.count());
                if (smooth_recursive(fg, fixed[c], sf, fs[c].data())) return -1;
                if (smooth_recursive(mg, moving[c], sm, ms[c].data())) return -1;
                fptr[c] = fs[c].data();
                mptr[c] = ms[c].data();
            } else {
                fptr[c] = fixed[c];
                mptr[c] = moving[c];
            }
        }
        int64_t n = lg.count();
        if (!have_prev) {
            f2m.assign(3 * n, 0.0);
            f2m_inv.assign(3 * n, 0.0);
            m2m.assign(3 * n, 0.0);
            m2m_inv.assign(3 * n, 0.0);
        } else {
            std::vector<double>* st[4] = {&f2m, &f2m_inv, &m2m, &m2m_inv};
            for (auto* v : st) {
                std::vector<double> nv(3 * n);
                resample_field(prev, v->data(), lg, nv.data());
                *v = std::move(nv);
            }
        }
        prev = lg;
        have_prev = true;
        Monitor monitor(r->convergence_window);
        bool converged = false;
        uint32_t current = 0;
        while (current < r->iterations[level] && !converged) {
            ++current;
            fwo_syn_iteration rec{};
            if (syn_iteration(r, lg, fg, fptr.data(), mg, mptr.data(), initial, masks, f2m.data(),
                              f2m_inv.data(), m2m.data(), m2m_inv.data(), nullptr, nullptr, &rec,
                              prior_grid, prior))
                return -1;
            monitor.add(rec.energy);
            rec.convergence_value = monitor.value();
            rec.level = level;
            if (rec.convergence_value < r->convergence_threshold) converged = true;
            if (records && nrec < cap) records[nrec] = rec;
            ++nrec;
        }
    }
    // syn.rs:969-970
    compose(prev, m2m_inv.data(), f2m.data(), warp);
    compose(prev, f2m_inv.data(), m2m.data(), inverse_warp);
    if (prior) {
        // syn.rs:761-774 (collapse): total = compose(P, W), total^-1 = compose(Winv, Pinv)
        const int64_t n3 = 3 * prev.count();
        std::vector<double> later(warp, warp + n3), later_inv(inverse_warp, inverse_warp + n3);
        compose(prev, prior, later.data(), warp);
        compose(prev, later_inv.data(), prior_inverse, inverse_warp);
    }
    if (count) *count = nrec;
    return 0;
}

}  // extern "C"

// ---- the linear-stage optimiser, crates/fastwarp-reg/src/optimizer.rs:142-435 -------------------

namespace {

int opt_nparams(const fwo_linear_transform& t) { return t.kind == 0 ? 6 : 12; }

void opt_apply(const fwo_linear_transform& t, const double* p, double* out) {
    fwo_affine a;
    linear_map(&t, &a);
    for (int r = 0; r < 3; ++r)
        out[r] = a.matrix[r * 3] * p[0] + a.matrix[r * 3 + 1] * p[1] + a.matrix[r * 3 + 2] * p[2] +
                 a.offset[r];
}

// optimizer.rs:168-183: the largest corner displacement caused by adding `delta`.
double opt_shift(const double* corners, const fwo_linear_transform& t, const double* delta) {
    fwo_linear_transform m = t;
    for (int i = 0; i < opt_nparams(t); ++i) m.parameters[i] += delta[i];
    double best = 0.0;
    for (int c = 0; c < 8; ++c) {
        double a[3], b[3];
        opt_apply(m, corners + 3 * c, a);
        opt_apply(t, corners + 3 * c, b);
        double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        best = std::max(best, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    return best;
}

}  // namespace

extern "C" {

// optimizer.rs:185-216
int fwo_estimate_scales(const double* corners, const fwo_linear_transform* t, double small,
                        double* scales) {
    const int n = opt_nparams(*t);
    double lo = DBL_MAX;
    for (int i = 0; i < n; ++i) {
        double d[12] = {0};
        d[i] = small;
        scales[i] = opt_shift(corners, *t, d);
        if (scales[i] > DBL_EPSILON && scales[i] < lo) lo = scales[i];
    }
    if (lo == DBL_MAX) {
        for (int i = 0; i < n; ++i) scales[i] = 1.0;
        return 0;
    }
    for (int i = 0; i < n; ++i) {
        scales[i] = scales[i] <= DBL_EPSILON ? lo * lo : scales[i] * scales[i];
        scales[i] *= 1.0 / (small * small);
    }
    return 0;
}

// optimizer.rs:218-231
double fwo_estimate_step_scale(const double* corners, const fwo_linear_transform* t,
                               const double* step, double small) {
    const int n = opt_nparams(*t);
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = std::max(mx, std::fabs(step[i]));
    if (mx <= DBL_EPSILON) return 0.0;
    const double f = small / mx;
    double s[12];
    for (int i = 0; i < n; ++i) s[i] = step[i] * f;
    return opt_shift(corners, *t, s) / f;
}

// optimizer.rs:236-309 (golden-section search) and :311-435 (the conjugate-gradient loop).
int fwo_cg_optimize_level(const fwo_cg_settings* st, const double* corners,
                          fwo_linear_transform* t, fwo_metric_value_fn value,
                          fwo_metric_value_derivative_fn value_derivative, void* user,
                          fwo_cg_trace* trace, double* values, int64_t cap) {
    const int n = opt_nparams(*t);
    const double resphi = 2.0 - 1.618034;
    double scales[12];
    fwo_estimate_scales(corners, t, st->small_parameter_variation, scales);
    fwo_linear_transform cur = *t, best = *t;
    double conj[12] = {0}, last[12] = {0}, g[12];
    double lr = st->max_step_mm;
    std::vector<double> window;
    double total = 0.0;
    double best_value = DBL_MAX;
    *trace = fwo_cg_trace{};
    trace->converged_value = std::numeric_limits<double>::quiet_NaN();
    for (int i = 0; i < n; ++i) trace->scales[i] = scales[i];
    trace->initial_learning_rate = lr;
    int it = 0;
    while (it < st->iterations) {
        double v;
        if (value_derivative(user, &cur, &v, g)) return fail("the metric failed");
        window.push_back(v);
        if ((int)window.size() > st->convergence_window) window.erase(window.begin());
        total += std::fabs(v);
        const double cv = fwo_convergence_value(window.data(), (int64_t)window.size(),
                                                st->convergence_window, total);
        if (cv <= st->convergence_threshold) {
            trace->converged = 1;
            trace->converged_value = v;
            break;
        }
        if (values && trace->nvalues < cap) values[trace->nvalues] = v;
        trace->nvalues++;
        for (int i = 0; i < n; ++i) g[i] *= 1.0 / scales[i];
        if (it == 0) {
            const double ss = fwo_estimate_step_scale(corners, &cur, g, st->small_parameter_variation);
            lr = ss <= DBL_EPSILON ? 1.0 : st->max_step_mm / ss;
            trace->initial_learning_rate = lr;
        }
        double gamma = 0.0, den = 0.0;
        for (int i = 0; i < n; ++i) den += last[i] * last[i];
        if (den > DBL_EPSILON) {
            double num = 0.0;
            for (int i = 0; i < n; ++i) num += (g[i] - last[i]) * g[i];
            gamma = num / den;
        }
        if (!(gamma >= 0.0 && gamma <= 5.0)) gamma = 0.0;
        for (int i = 0; i < n; ++i) {
            last[i] = g[i];
            conj[i] = g[i] + conj[i] * gamma;
        }
        // golden-section search over [lower, 1, upper] * lr
        double a = lr * st->lower_limit, b = lr, c = lr * st->upper_limit;
        double mb = DBL_MAX;
        int lsi = 0;
        auto at = [&](double step, double* out) {
            trace->line_search_evaluations++;
            fwo_linear_transform q = cur;
            for (int i = 0; i < n; ++i) q.parameters[i] = cur.parameters[i] + step * conj[i];
            return value(user, &q, out);
        };
        for (;;) {
            if (lsi > st->max_line_search_iterations) {
                lr = (c + a) / 2.0;
                break;
            }
            ++lsi;
            const double x = c - b > b - a ? b + resphi * (c - b) : b - resphi * (b - a);
            if (std::fabs(c - a) < st->epsilon * (std::fabs(b) + std::fabs(x))) {
                lr = (c + a) / 2.0;
                break;
            }
            double mx;
            if (at(x, &mx)) return fail("the metric failed");
            if (mb == DBL_MAX && at(b, &mb)) return fail("the metric failed");
            if (mx < mb) {
                if (c - b > b - a) {
                    a = b;
                    b = x;
                } else {
                    c = b;
                    b = x;
                }
                mb = mx;
            } else if (c - b > b - a) {
                c = x;
            } else if (mx == DBL_MAX) {
                c = b;
                b = x;
                mb = mx;
            } else {
                a = x;
            }
        }
        for (int i = 0; i < n; ++i) cur.parameters[i] += lr * conj[i];
        if (v < best_value) {
            best_value = v;
            best = cur;
        }
        ++it;
    }
    trace->iterations = it;
    trace->best_value = best_value;
    trace->final_learning_rate = lr;
    *t = best;
    return 0;
}

}  // extern "C"

// ---- image preparation: isotropic resampling and intensity preprocessing --------------------

namespace {

constexpr int PRE_BINS = 256;         // preprocess.rs:36
constexpr double PRE_MARGIN = 10.0;   // preprocess.rs:37 (marginal scale)

// The 256-bin histogram of the finite values (preprocess.rs:46-102): bin edges from float32
// interval arithmetic, the last bin widened by a tenth of a bin, counts per bin.
struct PreHistogram {
    double mn[PRE_BINS], mx[PRE_BINS], freq[PRE_BINS];

    bool build(const double* v, int64_t n) {
        double lo = DBL_MAX, hi = -DBL_MAX;
        int64_t finite = 0;
        for (int64_t i = 0; i < n; ++i) {
            if (!std::isfinite(v[i])) continue;
            ++finite;
            lo = std::min(lo, v[i]);
            hi = std::max(hi, v[i]);
        }
        if (finite == 0) return fail("preprocess: image has no finite values") == 0;
        const double margin = ((hi - lo) / PRE_BINS) / PRE_MARGIN;
        const double upper = hi + margin;
        const float interval = ((float)upper - (float)lo) / (float)PRE_BINS;
        for (int j = 0; j < PRE_BINS - 1; ++j) {
            mn[j] = lo + (double)((float)j * interval);
            mx[j] = lo + (double)((float)(j + 1) * interval);
        }
        mn[PRE_BINS - 1] = lo + (double)((float)(PRE_BINS - 1) * interval);
        mx[PRE_BINS - 1] = upper;
        std::vector<int64_t> counts(PRE_BINS, 0);
#pragma omp parallel
        {
            std::vector<int64_t> local(PRE_BINS, 0);
#pragma omp for schedule(static) nowait
            for (int64_t i = 0; i < n; ++i)
                if (std::isfinite(v[i])) ++local[index_of(v[i])];
#pragma omp critical
            for (int j = 0; j < PRE_BINS; ++j) counts[j] += local[j];
        }
        for (int j = 0; j < PRE_BINS; ++j) freq[j] = (double)counts[j];
        return true;
    }

    // preprocess.rs:104-113: the bin whose lower edge is the last one <= v.
    int index_of(double v) const {
        if (v < mn[0]) return 0;
        if (v >= mx[PRE_BINS - 1]) return PRE_BINS - 1;
        int lo = 0, hi = PRE_BINS;  // first j with mn[j] > v
        while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (mn[mid] <= v) lo = mid + 1;
            else hi = mid;
        }
        return lo > 0 ? lo - 1 : 0;
    }

    // preprocess.rs:115-161 (ITK Histogram::Quantile): walk the cumulative frequency from the
    // nearer end and interpolate linearly inside the bin that crosses p.
    double quantile(double p) const {
        double total = 0.0;
        for (int j = 0; j < PRE_BINS; ++j) total += freq[j];
        double cumulated = 0.0, p_prev = 0.0, f_n = 0.0;
        if (p < 0.5) {
            int n = 0;
            double p_n = 0.0;
            do {
                f_n = freq[n];
                cumulated += f_n;
                p_prev = p_n;
                p_n = cumulated / total;
                ++n;
            } while (n < PRE_BINS && p_n < p);
            const double proportion = f_n / total;
            const double lo = mn[n - 1], width = mx[n - 1] - lo;
            return lo + ((p - p_prev) / proportion) * width;
        }
        int n = PRE_BINS - 1, m = 0;
        double p_n = 1.0;
        do {
            f_n = freq[n];
            cumulated += f_n;
            p_prev = p_n;
            p_n = 1.0 - cumulated / total;
            --n;
            ++m;
        } while (m < PRE_BINS && p_n > p);
        const double proportion = f_n / total;
        const int bin = n + 1;
        const double top = mx[bin], width = top - mn[bin];
        return top - ((p_prev - p) / proportion) * width;
    }
};

// preprocess.rs:168-173: both quantiles, each rounded to float32.
bool quantile_window(const double* v, int64_t n, float lower, float upper, double out[2]) {
    PreHistogram* h = new PreHistogram;
    const bool ok = h->build(v, n);
    if (ok) {
        out[0] = (double)(float)h->quantile((double)lower);
        out[1] = (double)(float)h->quantile((double)upper);
    }
    delete h;
    return ok;
}

// register.rs:112-146: the isotropic grid (same origin and direction, mm spacing) and the
// source index every output index samples along each axis.
void isotropic_axes(const Grid& g, double mm, int64_t out_n[3], double ratio[3], double last[3]) {
    for (int a = 0; a < 3; ++a) {
        last[a] = (double)(g.n[a] - 1);
        ratio[a] = mm / g.sp[a];
        const int64_t t = (int64_t)std::floor(last[a] * g.sp[a] / mm + 1e-9) + 1;
        out_n[a] = std::max<int64_t>(t, 1);
    }
}

bool same_spacing(const Grid& g, double mm) {
    for (int a = 0; a < 3; ++a)
        if (!(std::fabs(g.sp[a] - mm) < 1e-6)) return false;
    return true;
}

// register.rs:82-108: trilinear sample at a continuous index, corners outside skipped.
double sample_linear_clamped(const double* data, const int64_t size[3], const double c[3]) {
    const double lo[3] = {std::floor(c[0]), std::floor(c[1]), std::floor(c[2])};
    const double fr[3] = {c[0] - lo[0], c[1] - lo[1], c[2] - lo[2]};
    double acc = 0.0;
    for (int corner = 0; corner < 8; ++corner) {
        int64_t idx[3];
        double w = 1.0;
        bool inside = true;
        for (int a = 0; a < 3; ++a) {
            const int bit = (corner >> a) & 1;
            const int64_t i = (int64_t)lo[a] + bit;
            if (i < 0 || i >= size[a]) {
                inside = false;
                break;
            }
            idx[a] = i;
            w *= bit ? fr[a] : 1.0 - fr[a];
        }
        if (w == 0.0 || !inside) continue;
        acc += w * data[idx[0] + size[0] * (idx[1] + size[1] * idx[2])];
    }
    return acc;
}

}  // namespace

extern "C" {

int fwo_quantile_window(const double* values, int64_t n, float lower, float upper,
                        double out[2]) {
    if (!values || !out || n < 0) return fail("null argument");
    return quantile_window(values, n, lower, upper, out) ? 0 : -1;
}

int fwo_preprocess(const double* values, int64_t n, float lower, float upper, double out_min,
                   double out_max, double* out) {
    if (!values || !out || n < 0) return fail("null argument");
    double w[2];
    if (!quantile_window(values, n, lower, upper, w)) return -1;
    const double lo = w[0], hi = w[1];
    if (!(hi > lo)) {
        char msg[160];
        std::snprintf(msg, sizeof(msg), "preprocess: degenerate intensity window [%.17g, %.17g]",
                      lo, hi);
        return fail(msg);
    }
    const double scale = (out_max - out_min) / (hi - lo);
    const double shift = out_min - lo * scale;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double x = values[i];
        out[i] = x < lo ? out_min : x > hi ? out_max : x * scale + shift;
    }
    return 0;
}

int fwo_isotropic_grid(const fwo_grid* grid, double mm, fwo_grid* out) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    if (!(std::isfinite(mm) && mm > 0.0)) return fail("isotropic spacing must be positive");
    if (same_spacing(g, mm)) {
        *out = *grid;
        return 0;
    }
    int64_t n[3];
    double ratio[3], last[3];
    isotropic_axes(g, mm, n, ratio, last);
    fwo_grid o = *grid;
    for (int a = 0; a < 3; ++a) {
        o.size[a] = n[a];
        o.spacing[a] = mm;
    }
    *out = o;
    return 0;
}

int fwo_resample_isotropic(const fwo_grid* grid, const double* img, double mm, double* out) {
    Grid g;
    if (!make_grid(grid, g)) return -1;
    if (!img || !out) return fail("null argument");
    if (!(std::isfinite(mm) && mm > 0.0)) return fail("isotropic spacing must be positive");
    if (same_spacing(g, mm)) {
        std::memcpy(out, img, sizeof(double) * g.count());
        return 0;
    }
    int64_t n[3];
    double ratio[3], last[3];
    isotropic_axes(g, mm, n, ratio, last);
    const int64_t count = n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < count; ++l) {
        const int64_t i = l % n[0], j = (l / n[0]) % n[1], k = l / (n[0] * n[1]);
        const double c[3] = {std::min((double)i * ratio[0], last[0]),
                             std::min((double)j * ratio[1], last[1]),
                             std::min((double)k * ratio[2], last[2])};
        out[l] = (double)(float)sample_linear_clamped(img, g.n, c);
    }
    return 0;
}

}  // extern "C"
