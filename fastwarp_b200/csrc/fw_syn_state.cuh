// fw_syn_state.cuh -- the device state of one SyN registration's iteration loop, shared by the
// single-registration driver (fw_syn.cu) and the batch driver (fw_batch.cu): the window
// convergence monitor (convergence.rs:47-126), the level start and the end-of-iteration record
// (syn.rs:941-958).
#pragma once

#include <cfloat>

#include "fw_internal.cuh"

namespace fw {

constexpr int MAX_WINDOW = 64;

struct SynDev {
    int done;        // iterations recorded over all levels (the trace's write position)
    int it;          // iterations done in this level
    int limit;       // iteration limit of this level
    int converged;
    int status;      // 0 ok, 1 gradient not finite, 2 field not finite, 3 cancelled,
                     // 4 no voxel inside the masks (CC), 10 + k a Mattes pair's status k
    int level;
    int window;
    int count;       // values in the window
    int head;
    double total;    // running sum of |energy| of every value added
    double values[MAX_WINDOW];
    double threshold;
    double step;
    int channels;
    int masked;      // the CC pairs take the masks' valid voxels
    double wnorm[FW_MAX_CHANNELS];
    int metric[FW_MAX_CHANNELS];  // FW_METRIC_CC or FW_METRIC_MATTES
};

// convergence.rs:91-126, the closed form of the two-control-point fit.
__device__ __forceinline__ double convergence_value(const SynDev& s) {
    if (s.count < s.window) return DBL_MAX;
    if (s.window < 2) return 0.0;
    const double spline_eps = 1e-3, domain_spacing = 0.1, domain_size = 11.0;
    double r = 1.0 / ((domain_size - 1.0) * domain_spacing);
    double epsilon = r * domain_spacing * spline_eps;
    double delta[2] = {0, 0}, omega[2] = {0, 0};
    for (int k = 0; k < s.count; ++k) {
        double e = s.values[(s.head + k) % s.window];
        double p = ((double)k / (double)(s.window - 1)) * r;
        if (fabs(p - 1.0) <= epsilon) p = 1.0 - epsilon;
        if (p < 0.0 && fabs(p) <= epsilon) p = 0.0;
        double t = p - floor(p);
        double w[2] = {1.0 - t, t};
        double w2 = w[0] * w[0] + w[1] * w[1];
        double v = e / s.total;
        for (int j = 0; j < 2; ++j) {
            omega[j] += w[j] * w[j];
            delta[j] += v * (w[j] * w[j] * w[j] / w2);
        }
    }
    double phi[2] = {0, 0};
    for (int j = 0; j < 2; ++j) {
        if (fabs(omega[j]) > DBL_EPSILON) {
            double q = delta[j] / omega[j];
            phi[j] = isfinite(q) ? q : 0.0;
        }
    }
    return phi[0] - phi[1];
}

// The start of a level: a subject whose status is not zero (a failed earlier level) runs no
// iteration (limit 0). Returns whether the level runs.
__device__ __forceinline__ int syn_level_begin(SynDev* s, int level, int limit) {
    s->it = 0;
    s->limit = s->status == 0 ? limit : 0;
    s->converged = 0;
    s->level = level;
    s->count = 0;
    s->head = 0;
    s->total = 0.0;
    return s->limit > 0;
}

// Per-channel scalars, CC_STRIDE doubles a channel: [value (fixed, moving), |dF|^2, |dM|^2,
// valid voxels (masked CC), value (moving, fixed) (Mattes), status (Mattes)].
constexpr int CC_STRIDE = 8;

// The end of an iteration (syn.rs:941-958): the energy of the channels' values, the checks of
// the gradients, update maxima and inversion errors, the window convergence monitor, the
// iteration's record at trace[s->done] and the cancel flag (mapped host memory, may be null).
// cc: the per-channel scalars; max_bits: [F side, M side]; inv: 4 loop states. Returns whether
// the level goes on.
__device__ __forceinline__ int syn_record_step(SynDev* s, const double* __restrict__ cc,
                                               const unsigned int* __restrict__ max_bits,
                                               const InvState* __restrict__ inv,
                                               fw_syn_iteration* trace, int trace_cap,
                                               const volatile int* cancel) {
    // the CC value is symmetric in its two images; Mattes gives one value per direction
    auto value_m = [&](int c) {
        return s->metric[c] == FW_METRIC_MATTES ? cc[CC_STRIDE * c + 4] : cc[CC_STRIDE * c];
    };
    double vF = cc[0], vM = value_m(0);
    double wF = 0.0, wM = 0.0;
    for (int c = 0; c < s->channels; ++c) {
        wF += cc[CC_STRIDE * c] * s->wnorm[c];
        wM += value_m(c) * s->wnorm[c];
    }
    if (s->channels == 1) {
        wF = vF;
        wM = vM;
    }
    for (int c = 0; c < s->channels && s->channels > 1; ++c)
        if (!isfinite(cc[CC_STRIDE * c + 1]) || !isfinite(cc[CC_STRIDE * c + 2])) s->status = 1;
    for (int c = 0; c < s->channels; ++c) {
        if (s->metric[c] == FW_METRIC_MATTES) {
            const int k = (int)cc[CC_STRIDE * c + 5];
            if (k != 0) s->status = 10 + k;
        } else if (s->masked && cc[CC_STRIDE * c + 3] == 0.0) {
            s->status = 4;
        }
    }
    float mF = __uint_as_float(max_bits[0]), mM = __uint_as_float(max_bits[1]);
    if (!isfinite(mF) || !isfinite(mM)) s->status = 1;
    for (int q = 0; q < 4; ++q)
        if (!isfinite(inv[q].mean) || !isfinite(inv[q].max)) s->status = s->status ? s->status : 2;
    double energy = 0.5 * (vF + vM);
    // WindowConvergenceMonitor::add_energy_value
    if (s->count < s->window) {
        s->values[(s->head + s->count) % s->window] = energy;
        s->count++;
    } else {
        s->values[s->head] = energy;
        s->head = (s->head + 1) % s->window;
    }
    s->total += fabs(energy);
    double cv = convergence_value(*s);
    if (cv < s->threshold) s->converged = 1;
    int it = s->it, rec = s->done;
    if (rec < trace_cap) {
        fw_syn_iteration r;
        r.level = s->level;
        r.energy = energy;
        r.energy_weighted = 0.5 * (wF + wM);
        r.convergence_value = cv;
        r.fixed_update_scale = mF > 0.0f ? s->step / (double)mF : s->step;
        r.moving_update_scale = mM > 0.0f ? s->step / (double)mM : s->step;
        for (int q = 0; q < 4; ++q) {
            r.inversions[q].iterations = inv[q].executed;
            r.inversions[q].mean_error_norm = inv[q].executed ? inv[q].mean : 0.0;
            r.inversions[q].max_error_norm = inv[q].executed ? inv[q].max : 0.0;
        }
        trace[rec] = r;
    }
    s->it = it + 1;
    s->done = rec + 1;
    if (cancel && *cancel) s->status = 3;
    return (s->it < s->limit) && !s->converged && s->status == 0;
}

}  // namespace fw
